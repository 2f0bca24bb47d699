"""CPU: the oracle's restatement of Sol_PCGPressure3DDevice (ocuequation/sol_pcgpressure3d.cu).

The operator L p = -div(c grad p) is checked independently here in numpy (face ghosts by the
Neumann / periodic rules, the reference's half-sum face coefficients), and the solver's pressure
must satisfy it to the requested tolerance for every preconditioner that is symmetric (none,
Jacobi, multigrid).  BFBT (multigrid then Jacobi) is not symmetric, so CG need not converge with
it; the reference's own behaviour is compared on the GPU (tests/test_gpu_pcg.py).
"""
import numpy as np
import pytest

from oracle import oracle_ctypes as O

BCS = {"neumann": 4, "periodic": 2}


def setup(n, dt, seed=1):
    L = O.layout(n, n, n)
    npd = np.float64 if dt == O.F64 else np.float32
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1, 1, (n, n, n))
    b -= b.mean()
    rhs = np.zeros(int(L.allocated), npd)
    O.interior(rhs, L)[:] = b
    x = (np.arange(n) + 0.5) / n
    c = (1 + 0.5 * np.sin(2 * np.pi * x))[:, None, None] * (1 + 0.25 * np.cos(2 * np.pi * x))[None, :, None]
    coef = np.zeros(int(L.allocated), npd)
    O.interior(coef, L)[:] = c * np.ones((n, n, n))
    return L, rhs, coef, b


def operator(p, c, h, periodic):
    """-div(c grad p) with the reference's face coefficients 0.5 (c_nbr + c)."""
    mode = "wrap" if periodic else "edge"
    P = np.pad(p, 1, mode=mode)
    Cp = np.pad(c, 1, mode=mode)
    out = np.zeros_like(p)
    cc = Cp[1:-1, 1:-1, 1:-1]
    pc = P[1:-1, 1:-1, 1:-1]
    for sl in [(slice(0, -2), slice(1, -1), slice(1, -1)), (slice(2, None), slice(1, -1), slice(1, -1)),
               (slice(1, -1), slice(0, -2), slice(1, -1)), (slice(1, -1), slice(2, None), slice(1, -1)),
               (slice(1, -1), slice(1, -1), slice(0, -2)), (slice(1, -1), slice(1, -1), slice(2, None))]:
        out -= (P[sl] - pc) * 0.5 * (Cp[sl] + cc) / (h * h)
    return out


@pytest.mark.parametrize("bcname", sorted(BCS))
@pytest.mark.parametrize("pc", [O.PRECOND_NONE, O.PRECOND_JACOBI, O.PRECOND_MULTIGRID])
def test_symmetric_preconditioners_solve_the_operator(bcname, pc):
    n = 16
    L, rhs, coef, b = setup(n, O.F64)
    prm = O.pcg_params(O.bcset_all(BCS[bcname], 0.0), pc)
    s = O.OraclePCG(O.F64, prm, n, n, n, 1 / n, 1 / n, 1 / n, rhs, coef, L)
    ok, res = s.solve(1e-8, 500)
    assert ok and res <= 1e-8
    p = O.interior(s.pressure(), L)
    r = b - operator(p, O.interior(coef, L), 1 / n, bcname == "periodic")
    rel = np.linalg.norm(r) / np.linalg.norm(b)
    assert rel <= 1e-6, rel
    if pc == O.PRECOND_MULTIGRID:  # multigrid preconditioning takes few iterations
        assert s.iterations <= 20, s.iterations


def test_unit_coefficient_matches_multigrid():
    n = 16
    L, rhs, coef, b = setup(n, O.F64, 3)
    O.interior(coef, L)[:] = 1.0
    prm = O.pcg_params(O.bcset_all(4, 0.0), O.PRECOND_MULTIGRID)
    s = O.OraclePCG(O.F64, prm, n, n, n, 1 / n, 1 / n, 1 / n, rhs, coef, L)
    ok, _ = s.solve(1e-10, 200)
    assert ok
    mp = O.MGParams()
    mp.bc = O.bcset_all(4, 0.0)
    mp.nu1 = mp.nu2 = 2
    mp.convergence = 0x05
    # the multigrid solves lap(p) = b; the CG operator is -lap
    neg = rhs.copy()
    O.interior(neg, L)[:] *= -1
    om = O.OracleMG("d", mp, n, n, n, 1 / n, 1 / n, 1 / n, neg, L)
    om.solve(1e-12, 50)
    x = O.interior(s.pressure(), L)
    y = O.interior(om.grid("u", 0)[0], L)
    x, y = x - x.mean(), y - y.mean()
    assert np.linalg.norm(x - y) / np.linalg.norm(y) <= 1e-7


def test_bad_arguments_and_boundary_types():
    n = 8
    L, rhs, coef, _ = setup(n, O.F32)
    with pytest.raises(RuntimeError):  # Dirichlet faces are refused (bc.check_type)
        O.OraclePCG(O.F32, O.pcg_params(O.bcset_all(3, 0.0)), n, n, n, 0.1, 0.1, 0.1, rhs, coef, L)
    s = O.OraclePCG(O.F32, O.pcg_params(O.bcset_all(4, 0.0), O.PRECOND_JACOBI), n, n, n, 0.1, 0.1, 0.1, rhs,
                    coef, L)
    assert s.solve(-1.0, 10) == (False, 0.0)
    assert s.solve(1e-3, 0) == (False, 0.0)
