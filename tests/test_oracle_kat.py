"""CPU: pin the oracle against the reference's own known answers and properties.

The reference ships no golden vectors; its tests pin tolerances and analytic answers.  Each
test below re-expresses one of them (file:line of the reference test in the docstring) against
the oracle, so that the oracle is trusted before it is used as the parity checker for the GPU.
"""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import oracle_ctypes as O
from tests.helpers import DIR, F32, F64, INFLOW, NEU, PER, MAC_BCS, bc_from, mg_params, npdt


def test_layout_rule():
    """Grid3DDevice<T>::init (grid3ddev.cu:358-400): pnz rounded to 16, 16-gz pre-padding."""
    L = O.layout(64, 64, 64)
    assert (L.pnx, L.pny, L.pnz) == (66, 66, 80)
    assert L.allocated == 348495
    assert L.shift == 1 * 80 * 66 + 1 * 80 + 16
    L = O.layout(256, 256, 256)
    assert L.pnz == 272 and L.allocated == 18105423
    # k = 0 of every row sits on a 16-element boundary
    assert (L.shift + 5 * L.xstride + 7 * L.ystride) % 16 == 0


@pytest.mark.parametrize("n,levels,coarsest", [(64, 5, 4), (256, 7, 4), (96, 5, 6), (48, 4, 6),
                                               (80, 4, 10), (32, 4, 4)])
def test_num_levels(n, levels, coarsest):
    """num_levels (sol_mgpressure3d.cpp:67-92)."""
    assert O.lib().orc_num_levels(n, n, n) == levels
    assert n // 2 ** (levels - 1) == coarsest


def test_optimal_omega():
    """Yavneh's omega (sol_mgpressure3d.cpp:94-109): isotropic h gives ~1.1459."""
    w = O.lib().orc_optimal_omega(1.0, 1.0, 1.0)
    c = 1 - 1 / 3
    assert abs(w - 2 / (1 + math.sqrt(1.0 - c * c))) < 1e-15
    assert abs(w - 1.1459) < 1e-4


def _cos_rhs(nx, ny, nz, hx, hy, hz, axis):
    """init_rhs of mgdoubletest.cpp:44-97: mean-removed cos(x) sin(y) cos(z)."""
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    x = (i - 0.5) * 2 * np.pi * hx
    y = (j - 0.5) * 2 * np.pi * hy
    z = (k - 0.5) * 2 * np.pi * hz
    if axis in (1, 2):
        x = np.zeros_like(x)
    if axis in (0, 2):
        y = np.full_like(y, np.pi / 2)
    if axis in (0, 1):
        z = np.zeros_like(z)
    f = np.cos(x) * np.sin(y) * np.cos(z)
    return f - f.mean()


@pytest.mark.parametrize("dt,tol", [(F64, 1e-8), (F32, 1e-3)])
@pytest.mark.parametrize("value", [0.0, 0.5, 1.0])
def test_all_dirichlet_zero_rhs(dt, tol, value):
    """run_all_dirichelet_test (mgdoubletest.cpp:199-227, mgtest.cpp:179-201): zero RHS with
    Dirichlet value v everywhere => p == v, from a hashed random initial guess."""
    n = 32
    L = O.layout(n, n, n)
    rhs = np.zeros(int(L.allocated), npdt(dt))
    m = O.OracleMG("d" if dt == F64 else "f", mg_params(O.bcset_all(DIR, value)), n, n, n,
                   4 / n, 4 / n, 4 / n, rhs, L)
    u, Lu = m.grid("u", 0)
    rng = np.random.default_rng(1)
    O.interior(u, Lu)[:] = (0.5 - rng.random((n, n, n))).astype(npdt(dt))
    ok, res = m.solve(tol, 15)
    assert ok and res < tol
    ui = O.interior(u, Lu)
    assert np.abs(ui - value).max() < max(tol, 1e-6) * 10


@pytest.mark.parametrize("dt,tol", [(F64, 1e-8), (F32, 1e-3)])
@pytest.mark.parametrize("axis,value", [(0, 0.0), (1, 1.0), (2, -1.0), (2, 0.321)])
@pytest.mark.parametrize("h", [(4 / 32, 4 / 32, 4 / 32), (4 / 32, 5 / 32, 6 / 32)])
def test_isotropic_dirichlet_axis(dt, tol, axis, value, h):
    """run_isotropic_test (mgdoubletest.cpp:150-197): Dirichlet on one axis, periodic on the
    others, cos*sin*cos RHS; the solve reaches the tolerance."""
    n = 32
    L = O.layout(n, n, n)
    rhs = np.zeros(int(L.allocated), npdt(dt))
    O.interior(rhs, L)[:] = _cos_rhs(n, n, n, *h, axis).astype(npdt(dt))
    faces = {f: (PER, 0.0) for f in ("xpos", "xneg", "ypos", "yneg", "zpos", "zneg")}
    names = [("xpos", "xneg"), ("ypos", "yneg"), ("zpos", "zneg")][axis]
    for f in names:
        faces[f] = (DIR, value)
    m = O.OracleMG("d" if dt == F64 else "f", mg_params(bc_from(faces)), n, n, n, *h, rhs, L)
    ok, res = m.solve(tol, 16)
    assert ok and res < tol


@pytest.mark.parametrize("dt,tol", [(F64, 1e-8), (F32, 1e-3)])
@pytest.mark.parametrize("kind", ["neumann", "periodic"])
@pytest.mark.parametrize("sym", [0, 1])
def test_neumann_and_periodic(dt, tol, kind, sym):
    """run_neumann_test / run_all_periodic_test (mgdoubletest.cpp:229-272), symmetric and not."""
    nx, ny, nz = 32, 16, 24
    h = (4 / 32, 4 / 16, 4 / 32)
    L = O.layout(nx, ny, nz)
    rhs = np.zeros(int(L.allocated), npdt(dt))
    O.interior(rhs, L)[:] = _cos_rhs(nx, ny, nz, *h, -1).astype(npdt(dt))
    t = NEU if kind == "neumann" else PER
    m = O.OracleMG("d" if dt == F64 else "f", mg_params(O.bcset_all(t, 0.0), sym=sym), nx, ny, nz, *h,
                   rhs, L)
    ok, res = m.solve(tol, 20)
    assert ok and res < tol


def test_fp32_config1_converges():
    """64^3 FP32 Neumann, U[-1,1] seed 0: reaches 1e-6 relative RMS residual within 20 cycles."""
    from tests.helpers import config1_rhs
    n = 64
    L = O.layout(n, n, n)
    rhs = np.zeros(int(L.allocated), np.float32)
    O.interior(rhs, L)[:] = config1_rhs(n).astype(np.float32)
    rms = float(np.sqrt(np.mean(O.interior(rhs, L).astype(np.float64) ** 2)))
    m = O.OracleMG("f", mg_params(O.bcset_all(NEU, 0.0)), n, n, n, 1 / n, 1 / n, 1 / n, rhs, L)
    ok, res = m.solve(1e-6 * rms, 20)
    assert ok and res / rms < 1e-6
    assert 3 <= m.vcycles <= 10


def test_mixed_and_ir_agree_with_fp64():
    """Reference mixed solver (mgmixedtest.cpp) and the IR solver both reach 1e-10 relative and
    agree with the plain FP64 solution (mean removed) to the FP64 solve's accuracy."""
    n = 32
    L = O.layout(n, n, n)
    rng = np.random.default_rng(4)
    b = rng.uniform(-1, 1, (n, n, n))
    b -= b.mean()
    rms = float(np.sqrt(np.mean(b ** 2)))
    sols = {}
    for kind in ("d", "mixed", "ir"):
        rhs = np.zeros(int(L.allocated), np.float64)
        O.interior(rhs, L)[:] = b
        m = O.OracleMG(kind, mg_params(O.bcset_all(NEU, 0.0)), n, n, n, 1 / n, 1 / n, 1 / n, rhs, L,
                       inner_cycles=3)
        ok, res = m.solve(1e-10 * rms, 30)
        assert ok and res <= 1e-10 * rms, (kind, res / rms)
        u = O.interior(m.grid("u", 0)[0], L).copy()
        sols[kind] = u - u.mean()
    scale = np.abs(sols["d"]).max()
    assert np.abs(sols["mixed"] - sols["d"]).max() < 1e-6 * scale
    assert np.abs(sols["ir"] - sols["d"]).max() < 1e-6 * scale


def _project_case(dt, nx, ny, nz, h, bc):
    """ProjectTest (projecttest.cpp:27-136): sine velocity field, project, max|div| small."""
    Lu = O.layout(nx + 1, ny, nz, 1, 1, 1, 0, 1, 1)
    bufs = [np.zeros(int(Lu.allocated), npdt(dt)) for _ in range(3)]
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    fields = [np.sin(k / nz * 4 * np.pi) + np.sin(j / ny * 4 * np.pi),
              np.sin(k / nz * 8 * np.pi) + np.sin(i / nx * 6 * np.pi),
              np.cos(j / ny * 8 * np.pi) + np.sin(k / nz * 6 * np.pi)]
    for buf, f in zip(bufs, fields):
        O.region(buf, Lu, 0, nx, 0, ny, 0, nz)[:] = f.astype(npdt(dt))
    lib = O.lib()
    s = "_d" if dt == F64 else "_f"
    getattr(lib, "orc_mac_bc_level1" + s)(*[O.ptr(b) for b in bufs], C.byref(Lu), nx, ny, nz, C.byref(bc), *h)
    p = lib.orc_project_create(dt, C.byref(bc), nx, ny, nz, *h, *[O.ptr(b) for b in bufs], C.byref(Lu))
    return lib, p, bufs, Lu


@pytest.mark.parametrize("dt,tol", [(F32, 2e-4), (F64, 1e-10)])
@pytest.mark.parametrize("bcname", ["periodic", "closed_noslip", "inflow"])
def test_projection_divergence_free(dt, tol, bcname):
    nx, ny, nz = 32, 16, 16
    h = (0.5, 0.5, 1.0)
    bc = bc_from(MAC_BCS[bcname])
    lib, p, bufs, Lu = _project_case(dt, nx, ny, nz, h, bc)
    assert lib.orc_project_solve(p, tol)
    lib.orc_project_solve_divergence_only(p)
    Ld = O.layout(nx, ny, nz, 1, 1, 1, Lu.pnx - nx - 2, Lu.pny - ny - 2, Lu.pnz - nz - 2)
    div = O.wrap(lib.orc_project_divergence(p), Ld, dt)
    assert np.abs(O.interior(div, Ld)).max() <= tol
    lib.orc_project_destroy(p)


def test_advection_symmetry_and_mass():
    """Advection3DTest (advection3dtest.cpp:159-213): an axis-symmetric blob advected by a
    uniform field gives mirror-symmetric dphi/dt; a divergence-free periodic field conserves
    mass (sum of dphi/dt is zero)."""
    n = 16
    Lt = O.layout(n, n, n, 1, 1, 1, 1, 1, 1)
    bufs = {c: np.zeros(int(Lt.allocated), np.float64) for c in "uvwp"}
    i, j, k = np.meshgrid(np.arange(n) + 0.5, np.arange(n) + 0.5, np.arange(n) + 0.5, indexing="ij")
    r2 = (i - n / 2) ** 2 + (j - n / 2) ** 2 + (k - n / 2) ** 2
    O.region(bufs["p"], Lt, -1, n + 1, -1, n + 1, -1, n + 1)[:] = 0
    O.interior(bufs["p"], Lt)[:] = np.exp(-r2 / 8)
    lib = O.lib()
    lib.orc_bc_level1_d(O.ptr(bufs["p"]), C.byref(Lt), C.byref(O.bcset_all(PER)), 1, 1, 1)
    for it in (1, 2):
        for axis, c in enumerate("uvw"):
            for cc in "uvw":
                bufs[cc][:] = 0
            bufs[c][:] = 1.0
            d = np.zeros(int(Lt.allocated), np.float64)
            lib.orc_advect_passive_d(*[O.ptr(bufs[x]) for x in "uvwp"], O.ptr(d), C.byref(Lt), n, n, n,
                                     1.0, 1.0, 1.0, it)
            di = O.interior(d, Lt)
            assert abs(di.sum()) < 1e-10
            # the two transverse axes stay mirror symmetric about the blob centre
            for ax in range(3):
                if ax != axis:
                    assert np.abs(di - np.flip(di, axis=ax)).max() < 1e-12


@pytest.mark.slow
def test_rayleigh_critical_number_free_slip_16():
    """RayleighTest (rayleigh.cpp:64-345): free-slip Rayleigh-Benard at resolution 16, vertical
    z; bracket the growth-rate sign change between Ra = 659 and 660 and interpolate.  The
    reference records Ra_c(16) = 659.693989 (rayleigh.cpp:338)."""
    from tests.rayleigh import critical_rayleigh_oracle
    ra = critical_rayleigh_oracle(16)
    # seeds 0..2 give 659.6931, 659.6929, 659.6932: the random start moves Ra_c by ~3e-4
    assert abs(ra - 659.693989) < 3e-3, ra
