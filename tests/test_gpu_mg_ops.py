"""GPU parity of the multigrid level operations and of every kernel path (fused ghost writes,
fused residual+restriction+norms, single-CTA tail, per-operation reference kernels) against the
CPU oracle, bit for bit."""
import numpy as np
import pytest

import opencurrent_b200 as ocu
from oracle import oracle_ctypes as O
from tests.helpers import F32, F64, SCALAR_BCS, bc_from, mg_params, npdt
from tests.test_gpu_parity import assert_same, dev_grid, to_ocu_bc

pytestmark = pytest.mark.gpu


def pair(dt, shape, h, bcname, seed=0, sym=0, disable_host=0, conv=0x05, **knobs):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    L = O.layout(nx, ny, nz)
    rhs = np.zeros(int(L.allocated), npdt(dt))
    b = rng.uniform(-1, 1, shape)
    b -= b.mean()
    O.interior(rhs, L)[:] = b.astype(npdt(dt))
    bc = bc_from(SCALAR_BCS[bcname])
    om = O.OracleMG("d" if dt == F64 else "f", mg_params(bc, sym=sym, disable_host=disable_host, conv=conv),
                    nx, ny, nz, *h, rhs, L)
    g = dev_grid(rhs, dt, L)
    dm = ocu.Sol_MultigridPressure3DDevice(dt)
    dm.bc = to_ocu_bc(bc)
    dm.make_symmetric_operator = bool(sym)
    dm.disable_relax_on_host = bool(disable_host)
    dm.convergence = conv
    for k, v in knobs.items():
        setattr(dm, k, v)
    dm.initialize_storage(nx, ny, nz, *h, g)
    dm._sync_params()
    # random initial guess with consistent ghosts on both sides
    u0 = rng.uniform(-1, 1, shape).astype(npdt(dt))
    ou, Lu = om.grid("u", 0)
    O.interior(ou, Lu)[:] = u0
    s = "_d" if dt == F64 else "_f"
    getattr(O.lib(), "orc_bc_level1" + s)(O.ptr(ou), __import__("ctypes").byref(Lu),
                                          __import__("ctypes").byref(bc), *h)
    dm.pressure().copy_from_host(ou)
    return om, dm, g


KNOBS = [dict(), dict(unfused=True), dict(tail_cells=-1), dict(tail_cells=40000), dict(tail_cells=4096),
         dict(store_residual_grids=True), dict(sweep_cells=1), dict(sweep_cells=-1)]


@pytest.mark.parametrize("dt", [F32, F64])
@pytest.mark.parametrize("bcname", ["neumann", "periodic", "mixed_all", "neumann_inhom", "dirichlet", "mixed_dn"])
@pytest.mark.parametrize("order", [0, 1, 2])
@pytest.mark.parametrize("sweep", [1, -1])
def test_relax_levels(dt, bcname, order, sweep):
    """Every level, both relax paths: the two-colour TMA pass (sweep_cells=1 puts every
    eligible level on it) and the per-colour launches."""
    om, dm, _ = pair(dt, (32, 32, 32), (0.03, 0.03, 0.03), bcname, seed=1, sweep_cells=sweep)
    lib = O.lib()
    for lev in range(om.num_levels):
        it = 3
        lib.orc_mg_relax(om.h, 0, lev, it, order)
        dm.relax(lev, it, order)
        dm.synchronize()
        assert_same(dm.read_u(lev).copy_to_host(), om.grid("u", lev)[0], f"relax level {lev}")


@pytest.mark.parametrize("dt", [F32, F64])
@pytest.mark.parametrize("knobs", range(len(KNOBS)))
def test_restrict_and_prolong(dt, knobs):
    om, dm, _ = pair(dt, (64, 32, 48), (0.02, 0.03, 0.02), "neumann_inhom", seed=2, **KNOBS[knobs])
    import ctypes as C
    lib = O.lib()
    for lev in range(om.num_levels - 1):
        l2o, lio = C.c_double(), C.c_double()
        lib.orc_mg_restrict_residuals(om.h, 0, lev, lev + 1, C.byref(l2o), C.byref(lio))
        l2d, lid = dm.restrict_residuals(lev, lev + 1, norms=True)
        assert (l2d, lid) == (l2o.value, lio.value), lev
        assert_same(dm.read_b(lev + 1).copy_to_host(), om.grid("b", lev + 1)[0], f"restricted b {lev + 1}")
        if KNOBS[knobs].get("store_residual_grids"):
            assert_same(dm.read_r(lev).copy_to_host(), om.grid("r", lev)[0], f"r {lev}")
    for lev in range(om.num_levels - 2, -1, -1):
        lib.orc_mg_prolong(om.h, 0, lev + 1, lev)
        dm.prolong(lev + 1, lev)
        dm.synchronize()
        assert_same(dm.read_u(lev).copy_to_host(), om.grid("u", lev)[0], f"prolong into {lev}")


# Rows of 128 and 256 cells take the FP32 float4 kernels (colour sweep: nz % 128 = 0; prolongation:
# coarse nz % 64 = 0), including their j/i-face rows, z-face ghosts and lane-edge neighbours.
LONG_ROWS = [(12, 20, 256), (20, 10, 128)]


@pytest.mark.parametrize("dt", [F32, F64])
@pytest.mark.parametrize("bcname", ["neumann", "periodic", "neumann_inhom", "dirichlet", "mixed_dn", "mixed_all"])
@pytest.mark.parametrize("shape", LONG_ROWS)
def test_relax_levels_long_rows(dt, bcname, shape):
    om, dm, _ = pair(dt, shape, (0.03, 0.02, 0.01), bcname, seed=4)
    lib = O.lib()
    for lev in range(om.num_levels):
        for order in (0, 1, 2):
            lib.orc_mg_relax(om.h, 0, lev, 2, order)
            dm.relax(lev, 2, order)
        dm.synchronize()
        assert_same(dm.read_u(lev).copy_to_host(), om.grid("u", lev)[0], f"relax level {lev}")


@pytest.mark.parametrize("dt", [F32, F64])
@pytest.mark.parametrize("bcname", ["neumann_inhom", "periodic", "dirichlet", "mixed_all"])
@pytest.mark.parametrize("shape", LONG_ROWS + [(80, 220, 128)])  # the last: float4 prolongation (coarse > 64^3 cells)
def test_restrict_and_prolong_long_rows(dt, bcname, shape):
    import ctypes as C
    om, dm, _ = pair(dt, shape, (0.03, 0.02, 0.01), bcname, seed=5)
    lib = O.lib()
    for lev in range(om.num_levels - 1):
        l2o, lio = C.c_double(), C.c_double()
        lib.orc_mg_restrict_residuals(om.h, 0, lev, lev + 1, C.byref(l2o), C.byref(lio))
        l2d, lid = dm.restrict_residuals(lev, lev + 1, norms=True)
        assert (l2d, lid) == (l2o.value, lio.value), lev
        assert_same(dm.read_b(lev + 1).copy_to_host(), om.grid("b", lev + 1)[0], f"restricted b {lev + 1}")
    rng = np.random.default_rng(6)
    for lev in range(om.num_levels - 2, -1, -1):
        # a nonzero coarse correction and fine guess, the same buffers (ghosts included) on both sides
        for q in (lev + 1, lev):
            ou, Lq = om.grid("u", q)
            O.interior(ou, Lq)[:] = rng.uniform(-1, 1, O.interior(ou, Lq).shape).astype(ou.dtype)
            dm.read_u(q).copy_from_host(ou)
        lib.orc_mg_prolong(om.h, 0, lev + 1, lev)
        dm.prolong(lev + 1, lev)
        dm.synchronize()
        assert_same(dm.read_u(lev).copy_to_host(), om.grid("u", lev)[0], f"prolong into {lev}")


@pytest.mark.parametrize("dt", [F32, F64])
@pytest.mark.parametrize("knobs", range(len(KNOBS)))
@pytest.mark.parametrize("case", [((64, 64, 64), "neumann", 0, 0), ((48, 32, 64), "periodic", 1, 0),
                                  ((32, 64, 32), "mixed_xdir", 0, 1), ((96, 48, 48), "mixed_all", 1, 1),
                                  ((40, 24, 48), "mixed_dn", 1, 0), ((64, 48, 56), "dirichlet", 0, 0)])
def test_kernel_paths_match_oracle(dt, knobs, case):
    shape, bcname, sym, disable_host = case
    om, dm, _ = pair(dt, shape, (0.02, 0.025, 0.02), bcname, seed=3, sym=sym, disable_host=disable_host,
                     **KNOBS[knobs])
    om.run_fmg(2)
    dm.run_fmg(2)
    assert_same(dm.pressure().copy_to_host(), om.grid("u", 0)[0], f"fmg {KNOBS[knobs]}")
    om.run_vcycles(3)
    dm.run_vcycles(3)
    assert_same(dm.pressure().copy_to_host(), om.grid("u", 0)[0], f"vcycles {KNOBS[knobs]}")
    tol = 1e-4 if dt == F32 else 1e-9
    ok_o, res_o = om.solve(tol, 20)
    ok_d, res_d = dm.solve(tol, 20)
    assert (ok_o, res_o) == (ok_d, res_d)
    assert_same(dm.pressure().copy_to_host(), om.grid("u", 0)[0], f"solve {KNOBS[knobs]}")


def test_odd_periodic_coarsest_device_relax():
    """disable_relax_on_host with an odd periodic coarsest level (10 -> 5): the ghost refresh
    between colours cannot ride along with the sweep, so the separate fill runs."""
    om, dm, _ = pair(F64, (40, 40, 40), (0.025,) * 3, "periodic", seed=4, disable_host=1)
    om.run_fmg(1)
    dm.run_fmg(1)
    assert_same(dm.pressure().copy_to_host(), om.grid("u", 0)[0], "odd periodic coarsest")


def test_rayleigh_critical_number_on_gpu():
    """RayleighTest protocol (rayleigh.cpp) through the CUDA path: Ra_c(16) = 659.693989."""
    from tests.rayleigh import critical_rayleigh_device
    ra = critical_rayleigh_device(16)
    assert abs(ra - 659.693989) < 3e-3, ra
