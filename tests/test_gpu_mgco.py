"""GPU: the multi-image multigrid solver (Sol_MultigridPressure3DDeviceCo, sol_mgpressure3dco.cu).

N images (slabs along x) share one device here and are driven in lockstep with device-to-device
halo copies ordered by events (on several devices the same copies cross NVLink).  Every per-cell
operation is the single-image solver's, so after a fixed number of FMG or V-cycles the images'
slabs put together equal, bit for bit, the oracle's solve of the whole grid, every level from
the cutoff down included.  Solves to a tolerance take as many cycles as the oracle's; the
residual norm is folded across images in image order, so it is compared within rounding.
"""
import numpy as np
import pytest

import opencurrent_b200 as ocu
from oracle import oracle_ctypes as O
from tests.helpers import SCALAR_BCS, bc_from, mg_params
from tests.test_gpu_parity import assert_same, dev_grid, to_ocu_bc

pytestmark = pytest.mark.gpu

F32, F64 = ocu.F32, ocu.F64
SINGULAR = {"neumann", "neumann_inhom", "periodic", "mixed_zneu"}

# (global shape, spacings, bc, images, cutoff cells): the cutoffs put 1 to 3 levels on the images
CASES = [
    ((64, 32, 32), (1 / 64, 1 / 32, 1 / 32), "neumann", 2, 512),
    ((64, 32, 32), (1 / 64, 1 / 32, 1 / 32), "neumann", 4, 512),
    ((32, 32, 32), (1 / 32,) * 3, "periodic", 2, 64 ** 3),
    ((64, 16, 24), (0.05, 0.04, 0.06), "dirichlet", 4, 1000),
    ((48, 32, 40), (0.03, 0.03, 0.06), "mixed_xdir", 2, 4000),
    ((32, 24, 48), (0.04, 0.05, 0.03), "mixed_zneu", 4, 2000),
    ((64, 32, 32), (0.02, 0.03, 0.03), "mixed_dn", 2, 512),
    ((40, 40, 20), (0.05, 0.05, 0.05), "neumann_inhom", 2, 4000),
]


def npdt(dt):
    return np.float64 if dt == F64 else np.float32


def rhs_field(shape, bcname, seed):
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1, 1, shape)
    if bcname in SINGULAR:
        b -= b.mean()
    return b


def co_solver(dt, shape, h, bcname, N, cutoff, b, **params):
    nxl = shape[0] // N
    Ls = O.layout(nxl, shape[1], shape[2])
    rhs = []
    for i in range(N):
        host = np.zeros(int(Ls.allocated), npdt(dt))
        O.interior(host, Ls)[:] = b[i * nxl:(i + 1) * nxl].astype(npdt(dt))
        rhs.append(dev_grid(host, dt, Ls))
    s = ocu.Sol_MultigridPressure3DDeviceCo(dt, N)
    s.bc = to_ocu_bc(bc_from(SCALAR_BCS[bcname]))
    s.grid_size_for_cutoff = cutoff
    for k, v in params.items():
        setattr(s, k, v)
    s.initialize_storage(nxl, shape[1], shape[2], *h, rhs)
    return s, Ls, rhs


def oracle_solver(dt, shape, h, bcname, b, **kw):
    L = O.layout(*shape)
    host = np.zeros(int(L.allocated), npdt(dt))
    O.interior(host, L)[:] = b.astype(npdt(dt))
    om = O.OracleMG("d" if dt == F64 else "f", mg_params(bc_from(SCALAR_BCS[bcname]), **kw), *shape, *h, host, L)
    return om, L, host


def whole(s, N, Ls):
    return np.concatenate([O.interior(s.co_pressure(i).copy_to_host(), Ls) for i in range(N)], axis=0)


@pytest.mark.parametrize("dt", [F32, F64])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_fixed_schedule_bit_identical_to_oracle(dt, case):
    shape, h, bcname, N, cutoff = CASES[case]
    b = rhs_field(shape, bcname, 40 + case)
    s, Ls, keep = co_solver(dt, shape, h, bcname, N, cutoff, b)
    om, L, keep_o = oracle_solver(dt, shape, h, bcname, b)
    assert s.stats.num_levels == om.num_levels
    assert 1 <= s.cutoff_level < om.num_levels
    s.run_fmg(2)
    om.run_fmg(2)
    assert_same(whole(s, N, Ls), O.interior(om.grid("u", 0)[0], L), f"fmg {bcname} N={N}")
    s.run_vcycles(2)
    om.run_vcycles(2)
    assert_same(whole(s, N, Ls), O.interior(om.grid("u", 0)[0], L), f"vcycles {bcname} N={N}")
    # the levels held whole by image 0, ghosts included
    for lev in range(s.cutoff_level, om.num_levels):
        assert_same(s.read_u(lev).copy_to_host(), om.grid("u", lev)[0], f"u level {lev}")
        assert_same(s.read_b(lev).copy_to_host(), om.grid("b", lev)[0], f"b level {lev}")


@pytest.mark.parametrize("dt", [F32, F64])
@pytest.mark.parametrize("case", [0, 2, 5, 7])
def test_unfused_kernels_bit_identical_to_oracle(dt, case):
    """The reference's separate kernels (ghost fill after every colour, residual stored, then
    restricted) instead of the fused ones: the same bits."""
    shape, h, bcname, N, cutoff = CASES[case]
    b = rhs_field(shape, bcname, 60 + case)
    s, Ls, keep = co_solver(dt, shape, h, bcname, N, cutoff, b, unfused=True)
    om, L, keep_o = oracle_solver(dt, shape, h, bcname, b)
    s.run_fmg(1)
    om.run_fmg(1)
    s.run_vcycles(1)
    om.run_vcycles(1)
    assert_same(whole(s, N, Ls), O.interior(om.grid("u", 0)[0], L), f"unfused {bcname} N={N}")


@pytest.mark.parametrize("dt,tol", [(F32, 1e-4), (F64, 1e-9)])
@pytest.mark.parametrize("conv", [0x05, 0x0A])
def test_solve_to_tolerance(dt, tol, conv):
    shape, h, bcname, N = (64, 64, 64), (1 / 64,) * 3, "neumann", 2
    b = rhs_field(shape, bcname, 9)
    s, Ls, keep = co_solver(dt, shape, h, bcname, N, 16 ** 3, b, convergence=conv)
    om, L, keep_o = oracle_solver(dt, shape, h, bcname, b, conv=conv)
    ok_d, res_d = s.solve(tol, 15)
    ok_o, res_o = om.solve(tol, 15)
    print(f"MGCO dt={dt} conv={conv:#x} res={res_d:.6e}/{res_o:.6e} vcycles={s.stats.vcycles}/{om.vcycles}")
    assert ok_d and ok_o
    assert s.stats.vcycles == om.vcycles
    assert abs(res_d - res_o) <= (1e-5 if dt == F32 else 1e-12) * res_o
    assert_same(whole(s, N, Ls), O.interior(om.grid("u", 0)[0], L), "solved pressure")
    # a second solve starts from the converged pressure and stops at once
    ok2, _ = s.solve(tol, 15)
    assert ok2 and s.stats.vcycles == 0


def test_one_image_equals_single_image_solver():
    shape, h, bcname = (32, 32, 32), (1 / 32,) * 3, "periodic"
    b = rhs_field(shape, bcname, 3)
    s, Ls, keep = co_solver(F64, shape, h, bcname, 1, 8 ** 3, b)
    L = O.layout(*shape)
    host = np.zeros(int(L.allocated), np.float64)
    O.interior(host, L)[:] = b
    g = dev_grid(host, F64, L)
    d = ocu.Sol_MultigridPressure3DDevice(F64)
    d.bc = to_ocu_bc(bc_from(SCALAR_BCS[bcname]))
    d.initialize_storage(*shape, *h, g)
    s.run_fmg(1)
    d.run_fmg(1)
    assert_same(whole(s, 1, Ls), O.interior(d.pressure().copy_to_host(), L), "one image")


def test_argument_errors():
    shape, h, bcname = (64, 32, 32), (1 / 64, 1 / 32, 1 / 32), "neumann"
    b = rhs_field(shape, bcname, 1)
    # 16 slabs of 2 cells: level 2 (8 cells along x) is above the cutoff and does not split
    with pytest.raises(ocu.OcuError, match="does not split"):
        co_solver(F64, (32, 64, 64), (1 / 32, 1 / 64, 1 / 64), bcname, 16, 256,
                  rhs_field((32, 64, 64), bcname, 1))
    # one rhs per image
    Ls = O.layout(32, 32, 32)
    g = dev_grid(np.zeros(int(Ls.allocated)), F64, Ls)
    s = ocu.Sol_MultigridPressure3DDeviceCo(F64, 2)
    with pytest.raises(ValueError):
        s.initialize_storage(32, 32, 32, *h, [g])
    # rhs dimensions must be the slab's
    with pytest.raises(ocu.OcuError):
        s.initialize_storage(16, 32, 32, *h, [g, g])
    # a cutoff no level reaches would split the coarsest level
    with pytest.raises(ocu.OcuError, match="coarsest level"):
        co_solver(F64, shape, h, bcname, 2, 1, b)
    # the single-image entry point refuses a multi-image handle
    s2, Ls2, keep = co_solver(F64, shape, h, bcname, 2, 512, b)
    lib = ocu.load()
    assert lib.ocu_mg_initialize_storage(s2._h, 64, 32, 32, *h, keep[0]._h) != 0
    assert lib.ocu_mgco_num_images(s2._h) == 2
    # level operations act on every image (core 0)
    s2.relax(0, 1, core=0)
    s2.restrict_residuals(0, 1, core=0)
    s2.prolong(1, 0, core=0)
    s2.synchronize()
