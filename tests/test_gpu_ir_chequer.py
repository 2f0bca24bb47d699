"""The refinement mixed solver with its split-layout FP32 correction solver (the default).

Its inner FP32 cycles are this library's own algorithm (red/black colour arrays, fused
multiply-adds), so the check is the one the mixed-precision config states: the solve reaches the
requested relative residual, and its solution is compared with an FP64 multigrid solution driven
well past that tolerance (the oracle's FP64 solver), with the difference printed per case
(`IRCHQ ...`, pytest -s) and bounded.
"""
import numpy as np
import pytest

import opencurrent_b200 as ocu
from oracle import oracle_ctypes as O
from tests.helpers import F64, SCALAR_BCS, bc_from, mg_params
from tests.test_gpu_parity import assert_same, dev_grid, to_ocu_bc

pytestmark = pytest.mark.gpu

SINGULAR = {"neumann", "neumann_inhom", "periodic", "mixed_zneu"}
CASES = [
    ((64, 64, 64), (1 / 64, 1 / 64, 1 / 64), "neumann"),
    ((64, 32, 48), (1 / 64, 1 / 32, 1 / 48), "dirichlet"),
    ((32, 32, 32), (1 / 32, 1 / 32, 1 / 32), "periodic"),
    ((48, 32, 40), (0.03, 0.03, 0.06), "mixed_xdir"),
    ((24, 24, 48), (0.04, 0.05, 0.03), "mixed_zneu"),
    ((40, 40, 24), (0.025, 0.025, 0.04), "mixed_all"),
    ((96, 96, 96), (1 / 96, 1 / 96, 1 / 96), "mixed_dn"),
]


def rel_l2(a, b, L, remove_mean):
    x = O.interior(a, L).astype(np.float64)
    y = O.interior(b, L).astype(np.float64)
    if remove_mean:
        x, y = x - x.mean(), y - y.mean()
    return float(np.linalg.norm(x - y) / np.linalg.norm(y))


def problem(shape, seed):
    L = O.layout(*shape)
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1, 1, shape)
    b -= b.mean()
    rhs = np.zeros(int(L.allocated), np.float64)
    O.interior(rhs, L)[:] = b
    return L, rhs, float(np.sqrt(np.mean(b * b)))


@pytest.mark.parametrize("case", range(len(CASES)))
def test_ir_split_inner_reaches_1e10(case):
    shape, h, bcname = CASES[case]
    L, rhs, rms = problem(shape, 700 + case)
    bc = bc_from(SCALAR_BCS[bcname])
    tol = 1e-10 * rms
    om = O.OracleMG("d", mg_params(bc), *shape, *h, rhs.copy(), L)
    ok_o, res_o = om.solve(1e-13 * rms, 60)  # to its FP64 floor
    assert res_o <= 2e-11 * rms, res_o / rms
    g = dev_grid(rhs, F64, L)
    dm = ocu.Sol_MultigridPressureMixed3DDeviceD("ir")
    dm.bc = to_ocu_bc(bc)
    dm.initialize_storage(*shape, *h, g)
    ok, res = dm.solve(tol, 20)
    e = rel_l2(dm.pressure().copy_to_host(), om.grid("u", 0)[0], L, bcname in SINGULAR)
    # the reference-layout inner solves on the same problem, for the refinement step count
    ge = dev_grid(rhs, F64, L)
    de = ocu.Sol_MultigridPressureMixed3DDeviceD("ir")
    de.bc = to_ocu_bc(bc)
    de.ir_inner_exact = True
    de.initialize_storage(*shape, *h, ge)
    ok_e, res_e = de.solve(tol, 20)
    print(f"IRCHQ {bcname} {shape} rel_res={res / rms:.3e} outer={dm.stats.outer_iterations} "
          f"fp32_cycles={dm.stats.vcycles} err_vs_fp64_oracle={e:.3e} "
          f"exact_inner_outer={de.stats.outer_iterations}")
    assert ok and res <= tol
    # the split solver carries the coarse solution up by nested iteration (smoothing per level)
    # instead of one V-cycle per level: cheaper steps, and on the harder boundary mixes up to
    # about half again as many of them
    assert dm.stats.outer_iterations <= 1.5 * de.stats.outer_iterations + 1
    assert e <= 1e-7


@pytest.mark.parametrize("shape", [(8, 8, 8), (16, 16, 16), (16, 8, 32)])
def test_ir_small_grids_through_the_tail(shape):
    """Grids whose split hierarchy lies wholly (8^3: 512 cells) or from level 1 on in the
    single-CTA tail: the correction then ends with x += e as its own pass (wholly in the tail)
    or in the last prolongation out of the tail; both reach 1e-10 and the FP64 solution."""
    L, rhs, rms = problem(shape, 800)
    bc = bc_from(SCALAR_BCS["neumann"])
    h = tuple(1.0 / n for n in shape)
    om = O.OracleMG("d", mg_params(bc), *shape, *h, rhs.copy(), L)
    ok_o, res_o = om.solve(1e-13 * rms, 60)
    assert res_o <= 2e-11 * rms
    dm = ocu.Sol_MultigridPressureMixed3DDeviceD("ir")
    dm.bc = to_ocu_bc(bc)
    dm.initialize_storage(*shape, *h, dev_grid(rhs, F64, L))
    ok, res = dm.solve(1e-10 * rms, 20)
    e = rel_l2(dm.pressure().copy_to_host(), om.grid("u", 0)[0], L, True)
    print(f"IRCHQ small {shape} rel_res={res / rms:.3e} outer={dm.stats.outer_iterations} err={e:.3e}")
    assert ok and res <= 1e-10 * rms
    assert e <= 1e-7


def test_ir_split_inner_second_solve_repeats_first():
    """A second solve from a zero guess replays the captured step and gives the same result."""
    shape, h, bcname = CASES[0]
    L, rhs, rms = problem(shape, 11)
    g = dev_grid(rhs, F64, L)
    dm = ocu.Sol_MultigridPressureMixed3DDeviceD("ir")
    dm.bc = to_ocu_bc(bc_from(SCALAR_BCS[bcname]))
    dm.initialize_storage(*shape, *h, g)
    ok1, r1 = dm.solve(1e-10 * rms, 20)
    p1 = dm.pressure().copy_to_host()
    dm.pressure().clear_zero()
    ok2, r2 = dm.solve(1e-10 * rms, 20)
    assert ok1 and ok2 and r1 == r2
    assert_same(dm.pressure().copy_to_host(), p1, "second solve")


def test_ir_odd_periodic_hierarchy_uses_exact_inner():
    """A periodic axis that is odd on a coarse level (20 -> 10 -> 5) is not taken by the split
    solver; the reference-layout inner solves run and reach the tolerance."""
    shape, h = (20, 40, 20), (0.05, 0.05, 0.05)
    L, rhs, rms = problem(shape, 12)
    bc = bc_from(SCALAR_BCS["periodic"])
    om = O.OracleMG("d", mg_params(bc), *shape, *h, rhs.copy(), L)
    om.solve(1e-13 * rms, 60)
    g = dev_grid(rhs, F64, L)
    dm = ocu.Sol_MultigridPressureMixed3DDeviceD("ir")
    dm.bc = to_ocu_bc(bc)
    dm.initialize_storage(*shape, *h, g)
    ok, res = dm.solve(1e-10 * rms, 20)
    e = rel_l2(dm.pressure().copy_to_host(), om.grid("u", 0)[0], L, True)
    print(f"IRCHQ odd-periodic fallback rel_res={res / rms:.3e} err_vs_fp64_oracle={e:.3e}")
    assert ok and res <= 1e-10 * rms
    assert e <= 1e-7


def test_split_level_operations_run_on_every_level():
    """The split hierarchy's level operations of the C ABI (core 2: a colour sweep, red-black
    iterations, residual + restriction into the next level, prolongation from it) launch on
    every level, and levels out of range or norms requested from the split hierarchy are refused."""
    shape, h, bcname = CASES[1]
    L, rhs, rms = problem(shape, 13)
    g = dev_grid(rhs, F64, L)
    dm = ocu.Sol_MultigridPressureMixed3DDeviceD("ir")
    dm.bc = to_ocu_bc(bc_from(SCALAR_BCS[bcname]))
    dm.initialize_storage(*shape, *h, g)
    levels = dm.stats.num_levels
    assert levels >= 3
    for lv in range(levels):
        dm.relax_sweep(lv, 0, core=2)
        dm.relax_sweep(lv, 1, core=2)
        dm.relax(lv, 2, order=1, core=2)
        if lv + 1 < levels:
            dm.restrict_residuals(lv, lv + 1, core=2)
            dm.prolong(lv + 1, lv, core=2)
    dm.synchronize()
    with pytest.raises(ocu.OcuError):
        dm.relax_sweep(levels, 0, core=2)
    with pytest.raises(ocu.OcuError):
        dm.restrict_residuals(0, 2, core=2)
    with pytest.raises(ocu.OcuError):
        dm.restrict_residuals(0, 1, norms=True, core=2)
    with pytest.raises(ocu.OcuError):
        dm.prolong(levels, levels - 1, core=2)
    # the solve afterwards is unaffected by the level operations (they work on its scratch levels)
    ok, res = dm.solve(1e-10 * rms, 20)
    assert ok and res <= 1e-10 * rms
