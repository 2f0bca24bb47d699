"""Failure paths on the GPU, exercised without faulting, trapping or hanging it.

* A bounded device wait that runs out: the two-colour TMA pass (opt-in) in its test mode first
  waits on a barrier nothing completes (ocu_mg_params.wait_limit < 0), gives up before issuing
  any load, and the solve reports OCU_ERR_TIMEOUT; the next solve with the default limit starts
  clean and matches the oracle bit for bit.
* A solve that cannot converge (max_iter exhausted, or a NaN in the right-hand side) returns
  "not converged" after the reference's retry from a zero guess (sol_mgpressure3d.cpp:348-364),
  without any hang, and the solver stays usable.
* A projection whose pressure solve does not converge reports failure and sets the sticky error
  (sol_project3ddev.cu:67-78, error_handler.h:27-57), as the reference's does.
"""
import numpy as np
import pytest

import opencurrent_b200 as ocu
from opencurrent_b200._capi import ERR_TIMEOUT
from oracle import oracle_ctypes as O
from tests.helpers import F32, MAC_BCS, SCALAR_BCS, bc_from, mg_params, rand_buffer
from tests.test_gpu_parity import assert_same, dev_grid, mac_setup, to_ocu_bc

pytestmark = pytest.mark.gpu


def neumann_problem(n=64, seed=0, dt=F32):
    L = O.layout(n, n, n)
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1, 1, (n, n, n))
    b -= b.mean()
    rhs = np.zeros(int(L.allocated), np.float64 if dt == ocu.F64 else np.float32)
    O.interior(rhs, L)[:] = b.astype(rhs.dtype)
    return L, rhs, float(np.sqrt(np.mean(b * b)))


def test_bounded_wait_timeout_reports_and_recovers():
    n = 64
    L, rhs, rms = neumann_problem(n, 1)
    bc = bc_from(SCALAR_BCS["neumann"])
    g = dev_grid(rhs, F32, L)
    s = ocu.Sol_MultigridPressure3DDevice(F32)
    s.bc = to_ocu_bc(bc)
    s.sweep_cells = 4096          # the TMA two-colour pass on every level with >= 4096 cells
    s.wait_limit = -1000          # test mode: its first wait runs out after 1000 polls
    s.initialize_storage(n, n, n, 1 / n, 1 / n, 1 / n, g)
    with pytest.raises(ocu.OcuError) as e:
        s.solve(1e-6 * rms, 10)
    assert e.value.status == ERR_TIMEOUT
    # the context is intact: the same solver, default limit, from a zero guess
    s.wait_limit = 0
    s.pressure().clear_zero()
    ok, res = s.solve(1e-6 * rms, 10)
    om = O.OracleMG("f", mg_params(bc), n, n, n, 1 / n, 1 / n, 1 / n, rhs.copy(), L)
    ok_o, res_o = om.solve(1e-6 * rms, 10)
    assert ok and ok_o and res == res_o
    assert_same(s.pressure().copy_to_host(), om.grid("u", 0)[0], "after timeout")


@pytest.mark.parametrize("dt", [ocu.F32, ocu.F64])
def test_max_iter_exhausted_returns_not_converged(dt):
    n = 32
    L, rhs, rms = neumann_problem(n, 2, dt)
    bc = bc_from(SCALAR_BCS["neumann"])
    g = dev_grid(rhs, dt, L)
    s = ocu.Sol_MultigridPressure3DDevice(dt)
    s.bc = to_ocu_bc(bc)
    s.initialize_storage(n, n, n, 1 / n, 1 / n, 1 / n, g)
    ok, res = s.solve(1e-30, 2)   # unreachable: two cycles, then the retry from zero, then give up
    assert not ok and np.isfinite(res) and res > 0
    om = O.OracleMG("d" if dt == ocu.F64 else "f", mg_params(bc), n, n, n, 1 / n, 1 / n, 1 / n, rhs.copy(), L)
    ok_o, res_o = om.solve(1e-30, 2)
    assert not ok_o and res == res_o
    assert_same(s.pressure().copy_to_host(), om.grid("u", 0)[0], "after the retry")
    # still usable
    ok2, res2 = s.solve(1e-5 * rms if dt == ocu.F32 else 1e-10 * rms, 20)
    assert ok2


def test_nan_rhs_does_not_converge_and_solver_recovers():
    n = 32
    L, rhs, rms = neumann_problem(n, 3)
    bad = rhs.copy()
    O.interior(bad, L)[5, 6, 7] = np.nan
    g = dev_grid(bad, F32, L)
    s = ocu.Sol_MultigridPressure3DDevice(F32)
    s.bc = to_ocu_bc(bc_from(SCALAR_BCS["neumann"]))
    s.initialize_storage(n, n, n, 1 / n, 1 / n, 1 / n, g)
    ok, res = s.solve(1e-6 * rms, 5)
    assert not ok and np.isnan(res)
    # a clean right-hand side in the same grid, a zero guess: converges
    g.copy_from_host(rhs)
    s.pressure().clear_zero()
    ok2, res2 = s.solve(1e-6 * rms, 20)
    assert ok2 and res2 <= 1e-6 * rms


def test_projection_not_converged_reports_failure():
    nx, ny, nz = 32, 16, 16
    rng, (Lu, Lv, Lw, Lt) = mac_setup(F32, nx, ny, nz, 24)
    hs = [rand_buffer(Lu, F32, rng) for _ in range(3)]
    gs = [dev_grid(hs[0], F32, Lu), dev_grid(hs[1], F32, Lv), dev_grid(hs[2], F32, Lw)]
    pr = ocu.Sol_ProjectDivergence3DDevice(F32)
    pr.bc = to_ocu_bc(bc_from(MAC_BCS["closed_noslip"]))
    pr.initialize_storage(nx, ny, nz, 0.5, 0.5, 1.0, *gs)
    assert not pr.solve(1e-30)      # FP32 cannot reach it: 15 cycles, the retry, failure
    assert pr.solve(1e-3)           # and the next projection succeeds
