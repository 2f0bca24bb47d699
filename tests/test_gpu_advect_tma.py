"""GPU: the TMA-fed self-advection inside the Boussinesq step (FP32).

On the bench grids the NS step takes the TMA form only where every CTA gets a long run of planes
(256x256x128 and up); OCU_B200_ADVECT_TMA=1 makes it take the form wherever it applies, so these
tests run it on small grids against the oracle, bit for bit: tiles cut short in y and in k,
rows of 32, 64, 96 and 128 cells, upwind and centred schemes, Euler and AB2.  The timeout path
is tested without a fault: OCU_B200_TMA_STALL_TEST makes the first wait of every CTA wait on a
barrier that nothing completes; the step's next CFL readback reports OCU_ERR_TIMEOUT, and the
solver keeps working afterwards.
"""
import ctypes as C

import pytest

import opencurrent_b200 as ocu
from oracle import oracle_ctypes as O
from tests.test_gpu_parity import assert_same, ns_init, ns_params_rb, to_ocu_bc

pytestmark = pytest.mark.gpu

F32 = ocu.F32


def ns_pair(nx, ny, nz, scheme, ts, seed):
    p = ns_params_rb(F32, nx, ny, nz, scheme, ts)
    Ls, bufs = ns_init(F32, nx, ny, nz, seed)
    on = O.lib().orc_ns_create(F32, C.byref(p), *[O.ptr(bufs[c]) for c in "uvwt"])
    eq = ocu.Eqn_IncompressibleNS3D(F32)
    pp = ocu.Eqn_IncompressibleNS3DParams(F32)
    pp.init_grids(nx, ny, nz)
    for k in ("hx", "hy", "hz", "max_divergence", "vertical_direction", "gravity", "bouyancy",
              "thermal_diffusion", "viscosity", "advection_scheme", "time_step", "cfl_factor"):
        setattr(pp, k, getattr(p, k))
    pp.temp_bc, pp.flow_bc = to_ocu_bc(p.temp_bc), to_ocu_bc(p.flow_bc)
    pp.init_u, pp.init_v, pp.init_w, pp.init_temp = (bufs[c] for c in "uvwt")
    eq.set_parameters(pp)
    return on, eq, Ls, bufs


@pytest.mark.parametrize("shape", [(32, 24, 32), (24, 40, 64), (20, 12, 96), (12, 16, 128)])
@pytest.mark.parametrize("scheme,ts", [(1, 1), (2, 2)])
def test_ns_steps_with_tma_advection_bit_identical_to_oracle(monkeypatch, shape, scheme, ts):
    monkeypatch.setenv("OCU_B200_ADVECT_TMA", "1")
    nx, ny, nz = shape
    on, eq, Ls, keep = ns_pair(nx, ny, nz, scheme, ts, 5)
    for step in range(3):
        dt_o = O.lib().orc_ns_get_max_stable_timestep(on)
        dt_d = eq.get_max_stable_timestep()
        assert dt_o == dt_d
        ok_o = bool(O.lib().orc_ns_advance_one_step(on, dt_o))
        ok_d = eq.advance_one_step(dt_d)
        assert ok_o == ok_d
    for c, get in zip("uvwt", (eq.get_u, eq.get_v, eq.get_w, eq.get_temperature)):
        ref = O.wrap(O.lib().orc_ns_grid(on, c.encode()), Ls[c], F32)
        assert_same(get().copy_to_host(), ref, f"ns {c} {shape} scheme={scheme}")
    O.lib().orc_ns_destroy(on)


def test_tma_advection_timeout_is_reported_and_solver_recovers(monkeypatch):
    monkeypatch.setenv("OCU_B200_ADVECT_TMA", "1")
    on, eq, Ls, keep = ns_pair(24, 40, 64, 1, 1, 6)
    O.lib().orc_ns_destroy(on)
    eq.advance_one_step(eq.get_max_stable_timestep())
    monkeypatch.setenv("OCU_B200_TMA_STALL_TEST", "64")
    eq.advance_one_step(eq.get_max_stable_timestep())  # its advection gives up
    monkeypatch.delenv("OCU_B200_TMA_STALL_TEST")
    with pytest.raises(ocu.OcuError, match="TIMEOUT|timeout|gave up"):
        eq.get_max_stable_timestep()
    # the word is cleared on report: the next steps run normally
    for _ in range(2):
        eq.advance_one_step(eq.get_max_stable_timestep())
    assert eq.get_max_stable_timestep() > 0
