"""GPU: the NS step's work before the projection replayed as CUDA graphs.

A state's first step (Euler, or Adams-Bashforth with either order of the history buffers) runs
as plain launches; from its second occurrence the tail is one graph replay whose time-step
coefficients a one-thread kernel writes to device memory first.  Over 10 steps every state is
replayed several times, and the fields stay bit-identical to the oracle and to the same run on
plain launches (OCU_B200_NS_GRAPH=0).  The legacy NULL stream (no stream set) replays on a
private blocking stream; a caller's stream replays on that stream.
"""
import ctypes as C

import pytest
import torch

import opencurrent_b200 as ocu
from oracle import oracle_ctypes as O
from tests.test_gpu_parity import assert_same, ns_init, ns_params_rb, to_ocu_bc

pytestmark = pytest.mark.gpu

F32, F64 = ocu.F32, ocu.F64
STEPS = 10


def make_eq(dt, p, bufs):
    eq = ocu.Eqn_IncompressibleNS3D(dt)
    pp = ocu.Eqn_IncompressibleNS3DParams(dt)
    pp.init_grids(p.nx, p.ny, p.nz)
    for k in ("hx", "hy", "hz", "max_divergence", "vertical_direction", "gravity", "bouyancy",
              "thermal_diffusion", "viscosity", "advection_scheme", "time_step", "cfl_factor"):
        setattr(pp, k, getattr(p, k))
    pp.temp_bc, pp.flow_bc = to_ocu_bc(p.temp_bc), to_ocu_bc(p.flow_bc)
    pp.init_u, pp.init_v, pp.init_w, pp.init_temp = (bufs[c] for c in "uvwt")
    eq.set_parameters(pp)
    return eq


def fields(eq):
    return [g().copy_to_host() for g in (eq.get_u, eq.get_v, eq.get_w, eq.get_temperature)]


@pytest.mark.parametrize("dt", [F32, F64])
@pytest.mark.parametrize("scheme,ts", [(1, 1), (2, 2), (1, 2)])
def test_graph_replayed_steps_bit_identical_to_oracle(dt, scheme, ts):
    nx, ny, nz = 32, 32, 16
    p = ns_params_rb(dt, nx, ny, nz, scheme, ts)
    Ls, bufs = ns_init(dt, nx, ny, nz, 11)
    on = O.lib().orc_ns_create(dt, C.byref(p), *[O.ptr(bufs[c]) for c in "uvwt"])
    eq = make_eq(dt, p, bufs)
    for _ in range(STEPS):
        dt_o = O.lib().orc_ns_get_max_stable_timestep(on)
        dt_d = eq.get_max_stable_timestep()
        assert dt_o == dt_d
        assert bool(O.lib().orc_ns_advance_one_step(on, dt_o)) == eq.advance_one_step(dt_d)
    for c, got in zip("uvwt", fields(eq)):
        assert_same(got, O.wrap(O.lib().orc_ns_grid(on, c.encode()), Ls[c], dt), f"ns {c} ts={ts}")
    O.lib().orc_ns_destroy(on)


@pytest.mark.parametrize("dt", [F32, F64])
def test_graph_and_plain_launches_same_bits_and_launch_counts(monkeypatch, dt):
    nx, ny, nz = 32, 24, 16
    p = ns_params_rb(dt, nx, ny, nz, 1, 2)
    runs = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("OCU_B200_NS_GRAPH", mode)
        Ls, bufs = ns_init(dt, nx, ny, nz, 12)
        eq = make_eq(dt, p, bufs)
        counts = []
        for _ in range(STEPS):
            h = eq.get_max_stable_timestep()
            n0 = ocu.kernel_launch_count()
            eq.advance_one_step(h)
            counts.append(ocu.kernel_launch_count() - n0)
        runs[mode] = (fields(eq), counts)
    for a, b, c in zip(runs["0"][0], runs["1"][0], "uvwt"):
        assert_same(b, a, f"graph vs plain {c}")
    # a replayed step counts its graph's kernels plus the coefficient kernel
    plain, graph = runs["0"][1], runs["1"][1]
    assert graph[:3] == plain[:3]
    assert all(g in (q, q + 1) for g, q in zip(graph[3:], plain[3:]))
    assert any(g == q + 1 for g, q in zip(graph[3:], plain[3:]))


def test_graph_replay_on_a_caller_stream():
    dt = F32
    nx, ny, nz = 32, 32, 16
    p = ns_params_rb(dt, nx, ny, nz, 1, 2)
    Ls, bufs = ns_init(dt, nx, ny, nz, 13)
    on = O.lib().orc_ns_create(dt, C.byref(p), *[O.ptr(bufs[c]) for c in "uvwt"])
    eq = make_eq(dt, p, bufs)
    s = torch.cuda.Stream()
    ocu._capi.check(ocu.load().ocu_ns_set_stream(eq._h, C.c_void_p(s.cuda_stream)))
    for _ in range(6):
        h = O.lib().orc_ns_get_max_stable_timestep(on)
        assert eq.get_max_stable_timestep() == h
        O.lib().orc_ns_advance_one_step(on, h)
        eq.advance_one_step(h)
    s.synchronize()
    for c, got in zip("uvwt", fields(eq)):
        assert_same(got, O.wrap(O.lib().orc_ns_grid(on, c.encode()), Ls[c], dt), f"ns {c} on a stream")
    O.lib().orc_ns_destroy(on)
