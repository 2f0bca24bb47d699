"""GPU parity at the benchmark configurations' own sizes.

* the 256^3 FP64 multigrid of the mixed-precision config, bit-identical to the oracle on a fixed
  schedule (the to-tolerance solves at this size are compared with the reference's own FP64
  solver in tests/test_gpu_ref_parity.py);
* the 128x128x64 Rayleigh-Benard flow config (Ra 1e6, Pr 0.71, upwind, forward Euler), 10 steps,
  bit-identical to the oracle;
* an ensemble with members of the ensemble config's sizes (32^3 to 96^3), each member
  bit-identical to the oracle's single solve;
* the differentiable-flow config (96^3 periodic, 32 steps, checkpoints every 8): the FP64
  adjoint against central differences on 8 seeded directions, the FP32 gradient against the
  FP64 one.
"""
import ctypes as C

import numpy as np
import pytest

import opencurrent_b200 as ocu
from oracle import oracle_ctypes as O
from tests.helpers import F32, F64, SCALAR_BCS, bc_from, mg_params
from tests.test_gpu_parity import assert_same, dev_grid, ns_init, ns_params_rb, to_ocu_bc

pytestmark = pytest.mark.gpu


def test_fp64_256cube_fixed_schedule_bit_identical_to_oracle():
    from opencurrent_b200.workloads import fourier_rhs
    n = 256
    L = O.layout(n, n, n)
    rhs = np.zeros(int(L.allocated), np.float64)
    O.interior(rhs, L)[:] = fourier_rhs(n)
    bc = bc_from(SCALAR_BCS["neumann"])
    O.lib().orc_ns_set_omp_threads(0)
    om = O.OracleMG("d", mg_params(bc), n, n, n, 1 / n, 1 / n, 1 / n, rhs.copy(), L)
    g = dev_grid(rhs, F64, L)
    dm = ocu.Sol_MultigridPressure3DDevice(F64)
    dm.bc = to_ocu_bc(bc)
    dm.initialize_storage(n, n, n, 1 / n, 1 / n, 1 / n, g)
    for s in (om, dm):
        s.run_fmg(1)
        s.run_vcycles(1)
    assert_same(dm.pressure().copy_to_host(), om.grid("u", 0)[0], "256^3 FP64")


def test_rayleigh_benard_config_10_steps_bit_identical_to_oracle():
    nx, ny, nz = 128, 128, 64
    p = ns_params_rb(F32, nx, ny, nz)
    Ls, bufs = ns_init(F32, nx, ny, nz, 11)
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
    for _ in range(10):
        dt_o = O.lib().orc_ns_get_max_stable_timestep(on)
        dt_d = eq.get_max_stable_timestep()
        assert dt_o == dt_d
        assert bool(O.lib().orc_ns_advance_one_step(on, dt_o)) == eq.advance_one_step(dt_d)
    for c, get in zip("uvwt", (eq.get_u, eq.get_v, eq.get_w, eq.get_temperature)):
        ref = O.wrap(O.lib().orc_ns_grid(on, c.encode()), Ls[c], F32)
        assert_same(get().copy_to_host(), ref, f"ns config {c}")
    O.lib().orc_ns_destroy(on)


def test_ensemble_with_the_configs_member_sizes():
    """Members of every size of the ensemble config (U[-1,1] right-hand sides, 1e-6 relative,
    max_iter 30).  A converged member matches the oracle's single solve; a member that stalls
    above its tolerance in FP32 runs its 31 cycles once (the ensemble does not retry from zero as
    the single solve does) and matches the oracle's FMG of 31 cycles."""
    from tests.test_gpu_ensemble import _members
    dims = [(96, 96, 96), (64, 64, 64), (48, 48, 48), (32, 32, 32), (96, 96, 96), (64, 64, 64)]
    bc = bc_from(SCALAR_BCS["neumann"])
    h = [(1.0 / d[0],) * 3 for d in dims]
    ens = ocu.PressureEnsemble(F32, dims, h, bc=to_ocu_bc(bc))
    mem = _members(F32, dims, 2000)
    tols = []
    for m, (L, rhs, rms) in enumerate(mem):
        ens.rhs(m).copy_from_host(rhs)
        tols.append(1e-6 * rms)
    ens.solve(tols, 30)
    assert sorted(c["dims"][0] for c in ens.classes()) == [32, 48, 64, 96]
    stalled = 0
    for m, (L, rhs, rms) in enumerate(mem):
        om = O.OracleMG("f", mg_params(bc), *dims[m], *h[m], rhs.copy(), L)
        ok, res = om.solve(tols[m], 30)
        st = ens.member_stats(m)
        if not ok:
            stalled += 1
            om = O.OracleMG("f", mg_params(bc), *dims[m], *h[m], rhs.copy(), L)
            om.run_fmg(30)
            assert st.vcycles == 31, (m, st.vcycles)
        else:
            assert st.vcycles == om.vcycles and st.last_l2 == res, (m, st.vcycles, om.vcycles, st.last_l2, res)
        assert_same(ens.pressure(m).copy_to_host(), om.grid("u", 0)[0], f"member {m} {dims[m]}")
    print(f"ENSEMBLE config sizes: {len(dims) - stalled} of {len(dims)} members converged")


def test_differentiable_flow_config_gradient():
    import torch
    import bench
    r = bench.run_differentiable(torch, ocu)
    print("ADJOINT", r)
    # central differences against the FP64 adjoint: upwinding's kinks limit the agreement
    assert r["adjoint_fd_max_rel_err_fp64"] <= 1e-3
    assert r["adjoint_fp32_vs_fp64_grad_rel_l2"] <= 1e-5
