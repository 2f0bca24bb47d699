"""GPU parity against OpenCurrent's own device solver (oracle/_ref, built by oracle/build_ref.sh).

The B200 library is bit-identical to the CPU oracle (tests/test_gpu_parity.py).  Here both are
compared with the reference's compiled device code on the same inputs.  The reference kernels
are built with nvcc's defaults, so their a*b+c may be fused to an FMA where the oracle and the
library round twice; results therefore agree to rounding, not bit for bit.  Tolerances
(relative L2 over the interior, mean removed when the operator has constants in its null
space): FP32 1e-5 and FP64 1e-12 for the same schedule; to-tolerance runs are compared the same
way when both sides run the same number of cycles, and every measured figure is printed
(`REFPARITY ...`, shown with pytest -s).
"""
import ctypes as C

import numpy as np
import pytest

import opencurrent_b200 as ocu
from oracle import oracle_ctypes as O
from oracle import ref_ctypes as R
from tests.helpers import F32, F64, MAC_BCS, SCALAR_BCS, bc_from, config1_rhs, mg_params, npdt, rand_buffer
from tests.test_gpu_parity import MG_CASES, dev_grid, mac_setup, ns_init, ns_params_rb, to_ocu_bc

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(),
                                 reason="oracle/_ref/libocu_ref.so not built (needs the reference tree)")]

TOL = {F32: 1e-5, F64: 1e-12}
SINGULAR = {"neumann", "neumann_inhom", "periodic", "mixed_zneu"}


def report(case, **kv):
    print("REFPARITY " + case + " " + " ".join(f"{k}={v:.3e}" if isinstance(v, float) else f"{k}={v}"
                                               for k, v in kv.items()))


def cells(L, nx, ny, nz):
    """Layout L restricted to its first nx*ny*nz cells (same strides and shift)."""
    c = O.Layout()
    C.pointer(c)[0] = L
    c.nx, c.ny, c.nz = nx, ny, nz
    return c


def seeded_rhs(shape, dt, L, seed):
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1, 1, shape)
    b -= b.mean()
    rhs = np.zeros(int(L.allocated), npdt(dt))
    O.interior(rhs, L)[:] = b.astype(npdt(dt))
    return rhs


def gpu_mg(dt, bc, sym, shape, h, rhs, L, conv=0x05):
    dm = ocu.Sol_MultigridPressure3DDevice(dt)
    dm.bc = to_ocu_bc(bc)
    dm.make_symmetric_operator = bool(sym)
    dm.convergence = conv
    g = dev_grid(rhs, dt, L)
    dm.initialize_storage(*shape, *h, g)
    return dm, g


@pytest.mark.parametrize("dt", [F32, F64])
@pytest.mark.parametrize("case", range(len(MG_CASES)))
def test_mg_fixed_schedule_vs_reference(dt, case):
    """run_fmg(2) then run_vcycles(2): B200 library, oracle and reference on one input."""
    shape, h, bcname, sym = MG_CASES[case]
    L = O.layout(*shape)
    rhs = seeded_rhs(shape, dt, L, 300 + case)
    bc = bc_from(SCALAR_BCS[bcname])
    prm = mg_params(bc, sym=sym)
    kind = "d" if dt == F64 else "f"
    ref = R.RefMG(kind, prm, *shape, *h, rhs, L)
    om = O.OracleMG(kind, prm, *shape, *h, rhs.copy(), L)
    dm, _g = gpu_mg(dt, bc, sym, shape, h, rhs, L)
    for s in (ref, om, dm):
        s.run_fmg(2)
        s.run_vcycles(2)
    pr = ref.pressure()
    e_gpu = R.rel_l2(dm.pressure().copy_to_host(), pr, L, bcname in SINGULAR)
    e_orc = R.rel_l2(om.grid("u", 0)[0], pr, L, bcname in SINGULAR)
    report(f"mg_fixed dt={dt} {bcname} {shape}", gpu=e_gpu, oracle=e_orc)
    assert e_gpu <= TOL[dt] and e_orc <= TOL[dt]


@pytest.mark.parametrize("dt", [F32, F64])
def test_mg_solve_to_tolerance_vs_reference(dt):
    """64^3 Neumann to 1e-6 (FP32, the pressure config) / 1e-10 (FP64) relative RMS residual."""
    n = 64
    L = O.layout(n, n, n)
    rhs = np.zeros(int(L.allocated), npdt(dt))
    O.interior(rhs, L)[:] = config1_rhs(n).astype(npdt(dt))
    rms = float(np.sqrt(np.mean(O.interior(rhs, L).astype(np.float64) ** 2)))
    tol = (1e-6 if dt == F32 else 1e-10) * rms
    bc = bc_from(SCALAR_BCS["neumann"])
    ref = R.RefMG("d" if dt == F64 else "f", mg_params(bc), n, n, n, 1 / n, 1 / n, 1 / n, rhs, L)
    dm, _g = gpu_mg(dt, bc, 0, (n, n, n), (1 / n,) * 3, rhs, L)
    ok_r, res_r = ref.solve(tol, 20)
    ok_d, res_d = dm.solve(tol, 20)
    e = R.rel_l2(dm.pressure().copy_to_host(), ref.pressure(), L, True)
    report(f"mg_solve dt={dt} 64^3", rel_l2=e, res_gpu=res_d / rms, res_ref=res_r / rms,
           cycles_gpu=dm.stats.vcycles)
    assert ok_r and ok_d
    assert res_d <= tol and res_r <= tol
    assert e <= TOL[dt]


def cosine_rhs(n, L, dt, seed=3):
    """The 256^3 mixed-precision config's RHS: 16 seeded cosine modes, mean removed."""
    from opencurrent_b200 import workloads
    b = workloads.fourier_rhs(n, seed)
    rhs = np.zeros(int(L.allocated), npdt(dt))
    O.interior(rhs, L)[:] = b.astype(npdt(dt))
    return rhs


def test_fp64_256cube_fixed_schedule_vs_reference():
    """The 256^3 grid of the mixed-precision config: FP64 run_fmg(1) + run_vcycles(2)."""
    n = 256
    L = O.layout(n, n, n)
    rhs = cosine_rhs(n, L, F64)
    bc = bc_from(SCALAR_BCS["neumann"])
    ref = R.RefMG("d", mg_params(bc), n, n, n, 1 / n, 1 / n, 1 / n, rhs, L)
    dm, _g = gpu_mg(F64, bc, 0, (n, n, n), (1 / n,) * 3, rhs, L)
    for s in (ref, dm):
        s.run_fmg(1)
        s.run_vcycles(2)
    e = R.rel_l2(dm.pressure().copy_to_host(), ref.pressure(), L, True)
    report("fp64_256_fixed", rel_l2=e)
    assert e <= TOL[F64]


def test_256cube_solves_vs_reference_fp64_oracle():
    """256^3, 1e-10 relative: the B200 FP64 multigrid, the refinement solver (FP32 cycles in
    FP64) and the reference-algorithm mixed solver, each against the reference's FP64 solver
    driven to 1e-12 (the FP64 multigrid oracle), and the reference-algorithm mixed solver
    against the reference's own mixed solver."""
    n = 256
    L = O.layout(n, n, n)
    rhs = cosine_rhs(n, L, F64)
    rms = float(np.sqrt(np.mean(O.interior(rhs, L) ** 2)))
    bc = bc_from(SCALAR_BCS["neumann"])
    oracle = R.RefMG("d", mg_params(bc), n, n, n, 1 / n, 1 / n, 1 / n, rhs, L)
    ok, res = oracle.solve(1e-12 * rms, 40)
    assert ok, res / rms
    p_oracle = oracle.pressure()
    del oracle
    errs = {}
    g = dev_grid(rhs, F64, L)
    for name, make in (("fp64_mg", lambda: ocu.Sol_MultigridPressure3DDevice(F64)),
                       ("mixed_ir", lambda: ocu.Sol_MultigridPressureMixed3DDeviceD("ir")),
                       ("mixed_warmstart", lambda: ocu.Sol_MultigridPressureMixed3DDeviceD("warmstart"))):
        dm = make()
        dm.bc = to_ocu_bc(bc)
        dm.initialize_storage(n, n, n, 1 / n, 1 / n, 1 / n, g)
        ok_d, res_d = dm.solve(1e-10 * rms, 30)
        assert ok_d and res_d <= 1e-10 * rms, (name, res_d / rms)
        errs[name] = R.rel_l2(dm.pressure().copy_to_host(), p_oracle, L, True)
        if name == "mixed_warmstart":
            p_ws = dm.pressure().copy_to_host()
        del dm
    ref_mixed = R.RefMG("mixed", mg_params(bc), n, n, n, 1 / n, 1 / n, 1 / n, rhs, L)
    ok_r, res_r = ref_mixed.solve(1e-10 * rms, 30)
    assert ok_r
    p_ref_mixed = ref_mixed.pressure()
    errs["ref_mixed"] = R.rel_l2(p_ref_mixed, p_oracle, L, True)
    e_same = R.rel_l2(p_ws, p_ref_mixed, L, True)
    report("256_to_1e-10_vs_fp64_oracle", **errs, warmstart_vs_ref_mixed=e_same)
    # to-tolerance solutions: each within 1e-7 of the FP64 oracle (stated per result above)
    assert max(errs.values()) <= 1e-7
    assert e_same <= TOL[F64]


@pytest.mark.parametrize("dt", [F32, F64])
@pytest.mark.parametrize("interp", [1, 2])
def test_advection_vs_reference(dt, interp):
    nx, ny, nz = 24, 20, 36
    rng, (Lu, Lv, Lw, Lt) = mac_setup(dt, nx, ny, nz, 31)
    u, v, w, phi = (rand_buffer(Lu, dt, rng) for _ in range(4))
    du, dv, dw, dphi = (np.zeros_like(u) for _ in range(4))
    h = (0.1, 0.15, 0.05)
    r_du, r_dv, r_dw = R.advect_self(dt, nx, ny, nz, h, interp, [u, v, w, du, dv, dw],
                                      [Lu, Lv, Lw, Lu, Lv, Lw])
    r_dphi = R.advect_passive(dt, nx, ny, nz, h, interp, [u, v, w, phi, dphi], [Lu, Lv, Lw, Lt, Lt])
    gu, gv, gw = dev_grid(u, dt, Lu), dev_grid(v, dt, Lv), dev_grid(w, dt, Lw)
    gdu, gdv, gdw = dev_grid(du, dt, Lu), dev_grid(dv, dt, Lv), dev_grid(dw, dt, Lw)
    gphi, gdphi = dev_grid(phi, dt, Lt), dev_grid(dphi, dt, Lt)
    adv = ocu.Sol_SelfAdvection3DDevice()
    adv.interp_type = interp
    adv.initialize_storage(nx, ny, nz, *h, gu, gv, gw, gdu, gdv, gdw)
    adv.solve()
    pas = ocu.Sol_PassiveAdvection3DDevice()
    pas.interp_type = interp
    pas.initialize_storage(nx, ny, nz, *h, gu, gv, gw, gphi, gdphi)
    pas.solve()
    # the reference writes all three derivatives on the cells i < nx, j < ny, k < nz
    # (sol_selfadvection3ddev.cu:149), so compare those cells in each face grid's own layout
    errs = {}
    for name, g, r, L in (("dudt", gdu, r_du, Lu), ("dvdt", gdv, r_dv, Lv), ("dwdt", gdw, r_dw, Lw)):
        errs[name] = R.rel_l2(g.copy_to_host(), r, cells(L, nx, ny, nz))
    errs["dphidt"] = R.rel_l2(gdphi.copy_to_host(), r_dphi, Lt)
    report(f"advection dt={dt} interp={interp}", **errs)
    assert max(errs.values()) <= TOL[dt]


@pytest.mark.parametrize("dt", [F32, F64])
@pytest.mark.parametrize("bcname", ["closed_noslip", "periodic", "rb"])
def test_projection_vs_reference(dt, bcname):
    nx, ny, nz = 32, 16, 16
    rng, (Lu, Lv, Lw, Lt) = mac_setup(dt, nx, ny, nz, 41)
    hs = [rand_buffer(Lu, dt, rng) for _ in range(3)]
    bc = bc_from(MAC_BCS[bcname])
    h = (0.5, 0.5, 1.0)
    tol = 1e-4 if dt == F32 else 1e-10
    ref = R.RefProject("d" if dt == F64 else "f", bc, nx, ny, nz, *h, hs, [Lu, Lv, Lw])
    ok_r = ref.solve(tol)
    gs = [dev_grid(hs[0], dt, Lu), dev_grid(hs[1], dt, Lv), dev_grid(hs[2], dt, Lw)]
    pr = ocu.Sol_ProjectDivergence3DDevice(dt)
    pr.bc = to_ocu_bc(bc)
    pr.initialize_storage(nx, ny, nz, *h, *gs)
    ok_d = pr.solve(tol)
    errs = {}
    for name, g, r, L in zip("uvw", gs, ref.fields(), (Lu, Lv, Lw)):
        errs[name] = R.rel_l2(g.copy_to_host(), r, L)
    report(f"projection dt={dt} {bcname}", ok_gpu=ok_d, ok_ref=ok_r, **errs)
    assert bool(ok_d) == ok_r
    assert max(errs.values()) <= TOL[dt]


@pytest.mark.parametrize("algorithm", ["warmstart", "ir"])
@pytest.mark.parametrize("bcname", ["closed_noslip", "periodic", "rb"])
def test_projection_mixed_vs_reference(algorithm, bcname):
    """Sol_ProjectDivergenceMixed3DDeviceD against the reference's own class (its mixed pressure
    solver is the FP32 warm start + FP64 FMG).  The warm-start variant runs the same algorithm
    (FP64 tolerance); the refinement variant reaches the same tolerance by another route, so its
    velocities are compared at the level the 1e-10 pressure tolerance allows."""
    nx, ny, nz = 32, 16, 16
    rng, (Lu, Lv, Lw, Lt) = mac_setup(F64, nx, ny, nz, 43)
    hs = [rand_buffer(Lu, F64, rng) for _ in range(3)]
    bc = bc_from(MAC_BCS[bcname])
    h = (0.5, 0.5, 1.0)
    ref = R.RefProject("mixed", bc, nx, ny, nz, *h, hs, [Lu, Lv, Lw])
    ok_r = ref.solve(1e-10)
    gs = [dev_grid(hs[0], F64, Lu), dev_grid(hs[1], F64, Lv), dev_grid(hs[2], F64, Lw)]
    pr = ocu.Sol_ProjectDivergenceMixed3DDeviceD(algorithm)
    pr.bc = to_ocu_bc(bc)
    pr.initialize_storage(nx, ny, nz, *h, *gs)
    ok_d = pr.solve(1e-10)
    errs = {name: R.rel_l2(g.copy_to_host(), r, L) for name, g, r, L in zip("uvw", gs, ref.fields(), (Lu, Lv, Lw))}
    report(f"projection_mixed {algorithm} {bcname}", ok_gpu=ok_d, ok_ref=ok_r, **errs)
    assert ok_d and ok_r
    assert max(errs.values()) <= (TOL[F64] if algorithm == "warmstart" else 1e-8)


def _gpu_ns(dt, p, nx, ny, nz, bufs):
    eq = ocu.Eqn_IncompressibleNS3D(dt)
    pp = ocu.Eqn_IncompressibleNS3DParams(dt)
    pp.init_grids(nx, ny, nz)
    for k in ("hx", "hy", "hz", "max_divergence", "vertical_direction", "gravity", "bouyancy",
              "thermal_diffusion", "viscosity", "advection_scheme", "time_step", "cfl_factor"):
        setattr(pp, k, getattr(p, k))
    pp.temp_bc, pp.flow_bc = to_ocu_bc(p.temp_bc), to_ocu_bc(p.flow_bc)
    pp.init_u, pp.init_v, pp.init_w, pp.init_temp = (bufs[c] for c in "uvwt")
    eq.set_parameters(pp)
    return eq


def _run_ns(dt, p, nx, ny, nz, bufs, steps):
    """The same steps through the reference and through the B200 library, each with the time
    step it computes itself.  Returns (reference fields, library fields, dt pairs)."""
    ref = R.RefNS(dt, p, *[bufs[c] for c in "uvwt"])
    eq = _gpu_ns(dt, p, nx, ny, nz, bufs)
    dts = []
    for _ in range(steps):
        dt_r = ref.max_stable_timestep()
        dt_d = eq.get_max_stable_timestep()
        dts.append((dt_r, dt_d))
        ref.advance_one_step(dt_r)
        eq.advance_one_step(dt_d)
    got = {c: g().copy_to_host() for c, g in zip("uvwt", (eq.get_u, eq.get_v, eq.get_w, eq.get_temperature))}
    return {c: ref.grid(c) for c in "uvwt"}, got, dts


def _one_ulp_up(bufs, Ls):
    """The same initial state with every interior temperature moved up by one unit in the last
    place: a perturbation at the level of one rounding."""
    out = {c: b.copy() for c, b in bufs.items()}
    T = O.interior(out["t"], Ls["t"])
    T[:] = np.nextafter(T, np.inf)
    return out


@pytest.mark.parametrize("dt", [F32, F64])
def test_ns_steps_vs_reference(dt):
    """Four convection steps at 32x32x16 (periodic x/y, no-slip z, Pr = 0.71) from a temperature
    perturbation of +-0.1 at Ra = 1e4.  The temperature must agree within the precision's
    tolerance; the velocity, which the projection takes out of a buoyancy force that is mostly
    hydrostatic, within that tolerance or within 4x of the reference's own change when its
    initial temperature moves by one ulp, whichever is larger."""
    nx, ny, nz = 32, 32, 16
    p = ns_params_rb(dt, nx, ny, nz)
    p.bouyancy = 1e4 * 0.71
    Ls, bufs = ns_init(dt, nx, ny, nz, 5)
    T = O.interior(bufs["t"], Ls["t"])
    z = (np.arange(nz) + 0.5) / nz
    T[:] = ((1.0 - z)[None, None, :] + np.random.default_rng(6).uniform(-0.1, 0.1, (nx, ny, nz))).astype(T.dtype)
    ref, got, dts = _run_ns(dt, p, nx, ny, nz, bufs, 4)
    ref_ulp, _got2, _ = _run_ns(dt, p, nx, ny, nz, _one_ulp_up(bufs, Ls), 4)
    for dt_r, dt_d in dts:
        assert abs(dt_r - dt_d) <= 1e-6 * dt_r
    errs = {c: R.rel_l2(got[c], ref[c], Ls[c]) for c in "uvwt"}
    noise = {c: R.rel_l2(ref_ulp[c], ref[c], Ls[c]) for c in "uvwt"}
    report(f"ns dt={dt}", **errs, **{f"ref_ulp_{c}": noise[c] for c in "uvwt"})
    assert errs["t"] <= TOL[dt]
    for c in "uvw":
        assert errs[c] <= max(TOL[dt], 4 * noise[c]), (c, errs[c], noise[c])


@pytest.mark.parametrize("dt", [F32, F64])
def test_ns_rayleigh_benard_config_vs_reference(dt):
    """The flow config's own case at its size: 128x128x64, Ra = 1e6, Pr = 0.71, T = 1 - z plus a
    +-1e-3 perturbation, 10 steps.  Starting from rest, the velocity is what the projection leaves
    of a buoyancy force that is hydrostatic to one part in 1e3, so any rounding is amplified by
    that cancellation, in the reference as much as here.  The test measures the amplification
    on the reference itself (its fields after the same steps from a temperature moved by one ulp)
    and requires the library to sit within 4x of that, with the temperature within the
    precision's tolerance."""
    nx, ny, nz = 128, 128, 64
    p = ns_params_rb(dt, nx, ny, nz)
    Ls, bufs = ns_init(dt, nx, ny, nz, 7)
    ref, got, dts = _run_ns(dt, p, nx, ny, nz, bufs, 10)
    ref_ulp, _got2, _ = _run_ns(dt, p, nx, ny, nz, _one_ulp_up(bufs, Ls), 10)
    errs = {c: R.rel_l2(got[c], ref[c], Ls[c]) for c in "uvwt"}
    noise = {c: R.rel_l2(ref_ulp[c], ref[c], Ls[c]) for c in "uvwt"}
    report(f"ns_config dt={dt} 128x128x64 10 steps", **{f"{c}": errs[c] for c in "uvwt"},
           **{f"ref_ulp_{c}": noise[c] for c in "uvwt"})
    assert errs["t"] <= 10 * TOL[dt]
    for c in "uvw":
        assert errs[c] <= 4 * max(noise[c], TOL[dt]), (c, errs[c], noise[c])
