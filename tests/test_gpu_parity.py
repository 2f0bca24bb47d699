"""GPU parity: every CUDA entry point against the CPU oracle on the same seeded inputs.

The library is built with --fmad=false and the oracle with -ffp-contract=off, both following the
reference's operation order, so the comparison is bit-exact (np.array_equal over the whole padded
buffer, ghosts included) unless a test states a tolerance.
"""
import ctypes as C

import numpy as np
import pytest

import opencurrent_b200 as ocu
from oracle import oracle_ctypes as O
from tests.helpers import (F32, F64, MAC_BCS, SCALAR_BCS, bc_from, config1_rhs, mg_params, npdt,
                           rand_buffer)

pytestmark = pytest.mark.gpu

DTYPES = [F32, F64]


def dev_grid(host, dt, L):
    g = ocu.Grid3DDevice(dt)
    g.init(L.nx, L.ny, L.nz, L.gx, L.gy, L.gz, L.pnx - (L.nx + 2 * L.gx), L.pny - (L.ny + 2 * L.gy),
           L.pnz - (L.nz + 2 * L.gz))
    assert g.layout.allocated == L.allocated and g.layout.shift == L.shift
    g.copy_from_host(host)
    return g


def to_ocu_bc(c_bcset):
    s = ocu.BoundaryConditionSet()
    for f in s.FACES:
        b = getattr(c_bcset, f)
        setattr(s, f, ocu.BoundaryCondition(b.type, b.value, b.aux_value))
    return s


def assert_same(a, b, what=""):
    if not np.array_equal(a, b, equal_nan=True):
        d = np.abs(a.astype(np.float64) - b.astype(np.float64))
        idx = int(np.nanargmax(d))
        raise AssertionError(f"{what}: {np.count_nonzero(d)} elements differ; max |d| = {d[idx]:.3e} at {idx}")


def test_library_loaded():
    lib = ocu.load()
    assert b"sm_100a" in lib.ocu_version()
    n0 = ocu.kernel_launch_count()
    g = ocu.Grid3DDevice(F32)
    g.init(8, 8, 8)
    g.clear(1.5)
    assert ocu.kernel_launch_count() > n0
    h = g.copy_to_host()
    assert np.all(h == np.float32(1.5))


# ---------------------------------------------------------------- ghost cells -----------------
@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("bcname", sorted(SCALAR_BCS))
@pytest.mark.parametrize("variant", [0, 1])
def test_scalar_bc(dt, bcname, variant):
    rng = np.random.default_rng(11)
    L = O.layout(12, 10, 14, padx=1, pady=2, padz=3)
    host = rand_buffer(L, dt, rng)
    bc = bc_from(SCALAR_BCS[bcname])
    g = dev_grid(host, dt, L)
    g.apply_boundary_conditions(to_ocu_bc(bc), 0.1, 0.2, 0.3, variant)
    ref = host.copy()
    lib = O.lib()
    s = "_d" if dt == F64 else "_f"
    fn = getattr(lib, ("orc_bc_level1" if variant == 0 else "orc_bc_nocorners_dev") + s)
    assert fn(O.ptr(ref), C.byref(L), C.byref(bc), 0.1, 0.2, 0.3)
    assert_same(g.copy_to_host(), ref, f"bc {bcname} variant {variant}")


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("bcname", sorted(MAC_BCS))
def test_mac_bc(dt, bcname):
    rng = np.random.default_rng(12)
    nx, ny, nz = 10, 12, 8
    Lu = O.layout(nx + 1, ny, nz, 1, 1, 1, 0, 1, 1)
    Lv = O.layout(nx, ny + 1, nz, 1, 1, 1, 1, 0, 1)
    Lw = O.layout(nx, ny, nz + 1, 1, 1, 1, 1, 1, 0)
    hs = [rand_buffer(Lu, dt, rng) for _ in range(3)]
    gs = [dev_grid(hs[0], dt, Lu), dev_grid(hs[1], dt, Lv), dev_grid(hs[2], dt, Lw)]
    bc = bc_from(MAC_BCS[bcname])
    ocu.apply_3d_mac_boundary_conditions_level1(*gs, to_ocu_bc(bc), 0.1, 0.1, 0.1)
    refs = [h.copy() for h in hs]
    s = "_d" if dt == F64 else "_f"
    assert getattr(O.lib(), "orc_mac_bc_level1" + s)(*[O.ptr(r) for r in refs], C.byref(Lu), nx, ny, nz,
                                                      C.byref(bc), 0.1, 0.1, 0.1)
    for g, r, name in zip(gs, refs, "uvw"):
        assert_same(g.copy_to_host(), r, f"mac {bcname} {name}")


# ---------------------------------------------------------------- reductions / axpy ---------
@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("shape", [(7, 5, 3), (64, 64, 64), (33, 70, 45), (128, 130, 40)])
def test_reductions(dt, shape):
    rng = np.random.default_rng(13)
    L = O.layout(*shape)
    host = rand_buffer(L, dt, rng, -3, 3)
    g = dev_grid(host, dt, L)
    s = "_d" if dt == F64 else "_f"
    for op, meth in enumerate(["reduce_maxabs", "reduce_max", "reduce_min", "reduce_sum",
                               "reduce_sqrsum", "reduce_checknan"]):
        ref = getattr(O.lib(), "orc_reduce" + s)(O.ptr(host), C.byref(L), op)
        got = getattr(g, meth)()
        assert got == ref, (meth, got, ref)


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("nz,pad", [(30, (0, 0, 0)), (31, (0, 0, 0)), (32, (1, 1, 14))])
def test_linear_combination(dt, nz, pad):
    """The interior-only sweep (these layouts are more than 3 % padding): rows that end in a
    partial 16-byte group (nz = 30 in FP32, 31 in both precisions) and whole groups."""
    rng = np.random.default_rng(14)
    L = O.layout(20, 18, nz, 1, 1, 1, *pad)
    a, b = rand_buffer(L, dt, rng), rand_buffer(L, dt, rng)
    ga, gb, gr = dev_grid(a, dt, L), dev_grid(b, dt, L), dev_grid(np.zeros_like(a), dt, L)
    gr.linear_combination(0.7, ga, -1.3, gb)
    ref = np.zeros_like(a)
    s = "_d" if dt == F64 else "_f"
    getattr(O.lib(), "orc_lincomb2" + s)(O.ptr(ref), C.byref(L), 0.7, O.ptr(a), -1.3, O.ptr(b))
    assert_same(gr.copy_to_host(), ref, "lincomb2")


# ---------------------------------------------------------------- stencils ------------------
def mac_setup(dt, nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    Lu = O.layout(nx + 1, ny, nz, 1, 1, 1, 0, 1, 1)
    Lv = O.layout(nx, ny + 1, nz, 1, 1, 1, 1, 0, 1)
    Lw = O.layout(nx, ny, nz + 1, 1, 1, 1, 1, 1, 0)
    Lt = O.layout(nx, ny, nz, 1, 1, 1, 1, 1, 1)
    return rng, (Lu, Lv, Lw, Lt)


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("interp", [1, 2])
def test_advection_and_stencils(dt, interp):
    nx, ny, nz = 24, 20, 36
    rng, (Lu, Lv, Lw, Lt) = mac_setup(dt, nx, ny, nz, 15)
    u, v, w, phi = (rand_buffer(Lu, dt, rng) for _ in range(4))
    du, dv, dw, dphi = (rand_buffer(Lu, dt, rng) for _ in range(4))
    gu, gv, gw = dev_grid(u, dt, Lu), dev_grid(v, dt, Lv), dev_grid(w, dt, Lw)
    gphi = dev_grid(phi, dt, Lt)
    gdu, gdv, gdw, gdphi = dev_grid(du, dt, Lu), dev_grid(dv, dt, Lv), dev_grid(dw, dt, Lw), dev_grid(dphi, dt, Lt)
    h = (0.1, 0.15, 0.05)
    lib = O.lib()
    s = "_d" if dt == F64 else "_f"
    # self-advection
    adv = ocu.Sol_SelfAdvection3DDevice()
    adv.interp_type = interp
    adv.initialize_storage(nx, ny, nz, *h, gu, gv, gw, gdu, gdv, gdw)
    adv.solve()
    rdu, rdv, rdw = du.copy(), dv.copy(), dw.copy()
    getattr(lib, "orc_advect_self" + s)(O.ptr(u), O.ptr(v), O.ptr(w), O.ptr(rdu), O.ptr(rdv), O.ptr(rdw),
                                        C.byref(Lu), nx, ny, nz, *h, interp)
    assert_same(gdu.copy_to_host(), rdu, "dudt")
    assert_same(gdv.copy_to_host(), rdv, "dvdt")
    assert_same(gdw.copy_to_host(), rdw, "dwdt")
    # passive advection
    pas = ocu.Sol_PassiveAdvection3DDevice()
    pas.interp_type = interp
    pas.initialize_storage(nx, ny, nz, *h, gu, gv, gw, gphi, gdphi)
    pas.solve()
    rdphi = dphi.copy()
    getattr(lib, "orc_advect_passive" + s)(O.ptr(u), O.ptr(v), O.ptr(w), O.ptr(phi), O.ptr(rdphi), C.byref(Lt),
                                           nx, ny, nz, *h, interp)
    assert_same(gdphi.copy_to_host(), rdphi, "dphidt")
    # Laplacian accumulate (u grid, nx+1 faces as in the NS viscosity term)
    lap = ocu.Sol_LaplacianCentered3DDevice()
    lap.coefficient = 0.71
    lap.initialize_storage(nx + 1, ny, nz, *h, gu, gdu)
    lap.solve()
    getattr(lib, "orc_laplacian" + s)(O.ptr(u), O.ptr(rdu), C.byref(Lu), nx + 1, ny, nz, *h,
                                      float(npdt(dt)(0.71)))
    assert_same(gdu.copy_to_host(), rdu, "laplacian")
    # divergence + gradient
    gdiv = dev_grid(np.zeros_like(phi), dt, Lt)
    ocu.check(ocu.load().ocu_divergence(gu.handle, gv.handle, gw.handle, gdiv.handle, nx, ny, nz, *h, None))
    rdiv = np.zeros_like(phi)
    getattr(lib, "orc_divergence" + s)(O.ptr(u), O.ptr(v), O.ptr(w), O.ptr(rdiv), C.byref(Lt), nx, ny, nz, *h)
    assert_same(gdiv.copy_to_host(), rdiv, "divergence")
    ocu.check(ocu.load().ocu_gradient_add(gu.handle, gv.handle, gw.handle, gphi.handle, -1.0, *h, None))
    ru, rv, rw = u.copy(), v.copy(), w.copy()
    getattr(lib, "orc_gradient" + s)(O.ptr(ru), O.ptr(rv), O.ptr(rw), O.ptr(phi), C.byref(Lt), nx, ny, nz, *h, -1.0)
    assert_same(gu.copy_to_host(), ru, "grad u")
    assert_same(gv.copy_to_host(), rv, "grad v")
    assert_same(gw.copy_to_host(), rw, "grad w")


# ---------------------------------------------------------------- multigrid -----------------
MG_CASES = [
    # (shape, h, bcname, sym)
    ((32, 32, 32), (1 / 32, 1 / 32, 1 / 32), "neumann", 0),
    ((32, 32, 32), (1 / 32, 1 / 32, 1 / 32), "periodic", 0),
    ((32, 16, 24), (0.05, 0.04, 0.06), "dirichlet", 0),
    ((48, 32, 40), (0.03, 0.03, 0.06), "mixed_xdir", 1),
    ((24, 24, 48), (0.04, 0.05, 0.03), "mixed_zneu", 0),
    ((20, 40, 20), (0.05, 0.05, 0.05), "neumann_inhom", 1),
]


def _mg_pair(dt, shape, h, bcname, sym, seed, disable_host=0, conv=0x05):
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
    g_rhs = dev_grid(rhs, dt, L)
    dm = ocu.Sol_MultigridPressure3DDevice(dt)
    dm.bc = to_ocu_bc(bc)
    dm.make_symmetric_operator = bool(sym)
    dm.disable_relax_on_host = bool(disable_host)
    dm.convergence = conv
    dm.initialize_storage(nx, ny, nz, *h, g_rhs)
    return om, dm, g_rhs, L


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("case", range(len(MG_CASES)))
def test_mg_fixed_schedule(dt, case):
    shape, h, bcname, sym = MG_CASES[case]
    om, dm, _, L = _mg_pair(dt, shape, h, bcname, sym, 100 + case)
    om.run_fmg(2)
    dm.run_fmg(2)
    assert_same(dm.pressure().copy_to_host(), om.grid("u", 0)[0], f"fmg {bcname}")
    om.run_vcycles(2)
    dm.run_vcycles(2)
    assert_same(dm.pressure().copy_to_host(), om.grid("u", 0)[0], f"vcycle {bcname}")
    # coarse levels too
    for lev in range(1, om.num_levels):
        assert_same(dm.read_u(lev).copy_to_host(), om.grid("u", lev)[0], f"u level {lev}")
        assert_same(dm.read_b(lev).copy_to_host(), om.grid("b", lev)[0], f"b level {lev}")


@pytest.mark.parametrize("dt", DTYPES)
def test_mg_device_coarse_relax_option(dt):
    om, dm, _, L = _mg_pair(dt, (32, 32, 32), (1 / 32,) * 3, "neumann", 0, 7, disable_host=1)
    om.run_fmg(1)
    dm.run_fmg(1)
    assert_same(dm.pressure().copy_to_host(), om.grid("u", 0)[0], "disable_relax_on_host")


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("conv", [0x05, 0x0A])
def test_mg_solve_to_tolerance(dt, conv):
    om, dm, _, L = _mg_pair(dt, (64, 64, 64), (1 / 64,) * 3, "neumann", 0, 0, conv=conv)
    tol = 1e-5 if dt == F32 else 1e-9
    ok_o, res_o = om.solve(tol, 15)
    ok_d, res_d = dm.solve(tol, 15)
    assert ok_o and ok_d
    assert res_d == res_o
    assert dm.stats.vcycles == om.vcycles
    assert_same(dm.pressure().copy_to_host(), om.grid("u", 0)[0], "solve")


def test_config1_fp32_64cubed_to_1e6_relative():
    """64^3 Neumann FP32, U[-1,1] seed 0, stop at 1e-6 relative RMS residual."""
    n = 64
    L = O.layout(n, n, n)
    b = config1_rhs(n)
    rhs = np.zeros(int(L.allocated), np.float32)
    O.interior(rhs, L)[:] = b.astype(np.float32)
    rms = float(np.sqrt(np.mean(O.interior(rhs, L).astype(np.float64) ** 2)))
    bc = bc_from(SCALAR_BCS["neumann"])
    om = O.OracleMG("f", mg_params(bc), n, n, n, 1 / n, 1 / n, 1 / n, rhs, L)
    g = dev_grid(rhs, F32, L)
    dm = ocu.Sol_MultigridPressure3DDevice(F32)
    dm.bc = to_ocu_bc(bc)
    dm.initialize_storage(n, n, n, 1 / n, 1 / n, 1 / n, g)
    ok, res = dm.solve(1e-6 * rms, 20)
    ok_o, res_o = om.solve(1e-6 * rms, 20)
    assert ok and ok_o and res / rms < 1e-6
    assert res == res_o and dm.stats.vcycles == om.vcycles
    assert_same(dm.pressure().copy_to_host(), om.grid("u", 0)[0], "config1")


@pytest.mark.parametrize("algorithm", ["warmstart", "ir"])
def test_mixed_solvers(algorithm):
    n = 32
    L = O.layout(n, n, n)
    rng = np.random.default_rng(5)
    b = rng.uniform(-1, 1, (n, n, n))
    b -= b.mean()
    rhs = np.zeros(int(L.allocated), np.float64)
    O.interior(rhs, L)[:] = b
    bc = bc_from(SCALAR_BCS["neumann"])
    prm = mg_params(bc)
    om = O.OracleMG("mixed" if algorithm == "warmstart" else "ir", prm, n, n, n, 1 / n, 1 / n, 1 / n, rhs, L,
                    inner_cycles=3)
    g = dev_grid(rhs, F64, L)
    dm = ocu.Sol_MultigridPressureMixed3DDeviceD(algorithm)
    dm.bc = to_ocu_bc(bc)
    dm.ir_inner_cycles = 3
    dm.ir_inner_exact = True  # the reference-layout inner solves, which the oracle restates
    dm.initialize_storage(n, n, n, 1 / n, 1 / n, 1 / n, g)
    rms = float(np.sqrt(np.mean(b ** 2)))
    ok_o, res_o = om.solve(1e-10 * rms, 20)
    ok_d, res_d = dm.solve(1e-10 * rms, 20)
    assert ok_o and ok_d and res_d == res_o
    assert_same(dm.pressure().copy_to_host(), om.grid("u", 0)[0], algorithm)
    if algorithm == "ir":
        assert dm.stats.outer_iterations == om.outer_iterations


# ---------------------------------------------------------------- projection / NS ------------
@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("bcname", ["closed_noslip", "periodic", "rb"])
def test_projection(dt, bcname):
    nx, ny, nz = 32, 16, 16
    rng, (Lu, Lv, Lw, Lt) = mac_setup(dt, nx, ny, nz, 21)
    hs = [rand_buffer(Lu, dt, rng) for _ in range(3)]
    gs = [dev_grid(hs[0], dt, Lu), dev_grid(hs[1], dt, Lv), dev_grid(hs[2], dt, Lw)]
    bc = bc_from(MAC_BCS[bcname])
    h = (0.5, 0.5, 1.0)
    pr = ocu.Sol_ProjectDivergence3DDevice(dt)
    pr.bc = to_ocu_bc(bc)
    pr.initialize_storage(nx, ny, nz, *h, *gs)
    refs = [x.copy() for x in hs]
    op = O.lib().orc_project_create(dt, C.byref(bc), nx, ny, nz, *h, *[O.ptr(r) for r in refs], C.byref(Lu))
    tol = 1e-4 if dt == F32 else 1e-10
    ok_d = pr.solve(tol)
    ok_o = O.lib().orc_project_solve(op, tol)
    assert bool(ok_d) == bool(ok_o)
    for g, r, name in zip(gs, refs, "uvw"):
        assert_same(g.copy_to_host(), r, f"projection {bcname} {name}")
    O.lib().orc_project_destroy(op)


@pytest.mark.parametrize("algorithm", ["warmstart", "ir"])
@pytest.mark.parametrize("bcname", ["closed_noslip", "periodic", "rb"])
def test_projection_mixed(algorithm, bcname):
    """Sol_ProjectDivergenceMixed3DDeviceD (sol_projectmixed3d.cu:24-94): FP64 fields, mixed
    pressure solver; bit-identical to the oracle's restatement of the same class (the refinement
    variant with the reference-layout inner solves, which the oracle restates)."""
    nx, ny, nz = 32, 16, 16
    rng, (Lu, Lv, Lw, Lt) = mac_setup(F64, nx, ny, nz, 23)
    hs = [rand_buffer(Lu, F64, rng) for _ in range(3)]
    gs = [dev_grid(hs[0], F64, Lu), dev_grid(hs[1], F64, Lv), dev_grid(hs[2], F64, Lw)]
    bc = bc_from(MAC_BCS[bcname])
    h = (0.5, 0.5, 1.0)
    pr = ocu.Sol_ProjectDivergenceMixed3DDeviceD(algorithm)
    pr.bc = to_ocu_bc(bc)
    pr.initialize_storage(nx, ny, nz, *h, *gs)
    if algorithm == "ir":
        ps = pr.pressure_solver
        ps.ir_inner_exact = True
        ps._sync_params()
    refs = [x.copy() for x in hs]
    op = O.lib().orc_project_create_kind(2 if algorithm == "warmstart" else 3, C.byref(bc), nx, ny, nz, *h,
                                         *[O.ptr(r) for r in refs], C.byref(Lu), 4)
    ok_d = pr.solve(1e-10)
    ok_o = O.lib().orc_project_solve(op, 1e-10)
    assert bool(ok_d) == bool(ok_o)
    for g, r, name in zip(gs, refs, "uvw"):
        assert_same(g.copy_to_host(), r, f"mixed projection {algorithm} {bcname} {name}")
    O.lib().orc_project_destroy(op)


def ns_params_rb(dt, nx, ny, nz, scheme=1, ts=1):
    p = O.NSParams()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.hx = p.hy = p.hz = 1.0 / nz
    p.max_divergence = 1e-5 if dt == F32 else 1e-9
    p.temp_bc = bc_from({"xpos": (2, 0), "xneg": (2, 0), "ypos": (2, 0), "yneg": (2, 0),
                         "zpos": (3, 0.0), "zneg": (3, 1.0)})
    p.flow_bc = bc_from(MAC_BCS["rb"])
    p.vertical_direction = 0x11
    p.gravity = -1.0
    p.bouyancy = 1e6 * 0.71
    p.thermal_diffusion = 1.0
    p.viscosity = 0.71
    p.advection_scheme = scheme
    p.time_step = ts
    p.cfl_factor = 0.5
    return p


def ns_init(dt, nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    Ls = {c: O.layout(*dims) for c, dims in
          {"u": (nx + 1, ny, nz, 1, 1, 1, 0, 1, 1), "v": (nx, ny + 1, nz, 1, 1, 1, 1, 0, 1),
           "w": (nx, ny, nz + 1, 1, 1, 1, 1, 1, 0), "t": (nx, ny, nz, 1, 1, 1, 1, 1, 1)}.items()}
    bufs = {c: np.zeros(int(Ls[c].allocated), npdt(dt)) for c in "uvwt"}
    h = 1.0 / nz
    T = O.interior(bufs["t"], Ls["t"])
    z = (np.arange(nz) + 0.5) * h
    T[:] = (1.0 - z)[None, None, :] + rng.uniform(-1e-3, 1e-3, (nx, ny, nz))
    return Ls, bufs


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("scheme,ts", [(1, 1), (2, 2)])
def test_ns_steps(dt, scheme, ts):
    nx, ny, nz = 32, 32, 16
    p = ns_params_rb(dt, nx, ny, nz, scheme, ts)
    Ls, bufs = ns_init(dt, nx, ny, nz, 3)
    on = O.lib().orc_ns_create(dt, C.byref(p), *[O.ptr(bufs[c]) for c in "uvwt"])
    eq = ocu.Eqn_IncompressibleNS3D(dt)
    pp = ocu.Eqn_IncompressibleNS3DParams(dt)
    pp.init_grids(nx, ny, nz)
    for k in ("hx", "hy", "hz", "max_divergence", "vertical_direction", "gravity", "bouyancy",
              "thermal_diffusion", "viscosity", "advection_scheme", "time_step", "cfl_factor"):
        setattr(pp, k, getattr(p, k))
    pp.temp_bc, pp.flow_bc = to_ocu_bc(p.temp_bc), to_ocu_bc(p.flow_bc)
    pp.init_u, pp.init_v, pp.init_w, pp.init_temp = (bufs[c] for c in "uvwt")
    eq.set_parameters(pp)
    for step in range(4):
        dt_o = O.lib().orc_ns_get_max_stable_timestep(on)
        dt_d = eq.get_max_stable_timestep()
        assert dt_o == dt_d
        ok_o = bool(O.lib().orc_ns_advance_one_step(on, dt_o))
        ok_d = eq.advance_one_step(dt_d)
        # FP32 cannot always reach an absolute 1e-5 divergence; both sides must agree on it
        assert ok_o == ok_d
    for c, get in zip("uvwt", (eq.get_u, eq.get_v, eq.get_w, eq.get_temperature)):
        ref = O.wrap(O.lib().orc_ns_grid(on, c.encode()), Ls[c], dt)
        assert_same(get().copy_to_host(), ref, f"ns {c}")
    O.lib().orc_ns_destroy(on)
