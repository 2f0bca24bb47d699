"""Rayleigh-Benard critical-number protocol of the reference's RayleighTest (tests/rayleigh.cpp),
driven either by the CPU oracle or by the CUDA library.

init_params (rayleigh.cpp:62-170): vertical z, nx = res, ny = res/2, nz = res on a
sqrt(2) x sqrt(2)/2 x 1 box (extents and spacings computed in float, as the reference does),
closed free-slip walls, Neumann temperature on the sides and Dirichlet top/bottom
(bottom = deltaT), unit viscosity/diffusivity/buoyancy, first-order upwind, forward Euler,
CFL 0.99, projection to 1e-12.  run_resolution_ra (:172-247): advance(0.01) until the log growth
ratios of max|u| and max|w| agree to 0.5% after more than 50 advances.  run_resolution
(:250-272): bracket Ra in 657..660 and interpolate the zero crossing.  The reference's random
perturbation uses rand(); here it is a seeded numpy draw of the same range.
"""
import ctypes as C
import math

import numpy as np

from oracle import oracle_ctypes as O

DIR_ZPOS = 0x11


def _params(res, delta_t, dt):
    nx, ny, nz = res, res // 2, res
    domain_x = np.float32(math.sqrt(2.0))
    domain_y = np.float32(domain_x * np.float32(0.5))
    domain_z = np.float32(1.0)
    hx, hy, hz = (float(np.float32(domain_x / np.float32(nx))), float(np.float32(domain_y / np.float32(ny))),
                  float(np.float32(domain_z / np.float32(nz))))
    p = O.NSParams()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.hx, p.hy, p.hz = hx, hy, hz
    p.max_divergence = 1e-12
    p.viscosity = 1.0
    p.thermal_diffusion = 1.0
    p.gravity = -1.0
    p.bouyancy = 1.0
    p.vertical_direction = DIR_ZPOS
    p.advection_scheme = 1
    p.time_step = 1
    p.cfl_factor = 0.99
    p.flow_bc = O.bcset_all(7, 0.0, 0.0)
    faces = {f: (4, 0.0) for f in ("xpos", "xneg", "ypos", "yneg")}
    faces["zpos"] = (3, 0.0)
    faces["zneg"] = (3, float(delta_t))
    p.temp_bc = O.bcset(**faces)
    return p, float(domain_z)


def _init_fields(p, delta_t, dt, seed):
    nx, ny, nz = p.nx, p.ny, p.nz
    Ls = {"u": O.layout(nx + 1, ny, nz, 1, 1, 1, 0, 1, 1), "v": O.layout(nx, ny + 1, nz, 1, 1, 1, 1, 0, 1),
          "w": O.layout(nx, ny, nz + 1, 1, 1, 1, 1, 1, 0), "t": O.layout(nx, ny, nz, 1, 1, 1, 1, 1, 1)}
    npdt = np.float64 if dt == O.F64 else np.float32
    bufs = {c: np.zeros(int(Ls[c].allocated), npdt) for c in "uvwt"}
    rng = np.random.default_rng(seed)
    k = np.arange(nz)
    y = (1 - ((k + 0.5) * np.float32(p.hz)) / np.float32(1.0)).astype(np.float32).astype(np.float64)
    O.region(bufs["t"], Ls["t"], 0, nx, 0, ny, 0, nz)[:] = (y * delta_t)[None, None, :]
    for c in "uvw":
        # rand_val(-1e-4, 1e-4) = -1e-4 + 2e-4 * U[0,1] (rayleigh.cpp:50-52)
        O.region(bufs[c], Ls[c], 0, nx, 0, ny, 0, nz)[:] = -1e-4 + 2e-4 * rng.random((nx, ny, nz))
    return bufs


class OracleEngine:
    def __init__(self, p, bufs, dt):
        self.lib = O.lib()
        self.h = self.lib.orc_ns_create(dt, C.byref(p), *[O.ptr(bufs[c]) for c in "uvwt"])
        self.p = p
        self.dt = dt
        nx, ny, nz = p.nx, p.ny, p.nz
        self.Ls = {"u": O.layout(nx + 1, ny, nz, 1, 1, 1, 0, 1, 1), "w": O.layout(nx, ny, nz + 1, 1, 1, 1, 1, 1, 0)}

    def advance(self, t):
        assert self.lib.orc_ns_advance(self.h, t)

    def maxabs(self, c):
        buf = self.lib.orc_ns_grid(self.h, c.encode())
        s = "_d" if self.dt == O.F64 else "_f"
        return getattr(self.lib, "orc_reduce" + s)(buf, C.byref(self.Ls[c]), 0)

    def close(self):
        self.lib.orc_ns_destroy(self.h)


class DeviceEngine:
    def __init__(self, p, bufs, dt):
        import opencurrent_b200 as ocu
        self.eq = ocu.Eqn_IncompressibleNS3D(dt)
        pp = ocu.Eqn_IncompressibleNS3DParams(dt)
        pp.init_grids(p.nx, p.ny, p.nz)
        for k in ("hx", "hy", "hz", "max_divergence", "vertical_direction", "gravity", "bouyancy",
                  "thermal_diffusion", "viscosity", "advection_scheme", "time_step", "cfl_factor"):
            setattr(pp, k, getattr(p, k))
        for name in ("temp_bc", "flow_bc"):
            src = getattr(p, name)
            s = ocu.BoundaryConditionSet()
            for f in s.FACES:
                b = getattr(src, f)
                setattr(s, f, ocu.BoundaryCondition(b.type, b.value, b.aux_value))
            setattr(pp, name, s)
        pp.init_u, pp.init_v, pp.init_w, pp.init_temp = (bufs[c] for c in "uvwt")
        self.eq.set_parameters(pp)

    def advance(self, t):
        self.eq.advance(t)

    def maxabs(self, c):
        return (self.eq.get_u() if c == "u" else self.eq.get_w()).reduce_maxabs()

    def close(self):
        pass


def growth_rate(engine_cls, res, delta_t, dt=O.F64, seed=0, max_count=1000):
    p, _ = _params(res, delta_t, dt)
    bufs = _init_fields(p, delta_t, dt, seed)
    eng = engine_cls(p, bufs, dt)
    count, last_u, last_w = 1, 0.0, 0.0
    try:
        while True:
            count += 1
            eng.advance(0.01)
            mu, mw = eng.maxabs("u"), eng.maxabs("w")
            with np.errstate(divide="ignore", invalid="ignore"):
                ur = math.log(mu / last_u) if last_u > 0 else float("inf")
                vr = math.log(mw / last_w) if last_w > 0 else float("inf")
            rel = abs((ur - vr) / ur) if math.isfinite(ur) and math.isfinite(vr) and ur != 0 else float("inf")
            if rel < 0.005 and count > 50:
                return 0.5 * (ur + vr)
            last_u, last_w = mu, mw
            if mu < 1e-10 or mu > 0.1 or count > max_count:
                raise RuntimeError(f"growth-rate run did not settle (max|u| = {mu}, count = {count})")
    finally:
        eng.close()


def critical_rayleigh(engine_cls, res, dt=O.F64):
    lb = ub = None
    for ra in (657.0, 658.0, 659.0, 660.0):
        rate = growth_rate(engine_cls, res, ra, dt)
        if rate < 0:
            lb = (ra, rate)
        else:
            ub = (ra, rate)
            break
    assert lb is not None and ub is not None
    return lb[0] - lb[1] / (ub[1] - lb[1])


def critical_rayleigh_oracle(res):
    return critical_rayleigh(OracleEngine, res)


def critical_rayleigh_device(res):
    return critical_rayleigh(DeviceEngine, res)
