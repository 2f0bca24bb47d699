"""Seeded synthetic inputs of the benchmark configurations (no datasets are involved).

  config1_rhs      64^3 FP32 pressure solve: RHS ~ U[-1,1] i.i.d. (seed 0), mean removed.
  fourier_rhs      256^3 mixed-precision solve: 16 cosine modes, wavenumbers U{1..16},
                   amplitudes N(0,1), mean removed.
  rayleigh_benard  128x128x64 Boussinesq flow: periodic x/y, no-slip z walls, T linear from 1
                   (bottom) to 0 (top) plus U[-1e-3,1e-3], Ra = 1e6, Pr = 0.71, upwind, forward
                   Euler, CFL 0.5, projection to 1e-5 (non-dimensional form of
                   tests/rayleightiming.cpp:86-89 in the reference: nu = Pr, kappa = 1,
                   buoyancy = Ra * Pr, gravity = -1).
  ensemble_sizes   batched ensemble: sizes drawn from {32,48,64,96}^3 (seed 1).
"""
import numpy as np


def interior(buf, L):
    """(nx, ny, nz) strided view of the interior of a flat padded buffer."""
    return region(buf, L, 0, L.nx, 0, L.ny, 0, L.nz)


def region(buf, L, i0, i1, j0, j1, k0, k1):
    base = int(L.shift) + i0 * L.xstride + j0 * L.ystride + k0
    s = buf.itemsize
    return np.lib.stride_tricks.as_strided(buf[base:], shape=(i1 - i0, j1 - j0, k1 - k0),
                                           strides=(L.xstride * s, L.ystride * s, s))


def padded(b, L, dtype):
    buf = np.zeros(int(L.allocated), dtype)
    interior(buf, L)[:] = b.astype(dtype)
    return buf


def config1_rhs(n=64, seed=0):
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1.0, 1.0, (n, n, n))
    b -= b.mean()
    return b


def fourier_rhs(n=256, seed=3, modes=16):
    rng = np.random.default_rng(seed)
    k = rng.integers(1, 17, size=(modes, 3))
    a = rng.standard_normal(modes)
    x = (np.arange(n) + 0.5) / n
    b = np.zeros((n, n, n))
    for m in range(modes):
        b += a[m] * (np.cos(k[m, 0] * np.pi * x)[:, None, None] * np.cos(k[m, 1] * np.pi * x)[None, :, None]
                     * np.cos(k[m, 2] * np.pi * x)[None, None, :])
    b -= b.mean()
    return b


def rayleigh_benard(ocu, nx=128, ny=128, nz=64, dtype=None, seed=0, ra=1e6, pr=0.71):
    """Eqn_IncompressibleNS3DParams for the Rayleigh-Benard workload."""
    dtype = ocu.F32 if dtype is None else dtype
    p = ocu.Eqn_IncompressibleNS3DParams(dtype)
    p.init_grids(nx, ny, nz)
    h = 1.0 / nz
    p.hx = p.hy = p.hz = h
    p.max_divergence = 1e-5
    per = ocu.BoundaryCondition(ocu.BC_PERIODIC)
    wall = ocu.BoundaryCondition(ocu.BC_FORCED_INFLOW_VARIABLE_SLIP, 0.0, 1.0)
    p.flow_bc = ocu.BoundaryConditionSet(per, zpos=wall, zneg=wall)
    p.temp_bc = ocu.BoundaryConditionSet(per, zpos=ocu.BoundaryCondition(ocu.BC_DIRICHELET, 0.0),
                                         zneg=ocu.BoundaryCondition(ocu.BC_DIRICHELET, 1.0))
    p.vertical_direction = ocu.DIR_ZPOS
    p.gravity = -1.0
    p.bouyancy = ra * pr
    p.thermal_diffusion = 1.0
    p.viscosity = pr
    p.advection_scheme = ocu.IT_FIRST_ORDER_UPWIND
    p.time_step = ocu.TS_FORWARD_EULER
    p.cfl_factor = 0.5
    rng = np.random.default_rng(seed)
    z = (np.arange(nz) + 0.5) * h
    t = (1.0 - z)[None, None, :] + rng.uniform(-1e-3, 1e-3, (nx, ny, nz))
    interior(p.init_temp, p.layouts["t"])[:] = t.astype(p.init_temp.dtype)
    return p


def ensemble_sizes(count=512, seed=1, choices=(32, 48, 64, 96)):
    rng = np.random.default_rng(seed)
    return [int(x) for x in rng.choice(np.array(choices), size=count)]
