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


def divergence_free_velocity(n, seed=5, kmax=8):
    """Periodic velocity on the MAC faces of an n^3 grid (h = 1/n): the curl of a vector
    potential with N(0,1) entries, low-passed to |k| <= kmax, evaluated spectrally at the face
    positions (u at (i, j+1/2, k+1/2) h, v at (i+1/2, j, k+1/2) h, w at (i+1/2, j+1/2, k) h) and
    scaled to max |velocity| = 1.  FP64; returns three (n, n, n) arrays."""
    rng = np.random.default_rng(seed)
    m = np.fft.fftfreq(n, d=1.0 / n)  # integer wavenumbers
    mx, my, mz = np.meshgrid(m, m, m, indexing="ij")
    keep = (mx ** 2 + my ** 2 + mz ** 2) <= kmax ** 2
    A = [np.fft.fftn(rng.standard_normal((n, n, n))) * keep for _ in range(3)]
    kx, ky, kz = (2 * np.pi * mx, 2 * np.pi * my, 2 * np.pi * mz)
    uh = 1j * (ky * A[2] - kz * A[1])
    vh = 1j * (kz * A[0] - kx * A[2])
    wh = 1j * (kx * A[1] - ky * A[0])

    def at(fh, sx, sy, sz):
        phase = np.exp(2j * np.pi * (mx * sx + my * sy + mz * sz) / n)
        return np.real(np.fft.ifftn(fh * phase))

    u, v, w = at(uh, 0, 0.5, 0.5), at(vh, 0.5, 0, 0.5), at(wh, 0.5, 0.5, 0)
    s = max(np.abs(u).max(), np.abs(v).max(), np.abs(w).max())
    return u / s, v / s, w / s


def gaussian_blob(n, center, sigma=0.1):
    """exp(-|x - c|^2 / (2 sigma^2)) at the cell centres of the periodic unit cube (periodic
    distance), FP64 (n, n, n)."""
    x = (np.arange(n) + 0.5) / n
    d = [np.minimum(np.abs(x - c), 1 - np.abs(x - c)) for c in center]
    dx, dy, dz = np.meshgrid(d[0], d[1], d[2], indexing="ij")
    return np.exp(-(dx ** 2 + dy ** 2 + dz ** 2) / (2 * sigma ** 2))
