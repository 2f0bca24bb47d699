"""TEST INFRASTRUCTURE ONLY: ctypes access to OpenCurrent's own device solver.

oracle/build_ref.sh compiles the reference sources (with the CUDA 12 texture shim and the
warp-reduction fix of oracle/ref/) into oracle/_ref/libocu_ref.so; this module loads it and
wraps the C entry layer of oracle/ref/ref_driver.cu.  Only tests/ use it.  The library is
built where the reference tree is present and travels to GPU machines as a file; when it is
missing, available() is False and the tests that need it say so.
"""
import ctypes as C
import os

import numpy as np

from oracle import oracle_ctypes as O

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libocu_ref.so")

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(LIB_PATH)
        _setup(_lib)
    return _lib


def _setup(L):
    P, d, i = C.c_void_p, C.c_double, C.c_int
    LP = C.POINTER(O.Layout)
    L.ref_grid_create.argtypes = [i] * 10
    L.ref_grid_create.restype = P
    L.ref_grid_destroy.argtypes = [P]
    L.ref_grid_layout.argtypes = [P, LP]
    L.ref_grid_upload.argtypes = [P, P]
    L.ref_grid_download.argtypes = [P, P]
    L.ref_mg_create.argtypes = [i, C.POINTER(O.MGParams), i, i, i, d, d, d, P]
    L.ref_mg_create.restype = P
    L.ref_mg_destroy.argtypes = [P]
    L.ref_mg_solve.argtypes = [P, C.POINTER(d), d, i]
    L.ref_mg_run_vcycles.argtypes = [P, i]
    L.ref_mg_run_fmg.argtypes = [P, i]
    L.ref_mg_pressure.argtypes = [P]
    L.ref_mg_pressure.restype = P
    L.ref_pcg_create.argtypes = [C.POINTER(O.PCGParams), i, i, i, d, d, d, P, P]
    L.ref_pcg_create.restype = P
    L.ref_pcg_solve.argtypes = [P, C.POINTER(d), d, i]
    L.ref_pcg_pressure.argtypes = [P]
    L.ref_pcg_pressure.restype = P
    L.ref_pcg_destroy.argtypes = [P]
    L.ref_project_create.argtypes = [i, C.POINTER(O.BCSet), i, i, i, d, d, d, P, P, P]
    L.ref_project_create.restype = P
    L.ref_project_destroy.argtypes = [P]
    L.ref_project_solve.argtypes = [P, d]
    L.ref_project_solve_divergence_only.argtypes = [P]
    L.ref_project_divergence.argtypes = [P]
    L.ref_project_divergence.restype = P
    L.ref_project_pressure.argtypes = [P]
    L.ref_project_pressure.restype = P
    L.ref_advect_self.argtypes = [i, i, i, i, d, d, d, i] + [P] * 6
    L.ref_advect_passive.argtypes = [i, i, i, i, d, d, d, i] + [P] * 5
    L.ref_ns_create.argtypes = [i, C.POINTER(O.NSParams), P, P, P, P]
    L.ref_ns_create.restype = P
    L.ref_ns_destroy.argtypes = [P]
    L.ref_ns_get_max_stable_timestep.argtypes = [P]
    L.ref_ns_get_max_stable_timestep.restype = d
    L.ref_ns_advance_one_step.argtypes = [P, d]
    L.ref_ns_download.argtypes = [P, C.c_char, P, LP]


class RefGrid:
    """A reference Grid3DDevice<T> with the layout of an oracle Layout (checked)."""

    def __init__(self, dtype, L, host=None, handle=None):
        self.dtype = dtype
        self.L = L
        if handle is not None:
            self.h, self.owned = handle, False
        else:
            pad = (L.pnx - L.nx - 2 * L.gx, L.pny - L.ny - 2 * L.gy, L.pnz - L.nz - 2 * L.gz)
            self.h = lib().ref_grid_create(dtype, L.nx, L.ny, L.nz, L.gx, L.gy, L.gz, *pad)
            self.owned = True
            if not self.h:
                raise RuntimeError("reference Grid3DDevice::init failed")
            got = O.Layout()
            lib().ref_grid_layout(self.h, C.byref(got))
            for f in ("pnx", "pny", "pnz", "xstride", "ystride", "shift", "allocated"):
                if getattr(got, f) != getattr(L, f):
                    raise RuntimeError(f"reference layout differs in {f}")
        if host is not None:
            self.upload(host)

    def upload(self, host):
        assert host.size == self.L.allocated
        if not lib().ref_grid_upload(self.h, O.ptr(np.ascontiguousarray(host))):
            raise RuntimeError("upload failed")

    def download(self):
        out = np.empty(int(self.L.allocated), O.np_dtype(self.dtype))
        if not lib().ref_grid_download(self.h, O.ptr(out)):
            raise RuntimeError("download failed")
        return out

    def __del__(self):
        try:
            if self.owned and self.h:
                lib().ref_grid_destroy(self.h)
                self.h = None
        except Exception:
            pass


class RefMG:
    """kind: 'f' / 'd' (Sol_MultigridPressure3DDevice<T>) or 'mixed'
    (Sol_MultigridPressureMixed3DDeviceD).  The rhs grid is borrowed and kept alive here."""

    KINDS = {"f": 0, "d": 1, "mixed": 2}

    def __init__(self, kind, prm, nx, ny, nz, hx, hy, hz, rhs_host, L):
        self.dtype = O.F32 if kind == "f" else O.F64
        self.rhs = RefGrid(self.dtype, L, rhs_host)
        self.L = L
        self.h = lib().ref_mg_create(self.KINDS[kind], C.byref(prm), nx, ny, nz, hx, hy, hz, self.rhs.h)
        if not self.h:
            raise RuntimeError("reference initialize_storage failed")

    def solve(self, tol, max_iter=4):
        r = C.c_double(0)
        ok = lib().ref_mg_solve(self.h, C.byref(r), tol, max_iter)
        return bool(ok), r.value

    def run_vcycles(self, n):
        return lib().ref_mg_run_vcycles(self.h, n)

    def run_fmg(self, n):
        return lib().ref_mg_run_fmg(self.h, n)

    def pressure(self):
        return RefGrid(self.dtype, self.L, handle=lib().ref_mg_pressure(self.h)).download()

    def __del__(self):
        try:
            if self.h:
                lib().ref_mg_destroy(self.h)
                self.h = None
        except Exception:
            pass


class RefPCG:
    """Sol_PCGPressure3DDevice<T> over reference grids made from host rhs / coefficient buffers."""

    def __init__(self, dtype, prm, nx, ny, nz, hx, hy, hz, rhs_host, coef_host, L):
        self.dtype = dtype
        self.rhs = RefGrid(dtype, L, rhs_host)
        self.coef = RefGrid(dtype, L, coef_host)
        self.L = L
        self.h = lib().ref_pcg_create(C.byref(prm), nx, ny, nz, hx, hy, hz, self.rhs.h, self.coef.h)
        if not self.h:
            raise RuntimeError("reference initialize_storage failed")

    def solve(self, tol, max_iter=1000):
        r = C.c_double(0)
        ok = lib().ref_pcg_solve(self.h, C.byref(r), tol, max_iter)
        return bool(ok), r.value

    def pressure(self):
        return RefGrid(self.dtype, self.L, handle=lib().ref_pcg_pressure(self.h)).download()

    def __del__(self):
        try:
            if self.h:
                lib().ref_pcg_destroy(self.h)
                self.h = None
        except Exception:
            pass


class RefProject:
    """kind 'f' / 'd' (Sol_ProjectDivergence3DDevice<T>) or 'mixed'
    (Sol_ProjectDivergenceMixed3DDeviceD) over reference MAC grids made from host buffers."""

    KINDS = {"f": 0, "d": 1, "mixed": 2}

    def __init__(self, kind, bc, nx, ny, nz, hx, hy, hz, hosts, layouts):
        self.dtype = O.F32 if kind == "f" else O.F64
        self.grids = [RefGrid(self.dtype, L, hst) for hst, L in zip(hosts, layouts)]
        self.h = lib().ref_project_create(self.KINDS[kind], C.byref(bc), nx, ny, nz, hx, hy, hz,
                                          *[g.h for g in self.grids])
        if not self.h:
            raise RuntimeError("reference projection initialize_storage failed")

    def solve(self, tol):
        return bool(lib().ref_project_solve(self.h, tol))

    def fields(self):
        return [g.download() for g in self.grids]

    def __del__(self):
        try:
            if self.h:
                lib().ref_project_destroy(self.h)
                self.h = None
        except Exception:
            pass


def advect_self(dtype, nx, ny, nz, h, interp, hosts, layouts):
    """hosts/layouts: u, v, w, dudt, dvdt, dwdt.  Returns the three derivative buffers."""
    gs = [RefGrid(dtype, L, x) for x, L in zip(hosts, layouts)]
    if not lib().ref_advect_self(dtype, nx, ny, nz, *h, interp, *[g.h for g in gs]):
        raise RuntimeError("reference self-advection failed")
    return [g.download() for g in gs[3:]]


def advect_passive(dtype, nx, ny, nz, h, interp, hosts, layouts):
    """hosts/layouts: u, v, w, phi, dphidt.  Returns dphidt."""
    gs = [RefGrid(dtype, L, x) for x, L in zip(hosts, layouts)]
    if not lib().ref_advect_passive(dtype, nx, ny, nz, *h, interp, *[g.h for g in gs]):
        raise RuntimeError("reference passive advection failed")
    return gs[4].download()


class RefNS:
    def __init__(self, dtype, prm, u, v, w, t):
        self.dtype = dtype
        self.h = lib().ref_ns_create(dtype, C.byref(prm), O.ptr(u), O.ptr(v), O.ptr(w), O.ptr(t))
        if not self.h:
            raise RuntimeError("reference Eqn_IncompressibleNS3D::set_parameters failed")
        self.sizes = {"u": u.size, "v": v.size, "w": w.size, "t": t.size}

    def max_stable_timestep(self):
        return lib().ref_ns_get_max_stable_timestep(self.h)

    def advance_one_step(self, dt):
        return bool(lib().ref_ns_advance_one_step(self.h, dt))

    def grid(self, which):
        out = np.empty(self.sizes[which], O.np_dtype(self.dtype))
        if not lib().ref_ns_download(self.h, which.encode(), O.ptr(out), None):
            raise RuntimeError("download failed")
        return out

    def __del__(self):
        try:
            if self.h:
                lib().ref_ns_destroy(self.h)
                self.h = None
        except Exception:
            pass


def rel_l2(a, b, L, remove_mean=False):
    """Relative L2 difference ||a - b|| / ||b|| over the interior cells of layout L."""
    x = O.interior(a, L).astype(np.float64)
    y = O.interior(b, L).astype(np.float64)
    if remove_mean:
        x = x - x.mean()
        y = y - y.mean()
    den = np.sqrt(np.sum(y * y))
    return float(np.sqrt(np.sum((x - y) ** 2)) / den) if den > 0 else float(np.sqrt(np.sum(x * x)))
