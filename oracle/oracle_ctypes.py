"""TEST INFRASTRUCTURE ONLY: ctypes loader for the CPU oracle (oracle/liboracle.so).

Imported by tests/, by the smoke check in __graft_entry__.py and by the CPU-baseline leg of
bench.py.  The product path (opencurrent_b200) never imports this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

F32, F64 = 0, 1


class Layout(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("gx", C.c_int), ("gy", C.c_int), ("gz", C.c_int),
                ("pnx", C.c_int), ("pny", C.c_int), ("pnz", C.c_int),
                ("xstride", C.c_int), ("ystride", C.c_int),
                ("shift", C.c_longlong), ("allocated", C.c_longlong)]


class BC(C.Structure):
    _fields_ = [("type", C.c_int), ("value", C.c_float), ("aux_value", C.c_float)]


class BCSet(C.Structure):
    _fields_ = [(n, BC) for n in ("xpos", "xneg", "ypos", "yneg", "zpos", "zneg")]


class MGParams(C.Structure):
    _fields_ = [("bc", BCSet), ("nu1", C.c_int), ("nu2", C.c_int), ("convergence", C.c_int),
                ("make_symmetric_operator", C.c_int), ("disable_relax_on_host", C.c_int)]


class PCGParams(C.Structure):
    _fields_ = [("bc", BCSet), ("convergence", C.c_int), ("preconditioner", C.c_int),
                ("multigrid_cycles", C.c_int), ("multigrid_use_fmg", C.c_int)]


class NSParams(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double),
                ("max_divergence", C.c_double), ("temp_bc", BCSet), ("flow_bc", BCSet),
                ("vertical_direction", C.c_int), ("gravity", C.c_double),
                ("bouyancy", C.c_double), ("thermal_diffusion", C.c_double),
                ("viscosity", C.c_double), ("advection_scheme", C.c_int),
                ("time_step", C.c_int), ("cfl_factor", C.c_double)]


def build():
    """Compile the oracle with its Makefile (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _setup(_lib)
    return _lib


def _setup(L):
    P = C.c_void_p
    LP = C.POINTER(Layout)
    BP = C.POINTER(BCSet)
    d = C.c_double
    i = C.c_int
    L.orc_layout.argtypes = [i] * 9 + [LP]
    L.orc_num_levels.argtypes = [i, i, i]
    L.orc_optimal_omega.argtypes = [d, d, d]
    L.orc_optimal_omega.restype = d
    for s in ("_f", "_d"):
        for n in ("orc_bc_level1", "orc_bc_nocorners_dev", "orc_bc_nocorners_host"):
            getattr(L, n + s).argtypes = [P, LP, BP, d, d, d]
        getattr(L, "orc_mac_bc_level1" + s).argtypes = [P, P, P, LP, i, i, i, BP, d, d, d]
        getattr(L, "orc_reduce" + s).argtypes = [P, LP, i]
        getattr(L, "orc_reduce" + s).restype = d
        getattr(L, "orc_lincomb1" + s).argtypes = [P, LP, d, P]
        getattr(L, "orc_lincomb2" + s).argtypes = [P, LP, d, P, d, P]
        getattr(L, "orc_divergence" + s).argtypes = [P, P, P, P, LP, i, i, i, d, d, d]
        getattr(L, "orc_gradient" + s).argtypes = [P, P, P, P, LP, i, i, i, d, d, d, d]
        getattr(L, "orc_laplacian" + s).argtypes = [P, P, LP, i, i, i, d, d, d, d]
        getattr(L, "orc_advect_self" + s).argtypes = [P, P, P, P, P, P, LP, i, i, i, d, d, d, i]
        getattr(L, "orc_advect_passive" + s).argtypes = [P, P, P, P, P, LP, i, i, i, d, d, d, i]
        getattr(L, "orc_thermal_force" + s).argtypes = [P, d, P, LP, i, i, i, i]
    MP = C.POINTER(MGParams)
    L.orc_mg_create.argtypes = [i, MP, i, i, i, d, d, d, P, LP]
    L.orc_mg_create.restype = P
    L.orc_mgmixed_create.argtypes = [MP, i, i, i, d, d, d, P, LP]
    L.orc_mgmixed_create.restype = P
    L.orc_mgir_create.argtypes = [MP, i, i, i, d, d, d, P, LP, i]
    L.orc_mgir_create.restype = P
    L.orc_mg_destroy.argtypes = [P]
    L.orc_mg_set_params.argtypes = [P, MP]
    L.orc_mg_solve.argtypes = [P, C.POINTER(d), d, i]
    L.orc_mg_run_vcycles.argtypes = [P, i]
    L.orc_mg_run_fmg.argtypes = [P, i]
    L.orc_mg_num_levels.argtypes = [P]
    L.orc_mg_relax.argtypes = [P, i, i, i, i]
    L.orc_mg_relax_sweep.argtypes = [P, i, i, i]
    L.orc_mg_restrict_residuals.argtypes = [P, i, i, i, C.POINTER(d), C.POINTER(d)]
    L.orc_mg_prolong.argtypes = [P, i, i, i]
    L.orc_mg_grid.argtypes = [P, C.c_char, i, LP]
    L.orc_mg_grid.restype = P
    L.orc_mg_vcycles.argtypes = [P]
    L.orc_mgir_outer_iterations.argtypes = [P]
    L.orc_mg_omega.argtypes = [P]
    L.orc_mg_omega.restype = d
    L.orc_project_create.argtypes = [i, BP, i, i, i, d, d, d, P, P, P, LP]
    L.orc_project_create.restype = P
    L.orc_project_create_kind.argtypes = [i, BP, i, i, i, d, d, d, P, P, P, LP, i]
    L.orc_project_create_kind.restype = P
    L.orc_project_destroy.argtypes = [P]
    L.orc_project_solve.argtypes = [P, d]
    L.orc_project_solve_divergence_only.argtypes = [P]
    L.orc_project_divergence.argtypes = [P]
    L.orc_project_divergence.restype = P
    L.orc_project_pressure_solver.argtypes = [P]
    L.orc_project_pressure_solver.restype = P
    NP = C.POINTER(NSParams)
    L.orc_ns_create.argtypes = [i, NP, P, P, P, P]
    L.orc_ns_create.restype = P
    L.orc_ns_destroy.argtypes = [P]
    L.orc_ns_get_max_stable_timestep.argtypes = [P]
    L.orc_ns_get_max_stable_timestep.restype = d
    L.orc_ns_advance_one_step.argtypes = [P, d]
    L.orc_ns_advance.argtypes = [P, d]
    L.orc_ns_grid.argtypes = [P, C.c_char]
    L.orc_ns_grid.restype = P
    L.orc_ns_layout.argtypes = [P, LP]
    L.orc_ns_set_omp_threads.argtypes = [i]
    for s in ("_f", "_d"):
        getattr(L, "orc_pcg_laplacian" + s).argtypes = [P, P, P, LP, d, d, d]
        getattr(L, "orc_pcg_diag" + s).argtypes = [P, P, P, LP, d, d, d]
        getattr(L, "orc_pcg_dot" + s).argtypes = [P, P, LP]
        getattr(L, "orc_pcg_dot" + s).restype = d
    L.orc_pcg_create.argtypes = [i, C.POINTER(PCGParams), i, i, i, d, d, d, P, P, LP]
    L.orc_pcg_create.restype = P
    L.orc_pcg_destroy.argtypes = [P]
    L.orc_pcg_solve.argtypes = [P, C.POINTER(d), d, i]
    L.orc_pcg_pressure.argtypes = [P]
    L.orc_pcg_pressure.restype = P
    L.orc_pcg_iterations.argtypes = [P]


def np_dtype(dtype):
    return np.float64 if dtype == F64 else np.float32


def ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def layout(nx, ny, nz, gx=1, gy=1, gz=1, padx=0, pady=0, padz=0):
    L = Layout()
    lib().orc_layout(nx, ny, nz, gx, gy, gz, padx, pady, padz, C.byref(L))
    return L


def wrap(addr, L, dtype):
    """numpy view (no copy) of an oracle-owned buffer."""
    n = int(L.allocated)
    ct = C.c_double if dtype == F64 else C.c_float
    return np.ctypeslib.as_array(C.cast(addr, C.POINTER(ct)), shape=(n,))


def bcset(**faces):
    """bcset(xpos=(type, value, aux), ...); faces not given default to BC_INVALID."""
    s = BCSet()
    for name, spec in faces.items():
        if isinstance(spec, int):
            spec = (spec, 0.0, 0.0)
        t, v, a = (list(spec) + [0.0, 0.0])[:3]
        setattr(s, name, BC(int(t), float(v), float(a)))
    return s


def bcset_all(t, value=0.0, aux=0.0):
    return bcset(**{n: (t, value, aux) for n in ("xpos", "xneg", "ypos", "yneg", "zpos", "zneg")})


class OracleMG:
    """Oracle multigrid solver; rhs buffer is borrowed (kept alive here)."""

    def __init__(self, kind, prm, nx, ny, nz, hx, hy, hz, rhs, L, inner_cycles=4):
        self.lib = lib()
        self.rhs = rhs
        self.L = L
        self.kind = kind
        if kind in ("f", "d"):
            self.h = self.lib.orc_mg_create(F64 if kind == "d" else F32, C.byref(prm), nx, ny, nz,
                                            hx, hy, hz, ptr(rhs), C.byref(L))
            self.dtype = F64 if kind == "d" else F32
        elif kind == "mixed":
            self.h = self.lib.orc_mgmixed_create(C.byref(prm), nx, ny, nz, hx, hy, hz, ptr(rhs),
                                                 C.byref(L))
            self.dtype = F64
        elif kind == "ir":
            self.h = self.lib.orc_mgir_create(C.byref(prm), nx, ny, nz, hx, hy, hz, ptr(rhs),
                                              C.byref(L), inner_cycles)
            self.dtype = F64
        else:
            raise ValueError(kind)
        if not self.h:
            raise RuntimeError("oracle MG create failed")

    def set_params(self, prm):
        self.lib.orc_mg_set_params(self.h, C.byref(prm))

    def solve(self, tol, max_iter=4):
        r = C.c_double(0)
        ok = self.lib.orc_mg_solve(self.h, C.byref(r), tol, max_iter)
        return bool(ok), r.value

    def run_vcycles(self, n):
        return self.lib.orc_mg_run_vcycles(self.h, n)

    def run_fmg(self, n):
        return self.lib.orc_mg_run_fmg(self.h, n)

    def grid(self, which="u", level=0, f32_core=False):
        L = Layout()
        w = which.upper() if f32_core else which
        addr = self.lib.orc_mg_grid(self.h, w.encode(), level, C.byref(L))
        dt = F32 if (f32_core or self.dtype == F32) else F64
        return wrap(addr, L, dt), L

    @property
    def num_levels(self):
        return self.lib.orc_mg_num_levels(self.h)

    @property
    def vcycles(self):
        return self.lib.orc_mg_vcycles(self.h)

    @property
    def outer_iterations(self):
        return self.lib.orc_mgir_outer_iterations(self.h)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.lib.orc_mg_destroy(self.h)
                self.h = None
        except Exception:
            pass


def interior(a, L):
    """(nx,ny,nz) view of the interior of a flat padded buffer."""
    base = int(L.shift)
    v = np.lib.stride_tricks.as_strided(
        a[base:], shape=(L.nx, L.ny, L.nz),
        strides=(L.xstride * a.itemsize, L.ystride * a.itemsize, a.itemsize))
    return v


def region(a, L, i0, i1, j0, j1, k0, k1):
    """view of cells i in [i0,i1), j in [j0,j1), k in [k0,k1) (ghost indices allowed)."""
    base = int(L.shift) + i0 * L.xstride + j0 * L.ystride + k0
    return np.lib.stride_tricks.as_strided(
        a[base:], shape=(i1 - i0, j1 - j0, k1 - k0),
        strides=(L.xstride * a.itemsize, L.ystride * a.itemsize, a.itemsize))


PRECOND_NONE, PRECOND_JACOBI, PRECOND_MULTIGRID, PRECOND_BFBT = 0, 1, 2, 3


def pcg_params(bc, preconditioner=PRECOND_BFBT, convergence=0x05, cycles=2, fmg=True):
    p = PCGParams()
    p.bc = bc
    p.convergence = convergence
    p.preconditioner = preconditioner
    p.multigrid_cycles = cycles
    p.multigrid_use_fmg = int(bool(fmg))
    return p


class OraclePCG:
    """Oracle preconditioned CG (Sol_PCGPressure3DDevice); rhs and coefficient are borrowed."""

    def __init__(self, dtype, prm, nx, ny, nz, hx, hy, hz, rhs, coef, L):
        self.lib = lib()
        self.rhs, self.coef, self.L, self.dtype = rhs, coef, L, dtype
        self.h = self.lib.orc_pcg_create(dtype, C.byref(prm), nx, ny, nz, hx, hy, hz, ptr(rhs), ptr(coef),
                                         C.byref(L))
        if not self.h:
            raise RuntimeError("oracle PCG create failed")

    def solve(self, tol, max_iter=1000):
        r = C.c_double(0)
        ok = self.lib.orc_pcg_solve(self.h, C.byref(r), tol, max_iter)
        return bool(ok), r.value

    def pressure(self):
        return wrap(self.lib.orc_pcg_pressure(self.h), self.L, self.dtype).copy()

    @property
    def iterations(self):
        return self.lib.orc_pcg_iterations(self.h)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.lib.orc_pcg_destroy(self.h)
                self.h = None
        except Exception:
            pass
