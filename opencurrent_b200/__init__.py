"""opencurrent_b200 -- B200-native (sm_100a) OpenCurrent projection-step hot path.

Python mirror of the reference's C++ API over the C ABI of libocu_b200.so
(include/ocu_b200.h).  Class and member names follow OpenCurrent (namespace ocu):
Grid3DDevice, BoundaryCondition(Set), Sol_MultigridPressure3DDevice,
Sol_MultigridPressureMixed3DDeviceD, Sol_ProjectDivergence3DDevice, Sol_SelfAdvection3DDevice,
Sol_PassiveAdvection3DDevice, Sol_LaplacianCentered3DDevice, Eqn_IncompressibleNS3D.
Where the reference returns bool and fills a double& (solve), the Python method returns
(ok, residual).  Every compute call runs on the device; nothing falls back to the CPU.
"""
import ctypes as C
import os

import numpy as np

from . import _capi
from ._capi import *  # noqa: F401,F403  (enums, structs)
from ._capi import OcuError, check, load

__all__ = [
    "NetCDFGrid3DWriter", "NetCDFGrid3DReader",
    "Sol_PCGPressure3DDevice",
    "PersistentEnsemble",
    "BoundaryCondition", "BoundaryConditionSet", "Grid3DDevice", "Sol_MultigridPressure3DDevice",
    "Sol_MultigridPressure3DDeviceF", "Sol_MultigridPressure3DDeviceD",
    "Sol_MultigridPressure3DDeviceCo", "mgco_plan",
    "Sol_MultigridPressureMixed3DDeviceD", "Sol_ProjectDivergence3DDevice",
    "Sol_SelfAdvection3DDevice", "Sol_PassiveAdvection3DDevice", "Sol_LaplacianCentered3DDevice",
    "Eqn_IncompressibleNS3DParams", "Eqn_IncompressibleNS3D", "layout", "OcuError",
    "kernel_launch_count",
]


def kernel_launch_count():
    return int(load().ocu_kernel_launch_count())


def _np_dtype(dt):
    return np.float64 if dt == F64 else np.float32


def layout(nx, ny, nz, gx=1, gy=1, gz=1, padx=0, pady=0, padz=0):
    """Grid3DDevice<T>::init layout rule (ocustorage/grid3ddev.cu:358-400)."""
    L = Layout()
    check(load().ocu_layout_compute(nx, ny, nz, gx, gy, gz, padx, pady, padz, C.byref(L)))
    return L


class BoundaryCondition:
    """ocuutil/boundary_condition.h:38-58 (value/aux_value are float32 in the reference)."""

    def __init__(self, type=BC_INVALID, value=0.0, aux_value=0.0):
        self.type, self.value, self.aux_value = int(type), float(value), float(aux_value)

    def to_c(self):
        return BC(self.type, self.value, self.aux_value)


class BoundaryConditionSet:
    FACES = ("xpos", "xneg", "ypos", "yneg", "zpos", "zneg")

    def __init__(self, all_faces=None, **faces):
        for f in self.FACES:
            src = faces.get(f, all_faces)
            if src is None:
                src = BoundaryCondition()
            setattr(self, f, BoundaryCondition(src.type, src.value, src.aux_value))

    def to_c(self):
        s = BCSet()
        for f in self.FACES:
            setattr(s, f, getattr(self, f).to_c())
        return s

    def make_homogeneous(self):
        for f in self.FACES:
            getattr(self, f).value = 0.0
            getattr(self, f).aux_value = 0.0


class Grid3DDevice:
    """Device grid in the Grid3DDevice<T> layout; owns its buffer unless it wraps a solver's."""

    def __init__(self, dtype=F32, _handle=None, _owner=None):
        self.dtype = dtype
        self._h = _handle
        self._owner = _owner  # keeps a parent solver alive for borrowed handles
        self._owned = _handle is None

    @classmethod
    def _borrow(cls, handle, owner):
        if not handle:
            return None
        lib = load()
        dt = C.c_int()
        check(lib.ocu_grid_info(handle, None, C.byref(dt), None))
        return cls(dt.value, _handle=handle, _owner=owner)

    def init(self, nx, ny, nz, gx=1, gy=1, gz=1, padx=0, pady=0, padz=0):
        h = C.c_void_p()
        check(load().ocu_grid_create(self.dtype, nx, ny, nz, gx, gy, gz, padx, pady, padz, C.byref(h)))
        self._h = h.value
        self._owned = True
        return True

    def init_congruent(self, other):
        L = other.layout
        return self.init(L.nx, L.ny, L.nz, L.gx, L.gy, L.gz, L.pnx - (L.nx + 2 * L.gx),
                         L.pny - (L.ny + 2 * L.gy), L.pnz - (L.nz + 2 * L.gz))

    @property
    def handle(self):
        return self._h

    @property
    def layout(self):
        L = Layout()
        check(load().ocu_grid_info(self._h, C.byref(L), None, None))
        return L

    @property
    def device_ptr(self):
        p = C.c_void_p()
        check(load().ocu_grid_info(self._h, None, None, C.byref(p)))
        return p.value

    nx = property(lambda self: self.layout.nx)
    ny = property(lambda self: self.layout.ny)
    nz = property(lambda self: self.layout.nz)

    def empty_host(self):
        return np.zeros(int(self.layout.allocated), dtype=_np_dtype(self.dtype))

    def copy_from_host(self, host):
        host = np.ascontiguousarray(host, dtype=_np_dtype(self.dtype))
        assert host.size == self.layout.allocated
        check(load().ocu_grid_upload(self._h, host.ctypes.data_as(C.c_void_p), None))

    def copy_to_host(self, out=None):
        if out is None:
            out = self.empty_host()
        check(load().ocu_grid_download(self._h, out.ctypes.data_as(C.c_void_p), None))
        return out

    def clear_zero(self):
        check(load().ocu_grid_clear(self._h, 0.0, None))
        return True

    def clear(self, value):
        check(load().ocu_grid_clear(self._h, float(value), None))
        return True

    def copy_all_data(self, other):
        check(load().ocu_grid_copy_all_data(self._h, other._h, None))
        return True

    def linear_combination(self, a1, g1, a2=None, g2=None):
        check(load().ocu_grid_linear_combination(self._h, float(a1), g1._h, float(a2 or 0.0),
                                                 g2._h if g2 is not None else None, None))
        return True

    def _reduce(self, op):
        r = C.c_double()
        check(load().ocu_grid_reduce(self._h, op, C.byref(r), None))
        return r.value

    def reduce_maxabs(self):
        return self._reduce(REDUCE_MAXABS)

    def reduce_max(self):
        return self._reduce(REDUCE_MAX)

    def reduce_min(self):
        return self._reduce(REDUCE_MIN)

    def reduce_sum(self):
        return self._reduce(REDUCE_SUM)

    def reduce_sqrsum(self):
        return self._reduce(REDUCE_SQRSUM)

    def reduce_checknan(self):
        return self._reduce(REDUCE_CHECKNAN)

    def apply_boundary_conditions(self, bc, hx, hy, hz, variant=BC_LEVEL1):
        c = bc.to_c()
        check(load().ocu_apply_boundary_conditions(self._h, C.byref(c), hx, hy, hz, variant, None))

    def __del__(self):
        try:
            if self._owned and self._h:
                load().ocu_grid_destroy(self._h)
                self._h = None
        except Exception:
            pass


def apply_3d_mac_boundary_conditions_level1(u, v, w, bc, hx, hy, hz):
    c = bc.to_c()
    check(load().ocu_apply_mac_boundary_conditions(u._h, v._h, w._h, C.byref(c), hx, hy, hz, None))
    return True


class _MGBase:
    kind = MG_F32

    def __init__(self):
        p = MGParams()
        load().ocu_mg_params_default(C.byref(p))
        self.bc = BoundaryConditionSet()
        self.nu1 = p.nu1
        self.nu2 = p.nu2
        self.convergence = p.convergence
        self.make_symmetric_operator = False
        self.disable_relax_on_host = False
        self.ir_inner_cycles = p.ir_inner_cycles
        self.store_residual_grids = False
        self.unfused = False
        self.tail_cells = 0
        self.sweep_cells = 0
        self.ir_inner_exact = False
        self.wait_limit = 0
        self._h = None
        self._rhs = None

    def _params(self):
        p = MGParams()
        p.bc = self.bc.to_c()
        p.nu1, p.nu2, p.convergence = self.nu1, self.nu2, self.convergence
        p.make_symmetric_operator = int(bool(self.make_symmetric_operator))
        p.disable_relax_on_host = int(bool(self.disable_relax_on_host))
        p.ir_inner_cycles = self.ir_inner_cycles
        p.store_residual_grids = int(bool(self.store_residual_grids))
        p.unfused = int(bool(self.unfused))
        p.tail_cells = int(self.tail_cells)
        p.sweep_cells = int(self.sweep_cells)
        p.ir_inner_exact = int(bool(self.ir_inner_exact))
        p.wait_limit = int(self.wait_limit)
        return p

    def initialize_storage(self, nx, ny, nz, hx, hy, hz, rhs):
        lib = load()
        h = C.c_void_p()
        p = self._params()
        check(lib.ocu_mg_create(self.kind, C.byref(p), C.byref(h)))
        self._h = h.value
        self._rhs = rhs  # borrowed, as in the reference
        check(lib.ocu_mg_initialize_storage(self._h, nx, ny, nz, hx, hy, hz, rhs._h))
        return True

    def _sync_params(self):
        p = self._params()
        check(load().ocu_mg_set_params(self._h, C.byref(p)))

    def solve(self, tolerance=1e-6, max_iter=4):
        """Base::solve (sol_mgpressure3d.cpp:332-370) -> (converged, residual)."""
        self._sync_params()
        r = C.c_double()
        st = check(load().ocu_mg_solve(self._h, C.byref(r), tolerance, max_iter),
                   allow=(ERR_NOT_CONVERGED,))
        return st == OK, r.value

    def run_vcycles(self, count):
        self._sync_params()
        check(load().ocu_mg_run_vcycles(self._h, count))
        return True

    def run_fmg(self, count):
        self._sync_params()
        check(load().ocu_mg_run_fmg(self._h, count))
        return True

    def pressure(self):
        return Grid3DDevice._borrow(load().ocu_mg_pressure(self._h), self)

    def read_u(self, level):
        return Grid3DDevice._borrow(load().ocu_mg_level_grid(self._h, b"u", level), self)

    def read_r(self, level):
        return Grid3DDevice._borrow(load().ocu_mg_level_grid(self._h, b"r", level), self)

    def read_b(self, level):
        return Grid3DDevice._borrow(load().ocu_mg_level_grid(self._h, b"b", level), self)

    @property
    def stats(self):
        s = MGStats()
        check(load().ocu_mg_get_stats(self._h, C.byref(s)))
        return s

    # level operations (protected in the reference; exposed for tests and kernel timing)
    def relax(self, level, iterations, order=0, core=0):
        check(load().ocu_mg_relax(self._h, core, level, iterations, order))

    def relax_sweep(self, level, color, core=0):
        check(load().ocu_mg_relax_sweep(self._h, core, level, color))

    def restrict_residuals(self, fine, coarse, norms=False, core=0):
        l2, linf = C.c_double(), C.c_double()
        check(load().ocu_mg_restrict_residuals(self._h, core, fine, coarse,
                                               C.byref(l2) if norms else None,
                                               C.byref(linf) if norms else None))
        return (l2.value, linf.value) if norms else None

    def prolong(self, coarse, fine, core=0):
        check(load().ocu_mg_prolong(self._h, core, coarse, fine))

    def synchronize(self):
        check(load().ocu_mg_synchronize(self._h))

    def __del__(self):
        try:
            if self._h:
                load().ocu_mg_destroy(self._h)
                self._h = None
        except Exception:
            pass


class Sol_MultigridPressure3DDevice(_MGBase):
    """Sol_MultigridPressure3DDevice<T> (ocuequation/sol_mgpressure3d.h:104-181)."""

    def __init__(self, dtype=F32):
        super().__init__()
        self.kind = MG_F64 if dtype == F64 else MG_F32


def Sol_MultigridPressure3DDeviceF():
    return Sol_MultigridPressure3DDevice(F32)


def Sol_MultigridPressure3DDeviceD():
    return Sol_MultigridPressure3DDevice(F64)


class Sol_MultigridPressure3DDeviceCo(_MGBase):
    """Sol_MultigridPressure3DDeviceCo<T> (sol_mgpressure3d.h:184-242, sol_mgpressure3dco.cu).

    The domain is split along x into `num_images` slabs, image i on device devices[i] (several
    images may share a device).  initialize_storage takes the slab size and one rhs grid per
    image; co_pressure(i) is image i's slab of the pressure.  One host thread drives every image:
    the x halo planes are copied device to device after each ghost refresh, and the levels of at
    most grid_size_for_cutoff cells are held whole by image 0.  solve / run_vcycles / run_fmg and
    the parameters are those of Sol_MultigridPressure3DDevice.
    """

    def __init__(self, dtype=F32, num_images=1, devices=None):
        super().__init__()
        self.kind = MG_F64 if dtype == F64 else MG_F32
        self.num_images = int(num_images)
        self.devices = [int(d) for d in devices] if devices is not None else [0] * self.num_images
        if len(self.devices) != self.num_images:
            raise ValueError("one device per image")
        self.grid_size_for_cutoff = 64 * 64 * 64

    def initialize_storage(self, nx, ny, nz, hx, hy, hz, rhs):
        """nx: the slab's cells along x; rhs: one grid per image (borrowed)."""
        rhs = list(rhs)
        if len(rhs) != self.num_images:
            raise ValueError("one rhs grid per image")
        lib = load()
        h = C.c_void_p()
        p = self._params()
        devs = (C.c_int * self.num_images)(*self.devices)
        check(lib.ocu_mgco_create(self.kind, C.byref(p), self.num_images, devs, C.byref(h)))
        self._h = h.value
        self._rhs = rhs
        check(lib.ocu_mgco_set_cutoff_cells(self._h, int(self.grid_size_for_cutoff)))
        arr = (C.c_void_p * self.num_images)(*[g._h for g in rhs])
        check(lib.ocu_mgco_initialize_storage(self._h, nx, ny, nz, hx, hy, hz, arr))
        return True

    def co_pressure(self, image=0):
        return Grid3DDevice._borrow(load().ocu_mgco_pressure(self._h, int(image)), self)

    @property
    def cutoff_level(self):
        return load().ocu_mgco_cutoff_level(self._h)


def mgco_plan(nx_local, ny, nz, num_images, image, bc, cutoff_cells=64 * 64 * 64):
    """The decomposition of one image of a Sol_MultigridPressure3DDeviceCo (host only):
    level count, cutoff level, x neighbours (-1 at the domain's face) and the image's faces."""
    out = _capi.MGCoPlan()
    b = bc.to_c()
    check(load().ocu_mgco_plan_compute(nx_local, ny, nz, num_images, image, int(cutoff_cells), C.byref(b),
                                       C.byref(out)))
    return {"num_levels": out.num_levels, "cutoff_level": out.cutoff_level, "neg_image": out.neg_image,
            "pos_image": out.pos_image,
            "local_bc": {f: getattr(out.local_bc, f).type for f in ("xpos", "xneg", "ypos", "yneg", "zpos", "zneg")}}


class PressureEnsemble:
    """Many independent pressure solves of uneven sizes run together (ocu_ens_* in the C ABI).

    Members with the same dimensions and spacings form a size class; every multigrid step of a
    class is one launch over all its members and convergence is decided per member on the
    device.  Each member's pressure is bit-identical to Sol_MultigridPressure3DDevice.solve on
    that member alone with the same parameters.
    """

    def __init__(self, dtype, dims, spacings, bc=None, nu1=2, nu2=2, make_symmetric_operator=False,
                 disable_relax_on_host=False):
        lib = load()
        n = len(dims)
        d = (C.c_int * (3 * n))(*[int(v) for t in dims for v in t])
        h = (C.c_double * (3 * n))(*[float(v) for t in spacings for v in t])
        p = MGParams()
        lib.ocu_mg_params_default(C.byref(p))
        p.bc = (bc or BoundaryConditionSet(BoundaryCondition(BC_NEUMANN, 0.0))).to_c()
        p.nu1, p.nu2 = nu1, nu2
        p.make_symmetric_operator = int(bool(make_symmetric_operator))
        p.disable_relax_on_host = int(bool(disable_relax_on_host))
        handle = C.c_void_p()
        check(lib.ocu_ens_create(dtype, n, d, h, C.byref(p), C.byref(handle)))
        self._h = handle.value
        self.dtype = dtype
        self.count = n

    def rhs(self, m):
        out = C.c_void_p()
        check(load().ocu_ens_rhs(self._h, m, C.byref(out)))
        return Grid3DDevice._borrow(out.value, self)

    def pressure(self, m):
        out = C.c_void_p()
        check(load().ocu_ens_pressure(self._h, m, C.byref(out)))
        return Grid3DDevice._borrow(out.value, self)

    def set_stream(self, stream_handle):
        check(load().ocu_ens_set_stream(self._h, C.c_void_p(stream_handle)))

    def solve(self, tol, max_iter=20):
        """tol: absolute L2 tolerance per member.  Returns the number of members converged."""
        t = (C.c_double * self.count)(*[float(v) for v in tol])
        conv = C.c_int()
        check(load().ocu_ens_solve(self._h, t, int(max_iter), C.byref(conv)), allow=(ERR_NOT_CONVERGED,))
        return conv.value

    def autotune(self, tol, max_iter=20):
        t = (C.c_double * self.count)(*[float(v) for v in tol])
        check(load().ocu_ens_autotune(self._h, t, int(max_iter)))

    def member_stats(self, m):
        st = MGStats()
        check(load().ocu_ens_member_stats(self._h, m, C.byref(st)))
        return st

    def classes(self):
        lib = load()
        n = C.c_int()
        check(lib.ocu_ens_num_classes(self._h, C.byref(n)))
        out = []
        for c in range(n.value):
            dims = (C.c_int * 3)()
            members = C.c_int()
            t = EnsTuning()
            check(lib.ocu_ens_class_info(self._h, c, dims, C.byref(members), C.byref(t)))
            out.append({"dims": tuple(dims), "members": members.value, "nu1": t.nu1, "nu2": t.nu2,
                        "relax_block": tuple(t.relax_block), "ms": t.ms})
        return out

    def set_tuning(self, cls, nu1, nu2, relax_block=(32, 4, 2)):
        t = EnsTuning()
        t.nu1, t.nu2 = nu1, nu2
        t.relax_block[:] = list(relax_block)
        check(load().ocu_ens_set_tuning(self._h, cls, C.byref(t)))

    def __del__(self):
        try:
            if self._h:
                load().ocu_ens_destroy(self._h)
                self._h = None
        except Exception:
            pass


class PersistentEnsemble:
    """Many independent pressure solves of uneven sizes in one persistent kernel launch
    (ocu_pens_* in the C ABI).

    Each block of the launch takes the next member (largest first) and runs its whole solve: an
    FP64 iterative refinement whose corrections are FP32 multigrid solves on the library's
    red/black split levels, until sqrt(sum r^2 / N) of the FP64 residual is at most the member's
    tolerance.  Right-hand sides and pressures are FP64 grids.
    """

    def __init__(self, dims, spacings, bc=None, nu1=2, nu2=2, cycles=2, ramp_iters=0, max_outer=10,
                 threads=512, dense=False, tail_cells=0):
        lib = load()
        n = len(dims)
        d = (C.c_int * (3 * n))(*[int(v) for t in dims for v in t])
        h = (C.c_double * (3 * n))(*[float(v) for t in spacings for v in t])
        p = PensParams()
        lib.ocu_pens_params_default(C.byref(p))
        if bc is not None:
            p.bc = bc.to_c()
        p.nu1, p.nu2, p.cycles, p.ramp_iters = nu1, nu2, cycles, ramp_iters
        p.max_outer, p.threads, p.dense, p.tail_cells = max_outer, threads, int(bool(dense)), tail_cells
        handle = C.c_void_p()
        check(lib.ocu_pens_create(n, d, h, C.byref(p), C.byref(handle)))
        self._h = handle.value
        self.count = n

    def rhs(self, m):
        out = C.c_void_p()
        check(load().ocu_pens_rhs(self._h, m, C.byref(out)))
        return Grid3DDevice._borrow(out.value, self)

    def pressure(self, m):
        out = C.c_void_p()
        check(load().ocu_pens_pressure(self._h, m, C.byref(out)))
        return Grid3DDevice._borrow(out.value, self)

    def set_stream(self, stream_handle):
        check(load().ocu_pens_set_stream(self._h, C.c_void_p(stream_handle)))

    def solve(self, tol):
        """tol: absolute L2 tolerance per member.  Returns the number of members converged."""
        t = (C.c_double * self.count)(*[float(v) for v in tol])
        conv = C.c_int()
        check(load().ocu_pens_solve(self._h, t, C.byref(conv)), allow=(ERR_NOT_CONVERGED,))
        return conv.value

    def member_stats(self, m):
        st = PensStats()
        check(load().ocu_pens_member_stats(self._h, m, C.byref(st)))
        return st

    def params(self):
        p = PensParams()
        check(load().ocu_pens_get_params(self._h, C.byref(p)))
        return p

    def set_params(self, **kw):
        p = self.params()
        for k, v in kw.items():
            setattr(p, k, v)
        check(load().ocu_pens_set_params(self._h, C.byref(p)))

    def launch_shape(self):
        b, t, s = C.c_int(), C.c_int(), C.c_longlong()
        check(load().ocu_pens_launch_shape(self._h, C.byref(b), C.byref(t), C.byref(s)))
        return b.value, t.value, s.value

    def autotune(self, tol):
        t = (C.c_double * self.count)(*[float(v) for v in tol])
        check(load().ocu_pens_autotune(self._h, t))

    def __del__(self):
        try:
            if self._h:
                load().ocu_pens_destroy(self._h)
                self._h = None
        except Exception:
            pass


class Sol_PCGPressure3DDevice:
    """Preconditioned conjugate gradients on L p = rhs, L = -div(c grad) with a cell coefficient
    grid c (Sol_PCGPressure3DDevice<T>, sol_pcgpressure3d.h:41-97).  preconditioner: one of
    PRECOND_NONE, PRECOND_JACOBI, PRECOND_MULTIGRID, PRECOND_BFBT (the reference's default);
    faces periodic or Neumann.  Bit-identical to the CPU oracle's restatement."""

    def __init__(self, dtype):
        p = PCGParams()
        load().ocu_pcg_params_default(C.byref(p))
        self.dtype = dtype
        self.bc = BoundaryConditionSet(BoundaryCondition(BC_NEUMANN, 0.0))
        self.convergence = p.convergence
        self.preconditioner = p.preconditioner
        self.multigrid_cycles = p.multigrid_cycles
        self.multigrid_use_fmg = bool(p.multigrid_use_fmg)
        self._h = None
        self._keep = ()

    def _params(self):
        p = PCGParams()
        p.bc = self.bc.to_c()
        p.convergence = int(self.convergence)
        p.preconditioner = int(self.preconditioner)
        p.multigrid_cycles = int(self.multigrid_cycles)
        p.multigrid_use_fmg = int(bool(self.multigrid_use_fmg))
        return p

    def initialize_storage(self, nx, ny, nz, hx, hy, hz, rhs, coefficient):
        lib = load()
        h = C.c_void_p()
        p = self._params()
        check(lib.ocu_pcg_create(self.dtype, C.byref(p), C.byref(h)))
        self._h = h.value
        self._keep = (rhs, coefficient)  # borrowed, as in the reference
        check(lib.ocu_pcg_initialize_storage(self._h, nx, ny, nz, hx, hy, hz, rhs._h, coefficient._h))
        return True

    def solve(self, tolerance=1e-6, max_iter=1000):
        """solve (sol_pcgpressure3d.cu:571-601) -> (converged, residual)."""
        p = self._params()
        check(load().ocu_pcg_set_params(self._h, C.byref(p)))
        r = C.c_double()
        st = check(load().ocu_pcg_solve(self._h, C.byref(r), tolerance, max_iter), allow=(ERR_NOT_CONVERGED,))
        return st == OK, r.value

    def pressure(self):
        out = C.c_void_p()
        check(load().ocu_pcg_pressure(self._h, C.byref(out)))
        return Grid3DDevice._borrow(out.value, self)

    @property
    def iterations(self):
        n = C.c_int()
        check(load().ocu_pcg_iterations(self._h, C.byref(n)))
        return n.value

    def set_stream(self, stream_handle):
        check(load().ocu_pcg_set_stream(self._h, C.c_void_p(stream_handle)))

    def __del__(self):
        try:
            if self._h:
                load().ocu_pcg_destroy(self._h)
                self._h = None
        except Exception:
            pass


_NC_NP = {NC_FLOAT: np.float32, NC_DOUBLE: np.float64, NC_INT: np.int32}


class NetCDFGrid3DWriter:
    """The reference's NetCDF grid files (ocustorage/gridnetcdf.h:67-123), written without
    libnetcdf in the NetCDF classic format.  add_data takes a Grid3DDevice or an (nx, ny, nz)
    numpy array of the variable's type; the file is written at close()."""

    def __init__(self):
        self._h = None

    def open(self, filename, nx, ny, nz, hx=1.0, hy=1.0, hz=1.0):
        h = C.c_void_p()
        check(load().ocu_nc_writer_open(os.fsencode(filename), nx, ny, nz, hx, hy, hz, C.byref(h)))
        self._h = h.value
        return True

    def is_open(self):
        return self._h is not None

    def define_variable(self, name, var_type, stag=GS_CENTER_POINT, offsetx=0.5, offsety=0.5, offsetz=0.5):
        check(load().ocu_nc_writer_define_variable(self._h, name.encode(), var_type, stag, offsetx, offsety, offsetz))
        return True

    def add_time_level(self, time):
        lvl = C.c_int()
        check(load().ocu_nc_writer_add_time_level(self._h, time, C.byref(lvl)))
        return lvl.value

    def add_data(self, name, grid, time_level=0):
        if isinstance(grid, Grid3DDevice):
            check(load().ocu_nc_writer_add_grid(self._h, name.encode(), grid._h, time_level))
            return True
        a = np.ascontiguousarray(grid)
        t = {np.dtype(np.float32): NC_FLOAT, np.dtype(np.float64): NC_DOUBLE, np.dtype(np.int32): NC_INT}[a.dtype]
        nx, ny, nz = a.shape
        check(load().ocu_nc_writer_add_data(self._h, name.encode(), a.ctypes.data_as(C.c_void_p), t, ny * nz, nz,
                                            nx, ny, nz, time_level))
        return True

    def close(self):
        h, self._h = self._h, None
        check(load().ocu_nc_writer_close(h))
        return True


class NetCDFGrid3DReader:
    """Reader of those files (ocustorage/gridnetcdf.h:126-183); read_variable returns an
    (nx, ny, nz) numpy array of the variable's type."""

    def __init__(self):
        self._h = None

    def open(self, filename):
        h = C.c_void_p()
        check(load().ocu_nc_reader_open(os.fsencode(filename), C.byref(h)))
        self._h = h.value
        nx, ny, nz, nt = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        hx, hy, hz = C.c_float(), C.c_float(), C.c_float()
        check(load().ocu_nc_reader_info(self._h, C.byref(nx), C.byref(ny), C.byref(nz), C.byref(hx), C.byref(hy),
                                        C.byref(hz), C.byref(nt)))
        self.nx, self.ny, self.nz = nx.value, ny.value, nz.value
        self.hx, self.hy, self.hz = hx.value, hy.value, hz.value
        self._nt = nt.value
        return True

    def is_open(self):
        return self._h is not None

    def num_time_levels(self):
        return self._nt

    def get_time(self, time_level):
        t = C.c_float()
        check(load().ocu_nc_reader_get_time(self._h, time_level, C.byref(t)))
        return t.value

    def _vars(self):
        n = C.c_int()
        check(load().ocu_nc_reader_num_variables(self._h, C.byref(n)))
        out = {}
        for q in range(n.value):
            buf = C.create_string_buffer(1024)
            t, x, y, z = C.c_int(), C.c_int(), C.c_int(), C.c_int()
            check(load().ocu_nc_reader_variable(self._h, q, buf, 1024, C.byref(t), C.byref(x), C.byref(y),
                                                C.byref(z)))
            out[buf.value.decode()] = (t.value, (x.value, y.value, z.value))
        return out

    def list_variables(self):
        return list(self._vars())

    def variable_type(self, name):
        return self._vars()[name][0]

    def variable_size(self, name):
        return self._vars()[name][1]

    def read_variable(self, name, time_level=0):
        t, (nx, ny, nz) = self._vars()[name]
        a = np.empty((nx, ny, nz), _NC_NP[t])
        check(load().ocu_nc_reader_read(self._h, name.encode(), a.ctypes.data_as(C.c_void_p), t, ny * nz, nz, nx, ny,
                                        nz, time_level))
        return a

    def close(self):
        if self._h:
            load().ocu_nc_reader_close(self._h)
            self._h = None
        return True

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Sol_MultigridPressureMixed3DDeviceD(_MGBase):
    """FP64-interface mixed solver.  algorithm='ir' (default): FP32 V-cycles inside FP64
    iterative refinement; algorithm='warmstart': the reference algorithm
    (sol_mgpressuremixed3ddevd.cpp:79-100)."""

    def __init__(self, algorithm="ir"):
        super().__init__()
        self.kind = MG_MIXED_IR if algorithm == "ir" else MG_MIXED_WARMSTART


class Sol_ProjectDivergence3DDevice:
    """Sol_ProjectDivergence3DDevice<T> (ocuequation/sol_project3d.h:74-93)."""

    def __init__(self, dtype=F32, _kind=None):
        self.dtype = dtype
        self.bc = BoundaryConditionSet()
        h = C.c_void_p()
        if _kind is None:
            check(load().ocu_project_create(dtype, C.byref(h)))
        else:
            check(load().ocu_project_create_with(_kind, C.byref(h)))
        self._h = h.value
        self._keep = None

    def initialize_storage(self, nx, ny, nz, hx, hy, hz, u, v, w):
        c = self.bc.to_c()
        self._keep = (u, v, w)
        check(load().ocu_project_initialize_storage(self._h, nx, ny, nz, hx, hy, hz, u._h, v._h, w._h,
                                                    C.byref(c)))
        return True

    def solve(self, tolerance=1e-5):
        st = check(load().ocu_project_solve(self._h, tolerance), allow=(ERR_NOT_CONVERGED,))
        return st == OK

    def solve_divergence_only(self):
        check(load().ocu_project_solve_divergence_only(self._h))
        return True

    @property
    def divergence(self):
        return Grid3DDevice._borrow(load().ocu_project_divergence(self._h), self)

    @property
    def pressure_solver(self):
        h = load().ocu_project_pressure_solver(self._h)
        p = MGParams()
        check(load().ocu_mg_get_params(h, C.byref(p)))
        return _BorrowedMG(h, self, p)

    def __del__(self):
        try:
            if self._h:
                load().ocu_project_destroy(self._h)
                self._h = None
        except Exception:
            pass


class Sol_ProjectDivergenceMixed3DDeviceD(Sol_ProjectDivergence3DDevice):
    """Sol_ProjectDivergenceMixed3DDeviceD (ocuequation/sol_projectmixed3d.h:28-45): FP64 fields,
    mixed-precision pressure solver.  algorithm "warmstart" is the reference's mixed solver (FP32
    FMG warm start + FP64 FMG); "ir" this library's FP32-in-FP64 refinement (the default, as for
    Sol_MultigridPressureMixed3DDeviceD)."""

    def __init__(self, algorithm="ir"):
        kind = MG_MIXED_IR if algorithm == "ir" else MG_MIXED_WARMSTART
        super().__init__(F64, _kind=kind)


class _BorrowedMG(_MGBase):
    """Pressure solver owned by a projection object (no destroy on collection)."""

    def __init__(self, handle, owner, p):
        _MGBase.__init__(self)
        self._h = handle
        self._owner = owner
        self.nu1, self.nu2, self.convergence = p.nu1, p.nu2, p.convergence
        bc = BoundaryConditionSet()
        for f in BoundaryConditionSet.FACES:
            b = getattr(p.bc, f)
            setattr(bc, f, BoundaryCondition(b.type, b.value, b.aux_value))
        self.bc = bc

    def __del__(self):
        pass


class Sol_SelfAdvection3DDevice:
    """Sol_SelfAdvection3DDevice<T> (sol_selfadvection3d.h:33-73)."""

    def __init__(self):
        self.interp_type = IT_FIRST_ORDER_UPWIND

    def initialize_storage(self, nx, ny, nz, hx, hy, hz, u, v, w, dudt, dvdt, dwdt):
        self.args = (nx, ny, nz, hx, hy, hz)
        self.g = (u, v, w, dudt, dvdt, dwdt)
        return True

    def solve(self):
        nx, ny, nz, hx, hy, hz = self.args
        u, v, w, du, dv, dw = self.g
        check(load().ocu_advect_self(u._h, v._h, w._h, du._h, dv._h, dw._h, nx, ny, nz, hx, hy, hz,
                                     self.interp_type, None))
        return True


class Sol_PassiveAdvection3DDevice:
    """Sol_PassiveAdvection3DDevice<T> (sol_passiveadvection3d.h:32-62)."""

    def __init__(self):
        self.interp_type = IT_FIRST_ORDER_UPWIND

    def initialize_storage(self, nx, ny, nz, hx, hy, hz, u, v, w, phi, dphidt):
        self.args = (nx, ny, nz, hx, hy, hz)
        self.g = (u, v, w, phi, dphidt)
        return True

    def solve(self):
        nx, ny, nz, hx, hy, hz = self.args
        u, v, w, phi, dphi = self.g
        check(load().ocu_advect_passive(u._h, v._h, w._h, phi._h, dphi._h, nx, ny, nz, hx, hy, hz,
                                        self.interp_type, None))
        return True


class Sol_LaplacianCentered3DDevice:
    """Sol_LaplacianCentered3DDevice<T> (sol_laplaciancent3d.h:28-58)."""

    def __init__(self):
        self.coefficient = 1.0

    def initialize_storage(self, nx, ny, nz, hx, hy, hz, phi, dphidt):
        self.args = (nx, ny, nz, hx, hy, hz)
        self.g = (phi, dphidt)
        return True

    def solve(self):
        nx, ny, nz, hx, hy, hz = self.args
        phi, dphi = self.g
        check(load().ocu_laplacian_add(phi._h, dphi._h, nx, ny, nz, hx, hy, hz, float(self.coefficient),
                                       None))
        return True


class Eqn_IncompressibleNS3DParams:
    """Eqn_IncompressibleNS3DParams<T> (eqn_incompressns3d.h:34-87); init_* are numpy host grids."""

    def __init__(self, dtype=F32):
        p = NSParams()
        load().ocu_ns_params_default(C.byref(p))
        self.dtype = dtype
        self.nx = self.ny = self.nz = 0
        self.hx = self.hy = self.hz = 0.0
        self.max_divergence = p.max_divergence
        self.temp_bc = BoundaryConditionSet()
        self.flow_bc = BoundaryConditionSet()
        self.vertical_direction = p.vertical_direction
        self.gravity = p.gravity
        self.bouyancy = p.bouyancy
        self.thermal_diffusion = p.thermal_diffusion
        self.viscosity = p.viscosity
        self.advection_scheme = p.advection_scheme
        self.time_step = p.time_step
        self.cfl_factor = p.cfl_factor
        # library option, not a reference field: FP64 pressure by FP32 V-cycles in FP64 refinement
        self.mixed_pressure = False
        self.init_u = self.init_v = self.init_w = self.init_temp = None
        self.layouts = {}

    def init_grids(self, nx, ny, nz):
        self.nx, self.ny, self.nz = nx, ny, nz
        for c in "uvwt":
            L = Layout()
            check(load().ocu_ns_init_layout(nx, ny, nz, c.encode(), C.byref(L)))
            self.layouts[c] = L
        dt = _np_dtype(self.dtype)
        self.init_u = np.zeros(int(self.layouts["u"].allocated), dt)
        self.init_v = np.zeros(int(self.layouts["v"].allocated), dt)
        self.init_w = np.zeros(int(self.layouts["w"].allocated), dt)
        self.init_temp = np.zeros(int(self.layouts["t"].allocated), dt)

    def to_c(self):
        p = NSParams()
        p.nx, p.ny, p.nz = self.nx, self.ny, self.nz
        p.hx, p.hy, p.hz = self.hx, self.hy, self.hz
        p.max_divergence = self.max_divergence
        p.temp_bc = self.temp_bc.to_c()
        p.flow_bc = self.flow_bc.to_c()
        p.vertical_direction = self.vertical_direction
        p.gravity, p.bouyancy = self.gravity, self.bouyancy
        p.thermal_diffusion, p.viscosity = self.thermal_diffusion, self.viscosity
        p.advection_scheme, p.time_step, p.cfl_factor = self.advection_scheme, self.time_step, self.cfl_factor
        p.mixed_pressure = int(bool(self.mixed_pressure))
        return p


class Eqn_IncompressibleNS3D:
    """Eqn_IncompressibleNS3D<T> (eqn_incompressns3d.h:138-177)."""

    def __init__(self, dtype=F32):
        self.dtype = dtype
        h = C.c_void_p()
        check(load().ocu_ns_create(dtype, C.byref(h)))
        self._h = h.value

    def set_parameters(self, params):
        p = params.to_c()
        dt = _np_dtype(self.dtype)
        arrs = [np.ascontiguousarray(a, dtype=dt) for a in
                (params.init_u, params.init_v, params.init_w, params.init_temp)]
        check(load().ocu_ns_set_parameters(self._h, C.byref(p),
                                           *[a.ctypes.data_as(C.c_void_p) for a in arrs]))
        return True

    def get_max_stable_timestep(self):
        d = C.c_double()
        check(load().ocu_ns_get_max_stable_timestep(self._h, C.byref(d)))
        return d.value

    def advance_one_step(self, dt):
        """advance_one_step (eqn_incompressns3d.cu:331-399).  Returns False, like the reference,
        when the projection's pressure solve stops above max_divergence; the state has still
        been advanced and projected with the last pressure iterate."""
        st = check(load().ocu_ns_advance_one_step(self._h, dt), allow=(ERR_NOT_CONVERGED,))
        return st == OK

    def advance(self, dt):
        """Equation::advance (equation.cpp:31-56): sub-steps at the stable time step; stops and
        returns False at the first sub-step that fails."""
        st = check(load().ocu_ns_advance(self._h, dt), allow=(ERR_NOT_CONVERGED,))
        return st == OK

    @property
    def num_steps(self):
        return load().ocu_ns_num_steps(self._h)

    def _grid(self, c):
        return Grid3DDevice._borrow(load().ocu_ns_grid(self._h, c.encode()), self)

    def get_u(self):
        return self._grid("u")

    def get_v(self):
        return self._grid("v")

    def get_w(self):
        return self._grid("w")

    def get_temperature(self):
        return self._grid("t")

    def get_deriv(self, c):
        return self._grid(c.upper())

    def get_pressure(self):
        return self._grid("p")

    def __del__(self):
        try:
            if self._h:
                load().ocu_ns_destroy(self._h)
                self._h = None
        except Exception:
            pass
