"""ctypes declarations of the libocu_b200.so C ABI (include/ocu_b200.h, include/ocu_types.h).

The library is loaded from this package directory only; there is no CPU fallback: if the
shared object is missing the import raises, and every compute call on a machine without a B200
returns OCU_ERR_CUDA, which the wrappers raise as OcuError.
"""
import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libocu_b200.so")

# ---- enums (ocu_types.h) ------------------------------------------------------------------
F32, F64 = 0, 1
BC_INVALID, BC_NONE, BC_PERIODIC, BC_DIRICHELET, BC_NEUMANN = 0, 1, 2, 3, 4
BC_SECOND_DERIV, BC_DIRICHELET_AND_NEUMANN, BC_FORCED_INFLOW_VARIABLE_SLIP, BC_SCALAR_SLIP = 5, 6, 7, 8
CONVERGENCE_CALC_L2, CONVERGENCE_CALC_LINF = 0x01, 0x02
CONVERGENCE_CRITERIA_L2, CONVERGENCE_CRITERIA_LINF, CONVERGENCE_CRITERIA_NONE = 0x04, 0x08, 0x10
CONVERGENCE_L2, CONVERGENCE_LINF, CONVERGENCE_NONE = 0x05, 0x0A, 0x10
CONVERGENCE_NONE_CALC_L2LINF = 0x13
IT_ERROR, IT_FIRST_ORDER_UPWIND, IT_SECOND_ORDER_CENTERED = 0, 1, 2
TS_ERROR, TS_FORWARD_EULER, TS_ADAMS_BASHFORD2 = 0, 1, 2
DIR_POSITIVE_FLAG, DIR_NEGATIVE_FLAG = 0x01, 0x02
DIR_XAXIS_FLAG, DIR_YAXIS_FLAG, DIR_ZAXIS_FLAG = 0x04, 0x08, 0x10
DIR_XPOS, DIR_XNEG, DIR_YPOS, DIR_YNEG, DIR_ZPOS, DIR_ZNEG = 0x05, 0x06, 0x09, 0x0A, 0x11, 0x12
REDUCE_MAXABS, REDUCE_MAX, REDUCE_MIN, REDUCE_SUM, REDUCE_SQRSUM, REDUCE_CHECKNAN = range(6)
BC_LEVEL1, BC_LEVEL1_NOCORNERS = 0, 1
MG_F32, MG_F64, MG_MIXED_IR, MG_MIXED_WARMSTART = 0, 1, 2, 3
PRECOND_NONE, PRECOND_JACOBI, PRECOND_MULTIGRID, PRECOND_BFBT = 0, 1, 2, 3
GS_CENTER_POINT, GS_U_FACE, GS_V_FACE, GS_W_FACE, GS_CUSTOM = 0, 1, 2, 3, 4
NC_INT, NC_FLOAT, NC_DOUBLE = 4, 5, 6

OK, ERR_INVALID_VALUE, ERR_LAYOUT, ERR_CUDA, ERR_NOT_CONVERGED = 0, 1, 2, 3, 4
ERR_NOT_INITIALIZED, ERR_ALLOC, ERR_UNSUPPORTED, ERR_TIMEOUT = 5, 6, 7, 8
STATUS_NAMES = {0: "OK", 1: "INVALID_VALUE", 2: "LAYOUT", 3: "CUDA", 4: "NOT_CONVERGED",
                5: "NOT_INITIALIZED", 6: "ALLOC", 7: "UNSUPPORTED", 8: "TIMEOUT"}


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
                ("make_symmetric_operator", C.c_int), ("disable_relax_on_host", C.c_int),
                ("ir_inner_cycles", C.c_int), ("store_residual_grids", C.c_int),
                ("unfused", C.c_int), ("tail_cells", C.c_int), ("sweep_cells", C.c_int),
                ("ir_inner_exact", C.c_int), ("wait_limit", C.c_int)]


class MGCoPlan(C.Structure):
    _fields_ = [("num_levels", C.c_int), ("cutoff_level", C.c_int), ("neg_image", C.c_int),
                ("pos_image", C.c_int), ("local_bc", BCSet)]


class MGStats(C.Structure):
    _fields_ = [("num_levels", C.c_int), ("vcycles", C.c_int), ("outer_iterations", C.c_int),
                ("last_l2", C.c_double), ("last_linf", C.c_double), ("omega", C.c_double)]


class EnsTuning(C.Structure):
    _fields_ = [("nu1", C.c_int), ("nu2", C.c_int), ("relax_block", C.c_int * 3), ("ms", C.c_double)]


class PensParams(C.Structure):
    _fields_ = [("bc", BCSet), ("nu1", C.c_int), ("nu2", C.c_int), ("cycles", C.c_int),
                ("ramp_iters", C.c_int), ("max_outer", C.c_int), ("threads", C.c_int),
                ("dense", C.c_int), ("tail_cells", C.c_int), ("ms", C.c_double)]


class PensStats(C.Structure):
    _fields_ = [("converged", C.c_int), ("corrections", C.c_int), ("vcycles", C.c_int), ("l2", C.c_double)]


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
                ("time_step", C.c_int), ("cfl_factor", C.c_double), ("mixed_pressure", C.c_int)]


# symbol -> (restype, argtypes); the exported-symbol test checks this table against the header
P, I, D = C.c_void_p, C.c_int, C.c_double
LP, BP = C.POINTER(Layout), C.POINTER(BCSet)
PP = C.POINTER(C.c_void_p)
SIGNATURES = {
    "ocu_last_error": (C.c_char_p, []),
    "ocu_version": (C.c_char_p, []),
    "ocu_kernel_launch_count": (C.c_ulonglong, []),
    "ocu_layout_compute": (I, [I] * 9 + [LP]),
    "ocu_grid_create": (I, [I] + [I] * 9 + [PP]),
    "ocu_grid_wrap": (I, [I, LP, P, PP]),
    "ocu_grid_destroy": (None, [P]),
    "ocu_grid_info": (I, [P, LP, C.POINTER(C.c_int), PP]),
    "ocu_grid_upload": (I, [P, P, P]),
    "ocu_grid_download": (I, [P, P, P]),
    "ocu_grid_upload_async": (I, [P, P, P]),
    "ocu_grid_download_async": (I, [P, P, P]),
    "ocu_grid_copy_all_data": (I, [P, P, P]),
    "ocu_grid_clear": (I, [P, D, P]),
    "ocu_grid_linear_combination": (I, [P, D, P, D, P, P]),
    "ocu_grid_reduce": (I, [P, I, C.POINTER(D), P]),
    "ocu_grid_reduce_noalloc": (I, [P, I, C.POINTER(D), P]),
    "ocu_apply_boundary_conditions": (I, [P, BP, D, D, D, I, P]),
    "ocu_apply_mac_boundary_conditions": (I, [P, P, P, BP, D, D, D, P]),
    "ocu_divergence": (I, [P, P, P, P, I, I, I, D, D, D, P]),
    "ocu_gradient_add": (I, [P, P, P, P, D, D, D, D, P]),
    "ocu_advect_self": (I, [P, P, P, P, P, P, I, I, I, D, D, D, I, P]),
    "ocu_advect_passive": (I, [P, P, P, P, P, I, I, I, D, D, D, I, P]),
    "ocu_laplacian_add": (I, [P, P, I, I, I, D, D, D, D, P]),
    "ocu_mg_params_default": (None, [C.POINTER(MGParams)]),
    "ocu_mg_create": (I, [I, C.POINTER(MGParams), PP]),
    "ocu_mg_destroy": (None, [P]),
    "ocu_mg_set_params": (I, [P, C.POINTER(MGParams)]),
    "ocu_mg_get_params": (I, [P, C.POINTER(MGParams)]),
    "ocu_mg_set_stream": (I, [P, P]),
    "ocu_mg_initialize_storage": (I, [P, I, I, I, D, D, D, P]),
    "ocu_mg_solve": (I, [P, C.POINTER(D), D, I]),
    "ocu_mg_run_vcycles": (I, [P, I]),
    "ocu_mg_run_fmg": (I, [P, I]),
    "ocu_mg_pressure": (P, [P]),
    "ocu_mg_level_grid": (P, [P, C.c_char, I]),
    "ocu_mg_get_stats": (I, [P, C.POINTER(MGStats)]),
    "ocu_mg_relax": (I, [P, I, I, I, I]),
    "ocu_mg_relax_sweep": (I, [P, I, I, I]),
    "ocu_mg_restrict_residuals": (I, [P, I, I, I, C.POINTER(D), C.POINTER(D)]),
    "ocu_mg_prolong": (I, [P, I, I, I]),
    "ocu_mg_synchronize": (I, [P]),
    "ocu_mgco_plan_compute": (I, [I, I, I, I, I, C.c_longlong, C.POINTER(BCSet), C.POINTER(MGCoPlan)]),
    "ocu_mgco_create": (I, [I, C.POINTER(MGParams), I, C.POINTER(C.c_int), PP]),
    "ocu_mgco_set_cutoff_cells": (I, [P, C.c_longlong]),
    "ocu_mgco_initialize_storage": (I, [P, I, I, I, D, D, D, C.POINTER(P)]),
    "ocu_mgco_pressure": (P, [P, I]),
    "ocu_mgco_num_images": (I, [P]),
    "ocu_mgco_cutoff_level": (I, [P]),
    "ocu_advect_passive_adjoint": (I, [P] * 9 + [I, I, I, D, D, D, D, I, P]),
    "ocu_advect_self_adjoint": (I, [P] * 9 + [I, I, I, D, D, D, D, I, P]),
    "ocu_adj_create": (I, [I, I, I, I, D, D, D, I, I, D, I, D, PP]),
    "ocu_adj_destroy": (None, [P]),
    "ocu_adj_set_stream": (I, [P, P]),
    "ocu_adj_layout": (I, [P, C.c_char, LP]),
    "ocu_adj_forward": (I, [P, P, P, P, P, P]),
    "ocu_adj_backward": (I, [P, P, P, P, P, P]),
    "ocu_ens_create": (I, [I, I, C.POINTER(C.c_int), C.POINTER(D), C.POINTER(MGParams), PP]),
    "ocu_ens_destroy": (None, [P]),
    "ocu_ens_set_stream": (I, [P, P]),
    "ocu_ens_rhs": (I, [P, I, PP]),
    "ocu_ens_pressure": (I, [P, I, PP]),
    "ocu_ens_solve": (I, [P, C.POINTER(D), I, C.POINTER(C.c_int)]),
    "ocu_ens_member_stats": (I, [P, I, C.POINTER(MGStats)]),
    "ocu_ens_num_classes": (I, [P, C.POINTER(C.c_int)]),
    "ocu_ens_class_info": (I, [P, I, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(EnsTuning)]),
    "ocu_ens_set_tuning": (I, [P, I, C.POINTER(EnsTuning)]),
    "ocu_ens_autotune": (I, [P, C.POINTER(D), I]),
    "ocu_nc_writer_open": (I, [C.c_char_p, I, I, I, C.c_float, C.c_float, C.c_float, PP]),
    "ocu_nc_writer_define_variable": (I, [P, C.c_char_p, I, I, C.c_float, C.c_float, C.c_float]),
    "ocu_nc_writer_add_time_level": (I, [P, C.c_float, C.POINTER(C.c_int)]),
    "ocu_nc_writer_add_data": (I, [P, C.c_char_p, P, I, C.c_longlong, C.c_longlong, I, I, I, I]),
    "ocu_nc_writer_add_grid": (I, [P, C.c_char_p, P, I]),
    "ocu_nc_writer_close": (I, [P]),
    "ocu_nc_reader_open": (I, [C.c_char_p, PP]),
    "ocu_nc_reader_close": (None, [P]),
    "ocu_nc_reader_info": (I, [P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                               C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                               C.POINTER(C.c_int)]),
    "ocu_nc_reader_get_time": (I, [P, I, C.POINTER(C.c_float)]),
    "ocu_nc_reader_num_variables": (I, [P, C.POINTER(C.c_int)]),
    "ocu_nc_reader_variable": (I, [P, I, C.c_char_p, I, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                   C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "ocu_nc_reader_read": (I, [P, C.c_char_p, P, I, C.c_longlong, C.c_longlong, I, I, I, I]),
    "ocu_pcg_params_default": (None, [C.POINTER(PCGParams)]),
    "ocu_pcg_create": (I, [I, C.POINTER(PCGParams), PP]),
    "ocu_pcg_destroy": (None, [P]),
    "ocu_pcg_set_stream": (I, [P, P]),
    "ocu_pcg_set_params": (I, [P, C.POINTER(PCGParams)]),
    "ocu_pcg_initialize_storage": (I, [P, I, I, I, C.c_float, C.c_float, C.c_float, P, P]),
    "ocu_pcg_solve": (I, [P, C.POINTER(D), D, I]),
    "ocu_pcg_pressure": (I, [P, PP]),
    "ocu_pcg_iterations": (I, [P, C.POINTER(C.c_int)]),
    "ocu_pens_params_default": (None, [C.POINTER(PensParams)]),
    "ocu_pens_create": (I, [I, C.POINTER(C.c_int), C.POINTER(D), C.POINTER(PensParams), PP]),
    "ocu_pens_destroy": (None, [P]),
    "ocu_pens_set_stream": (I, [P, P]),
    "ocu_pens_rhs": (I, [P, I, PP]),
    "ocu_pens_pressure": (I, [P, I, PP]),
    "ocu_pens_solve": (I, [P, C.POINTER(D), C.POINTER(C.c_int)]),
    "ocu_pens_member_stats": (I, [P, I, C.POINTER(PensStats)]),
    "ocu_pens_get_params": (I, [P, C.POINTER(PensParams)]),
    "ocu_pens_set_params": (I, [P, C.POINTER(PensParams)]),
    "ocu_pens_launch_shape": (I, [P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
    "ocu_pens_autotune": (I, [P, C.POINTER(D)]),
    "ocu_project_create": (I, [I, PP]),
    "ocu_project_create_with": (I, [I, PP]),
    "ocu_project_create_fields": (I, [I, I, PP]),
    "ocu_project_destroy": (None, [P]),
    "ocu_project_set_stream": (I, [P, P]),
    "ocu_project_initialize_storage": (I, [P, I, I, I, D, D, D, P, P, P, BP]),
    "ocu_project_solve": (I, [P, D]),
    "ocu_project_solve_divergence_only": (I, [P]),
    "ocu_project_divergence": (P, [P]),
    "ocu_project_pressure_solver": (P, [P]),
    "ocu_ns_params_default": (None, [C.POINTER(NSParams)]),
    "ocu_ns_init_layout": (I, [I, I, I, C.c_char, LP]),
    "ocu_ns_create": (I, [I, PP]),
    "ocu_ns_destroy": (None, [P]),
    "ocu_ns_set_stream": (I, [P, P]),
    "ocu_ns_set_parameters": (I, [P, C.POINTER(NSParams), P, P, P, P]),
    "ocu_ns_get_max_stable_timestep": (I, [P, C.POINTER(D)]),
    "ocu_ns_advance_one_step": (I, [P, D]),
    "ocu_ns_advance": (I, [P, D]),
    "ocu_ns_grid": (P, [P, C.c_char]),
    "ocu_ns_num_steps": (I, [P]),
}

_lib = None


def load():
    """Load libocu_b200.so from the package directory (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} not found: build it with `python -m opencurrent_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class OcuError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def check(status, allow=()):
    if status != OK and status not in allow:
        raise OcuError(status, load().ocu_last_error().decode(errors="replace"))
    return status
