"""CPU: the C ABI library loads, exports every symbol include/ocu_b200.h declares, and its
host-only logic (layout rule, parameter defaults, argument validation) behaves like the
reference.  No kernel is launched here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import opencurrent_b200 as ocu
from opencurrent_b200 import _capi
from oracle import oracle_ctypes as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "ocu_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ocu_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ocu.load()
    names = declared_symbols()
    assert len(names) >= 50
    for n in names:
        assert hasattr(lib, n), n
        assert n in _capi.SIGNATURES, f"{n} missing from the ctypes table"


def test_version_and_counter():
    lib = ocu.load()
    assert b"sm_100a" in lib.ocu_version()
    assert ocu.kernel_launch_count() >= 0


@pytest.mark.parametrize("dims", [(64, 64, 64, 1, 1, 1, 0, 0, 0), (129, 128, 64, 1, 1, 1, 0, 1, 1),
                                  (7, 5, 3, 2, 2, 2, 1, 2, 3), (256, 256, 256, 1, 1, 1, 0, 0, 0)])
def test_layout_matches_oracle(dims):
    a = ocu.layout(*dims)
    b = O.layout(*dims)
    for f, _ in _capi.Layout._fields_:
        assert getattr(a, f) == getattr(b, f), f


def test_ns_init_layouts_congruent():
    """init_grids (eqn_incompressns3d.h:75-83) pads u, v, w, temp to one layout."""
    lib = ocu.load()
    Ls = []
    for c in b"uvwt":
        L = _capi.Layout()
        assert lib.ocu_ns_init_layout(128, 128, 64, bytes([c]), C.byref(L)) == 0
        Ls.append(L)
    assert len({(L.pnx, L.pny, L.pnz, L.shift, L.allocated) for L in Ls}) == 1
    assert (Ls[0].nx, Ls[1].ny, Ls[2].nz) == (129, 129, 65)


def test_defaults_match_reference_constructors():
    p = _capi.MGParams()
    ocu.load().ocu_mg_params_default(C.byref(p))
    # Sol_MultigridPressure3DBase() (sol_mgpressure3d.cpp:26-40)
    assert (p.nu1, p.nu2, p.convergence, p.make_symmetric_operator) == (2, 2, _capi.CONVERGENCE_L2, 0)
    q = _capi.NSParams()
    ocu.load().ocu_ns_params_default(C.byref(q))
    # Eqn_IncompressibleNS3DParams() (eqn_incompressns3d.h:62-73)
    assert q.advection_scheme == _capi.IT_FIRST_ORDER_UPWIND and q.max_divergence == 1e-5
    assert q.cfl_factor == 1 and q.gravity == -9.8 and q.bouyancy == 1
    assert q.time_step == _capi.TS_FORWARD_EULER and q.vertical_direction == _capi.DIR_YPOS


def test_argument_validation_without_gpu():
    lib = ocu.load()
    h = C.c_void_p()
    assert lib.ocu_mg_create(_capi.MG_F32, None, C.byref(h)) == 0
    r = C.c_double()
    # solve before initialize_storage
    assert lib.ocu_mg_solve(h, C.byref(r), 1e-6, 4) == _capi.ERR_NOT_INITIALIZED
    assert b"not initialized" in lib.ocu_last_error()
    # null rhs, garbage h (check_float, sol_mgpressure3d.cpp:405-408)
    assert lib.ocu_mg_initialize_storage(h, 8, 8, 8, float("nan"), 1.0, 1.0, None) == _capi.ERR_INVALID_VALUE
    assert lib.ocu_mg_initialize_storage(h, 8, 8, 8, 1.0, 1.0, 1.0, None) == _capi.ERR_INVALID_VALUE
    lib.ocu_mg_destroy(h)
    assert lib.ocu_mg_create(9, None, C.byref(h)) == _capi.ERR_INVALID_VALUE
    L = _capi.Layout()
    assert lib.ocu_layout_compute(-1, 2, 2, 1, 1, 1, 0, 0, 0, C.byref(L)) == _capi.ERR_INVALID_VALUE


def test_ns_parameter_validation():
    """set_base_parameters rejects bad inputs before touching the device
    (eqn_incompressns3d.cu:67-117)."""
    eq = ocu.Eqn_IncompressibleNS3D(ocu.F32)
    pp = ocu.Eqn_IncompressibleNS3DParams(ocu.F32)
    pp.init_grids(8, 8, 8)
    pp.hx = pp.hy = pp.hz = 0.1
    pp.temp_bc = ocu.BoundaryConditionSet(ocu.BoundaryCondition(ocu.BC_PERIODIC))
    pp.flow_bc = ocu.BoundaryConditionSet(ocu.BoundaryCondition(ocu.BC_PERIODIC))
    for field, bad in (("max_divergence", 2.0), ("cfl_factor", -1.0), ("time_step", 7),
                       ("vertical_direction", 3), ("hx", 0.0), ("viscosity", -1.0)):
        old = getattr(pp, field)
        setattr(pp, field, bad)
        with pytest.raises(ocu.OcuError) as e:
            eq.set_parameters(pp)
        assert e.value.status == _capi.ERR_INVALID_VALUE
        setattr(pp, field, old)


def test_compute_entry_points_fail_loudly_without_gpu():
    """On a machine without a B200 there is no CPU fallback: device calls raise."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    g = ocu.Grid3DDevice(ocu.F32)
    with pytest.raises(ocu.OcuError) as e:
        g.init(8, 8, 8)
    assert e.value.status in (_capi.ERR_CUDA, _capi.ERR_ALLOC)


def test_ensemble_argument_validation_without_gpu():
    """ocu_ens_create checks its arguments before touching the device."""
    lib = ocu.load()
    h = C.c_void_p()
    dims = (C.c_int * 6)(32, 32, 32, 16, 16, 16)
    sp = (C.c_double * 6)(*([1 / 32] * 3 + [1 / 16] * 3))
    assert lib.ocu_ens_create(_capi.F32, 0, dims, sp, None, C.byref(h)) == _capi.ERR_INVALID_VALUE
    bad = (C.c_int * 6)(32, 32, 32, 1, 16, 16)
    assert lib.ocu_ens_create(_capi.F32, 2, bad, sp, None, C.byref(h)) == _capi.ERR_INVALID_VALUE
    assert b"member 1" in lib.ocu_last_error()
    badh = (C.c_double * 6)(*([1 / 32] * 3 + [0.0] * 3))
    assert lib.ocu_ens_create(_capi.F32, 2, dims, badh, None, C.byref(h)) == _capi.ERR_INVALID_VALUE
    assert lib.ocu_ens_solve(None, None, 4, None) == _capi.ERR_INVALID_VALUE
    p = _capi.MGParams()
    lib.ocu_mg_params_default(C.byref(p))
    p.convergence = _capi.CONVERGENCE_LINF
    assert lib.ocu_ens_create(_capi.F32, 2, dims, sp, C.byref(p), C.byref(h)) == _capi.ERR_UNSUPPORTED
    assert not h.value


def test_adjoint_chain_argument_validation_without_gpu():
    lib = ocu.load()
    h = C.c_void_p()
    args = (_capi.F32, 16, 16, 16, 1 / 16, 1 / 16, 1 / 16)
    assert lib.ocu_adj_create(*args, 0, 2, 0.01, _capi.IT_FIRST_ORDER_UPWIND, 1e-6, C.byref(h)) == \
        _capi.ERR_INVALID_VALUE  # no steps
    assert lib.ocu_adj_create(*args, 4, 2, -0.01, _capi.IT_FIRST_ORDER_UPWIND, 1e-6, C.byref(h)) == \
        _capi.ERR_INVALID_VALUE  # negative dt
    assert lib.ocu_adj_create(*args, 4, 2, 0.01, 7, 1e-6, C.byref(h)) == _capi.ERR_INVALID_VALUE
    assert b"interpolation" in lib.ocu_last_error()
    assert lib.ocu_adj_forward(None, None, None, None, None, None) == _capi.ERR_INVALID_VALUE
    assert not h.value
