"""CPU: the host-side decomposition of the multi-image multigrid solver (ocu_mgco_plan_compute),
against the rules of Sol_MultigridPressure3DDeviceCo::initialize_storage
(sol_mgpressure3dco.cu:262-300 cutoff and neighbours, 420-435 faces), restated here."""
import pytest

import opencurrent_b200 as ocu
from opencurrent_b200 import _capi

NEU, DIR, PER, NONE = ocu.BC_NEUMANN, ocu.BC_DIRICHELET, ocu.BC_PERIODIC, ocu.BC_NONE
FACES = ("xpos", "xneg", "ypos", "yneg", "zpos", "zneg")


def num_levels(nx, ny, nz):
    # Sol_MultigridPressure3DBase::num_levels (sol_mgpressure3d.cpp:67-92)
    c = [nx // 2, ny // 2, nz // 2]
    n = [nx, ny, nz]
    levels = 0
    while all(2 * c[a] == n[a] for a in range(3)):
        levels += 1
        n = list(c)
        c = [v // 2 for v in c]
        if any(c[a] < 2 or n[a] in (5, 7) for a in range(3)):
            break
    return levels


def expected(nxl, ny, nz, N, image, cells, faces):
    L = num_levels(nxl * N, ny, nz)
    cutoff = L
    d = [nxl * N, ny, nz]
    for lev in range(1, L):
        d = [v // 2 for v in d]
        if d[0] * d[1] * d[2] <= cells:
            cutoff = lev
            break
    neg = (image - 1 + N) % N
    pos = (image + 1) % N
    if image == 0 and faces["xneg"] != PER:
        neg = -1
    if image == N - 1 and faces["xpos"] != PER:
        pos = -1
    local = dict(faces)
    if neg != -1:
        local["xneg"] = NONE
    if pos != -1:
        local["xpos"] = NONE
    return {"num_levels": L, "cutoff_level": cutoff, "neg_image": neg, "pos_image": pos, "local_bc": local}


FACE_SETS = {
    "neumann": dict.fromkeys(FACES, NEU),
    "periodic": dict.fromkeys(FACES, PER),
    "x_dirichlet_rest_periodic": {"xpos": DIR, "xneg": DIR, "ypos": PER, "yneg": PER, "zpos": PER, "zneg": PER},
    "mixed": {"xpos": DIR, "xneg": NEU, "ypos": NEU, "yneg": DIR, "zpos": NONE, "zneg": DIR},
}


@pytest.mark.parametrize("name", sorted(FACE_SETS))
@pytest.mark.parametrize("dims,N,cells", [((128, 256, 256), 2, 64 ** 3), ((16, 64, 64), 4, 64 ** 3),
                                          ((32, 32, 32), 1, 512), ((8, 48, 40), 8, 1000),
                                          ((40, 40, 20), 2, 4000), ((64, 32, 32), 3, 1)])
def test_plan_matches_reference_rules(name, dims, N, cells):
    faces = FACE_SETS[name]
    bc = ocu.BoundaryConditionSet()
    for f, t in faces.items():
        setattr(bc, f, ocu.BoundaryCondition(t, 0.0))
    for image in range(N):
        got = ocu.mgco_plan(*dims, N, image, bc, cells)
        assert got == expected(*dims, N, image, cells, faces), (name, dims, N, image)


def test_plan_argument_errors():
    bc = ocu.BoundaryConditionSet(ocu.BoundaryCondition(NEU, 0.0))
    for args in [(0, 8, 8, 2, 0), (8, 8, 8, 0, 0), (8, 8, 8, 2, 2), (8, 8, 8, 2, -1)]:
        with pytest.raises(ocu.OcuError):
            ocu.mgco_plan(*args, bc)
    with pytest.raises(ocu.OcuError):
        ocu.mgco_plan(8, 8, 8, 2, 0, bc, cutoff_cells=0)


def test_create_refuses_other_kinds_and_counts():
    lib = ocu.load()
    import ctypes as C
    h = C.c_void_p()
    p = _capi.MGParams()
    lib.ocu_mg_params_default(C.byref(p))
    assert lib.ocu_mgco_create(_capi.MG_MIXED_IR, C.byref(p), 2, None, C.byref(h)) != 0
    assert lib.ocu_mgco_create(_capi.MG_F64, C.byref(p), 0, None, C.byref(h)) != 0
    # a handle is created without touching a device; the cutoff is set before initialization
    assert lib.ocu_mgco_create(_capi.MG_F64, C.byref(p), 2, None, C.byref(h)) == 0
    assert lib.ocu_mgco_num_images(h) == 2
    assert lib.ocu_mgco_cutoff_level(h) == -1
    assert lib.ocu_mgco_set_cutoff_cells(h, 0) != 0
    assert lib.ocu_mgco_set_cutoff_cells(h, 4096) == 0
    assert lib.ocu_mgco_pressure(h, 0) is None
    lib.ocu_mg_destroy(h)
