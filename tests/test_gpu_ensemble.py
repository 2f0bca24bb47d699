"""GPU: ensembles of independent pressure solves (ocu_ens_*).

Every member of a batched solve must be bit-identical -- pressure (ghosts included), cycle count
and final L2 residual -- to the oracle's single solve of that member with the same parameters
(sol_mgpressure3d.cpp:332-370 per member).  Uneven sizes, several size classes, BC mixes, the
symmetric operator, the device coarse relaxation, members that converge before any cycle, and
the autotuner's chosen settings are covered.
"""
import numpy as np
import pytest

import opencurrent_b200 as ocu
from oracle import oracle_ctypes as O
from tests.helpers import F32, F64, SCALAR_BCS, bc_from, mg_params, npdt
from tests.test_gpu_parity import assert_same, to_ocu_bc

pytestmark = pytest.mark.gpu


def _members(dt, dims, seed0, zero=()):
    """Per member: layout, padded rhs (uniform[-1,1], FP64 mean removed, cast) and its RMS."""
    out = []
    for m, d in enumerate(dims):
        L = O.layout(*d)
        rhs = np.zeros(int(L.allocated), npdt(dt))
        if m in zero:
            b = np.zeros(d)
        else:
            b = np.random.default_rng(seed0 + m).uniform(-1, 1, d)
            b -= b.mean()
        O.interior(rhs, L)[:] = b.astype(npdt(dt))
        rms = float(np.sqrt(np.mean(b ** 2)))
        out.append((L, rhs, rms))
    return out


def _check(dt, dims, bcname="neumann", sym=0, disable_host=0, nu=(2, 2), rel=1e-6, zero=(), max_iter=20,
           tune=None, seed0=1000):
    bc = bc_from(SCALAR_BCS[bcname])
    h = [(1.0 / d[0], 1.0 / d[1], 1.0 / d[2]) for d in dims]
    ens = ocu.PressureEnsemble(dt, dims, h, bc=to_ocu_bc(bc), nu1=nu[0], nu2=nu[1],
                               make_symmetric_operator=sym, disable_relax_on_host=disable_host)
    mem = _members(dt, dims, seed0, zero)
    tols = []
    for m, (L, rhs, rms) in enumerate(mem):
        ens.rhs(m).copy_from_host(rhs)
        tols.append(rel * rms if rms > 0 else 1e-8)
    if tune is not None:
        tune(ens, tols)
    classes = {c["dims"]: c for c in ens.classes()}
    conv = ens.solve(tols, max_iter)
    assert conv == len(dims)
    for m, (L, rhs, rms) in enumerate(mem):
        c = classes[tuple(dims[m])]
        om = O.OracleMG("d" if dt == F64 else "f",
                        mg_params(bc, nu1=c["nu1"], nu2=c["nu2"], sym=sym, disable_host=disable_host),
                        *dims[m], *h[m], rhs, L)
        ok, res = om.solve(tols[m], max_iter)
        assert ok, m
        st = ens.member_stats(m)
        assert st.vcycles == om.vcycles, (m, st.vcycles, om.vcycles)
        assert st.last_l2 == res, (m, st.last_l2, res)
        assert_same(ens.pressure(m).copy_to_host(), om.grid("u", 0)[0], f"member {m} {dims[m]}")
    return ens


def test_uneven_sizes_fp32_match_single_solves():
    dims = [(32, 32, 32), (48, 48, 48), (32, 32, 32), (16, 16, 16), (32, 16, 48), (48, 48, 48), (24, 24, 24)]
    ens = _check(F32, dims)
    cl = ens.classes()
    assert sorted(c["members"] for c in cl) == [1, 1, 1, 2, 2]
    # largest class first
    assert cl[0]["dims"] == (48, 48, 48)


def test_second_solve_from_converged_state():
    """A second solve starts from the converged pressures (the reference keeps the initial guess)."""
    dims = [(32, 32, 32), (16, 16, 16)]
    ens = _check(F32, dims, rel=1e-3)
    bc = bc_from(SCALAR_BCS["neumann"])
    mem = _members(F32, dims, 1000)
    tols = [1e-6 * rms for (_, _, rms) in mem]
    assert ens.solve(tols, 20) == 2
    for m, d in enumerate(dims):
        L, rhs, _ = mem[m]
        om = O.OracleMG("f", mg_params(bc), *d, 1.0 / d[0], 1.0 / d[1], 1.0 / d[2], rhs, L)
        om.solve(1e-3 * mem[m][2], 20)
        ok, res = om.solve(tols[m], 20)
        assert ok and ens.member_stats(m).last_l2 == res
        assert_same(ens.pressure(m).copy_to_host(), om.grid("u", 0)[0], f"second solve member {m}")


@pytest.mark.parametrize("bcname,sym,disable_host", [("mixed_dn", 1, 0), ("dirichlet", 0, 1), ("periodic", 0, 0),
                                                     ("mixed_xdir", 1, 1)])
def test_bc_and_operator_variants_fp64(bcname, sym, disable_host):
    dims = [(32, 32, 32), (16, 32, 16), (32, 32, 32), (24, 24, 24)]
    _check(F64, dims, bcname=bcname, sym=sym, disable_host=disable_host, rel=1e-10, max_iter=30)


def test_members_converged_before_any_cycle():
    """A zero right-hand side meets its tolerance at the initial check: no cycle runs for it."""
    dims = [(32, 32, 32), (32, 32, 32), (16, 16, 16)]
    ens = _check(F32, dims, zero=(1,))
    assert ens.member_stats(1).vcycles == 0
    assert ens.member_stats(0).vcycles > 0


@pytest.mark.parametrize("nu", [(1, 1), (3, 2)])
def test_smoothing_counts(nu):
    _check(F32, [(32, 32, 32), (48, 48, 48), (16, 16, 16)], nu=nu)


def test_autotuned_settings_still_match_single_solves():
    def tune(ens, tols):
        ens.autotune(tols, 20)
        for c in ens.classes():
            assert c["ms"] > 0 and c["nu1"] >= 1
            bx, by, bz = c["relax_block"]
            assert bx * by * bz <= 256
    _check(F32, [(32, 32, 32), (48, 48, 48), (32, 32, 32), (16, 16, 16)], tune=tune)


def test_set_tuning_block_shape_only_changes_speed():
    def tune(ens, tols):
        for c in range(len(ens.classes())):
            ens.set_tuning(c, 2, 2, (16, 8, 2))
    _check(F32, [(32, 32, 32), (48, 48, 48)], tune=tune)


def test_rejects_unsupported_configurations():
    none = bc_from(SCALAR_BCS["mixed_all"])  # has a BC_NONE face
    with pytest.raises(ocu.OcuError):
        ocu.PressureEnsemble(F32, [(32, 32, 32)], [(1 / 32,) * 3], bc=to_ocu_bc(none))
    with pytest.raises(ocu.OcuError):
        ocu.PressureEnsemble(F32, [(6, 6, 6)], [(1 / 6,) * 3])  # a single multigrid level
