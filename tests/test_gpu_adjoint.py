"""GPU: hand-written adjoints of advection + projection, and the torch.autograd binding.

Dot-product tests pin each transposed stencil against central differences of the forward
kernels (FP64, upwind choice frozen: random velocities keep clear of zero); the chain's
gradient is checked against central finite differences of the whole chain on random
directions (FP64) and the FP32 chain's gradient against the FP64 one.  The torch binding must
give the same gradient as the chain called directly.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import opencurrent_b200 as ocu  # noqa: E402
from opencurrent_b200 import _capi  # noqa: E402
from opencurrent_b200.autograd import AdvectProject, AdvectProjectChain  # noqa: E402
from opencurrent_b200.workloads import divergence_free_velocity, gaussian_blob  # noqa: E402

pytestmark = pytest.mark.gpu

UP, CEN = _capi.IT_FIRST_ORDER_UPWIND, _capi.IT_SECOND_ORDER_CENTERED


def _mac_grids(n, dt, fill):
    """u, v, w, phi device grids (NS layouts) with interiors from fill(which), periodic ghosts."""
    lib = ocu.load()
    out = {}
    for which in "uvwt":
        L = _capi.Layout()
        _capi.check(lib.ocu_ns_init_layout(n, n, n, which.encode(), C.byref(L)))
        g = ocu.Grid3DDevice(dt)
        pad = {"u": (0, 1, 1), "v": (1, 0, 1), "w": (1, 1, 0), "t": (1, 1, 1)}[which]
        dims = {"u": (n + 1, n, n), "v": (n, n + 1, n), "w": (n, n, n + 1), "t": (n, n, n)}[which]
        g.init(*dims, 1, 1, 1, *pad)
        host = g.empty_host()
        view = np.lib.stride_tricks.as_strided(host[int(L.shift):], (n, n, n),
                                               (L.xstride * host.itemsize, L.ystride * host.itemsize, host.itemsize))
        view[...] = fill(which)
        g.copy_from_host(host)
        out[which] = g
    periodic = ocu.BoundaryConditionSet(ocu.BoundaryCondition(ocu.BC_PERIODIC))
    _capi.check(lib.ocu_apply_mac_boundary_conditions(out["u"].handle, out["v"].handle, out["w"].handle,
                                                      C.byref(periodic.to_c()), 1.0 / n, 1.0 / n, 1.0 / n, None))
    _capi.check(lib.ocu_apply_boundary_conditions(out["t"].handle, C.byref(periodic.to_c()), 1.0 / n, 1.0 / n,
                                                  1.0 / n, 0, None))
    return out


def _interior(g, n):
    L = g.layout
    host = g.copy_to_host()
    return np.lib.stride_tricks.as_strided(host[int(L.shift):], (n, n, n),
                                           (L.xstride * host.itemsize, L.ystride * host.itemsize,
                                            host.itemsize)).copy()


def _random_fields(n, seed, sign=None):
    """|velocity| >= 0.2 so the upwind choice cannot flip under the difference quotient; with
    `sign` all components share one sign (the self-advection fluxes average two velocities)."""
    rng = np.random.default_rng(seed)
    f = {}
    for which in "uvw":
        s = rng.choice([-1.0, 1.0], (n, n, n)) if sign is None else sign
        f[which] = rng.uniform(0.2, 1.0, (n, n, n)) * s
    f["t"] = rng.uniform(-1, 1, (n, n, n))
    return f


@pytest.mark.parametrize("interp", [UP, CEN])
def test_passive_advection_adjoint_dot_product(interp):
    n, h, c = 12, 1.0 / 12, 0.37
    lib = ocu.load()
    base = _random_fields(n, 1)
    rng = np.random.default_rng(2)
    dirs = {w: rng.standard_normal((n, n, n)) for w in "uvwt"}
    lam = rng.standard_normal((n, n, n))

    def forward(eps):
        g = _mac_grids(n, ocu.F64, lambda w: base[w] + eps * dirs[w])
        d = ocu.Grid3DDevice(ocu.F64)
        d.init_congruent(g["t"])
        _capi.check(lib.ocu_advect_passive(g["u"].handle, g["v"].handle, g["w"].handle, g["t"].handle, d.handle,
                                           n, n, n, h, h, h, interp, None))
        return _interior(d, n)

    eps = 1e-6
    jvp = (forward(eps) - forward(-eps)) / (2 * eps)
    g = _mac_grids(n, ocu.F64, lambda w: base[w])
    lg = _mac_grids(n, ocu.F64, lambda w: lam if w == "t" else np.zeros((n, n, n)))
    out = _mac_grids(n, ocu.F64, lambda w: np.zeros((n, n, n)))
    _capi.check(lib.ocu_advect_passive_adjoint(g["u"].handle, g["v"].handle, g["w"].handle, g["t"].handle,
                                               lg["t"].handle, out["t"].handle, out["u"].handle, out["v"].handle,
                                               out["w"].handle, n, n, n, c, h, h, h, interp, None))
    adj = {w: _interior(out[w], n) for w in "uvwt"}
    adj["t"] = adj["t"] - lam  # remove the identity part
    lhs = c * float(np.sum(lam * jvp))
    rhs = sum(float(np.sum(adj[w] * dirs[w])) for w in "uvwt")
    assert abs(lhs - rhs) <= 1e-7 * abs(lhs), (lhs, rhs)


@pytest.mark.parametrize("interp,sign", [(UP, 1.0), (UP, -1.0), (CEN, None)])
def test_self_advection_adjoint_dot_product(interp, sign):
    n, h, c = 12, 1.0 / 12, 0.29
    lib = ocu.load()
    base = _random_fields(n, 3, sign)
    rng = np.random.default_rng(4)
    dirs = {w: rng.standard_normal((n, n, n)) for w in "uvw"}
    lam = {w: rng.standard_normal((n, n, n)) for w in "uvw"}

    def forward(eps):
        g = _mac_grids(n, ocu.F64, lambda w: base[w] + (eps * dirs[w] if w in dirs else 0))
        d = {w: ocu.Grid3DDevice(ocu.F64) for w in "uvw"}
        for w in "uvw":
            d[w].init_congruent(g[w])
        _capi.check(lib.ocu_advect_self(g["u"].handle, g["v"].handle, g["w"].handle, d["u"].handle, d["v"].handle,
                                        d["w"].handle, n, n, n, h, h, h, interp, None))
        return {w: _interior(d[w], n) for w in "uvw"}

    eps = 1e-6
    fp, fm = forward(eps), forward(-eps)
    jvp = {w: (fp[w] - fm[w]) / (2 * eps) for w in "uvw"}
    g = _mac_grids(n, ocu.F64, lambda w: base[w])
    lg = _mac_grids(n, ocu.F64, lambda w: lam[w] if w in lam else np.zeros((n, n, n)))
    out = _mac_grids(n, ocu.F64, lambda w: np.zeros((n, n, n)))
    _capi.check(lib.ocu_advect_self_adjoint(g["u"].handle, g["v"].handle, g["w"].handle, lg["u"].handle,
                                            lg["v"].handle, lg["w"].handle, out["u"].handle, out["v"].handle,
                                            out["w"].handle, n, n, n, c, h, h, h, interp, None))
    lhs = c * sum(float(np.sum(lam[w] * jvp[w])) for w in "uvw")
    rhs = sum(float(np.sum(_interior(out[w], n) * dirs[w])) for w in "uvw")
    assert abs(lhs - rhs) <= 1e-7 * abs(lhs), (lhs, rhs)


def _flow_inputs(chain, n, seed=5):
    u, v, w = divergence_free_velocity(n, seed=seed, kmax=4)
    phi = gaussian_blob(n, (0.4, 0.55, 0.5), 0.15)
    ts = []
    for which, x in zip("uvwt", (u, v, w, phi)):
        t = chain.empty(which)
        chain.interior(t, which).copy_(torch.from_numpy(x).to(t.dtype))
        ts.append(t)
    target = chain.empty("t")
    chain.interior(target, "t").copy_(torch.from_numpy(gaussian_blob(n, (0.6, 0.45, 0.5), 0.15)).to(target.dtype))
    return ts, target


def _loss(chain, ins, target):
    out = chain.forward(*ins)
    d = chain.interior(out, "t") - chain.interior(target, "t")
    return 0.5 * float((d.double() ** 2).sum()), out


@pytest.mark.parametrize("steps,every,interp,tol", [(6, 2, UP, 1e-4), (7, 3, UP, 1e-4), (5, 5, CEN, 1e-6)])
def test_chain_gradient_matches_finite_differences_fp64(steps, every, interp, tol):
    """The upwind chain is piecewise smooth (continuous fluxes, kinks where a velocity changes
    sign), so its difference quotients carry a small kink error; the centred chain is smooth."""
    n = 16
    chain = AdvectProjectChain((n, n, n), (1 / n,) * 3, steps, dt=0.25 / n, checkpoint_every=every,
                               dtype=_capi.F64, interp=interp, proj_tol=1e-12)
    ins, target = _flow_inputs(chain, n)
    loss, out = _loss(chain, ins, target)
    lam = out - target
    lam_i = chain.empty("t")
    chain.interior(lam_i, "t").copy_(chain.interior(lam, "t"))
    grads = chain.backward(lam_i)
    rng = np.random.default_rng(7)
    worst = 0.0
    for _ in range(4):
        dirs = []
        for which in "uvwt":
            d = chain.empty(which)
            chain.interior(d, which).copy_(torch.from_numpy(rng.standard_normal((n, n, n))))
            dirs.append(d)
        eps = 1e-5
        lp, _ = _loss(chain, [x + eps * d for x, d in zip(ins, dirs)], target)
        lm, _ = _loss(chain, [x - eps * d for x, d in zip(ins, dirs)], target)
        fd = (lp - lm) / (2 * eps)
        ad = sum(float((g * d).sum()) for g, d in zip(grads, dirs))
        worst = max(worst, abs(fd - ad) / max(abs(fd), 1e-30))
    assert worst < tol, worst


def test_fp32_gradient_close_to_fp64_gradient():
    n, steps = 16, 6
    grads = {}
    for dt in (_capi.F32, _capi.F64):
        chain = AdvectProjectChain((n, n, n), (1 / n,) * 3, steps, dt=0.25 / n, checkpoint_every=3, dtype=dt,
                                   proj_tol=1e-6 if dt == _capi.F32 else 1e-12)
        ins, target = _flow_inputs(chain, n)
        out = chain.forward(*ins)
        lam = chain.empty("t")
        chain.interior(lam, "t").copy_(chain.interior(out - target, "t"))
        grads[dt] = [g.double().cpu() for g in chain.backward(lam)]
    num = sum(float(((a - b) ** 2).sum()) for a, b in zip(grads[_capi.F32], grads[_capi.F64]))
    den = sum(float((b ** 2).sum()) for b in grads[_capi.F64])
    rel = (num / den) ** 0.5
    assert rel < 5e-3, rel


def test_autograd_function_matches_direct_backward():
    n, steps = 16, 4
    chain = AdvectProjectChain((n, n, n), (1 / n,) * 3, steps, dt=0.25 / n, checkpoint_every=2, dtype=_capi.F64,
                               proj_tol=1e-12)
    ins, target = _flow_inputs(chain, n)
    leaves = [x.clone().requires_grad_(True) for x in ins]
    out = AdvectProject.apply(*leaves, chain)
    d = chain.interior(out, "t") - chain.interior(target, "t")
    loss = 0.5 * (d ** 2).sum()
    loss.backward()
    lam = chain.empty("t")
    chain.interior(lam, "t").copy_(d.detach())
    chain.forward(*ins)
    direct = chain.backward(lam)
    for leaf, g in zip(leaves, direct):
        assert torch.equal(leaf.grad, g)


def test_chain_rejects_foreign_layouts():
    n = 8
    chain = AdvectProjectChain((n, n, n), (1 / n,) * 3, 2, dt=0.01, checkpoint_every=1, dtype=_capi.F32)
    u = chain.empty("u")
    bad = torch.zeros(10, dtype=torch.float32, device="cuda")
    with pytest.raises(AssertionError):
        chain.forward(u, chain.empty("v"), chain.empty("w"), bad)
