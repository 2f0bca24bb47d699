"""torch.autograd binding of the differentiable advection + projection chain (ocu_adj_*).

The chain runs `steps` forward-Euler steps of passive-scalar advection, velocity self-advection
and projection on a periodic MAC grid; its backward pass is the library's hand-written adjoint
(transposed upwind stencils, the self-adjoint projection reused), checkpointed every
`checkpoint_every` steps.  Tensors are flat CUDA tensors in the library's padded grid layout
(`AdvectProjectChain.empty`); `AdvectProjectChain.interior` gives the (nx, ny, nz)-shaped view.
"""
import ctypes as C

import torch

from . import _capi
from ._capi import Layout, check, load

_TORCH = {_capi.F32: torch.float32, _capi.F64: torch.float64}


class AdvectProjectChain:
    def __init__(self, n, h, steps, dt, checkpoint_every=8, dtype=_capi.F32,
                 interp=_capi.IT_FIRST_ORDER_UPWIND, proj_tol=1e-6):
        lib = load()
        self.n = tuple(int(x) for x in n)
        self.dtype = dtype
        handle = C.c_void_p()
        check(lib.ocu_adj_create(dtype, *self.n, *[float(x) for x in h], int(steps), int(checkpoint_every),
                                 float(dt), int(interp), float(proj_tol), C.byref(handle)))
        self._h = handle.value
        self.layouts = {}
        for w in "uvwt":
            L = Layout()
            check(lib.ocu_adj_layout(self._h, w.encode(), C.byref(L)))
            self.layouts[w] = L

    def empty(self, which="t"):
        """Zeroed flat CUDA tensor in the layout of grid `which` ('u', 'v', 'w' or 't')."""
        return torch.zeros(int(self.layouts[which].allocated), dtype=_TORCH[self.dtype], device="cuda")

    def interior(self, t, which="t"):
        """(nx, ny, nz) view of the cells (or faces [0, n)) of a flat layout tensor."""
        L = self.layouts[which]
        return t.as_strided(self.n, (L.xstride, L.ystride, 1), int(L.shift))

    def _wrap(self, t, which):
        assert t.is_cuda and t.dtype == _TORCH[self.dtype] and t.is_contiguous()
        assert t.numel() == self.layouts[which].allocated
        g = C.c_void_p()
        L = self.layouts[which]
        check(load().ocu_grid_wrap(self.dtype, C.byref(L), C.c_void_p(t.data_ptr()), C.byref(g)))
        return g.value

    def _call(self, fn, tensors):
        lib = load()
        check(lib.ocu_adj_set_stream(self._h, C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        handles = [self._wrap(t, w) for t, w in tensors]
        try:
            check(fn(self._h, *handles))
        finally:
            for g in handles:
                lib.ocu_grid_destroy(g)

    def forward(self, u0, v0, w0, phi0):
        out = self.empty("t")
        self._call(load().ocu_adj_forward, [(u0, "u"), (v0, "v"), (w0, "w"), (phi0, "t"), (out, "t")])
        return out

    def backward(self, lam_phi):
        outs = [self.empty(w) for w in "uvwt"]
        self._call(load().ocu_adj_backward, [(lam_phi.contiguous(), "t")] + list(zip(outs, "uvwt")))
        return tuple(outs)

    def __del__(self):
        try:
            if self._h:
                load().ocu_adj_destroy(self._h)
                self._h = None
        except Exception:
            pass


class AdvectProject(torch.autograd.Function):
    """phi_final = chain(u0, v0, w0, phi0); gradients from the hand-written adjoint."""

    @staticmethod
    def forward(ctx, u0, v0, w0, phi0, chain):
        ctx.chain = chain
        return chain.forward(u0.contiguous(), v0.contiguous(), w0.contiguous(), phi0.contiguous())

    @staticmethod
    def backward(ctx, grad_phi):
        lu, lv, lw, lphi = ctx.chain.backward(grad_phi)
        return lu, lv, lw, lphi, None
