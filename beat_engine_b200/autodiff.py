"""Reverse-mode differentiation of the far field through the library's adjoint.

``FarFieldSolve`` is a ``torch.autograd.Function`` (the Python counterpart of
the ``ChainRulesCore.rrule`` a Julia caller puts over the same entry points):

    p_inf = farfield_solve(ctx, faces, k_signed, eta, dirs, q0, a, vertices)

forward: (optionally) ``beat_b200_set_mesh`` with ``vertices``,
``beat_b200_set_admittance`` with ``a``, one ``beat_b200_solve`` with the
cached right-hand-side mapping and ``beat_b200_farfield``; backward: one
``beat_b200_adjoint`` (or ``beat_b200_adjoint_shape`` when the vertices need a
gradient), which reuses the forward solve's LU factors.

Gradient convention.  For a real loss L, torch stores the gradient of a
complex tensor z as 2 dL/d conj(z) and of a real tensor as dL/dz.  The
library's adjoint takes g = dJ/d conj(p_inf) and returns dJ/d conj(q0),
dJ/d conj(a) and dJ/dX, each linear in g.  So torch's grad_output (= 2 g) goes
in as it is: the complex outputs come back in torch's convention, and the real
vertex gradient is halved.

The forward solve leaves its factors on the context.  If any other library
call ran on the same context before ``backward`` (another forward call, a
solve, a field evaluation), backward solves the forward problem again first,
so the adjoint always uses the factors of the operator it differentiates.

The reference has no adjoint (its exterior path has no admittance or gradient
at all); the gradients are pinned by central differences of the forward solve
in ``tests/test_autodiff.py``.
"""
from __future__ import annotations

import numpy as np

from . import _lib


def _numpy(t):
    return t.detach().cpu().numpy()


def _forward(ctx, faces, k_signed, eta, dirs, q0, a, vertices, opts):
    if vertices is not None:
        ctx.set_mesh(vertices, faces, ctx.quad_order, ctx.singular_order)
    ctx.set_admittance(a)
    p, _ = ctx.solve(k_signed, eta, q0, opts)
    pinf = ctx.farfield(k_signed, dirs, p, q0)
    return p, pinf


def _function():
    import torch

    class FarFieldSolve(torch.autograd.Function):
        @staticmethod
        def forward(fctx, ctx, faces, k_signed, eta, dirs, precision, q0, a, vertices):
            opts = _lib.Context.opts(precision, flags=_lib.FLAG_RHS_CACHED)
            qn = np.asfortranarray(_numpy(q0).astype(np.complex128))
            an = None if a is None else _numpy(a).astype(np.complex128)
            xn = None if vertices is None else _numpy(vertices).astype(np.float64)
            p, pinf = _forward(ctx, faces, k_signed, eta, dirs, qn, an, xn, opts)
            fctx.state = (ctx, faces, k_signed, eta, np.asarray(dirs, np.float64), opts, qn, an, xn, p,
                          ctx.generation)
            fctx.has_a, fctx.has_x = a is not None, vertices is not None
            return torch.from_numpy(np.ascontiguousarray(pinf)).to(q0.device)

        @staticmethod
        def backward(fctx, grad):
            ctx, faces, k_signed, eta, dirs, opts, qn, an, xn, p, token = fctx.state
            if ctx.generation != token:  # another library call ran since: re-make this solve's factors
                p, _ = _forward(ctx, faces, k_signed, eta, dirs, qn, an, xn, opts)
            g = np.asfortranarray(_numpy(grad).astype(np.complex128))
            gx = None
            # needs_input_grad follows forward's inputs: ctx, faces, k, eta, dirs, precision, q0 (6), a (7),
            # vertices (8)
            if fctx.has_x and fctx.needs_input_grad[8]:
                w, ga, gx = ctx.adjoint_shape(k_signed, dirs, p, qn, g, opts)
                gx = 0.5 * gx  # real input: dL/dX, not 2 dL/dX
            else:
                w, ga = ctx.adjoint(k_signed, dirs, p, g, opts, want_admittance=fctx.has_a)
            dev = grad.device
            gq = torch.from_numpy(np.ascontiguousarray(w)).to(dev) if fctx.needs_input_grad[6] else None
            gan = torch.from_numpy(np.ascontiguousarray(ga)).to(dev) if (fctx.has_a and fctx.needs_input_grad[7]) \
                else None
            gxt = torch.from_numpy(np.ascontiguousarray(gx)).to(dev) if gx is not None else None
            return None, None, None, None, None, None, gq, gan, gxt

    return FarFieldSolve


_FN = None


def farfield_solve(ctx, faces, k_signed, eta, dirs, q0, a=None, vertices=None, precision=_lib.FP64):
    """Far field (M x R complex128 tensor) of the exterior solve with Neumann
    data ``q0`` (F x R complex128 tensor), per-face admittance coefficients
    ``a`` (F complex128 tensor, or None) and vertex positions ``vertices``
    (V x 3 float64 tensor, or None to keep the context's mesh), differentiable
    with respect to all three.  ``faces`` are the mesh's 0-based faces (used
    when ``vertices`` is given)."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(ctx, faces, float(k_signed), float(eta), dirs, int(precision), q0, a, vertices)
