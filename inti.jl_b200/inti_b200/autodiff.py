"""Reverse-mode rules for the operator product u = A σ.

Inti.jl differentiates only in forward mode (ForwardDiff through the element
maps, src/reference_interpolation.jl:36-39; the kernel derivative pattern of
test/kernels_test.jl:41-67).  This module gives the reverse rule of the
product, the Python counterpart of the ChainRules ``rrule`` of the Julia
binding (julia/IntiB200.jl): ``rrule(A, σ)`` returns ``u`` and a pullback
that maps the cotangent ``ū = ∂J/∂u`` to the cotangents of σ and of the
source quadrature (node coordinates, normals, weights).

* ∂J/∂σ is ``Aᴴ ū``: the transpose apply (``inti_op_apply_transpose``,
  correction rows included), conjugated for complex operators.
* The source-geometry cotangents come from the hand-written adjoint kernel
  (``inti_op_grad_sources``), which recomputes the kernel tiles instead of
  storing the M×N operator.  They cover the on-the-fly pair terms of the
  Laplace single and double layer: the off-surface potentials (no
  correction) are differentiated exactly.  A DIM correction is a constant
  of the rule: its dependence on the geometry (the least-squares weights of
  src/bdim.jl:154-185) is not differentiated, so operators carrying one
  report the geometry cotangents of their pair part only, and say so in the
  pullback's ``"geometry"`` entry.
* ``TorchPotential`` wraps the same rule as a ``torch.autograd.Function``
  over host or device tensors (σ, coordinates, normals, weights), rebuilding
  the operator from the given geometry in its forward pass.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .core import DoubleLayerKernel, GpuOperator, Laplace, SingleLayerKernel


def rrule(A: GpuOperator, sigma):
    """``(u, pullback)`` for ``u = A @ sigma``.

    ``pullback(ubar)`` returns a dict with ``"sigma"`` (∂J/∂σ), and, for the
    Laplace single and double layer, ``"coords"``, ``"normals"`` and
    ``"weights"`` of the source quadrature (``(n, dim)``, ``(n, dim)``,
    ``(n,)``); other kernels give ``None`` there.  ``"geometry"`` names what
    the geometry cotangents cover.
    """
    sigma = np.asarray(sigma)
    u = A @ sigma
    geometric = (not A.is_complex and A.kernel.op.pde == L.LAPLACE
                 and isinstance(A.kernel, (SingleLayerKernel, DoubleLayerKernel)) and A.precision == "fp64")

    def pullback(ubar):
        ubar = np.asarray(ubar)
        if ubar.shape != u.shape:
            raise L.DimensionMismatch(L.E_SHAPE, f"cotangent has shape {ubar.shape}, expected {u.shape}")
        out = {"coords": None, "normals": None, "weights": None}
        if A.is_complex:
            # conjugate transpose: Aᴴ ū = conj(Aᵀ conj(ū))
            out["sigma"] = np.conj(A.rmatvec(np.conj(ubar)))
            out["geometry"] = "not differentiated (Laplace single and double layer only)"
            return out
        if not geometric:
            out["sigma"] = A.rmatvec(ubar)
            out["geometry"] = "not differentiated (Laplace single and double layer only)"
            return out
        g = A.grad_sources(np.ascontiguousarray(ubar, dtype=np.float64), sigma)
        if A.correction is not None:
            # (A + C)ᵀ ū: the transpose apply carries the correction rows
            out["sigma"] = A.rmatvec(ubar)
            out["geometry"] = "pair terms only (the DIM correction is held constant)"
        else:
            out["sigma"] = g["sigma"]
            out["geometry"] = "exact"
        out["coords"], out["normals"], out["weights"] = g["coords"], g["normals"], g["weights"]
        return out

    return u, pullback


def _torch_function():
    import torch

    from .geometry import Quadrature

    class _Potential(torch.autograd.Function):
        @staticmethod
        def forward(fctx, sigma, coords, normals, weights, targets, kind, ctx):
            src = Quadrature(coords.detach().cpu().double().numpy(), normals.detach().cpu().double().numpy(),
                             weights.detach().cpu().double().numpy(), 0)
            from .geometry import points

            tgt = points(targets.detach().cpu().double().numpy())
            K = DoubleLayerKernel if kind == "DL" else SingleLayerKernel
            A = GpuOperator(K(Laplace(dim=src.dim)), tgt, src, None, "fp64", ctx)
            u, pb = rrule(A, sigma.detach().cpu().double().numpy())
            fctx.pullback = pb
            fctx.devs = (sigma.device, coords.device, normals.device, weights.device)
            return torch.from_numpy(u).to(sigma.device)

        @staticmethod
        def backward(fctx, ubar):
            g = fctx.pullback(ubar.detach().cpu().double().numpy())
            ds, dc, dn, dw = fctx.devs
            return (torch.from_numpy(g["sigma"]).to(ds), torch.from_numpy(g["coords"]).to(dc),
                    torch.from_numpy(g["normals"]).to(dn), torch.from_numpy(g["weights"]).to(dw),
                    None, None, None)

    return _Potential


_TORCH_FN = None


def TorchPotential(sigma, coords, normals, weights, targets, kind: str = "DL", ctx=None):
    """Laplace layer potential ``u(x_t) = Σ_j K(x_t, y_j) w_j σ_j`` at
    ``targets`` as a differentiable torch operation of σ and the source
    quadrature (coordinates ``(n, dim)``, normals ``(n, dim)``, weights
    ``(n,)``): its backward pass is the hand-written adjoint kernel."""
    global _TORCH_FN
    if kind not in ("SL", "DL"):
        raise L.ArgumentError(L.E_ARG, f"unknown potential kind {kind!r}")
    if _TORCH_FN is None:
        _TORCH_FN = _torch_function()
    return _TORCH_FN.apply(sigma, coords, normals, weights, targets, kind, ctx)
