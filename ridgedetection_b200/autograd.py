"""Evolve adjoint: C-ABI wrapper and a torch.autograd.Function for validation.

``evolve_adjoint`` calls ``rd_evolve_adjoint`` (no reference counterpart): a
forward of `iters` evolve passes without the movement test (each non-empty
cluster moves to the FP32 mean of its members, empty clusters keep their
point, decimation frozen) and the FP64 reverse pass of L = sum_k <W_k, S_k>
with the assignments frozen.

``EvolveFunction`` makes the final chosen points a differentiable function of
the cloud: S_final = F(P), with S0 = P[chosen_idx] (copies of cloud points, as
choose produces them), so dL/dP gets both the cluster-mean path and the path
through S0 of clusters that stayed empty.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L


def evolve_adjoint(P, S0, r1: float, iters: int, W, checkpoint_every: int = 0):
    """Host arrays in, host arrays out: (S_final f32, grad_P f64, grad_S0 f64)."""
    P = np.ascontiguousarray(P, dtype=np.float32)
    S0 = np.ascontiguousarray(S0, dtype=np.float32)
    W = np.ascontiguousarray(W, dtype=np.float64)
    n, dim = P.shape
    ns = S0.shape[0]
    if W.shape != S0.shape:
        raise ValueError("W must have the shape of S0")
    Sf = np.empty_like(S0)
    gP = np.empty((n, dim), np.float64)
    gS = np.empty((ns, dim), np.float64)
    vp = ctypes.c_void_p
    L.check(L.lib().rd_evolve_adjoint(dim, vp(P.ctypes.data), n, vp(S0.ctypes.data), ns,
                                      float(r1), int(iters), int(checkpoint_every),
                                      vp(W.ctypes.data), vp(Sf.ctypes.data), vp(gP.ctypes.data),
                                      vp(gS.ctypes.data), 0, vp(0)))
    return Sf, gP, gS


def evolve_adjoint_device(P, S0, r1: float, iters: int, W, checkpoint_every: int = 0):
    """CUDA tensors in (P f32 [n,dim], S0 f32 [ns,dim], W f64 [ns,dim]);
    returns (S_final, grad_P, grad_S0) as CUDA tensors."""
    import torch
    n, dim = P.shape
    ns = S0.shape[0]
    P, S0, W = P.contiguous(), S0.contiguous(), W.contiguous().to(torch.float64)
    Sf = torch.empty_like(S0)
    gP = torch.empty((n, dim), dtype=torch.float64, device=P.device)
    gS = torch.empty((ns, dim), dtype=torch.float64, device=P.device)
    vp = ctypes.c_void_p
    st = vp(torch.cuda.current_stream(P.device).cuda_stream)
    L.check(L.lib().rd_evolve_adjoint(dim, vp(P.data_ptr()), n, vp(S0.data_ptr()), ns,
                                      float(r1), int(iters), int(checkpoint_every),
                                      vp(W.data_ptr()), vp(Sf.data_ptr()), vp(gP.data_ptr()),
                                      vp(gS.data_ptr()), 1, st))
    return Sf, gP, gS


def _autograd_function():
    import torch

    class EvolveFunction(torch.autograd.Function):
        """S_final = evolve^iters(P, S0 = P[chosen_idx]) on the GPU."""

        @staticmethod
        def forward(ctx, P, chosen_idx, r1, iters, checkpoint_every=0):
            S0 = P.detach()[chosen_idx].contiguous()
            W0 = torch.zeros(S0.shape, dtype=torch.float64, device=P.device)
            Sf, _, _ = evolve_adjoint_device(P.detach(), S0, r1, iters, W0, checkpoint_every)
            ctx.save_for_backward(P.detach(), chosen_idx)
            ctx.r1, ctx.iters, ctx.ckpt = r1, iters, checkpoint_every
            return Sf

        @staticmethod
        def backward(ctx, grad_out):
            P, chosen_idx = ctx.saved_tensors
            S0 = P[chosen_idx].contiguous()
            _, gP, gS = evolve_adjoint_device(P, S0, ctx.r1, ctx.iters,
                                              grad_out.to(torch.float64), ctx.ckpt)
            gP = gP.index_add(0, chosen_idx, gS)
            return gP.to(P.dtype), None, None, None, None

    return EvolveFunction


def evolve_function():
    """The torch.autograd.Function class (torch imported lazily)."""
    return _autograd_function()
