"""Differentiable personalised PageRank on the GPU (torch.autograd.Function over
the C ABI's mg_ppr_forward / mg_ppr_backward).

    R = ppr(graph, edge_weights, teleport)          # R: [V, nvec], float32, CUDA
    R = (1 - d) * teleport + d * P^T R,   P[u, v] = edge_weights[e(u, v)]

edge_weights holds one FP32 weight per CSR edge of the graph (row-normalise
them first, e.g. with torch ops, if P must be stochastic; gradients flow
through that normalisation by ordinary autograd). The forward pass saves only
the converged rank matrix; the backward pass solves the adjoint system
lambda = dL/dR + d P lambda by power iteration over the out-edges and returns
dL/dedge_weights[e(u,v)] = d <lambda[v,:], R[u,:]> and dL/dteleport = (1-d) lambda.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import check, default_options, lib


class _PPR(torch.autograd.Function):
    @staticmethod
    def forward(ctx, edge_weights, teleport, graph, damping, tol, max_iter, extra):
        w = edge_weights.detach().contiguous()
        t = teleport.detach().contiguous()
        if w.dtype != torch.float32 or t.dtype != torch.float32 or not w.is_cuda or not t.is_cuda:
            raise TypeError("edge_weights and teleport must be float32 CUDA tensors")
        if w.numel() != graph.edges or t.dim() != 2 or t.shape[0] != graph.nodes:
            raise ValueError("edge_weights must be [E], teleport [V, nvec]")
        nvec = int(t.shape[1])
        out = torch.empty_like(t)
        o = default_options(damping=damping, tolerance=tol, iter_num=max_iter,
                            stream=torch.cuda.current_stream().cuda_stream, **extra)
        st = _lib.Stats()
        check(lib.mg_ppr_forward(graph.handle, w.data_ptr(), t.data_ptr(), nvec, out.data_ptr(), C.byref(st),
                                 C.byref(o)), "mg_ppr_forward")
        ctx.graph, ctx.damping, ctx.tol, ctx.max_iter, ctx.extra = graph, damping, tol, max_iter, extra
        ctx.forward_stats = st.as_dict()
        ctx.save_for_backward(w, out)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        w, R = ctx.saved_tensors
        g = grad_out.contiguous().float()
        nvec = int(R.shape[1])
        need_w, need_t = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        gw = torch.empty_like(w) if need_w else None
        gt = torch.empty_like(R) if need_t else None
        o = default_options(damping=ctx.damping, tolerance=ctx.tol, iter_num=ctx.max_iter,
                            stream=torch.cuda.current_stream().cuda_stream, **ctx.extra)
        st = _lib.Stats()
        check(lib.mg_ppr_backward(ctx.graph.handle, w.data_ptr(), R.data_ptr(), g.data_ptr(), nvec,
                                  gw.data_ptr() if gw is not None else None,
                                  gt.data_ptr() if gt is not None else None, C.byref(st), C.byref(o)),
              "mg_ppr_backward")
        return gw, gt, None, None, None, None, None


def ppr(graph, edge_weights: torch.Tensor, teleport: torch.Tensor, damping: float = 0.85, tol: float = 1e-7,
        max_iter: int = 10000, **options) -> torch.Tensor:
    """Personalised PageRank of every teleport column; differentiable in both inputs.
    `options`: further mg_options fields for both passes (e.g. use_cuda_graph=0)."""
    return _PPR.apply(edge_weights, teleport, graph, damping, tol, max_iter, dict(options))
