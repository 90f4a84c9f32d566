"""Differentiable weighted PageRank for PyTorch.

    x = knappnet_b200.autograd.pagerank(weights, graph, damping=0.85)
    loss = ((x - target) ** 2).sum()
    loss.backward()          # weights.grad = dL/dweights

`weights` is a CUDA float64 tensor of the graph's m edge weights (input edge
order). The forward pass is the library's weighted PageRank on the graph's
structure with these weights (net_pagerank_weights_device); the backward pass
is its hand-written adjoint (net_pagerank_grad_device): one transpose solve
(I - d M - d jump 1_D^T)^T lambda = dL/dx on the device, then per edge
dL/dw_e = d f_e (x_j / s_j) (lambda_i - (M^T lambda)_j), which includes the
derivative of the out-strength normalisation.

The library runs on its own CUDA stream; this binding waits for torch's
current stream before each call, and each call returns only once its results
are in device memory, so the tensors are ready for torch afterwards.
"""
from __future__ import annotations

import ctypes

import torch

from . import ERR_LEN, NetSolveInfo, _check, lib


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class PageRankFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, weights, graph, damping, directed, personalization, dangling, loops, tol,
                max_iter, precision):
        if not weights.is_cuda:
            raise ValueError("weights must be a CUDA tensor")
        if weights.numel() != graph.m:
            raise ValueError(f"weights has {weights.numel()} values; the graph has {graph.m} edges")
        w = weights.detach().to(torch.float64).contiguous()
        p = None
        if personalization is not None:
            p = personalization.detach().to(device=w.device, dtype=torch.float64).contiguous()
        out = torch.empty(graph.n, dtype=torch.float64, device=w.device)
        torch.cuda.current_stream(w.device).synchronize()
        info = NetSolveInfo()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_pagerank_weights_device(graph.h, _ptr(w), damping, int(directed),
                                                 _ptr(p), dangling, loops, tol, max_iter,
                                                 precision, _ptr(out), ctypes.byref(info), err,
                                                 ERR_LEN), err)
        ctx.save_for_backward(w, out)
        ctx.graph = graph
        ctx.p = p
        ctx.opts = (damping, directed, dangling, loops, tol, max_iter)
        ctx.info = info
        return out

    @staticmethod
    def backward(ctx, grad_out):
        w, x = ctx.saved_tensors
        damping, directed, dangling, loops, tol, max_iter = ctx.opts
        g = grad_out.detach().to(torch.float64).contiguous()
        gw = torch.empty_like(w)
        torch.cuda.current_stream(w.device).synchronize()
        info = NetSolveInfo()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_pagerank_grad_device(ctx.graph.h, _ptr(w), _ptr(x), _ptr(g), damping,
                                              int(directed), _ptr(ctx.p), dangling, loops, tol,
                                              max_iter, _ptr(gw), None, ctypes.byref(info), err,
                                              ERR_LEN), err)
        return gw, None, None, None, None, None, None, None, None, None


def pagerank(weights: torch.Tensor, graph, damping: float = 0.85, directed: bool = True,
             personalization: torch.Tensor | None = None, dangling: int = 0, loops: int = 0,
             tol: float = 0.0, max_iter: int = 0, precision: int = 0) -> torch.Tensor:
    """Weighted PageRank of `graph`'s structure with edge weights `weights`,
    differentiable with respect to the weights."""
    return PageRankFunction.apply(weights, graph, damping, directed, personalization, dangling,
                                  loops, tol, max_iter, precision)
