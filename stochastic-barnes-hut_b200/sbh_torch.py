"""Differentiable evaluation: torch.autograd.Function over sbh_eval_grad_device.

PyTorch supplies only the autograd plumbing, device tensors and the stream; the
values and the query-position gradients come from the library's adjoint kernels
(csrc/adjoint.cu) through the C ABI.  The forward call computes the gradient in
the same pass when the queries require it -- for the stochastic method that is
the gradient over the very paths the value was estimated from -- and backward
scales it by the incoming gradient.

    import sbh_capi as C, sbh_torch
    tree = C.GpuTree(C.HostTree(points, normals, masses, lo, hi, alpha=100.0,
                                dim_split_log=2))
    q = torch.rand(n, 3, device="cuda", requires_grad=True)
    d = sbh_torch.smooth_distance(tree, q, method="stochastic", budget=128)
    d.sum().backward()      # q.grad = dD/dq

Kernels: "gravity" and "plummer" (the potential), "smooth" (the smooth distance
-log(sum exp(-alpha r)) / alpha).  Methods: "brute_force", "barnes_hut",
"barnes_hut_vote", "stochastic".
"""
from __future__ import annotations

import torch

import sbh_capi as C

_KERNELS = {"gravity": C.GRAVITY, "plummer": C.PLUMMER, "smooth": C.SMOOTH_DIST}
_METHODS = {"brute_force": C.BRUTE_FORCE, "barnes_hut": C.BARNES_HUT,
            "barnes_hut_vote": C.BARNES_HUT_VOTE, "stochastic": C.STOCHASTIC}


class _Evaluate(torch.autograd.Function):
    @staticmethod
    def forward(ctx, queries, tree, params):
        if queries.dtype != torch.float32 or not queries.is_cuda:
            raise TypeError("queries must be a float32 CUDA tensor")
        if queries.dim() != 2 or queries.shape[1] != tree.dim:
            raise ValueError(f"queries must be (n, {tree.dim})")
        if queries.device.index != tree.device:
            raise ValueError(f"queries are on {queries.device}, the tree on cuda:{tree.device}")
        n = queries.shape[0]
        soa = queries.detach().t().contiguous()  # [dim][n]
        values = torch.empty(n, dtype=torch.float32, device=queries.device)
        need = ctx.needs_input_grad[0]
        grads = torch.empty((tree.dim, n), dtype=torch.float32, device=queries.device) if need else None
        stream = torch.cuda.current_stream(queries.device).cuda_stream
        tree.eval_grad_device(soa.data_ptr(), n, values.data_ptr(),
                              grads.data_ptr() if need else 0, params, stream=stream)
        if need:
            ctx.save_for_backward(grads)
        return values

    @staticmethod
    def backward(ctx, grad_values):
        (grads,) = ctx.saved_tensors
        return (grads * grad_values.unsqueeze(0)).t(), None, None


def evaluate(tree: C.GpuTree, queries: torch.Tensor, kernel: str = "gravity",
             method: str = "barnes_hut", beta: float = 2.0, samples_per_subdomain: int | None = None,
             budget: int | None = None, seed: int = 0, alpha: float | None = None,
             eps: float = 1e-3) -> torch.Tensor:
    """Values at `queries` (n, dim), differentiable in the queries.

    For the stochastic method give `samples_per_subdomain` (paths per root child,
    the reference's knob) or `budget` (paths per query in total, spread over the
    root's children)."""
    if kernel not in _KERNELS:
        raise ValueError(f"kernel must be one of {sorted(_KERNELS)}")
    if method not in _METHODS:
        raise ValueError(f"method must be one of {sorted(_METHODS)}")
    if samples_per_subdomain is None:
        rc = max(1, tree.info.root_children)
        samples_per_subdomain = max(1, int(round(budget / rc))) if budget else 1
    p = C.params(method=_METHODS[method], kernel=_KERNELS[kernel], beta=beta,
                 samples_per_subdomain=samples_per_subdomain, seed=seed, alpha=alpha, eps=eps)
    return _Evaluate.apply(queries, tree, p)


def smooth_distance(tree: C.GpuTree, queries: torch.Tensor, **kw) -> torch.Tensor:
    """-log(sum_i exp(-alpha |p_i - q|)) / alpha, max-shifted, differentiable."""
    return evaluate(tree, queries, kernel="smooth", **kw)


def gravity_potential(tree: C.GpuTree, queries: torch.Tensor, **kw) -> torch.Tensor:
    """sum_i -m_i / (|p_i - q| + 0.1), differentiable."""
    return evaluate(tree, queries, kernel="gravity", **kw)
