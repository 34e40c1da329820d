"""PyTorch wrapper: K2 as a differentiable function of the offset delta and of k.

    evaluator = K2Torch(table, T=1.3e6, tol=1e-10)
    val = evaluator(v_int, v_frac, delta, k)     # CUDA tensors; delta (float64) and k may need grad
    val.sum().backward()                          # delta.grad = dK2/ddelta, k.grad = sum dK2/dk

v = v_int + v_frac 2^-64 + delta: the exact 64.64 base (int64 tensors holding the u64 bits) and
an FP64 offset.  The forward pass runs the chosen-form plan, whose kernel produces K2,
dK2/ddelta and dK2/dk in one pass; backward only multiplies them by the incoming gradient.
PyTorch is used here for the autograd plumbing and device buffers only.
"""
from __future__ import annotations

import math

import torch

from . import k2
from ._lib import check, lib


def _dev_ptr(t: torch.Tensor) -> int:
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("tensors must be contiguous CUDA tensors")
    return t.data_ptr()


class K2Torch:
    """K2(v, T, k) over a resident table, with a plan cached per (P, k)."""

    def __init__(self, table: k2.ZeroTable, T: float = math.inf, tol: float = 1e-10):
        self.table, self.T, self.tol = table, float(T), float(tol)
        self._plans: dict[tuple[int, float], k2.Plan] = {}

    def plan(self, P: int, k: float) -> k2.Plan:
        key = (int(P), float(k))
        p = self._plans.get(key)
        if p is None:
            p = k2.Plan(self.table, [P], [k], [self.T], tol=self.tol)
            self._plans[key] = p
        return p

    def evaluate(self, v_int, v_frac, delta, k: float):
        """(val, dd, dk) tensors, no autograd."""
        P = v_int.shape[0]
        out = torch.empty(3, P, dtype=torch.float64, device=v_int.device)
        stream = torch.cuda.current_stream(v_int.device).cuda_stream
        self.plan(P, k).run_dev(_dev_ptr(v_int), _dev_ptr(v_frac), _dev_ptr(delta), out[0].data_ptr(),
                                out[1].data_ptr(), out[2].data_ptr(), stream)
        return out[0], out[1], out[2]

    def __call__(self, v_int, v_frac, delta, k):
        if not torch.is_tensor(k):
            k = torch.tensor(float(k), dtype=torch.float64, device=delta.device)
        return _K2Fn.apply(delta, k, v_int, v_frac, self)

    def newton(self, v_int, v_frac, delta, k: float, iters: int = 8, max_step: float = 1e-4):
        """Batched Newton polish of delta (in place); returns (h0, val, dd, dk) at the kept point."""
        P = v_int.shape[0]
        out = torch.empty(4, P, dtype=torch.float64, device=v_int.device)
        stream = torch.cuda.current_stream(v_int.device).cuda_stream
        check(lib().mb_plan_newton_dev(self.plan(P, k).handle, _dev_ptr(v_int), _dev_ptr(v_frac), _dev_ptr(delta),
                                       int(iters), float(max_step), out[0].data_ptr(), out[1].data_ptr(),
                                       out[2].data_ptr(), out[3].data_ptr(), stream))
        return out[0], out[1], out[2], out[3]

    def close(self):
        for p in self._plans.values():
            p.close()
        self._plans.clear()


class _K2Fn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, delta, k, v_int, v_frac, ev: K2Torch):
        val, dd, dk = ev.evaluate(v_int, v_frac, delta.detach().contiguous(), float(k.item()))
        ctx.save_for_backward(dd, dk)
        ctx.k_shape = k.shape
        return val

    @staticmethod
    def backward(ctx, g):
        dd, dk = ctx.saved_tensors
        grad_delta = g * dd if ctx.needs_input_grad[0] else None
        grad_k = (g * dk).sum().reshape(ctx.k_shape) if ctx.needs_input_grad[1] else None
        return grad_delta, grad_k, None, None, None
