"""Differentiable effective stiffness: ``torch.autograd.Function`` over the CUDA solver.

Forward: the six unit-load solves of one microstructure as one batch; returns M (6x6),
row k = mean stress for the unit macroscopic strain e_k (as ``c_eff``). Backward: the
hand-written gradient kernel ``lsb_ceff_gradient``; the Lippmann-Schwinger operator is
self-adjoint in the energy inner product, so the six forward strain fields are also the
adjoint fields and the gradient with respect to lambda(x), mu(x) is a pointwise product
of them (see ``jaxmaterials_b200/csrc/gradient.cu``). The reference only offers
forward-mode ``jax.jacfwd`` through its while loop (``src/driver.py:73-76``).
"""

from __future__ import annotations

import ctypes

import numpy as np

from .. import _lib
from .lippmann_schwinger import RULE_CUDA, _cached_solver

__all__ = ["EffectiveStiffness", "c_eff_autograd"]


def _torch():
    import torch

    return torch


class EffectiveStiffness(_torch().autograd.Function):
    @staticmethod
    def forward(ctx, lmbda, mu, solver, rtol, atol, maxiter):
        torch = _torch()
        f64 = lmbda.dtype == torch.float64
        r = solver.solve(lmbda.detach(), mu.detach(), np.eye(6), rtol=rtol, atol=atol,
                         maxiter=maxiter, rule=RULE_CUDA, want_sigma=False,
                         dtype=np.float64 if f64 else np.float32)
        if not np.all(r.status == 1):
            raise RuntimeError(f"effective stiffness: solves did not converge (status {r.status})")
        ctx.save_for_backward(r.epsilon)
        ctx.grid = solver.grid_spec
        return torch.as_tensor(r.mean_sigma, dtype=lmbda.dtype, device=lmbda.device)

    @staticmethod
    def backward(ctx, grad_m):
        torch = _torch()
        (eps,) = ctx.saved_tensors
        g = ctx.grid
        lib = _lib.load()
        f64 = eps.dtype == torch.float64
        dl = torch.empty(g.shape, dtype=eps.dtype, device=eps.device)
        dm = torch.empty_like(dl)
        gm = np.ascontiguousarray(grad_m.detach().double().cpu().numpy())
        voxels = np.array(g.shape, dtype=np.int32)
        fn = lib.lsb_ceff_gradient_f64 if f64 else lib.lsb_ceff_gradient
        stream = torch.cuda.current_stream(eps.device).cuda_stream
        _lib.check(fn(voxels.ctypes.data_as(_lib.c_int_p), ctypes.c_void_p(eps.data_ptr()),
                      gm.ctypes.data_as(_lib.c_double_p), ctypes.c_void_p(dl.data_ptr()),
                      ctypes.c_void_p(dm.data_ptr()), ctypes.c_void_p(stream)),
                   "lsb_ceff_gradient")
        return dl, dm, None, None, None, None


def c_eff_autograd(lmbda, mu, grid_spec, rtol=1e-6, atol=1e-20, maxiter=5000, depth=5,
                   precision=None):
    """M(lambda, mu) as a differentiable torch tensor (CUDA tensors in, float32 or float64).

    float32 inputs run mixed precision, float64 inputs FP64 fields throughout."""
    torch = _torch()
    s = _cached_solver(grid_spec, 6, depth)
    s.set_precision(precision or ("fp64" if lmbda.dtype == torch.float64 else "mixed"))
    return EffectiveStiffness.apply(lmbda, mu, s, rtol, atol, maxiter)
