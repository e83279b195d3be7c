"""
Adjoint-state gradient of the solve behind ``torch.autograd.Function``.

The converged field satisfies A E = s / k0^2 with A = -laplacian - eps (k0-scaled units; for vector fields the
curl-curl operator): this is the fixed point of the preconditioned iteration (reference solver.py:1070-1075,
E = G (chi E + s') with chi = i (eps - alpha) / alpha_i, s' = i s / alpha_i, g = -i alpha_i / (k^2 - alpha)).  A is
complex symmetric for isotropic (and for symmetric anisotropic) permittivity, so for a real loss L with torch
gradient g = dL/dRe(E) + i dL/dIm(E):

    nu = A^{-1} conj(g)          -- the same fused solve with source conj(g), same material and alpha
    dL/d eps = conj(sum_c nu_c E_c)           (k0^2-scaled fields; fused kernel mmx_adjoint_grad)
    dL/d s   = conj(nu) / k0^2

No iteration history is stored: the backward pass needs only the forward field and one adjoint field.  The
reference has no adjoint; its only gradient path back-propagates through an unrolled torch restatement of the
iteration (examples/scattering_neural_network.py:206-300).

``precision='mixed'`` runs both solves as complex64 inner iterations inside the FP64 defect-correction loop
(``mixed.MixedSolution``): the fields, and so the gradient, are then accurate to the FP64 solve's residue instead of
complex64's (whose iteration stalls between 1e-7 and 1e-6 on some sources), at about twice the solve time.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from . import _native as nat
from .batch import BatchSolution
from .grid import Grid


def _ptr(t):
    return nat.device_ptr(t)


def _now() -> float:
    """Host time after the device has finished the work queued so far (solve-phase timing in ``stats``)."""
    torch.cuda.synchronize()
    return time.perf_counter()


def _stream():
    s = torch.cuda.current_stream().cuda_stream
    return ctypes.c_void_p(s) if s else None


class _SolveFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, epsilon, sources, problem):
        grid, k0 = problem['grid'], problem['wavenumber']
        # the permittivity goes to the host for the FP64 preconditioner set-up (as in the reference); the sources
        # stay on the device
        eps_np = epsilon.detach().cpu().numpy()
        if problem.get('precision') == 'mixed':
            return _SolveFn._forward_mixed(ctx, epsilon, sources, problem, eps_np)
        bs = BatchSolution(grid, sources.detach(), eps_np, bound=problem.get('bound'), wavenumber=k0,
                           dtype=problem.get('dtype', np.complex64), device=sources.device)
        if problem.get('variant') is not None:  # the pass-kernel variant for both solves (e.g. the autotuner's)
            from . import autotune
            autotune.set_variant(bs.engine, int(problem['variant']))
        t0 = _now()
        bs.solve(problem.get('rtol', 1e-6), problem.get('maxiter', 100000))
        problem.setdefault('stats', {})['forward_iterations'] = bs.iterations
        problem['stats']['forward_solve_s'] = _now() - t0
        E = bs.E_device.clone()  # [B, C, N], k0^2-scaled
        ctx.bs = bs
        ctx.problem = problem
        ctx.eps_is_complex = torch.is_complex(epsilon)
        ctx.eps_shape = epsilon.shape
        ctx.save_for_backward(E)
        return (E * (1.0 / k0 ** 2)).reshape(bs.batch, bs.ncomp, *(int(n) for n in grid.shape))

    @staticmethod
    def _forward_mixed(ctx, epsilon, sources, problem, eps_np):
        from .mixed import MixedSolution
        grid, k0 = problem['grid'], problem['wavenumber']
        src = sources.detach().cpu().numpy()
        ms = MixedSolution(grid, src, eps_np, bound=problem.get('bound'), wavenumber=k0, device=sources.device)
        t0 = _now()
        ms.solve(rtol=problem.get('rtol', 1e-10))
        problem.setdefault('stats', {})['forward_iterations'] = np.array([ms.total_inner_iterations])
        problem['stats']['forward_solve_s'] = _now() - t0
        problem['stats']['forward_residue'] = float(ms.residues.max())
        E = ms.x.clone()  # [B, C, N] complex128, k0^2-scaled
        B, C = ms.batch, ms.ncomp
        ms.close()
        ctx.bs = None
        ctx.problem = problem
        ctx.eps_np = eps_np
        ctx.eps_is_complex = torch.is_complex(epsilon)
        ctx.eps_shape = epsilon.shape
        ctx.eps_dtype = epsilon.dtype
        ctx.src_dtype = sources.dtype
        ctx.save_for_backward(E)
        return (E * (1.0 / k0 ** 2)).reshape(B, C, *(int(n) for n in grid.shape))

    @staticmethod
    def _backward_mixed(ctx, grad_E):
        from .mixed import MixedSolution
        (E,) = ctx.saved_tensors
        problem = ctx.problem
        grid, k0 = problem['grid'], problem['wavenumber']
        B, C, N = E.shape
        # the adjoint system A nu = conj(g) with the same material, solved in mixed precision
        g = grad_E.detach().reshape(B, C, *(int(n) for n in grid.shape))
        ms = MixedSolution(grid, torch.conj(g).cpu().numpy(), ctx.eps_np, bound=problem.get('bound'), wavenumber=k0,
                           device=E.device)
        t0 = _now()
        ms.solve(rtol=problem.get('rtol', 1e-10))
        problem['stats']['adjoint_iterations'] = np.array([ms.total_inner_iterations])
        problem['stats']['adjoint_solve_s'] = _now() - t0
        nu = ms.x
        grad_eps = grad_src = None
        if ctx.needs_input_grad[0]:
            gb = torch.empty((B, N), dtype=torch.complex128, device=E.device)
            nat.call('mmx_adjoint_grad', _ptr(E), _ptr(nu), _ptr(gb), B, C, N, nat.MMX_C128, 1.0, _stream())
            gsum = gb.sum(dim=0).reshape(tuple(int(n) for n in grid.shape)) * (1.0 / k0 ** 2)
            grad_eps = (gsum if ctx.eps_is_complex else gsum.real).reshape(ctx.eps_shape).to(ctx.eps_dtype)
        if ctx.needs_input_grad[1]:
            grad_src = (torch.conj(nu) * (1.0 / k0 ** 2)).reshape(B, C, *(int(n) for n in grid.shape))
            grad_src = grad_src.to(ctx.src_dtype)
        ms.close()
        return grad_eps, grad_src, None

    @staticmethod
    def backward(ctx, grad_E):
        if ctx.problem.get('precision') == 'mixed':
            return _SolveFn._backward_mixed(ctx, grad_E)
        (E,) = ctx.saved_tensors
        bs, problem = ctx.bs, ctx.problem
        k0 = problem['wavenumber']
        B, C, N = bs.batch, bs.ncomp, bs.engine.N
        g = grad_E.detach().reshape(B, C, N)
        # adjoint solve A nu = conj(g): the engine's field F for source s satisfies A F = s, so the source conj(g)
        # gives nu directly.  It starts again from alpha0: the forward solve may have raised alpha (divergence
        # guard), and the fixed point does not depend on alpha.
        bs.engine.set_sources(torch.conj(g).to(bs.engine.torch_dtype) * (1.0j / bs.pre.alpha.imag / bs.pre.beta))
        bs.engine.reset_alpha()
        bs.engine.reset_update_norm()
        bs.set_fields(0.0)
        t0 = _now()
        bs.solve(problem.get('rtol', 1e-6), problem.get('maxiter', 100000))
        problem['stats']['adjoint_iterations'] = bs.iterations
        problem['stats']['adjoint_solve_s'] = _now() - t0
        nu = bs.E_device  # [B, C, N]
        grad_eps = grad_src = None
        if ctx.needs_input_grad[0]:
            gb = torch.empty((B, N), dtype=E.dtype, device=E.device)
            nat.call('mmx_adjoint_grad', _ptr(E), _ptr(nu), _ptr(gb), B, C, N,
                     nat.MMX_C64 if E.dtype == torch.complex64 else nat.MMX_C128, 1.0, _stream())
            # E is k0^2-scaled, the returned field is E / k0^2: dE_phys = A^{-1}(d eps E_phys)
            gsum = gb.sum(dim=0).reshape(tuple(int(n) for n in bs.grid.shape)) * (1.0 / k0 ** 2)
            grad_eps = gsum if ctx.eps_is_complex else gsum.real
            grad_eps = grad_eps.reshape(ctx.eps_shape)
        if ctx.needs_input_grad[1]:
            grad_src = (torch.conj(nu) * (1.0 / k0 ** 2)).reshape(B, C, *(int(n) for n in bs.grid.shape))
        bs.close()
        return grad_eps, grad_src, None


def solve(epsilon: torch.Tensor, sources: torch.Tensor, grid: Grid, wavenumber: float, bound=None,
          dtype=np.complex64, rtol: float = 1e-6, maxiter: int = 100000, stats: dict | None = None,
          precision: str = 'single', variant: int | None = None) -> torch.Tensor:
    """
    Differentiable solve: E [B, 1|3, *grid] for the isotropic permittivity ``epsilon`` [*grid] (real or complex)
    and sources [B, 1|3, *grid] (``source_distribution`` units).  Gradients flow to epsilon and sources through the
    adjoint solve above.  ``precision``: 'single' solves in ``dtype``; 'mixed' solves with complex64 inner iterations
    and FP64 defect correction to ``rtol`` (the fields are complex128).  ``variant``: the MMX_VARIANT_* pass-kernel
    flags of the forward and adjoint solves in single precision (None: the plan's default), e.g. the choice of
    ``autotune.tune`` on a batch of the same problem.
    """
    if precision not in ('single', 'mixed'):
        raise ValueError("precision must be 'single' or 'mixed'")
    problem = dict(grid=grid, wavenumber=float(wavenumber), bound=bound, dtype=dtype, rtol=rtol, maxiter=maxiter,
                   precision=precision, variant=variant)
    if stats is not None:
        problem['stats'] = stats
    if sources.dim() == grid.ndim + 1:
        sources = sources.unsqueeze(0)
    return _SolveFn.apply(epsilon, sources, problem)
