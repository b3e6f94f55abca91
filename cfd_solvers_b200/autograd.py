"""torch.autograd binding of the gray-LBM forward and its discrete adjoint.

``GrayLbm.apply(ns, tau, solver, steps, interval, init)`` runs ``steps`` steps
of ``solver`` (an :class:`EsotericPullCudaSolver` configured for BGK/TRT, with
optional force and stationary walls) from the state ``init(solver)`` sets up,
with the per-cell solid fraction ``ns`` (a CUDA tensor of N values) and the
relaxation time ``tau`` (a 0-d tensor), and returns the final density and
velocity as CUDA tensors ``rho`` (N) and ``u`` (3, N), the fields
``compute_macroscopic`` reports.  Its backward is the hand-written discrete
adjoint of the library (``cfdx_lbm_adjoint_backward``): transposed
Esoteric-Pull streaming and the per-cell collision Jacobian, with the forward
re-computed segment by segment from checkpoints kept every ``interval``
steps.  Gradients w.r.t. ``ns`` and ``tau`` are accumulated in FP64 on the GPU.

The reference has no differentiable path; its Python package is a ctypes
wrapper (python/cfd_solvers/bindings.py), which this module extends.
"""
from __future__ import annotations

import ctypes

import torch

from . import bindings as B
from .lbm import EsotericPullCudaSolver


def device_fields(solver: EsotericPullCudaSolver, device) -> tuple[torch.Tensor, torch.Tensor]:
    """rho (N) and u (3, N) of the solver's current state as CUDA tensors:
    float64 for FP64 storage, float32 otherwise."""
    n = solver.cells()
    f64 = solver.config.storage == "fp64"
    dt = torch.float64 if f64 else torch.float32
    rho = torch.empty(n, dtype=dt, device=device)
    u = torch.empty((3, n), dtype=dt, device=device)
    torch.cuda.current_stream(device).synchronize()
    solver.library.call("cfdx_lbm_macroscopic_f64" if f64 else "cfdx_lbm_macroscopic", solver.handle,
                        ctypes.c_void_p(rho.data_ptr()), ctypes.c_void_p(u[0].data_ptr()),
                        ctypes.c_void_p(u[1].data_ptr()), ctypes.c_void_p(u[2].data_ptr()), B.DEVICE)
    return rho, u


class GrayLbm(torch.autograd.Function):
    """(ns, tau) -> (rho(T), u(T)) through the B200 gray-LBM step; backward = discrete adjoint."""

    @staticmethod
    def forward(ctx, ns, tau, solver, steps, interval, init, subinterval=0):
        if not ns.is_cuda:
            raise ValueError("ns must be a CUDA tensor")
        solver.set_solid_fraction(ns.detach().to(torch.float32).contiguous())
        solver.set_tau(float(tau))
        init(solver)
        solver.adjoint_forward(int(steps), int(interval), int(subinterval))
        rho, u = device_fields(solver, ns.device)
        ctx.solver = solver
        ctx.ns_dtype = ns.dtype
        ctx.tau_like = tau
        return rho, u

    @staticmethod
    def backward(ctx, g_rho, g_u):
        solver = ctx.solver
        n = solver.cells()
        dev = g_u.device if g_u is not None else g_rho.device
        if g_u is None:
            g_u = torch.zeros((3, n), dtype=torch.float32, device=dev)
        g_u = g_u.to(torch.float32).contiguous()
        g_r = None if g_rho is None else g_rho.to(torch.float32).contiguous()
        grad = torch.empty(n, dtype=torch.float64, device=dev)
        grad, gtau = solver.adjoint_backward(g_u[0], g_u[1], g_u[2], g_rho=g_r, grad_ns_out=grad)
        tau = ctx.tau_like
        gt = torch.tensor(gtau, dtype=tau.dtype if torch.is_tensor(tau) else torch.float64,
                          device=tau.device if torch.is_tensor(tau) else dev)
        return grad.to(ctx.ns_dtype), gt, None, None, None, None, None


def gray_lbm(ns: torch.Tensor, tau, solver: EsotericPullCudaSolver, steps: int, interval: int = 64, init=None,
             subinterval: int = 0):
    """Functional form of :class:`GrayLbm`; ``init`` defaults to rest at rho = 1.

    ``subinterval`` > 0 reverses each checkpoint segment in two levels of recompute
    (see ``EsotericPullCudaSolver.adjoint_forward``); the gradients are the same.
    """
    if init is None:
        init = lambda s: s.initialize_uniform()  # noqa: E731
    if not torch.is_tensor(tau):
        tau = torch.tensor(float(tau), dtype=torch.float64, device=ns.device)
    return GrayLbm.apply(ns, tau, solver, steps, interval, init, subinterval)
