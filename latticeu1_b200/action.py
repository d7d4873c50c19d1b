"""Differentiable U(1) Wilson action: torch.autograd over the CUDA library.

    S(theta) = beta * sum_x sum_{mu<nu} w_{mu nu} (1 - cos theta_P(x)),
    dS/dtheta_mu(x) = beta * sum_{nu != mu} w [sin theta_{mu nu}(x) - sin theta_{mu nu}(x - nu)],

with w = 1/xi for spatial-spatial and xi for space-time plaquettes (the
reference's staple weights, include/staple.h:75-102).  theta is a CUDA tensor
of shape (V*d,) or (B, V*d) in the reference's angle layout
theta[mu*V + parity*V/2 + eo] (include/index.h:114-153), float32 or float64.
Forward and backward are the library's kernels (u1_wilson_action and its
adjoint u1_wilson_action_grad) queued on torch's current stream; the action
is summed in FP64 in a fixed order, so results are deterministic.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import torch

from ._lib import check, lib, u1_geom

__all__ = ["WilsonAction", "wilson_action", "topological_charge"]


def make_geom(dims: int, N: Sequence[int], beta: float, aniso: float = 1.0) -> tuple[u1_geom, int]:
    """The ABI geometry and the link count V*dims (validated by the library)."""
    N = list(N) + [0] * (4 - len(N))
    g = u1_geom(dims=int(dims), N=(C.c_int * 4)(*[int(n) for n in N[:4]]), beta=float(beta), aniso=float(aniso))
    info = (C.c_int64 * 8)()
    check(lib.u1_geom_validate(C.byref(g), info), "u1_geom_validate")
    return g, int(info[0]) * int(dims)


def _dtype_code(t: torch.Tensor) -> int:
    if t.dtype == torch.float32:
        return 0
    if t.dtype == torch.float64:
        return 1
    raise TypeError(f"theta must be float32 or float64, got {t.dtype}")


def _as_batch(theta: torch.Tensor, nlinks: int) -> torch.Tensor:
    if not theta.is_cuda:
        raise ValueError("theta must be a CUDA tensor")
    t = theta.reshape(1, -1) if theta.dim() == 1 else theta
    if t.dim() != 2 or t.shape[1] != nlinks:
        raise ValueError(f"theta must have shape (V*d,) or (B, V*d) with V*d = {nlinks}, got {tuple(theta.shape)}")
    return t.contiguous()


def _forward_raw(g: u1_geom, theta: torch.Tensor) -> torch.Tensor:
    """(B, 2) float64: action and (2D) topological charge per configuration."""
    B = theta.shape[0]
    nbytes = C.c_size_t()
    check(lib.u1_action_workspace_bytes(C.byref(g), B, C.byref(nbytes)), "u1_action_workspace_bytes")
    with torch.cuda.device(theta.device):
        ws = torch.empty(max(1, nbytes.value // 8), dtype=torch.float64, device=theta.device)
        out = torch.empty((B, 2), dtype=torch.float64, device=theta.device)
        stream = torch.cuda.current_stream(theta.device).cuda_stream
        check(lib.u1_wilson_action(C.byref(g), C.c_void_p(theta.data_ptr()), _dtype_code(theta), B,
                                   C.c_void_p(ws.data_ptr()), C.c_void_p(out.data_ptr()), C.c_void_p(stream)),
              "u1_wilson_action")
    return out


class _WilsonActionFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta: torch.Tensor, g: u1_geom):
        out = _forward_raw(g, theta)
        ctx.save_for_backward(theta)
        ctx.g = g
        return out[:, 0].clone()

    @staticmethod
    def backward(ctx, grad_s: torch.Tensor):
        (theta,) = ctx.saved_tensors
        scale = grad_s.detach().to(torch.float64).contiguous()
        grad = torch.empty_like(theta)
        with torch.cuda.device(theta.device):
            stream = torch.cuda.current_stream(theta.device).cuda_stream
            check(lib.u1_wilson_action_grad(C.byref(ctx.g), C.c_void_p(theta.data_ptr()), _dtype_code(theta),
                                            theta.shape[0], C.c_void_p(scale.data_ptr()),
                                            C.c_void_p(grad.data_ptr()), C.c_void_p(stream)),
                  "u1_wilson_action_grad")
        return grad, None


class WilsonAction(torch.nn.Module):
    """S(theta) per configuration, differentiable in theta (hand-written adjoint)."""

    def __init__(self, dims: int, N: Sequence[int], beta: float, aniso: float = 1.0):
        super().__init__()
        self.geom, self.nlinks = make_geom(dims, N, beta, aniso)
        self.dims = int(dims)
        self.beta = float(beta)
        self.aniso = float(aniso)

    def forward(self, theta: torch.Tensor) -> torch.Tensor:
        single = theta.dim() == 1
        t = _as_batch(theta, self.nlinks)
        s = _WilsonActionFn.apply(t, self.geom)
        return s[0] if single else s

    def charge(self, theta: torch.Tensor) -> torch.Tensor:
        """2D topological charge Q = (1/2pi) sum_x wrap(theta_P(x)) (0 in 3D/4D)."""
        single = theta.dim() == 1
        q = _forward_raw(self.geom, _as_batch(theta.detach(), self.nlinks))[:, 1]
        return q[0] if single else q


def wilson_action(theta: torch.Tensor, dims: int, N: Sequence[int], beta: float, aniso: float = 1.0) -> torch.Tensor:
    return WilsonAction(dims, N, beta, aniso)(theta)


def topological_charge(theta: torch.Tensor, N: Sequence[int]) -> torch.Tensor:
    """2D only: N = (Nx, Nt)."""
    return WilsonAction(2, (N[0], 0, 0, N[1]), 1.0).charge(theta)
