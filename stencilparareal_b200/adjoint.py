"""Differentiable RK4 propagation: a torch.autograd.Function over the C ABI.

Forward: n FP64 RK4 steps (Convection::DoRK4, src/Convection/Convection.cpp:292-303)
of q0 with diffusivity nu0 and velocity (cx, cy, cz).  Backward: the
hand-written discrete adjoint of the RK4 stages (sp_adjoint_rk4) with
sqrt(n) checkpointing and recompute, giving dL/dq0 and dL/d(nu0, cx, cy, cz)
for any scalar loss L of the final field.  Both directions run in
libstencilparareal.so, loaded with ctypes; PyTorch only holds the tensors.
"""
from __future__ import annotations

import ctypes as C
from typing import Tuple

import torch

from . import _lib as L
from .convection import Convection


class _Grid:
    """Propagator handle and staging fields for one set of PDE parameters."""

    def __init__(self, shape, dx, params, nufreq, upwind, device):
        nk, nj, ni = shape
        nu0, cx, cy, cz = (float(v) for v in params)
        self.conv = Convection(ni, nj, nk, dx, nu0, nufreq, cx, cy, cz, upwind=upwind, device=device)
        self.fields = [self.conv.field() for _ in range(3)]

    def to_field(self, dense: torch.Tensor, f):
        d = dense.detach().to(torch.float64).contiguous()
        self.conv.call(L.lib().sp_field_import, self.conv.handle, C.c_void_p(d.data_ptr()), C.c_void_p(f.ptr),
                       L.SP_F64, 0)
        return f

    def from_field(self, f) -> torch.Tensor:
        return f.interior().clone()

    def close(self):
        self.conv.close()


def _check_q0(q0: torch.Tensor):
    if q0.dim() != 3 or not q0.is_cuda or q0.dtype != torch.float64:
        raise TypeError("q0 must be a (nk, nj, ni) float64 CUDA tensor")


class RK4Propagate(torch.autograd.Function):
    """q_n = RK4^n(q0; nu0, c).  params = tensor([nu0, cx, cy, cz]) (float64)."""

    @staticmethod
    def forward(ctx, q0: torch.Tensor, params: torch.Tensor, dx: float, tStart: float, dt: float, n: int,
                checkpoint_every: int = 0, nufreq: float = 0.0, upwind: bool = True) -> torch.Tensor:
        _check_q0(q0)
        p = params.detach().to(torch.float64).cpu()
        g = _Grid(tuple(q0.shape), dx, p.tolist(), nufreq, upwind, q0.device.index or 0)
        fin, fout, _ = g.fields
        g.to_field(q0, fin)
        g.conv.DoRK4(fin, fout, tStart, dt, int(n))
        out = g.from_field(fout if n > 0 else fin)
        g.conv.synchronize()
        ctx.save_for_backward(q0.detach(), params.detach())
        ctx.cfg = (dx, tStart, dt, int(n), int(checkpoint_every), nufreq, upwind)
        g.close()
        return out

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        q0, params = ctx.saved_tensors
        dx, tStart, dt, n, ck, nufreq, upwind = ctx.cfg
        g = _Grid(tuple(q0.shape), dx, params.detach().cpu().tolist(), nufreq, upwind, q0.device.index or 0)
        fq0, flam, fgrad = g.fields
        g.to_field(q0, fq0)
        g.to_field(grad_out, flam)
        gp = (C.c_double * 4)()
        J = C.c_double(0.0)
        g.conv.call(L.lib().sp_adjoint_rk4, g.conv.handle, C.c_void_p(fq0.ptr), None, C.c_void_p(flam.ptr),
                    tStart, dt, n, ck, C.byref(J), C.c_void_p(fgrad.ptr), gp)
        grad_q0 = g.from_field(fgrad)
        grad_par = torch.tensor(list(gp), dtype=torch.float64, device=params.device)
        g.conv.synchronize()
        g.close()
        return grad_q0, grad_par, None, None, None, None, None, None, None


def rk4_propagate(q0: torch.Tensor, params: torch.Tensor, dx: float, tStart: float, dt: float, n: int,
                  checkpoint_every: int = 0, nufreq: float = 0.0, upwind: bool = True) -> torch.Tensor:
    return RK4Propagate.apply(q0, params, dx, tStart, dt, n, checkpoint_every, nufreq, upwind)


def misfit_gradient(conv: Convection, q0_field, target_field, tStart: float, dt: float, n: int,
                    checkpoint_every: int = 0) -> Tuple[float, object, list]:
    """J = 0.5||q_n - q_target||^2 and its gradient, straight through the C ABI.

    Returns (J, grad_q0 field, [dJ/dnu0, dJ/dcx, dJ/dcy, dJ/dcz])."""
    grad = conv.field()
    gp = (C.c_double * 4)()
    J = C.c_double(0.0)
    conv.call(L.lib().sp_adjoint_rk4, conv.handle, C.c_void_p(q0_field.ptr), C.c_void_p(target_field.ptr), None,
              tStart, dt, int(n), int(checkpoint_every), C.byref(J), C.c_void_p(grad.ptr), gp)
    return J.value, grad, list(gp)
