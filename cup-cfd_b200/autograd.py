"""torch.autograd.Function bindings of the face loops, used only to check the
hand-written adjoint kernels (torch.autograd.gradcheck) -- not a compute path.

Tensors are CUDA, FP64, in the mesh's internal numbering:
  phi [nCells], phiB [nBoundaries]  ->  gradient [3, nCells]
  state [4, nCells] (rho, u, v, w)  ->  massFlux [nFaces] (boundary entries 0)
Forward and backward both run the CUDA library (no CPU fallback).
"""
from __future__ import annotations

import torch

import cupcfd_b200 as cg


class _Gradient(torch.autograd.Function):
    @staticmethod
    def forward(ctx, phi, phiB, mesh, sign_mode):
        grad = torch.empty(3, mesh.nCells, dtype=torch.float64, device=phi.device)
        cg.dev_gradient(mesh, cg.PREC_F64, phi.contiguous(), phiB.contiguous(), grad, sign_mode=sign_mode,
                        stream=torch.cuda.current_stream())
        ctx.mesh, ctx.sign_mode = mesh, sign_mode
        return grad

    @staticmethod
    def backward(ctx, gbar):
        mesh = ctx.mesh
        phibar = torch.empty(mesh.nCells, dtype=torch.float64, device=gbar.device)
        phibbar = torch.empty(max(mesh.nBoundaries, 1), dtype=torch.float64, device=gbar.device)
        cg.dev_gradient_adjoint(mesh, cg.PREC_F64, gbar.contiguous(), phibar, phibbar, sign_mode=ctx.sign_mode,
                                stream=torch.cuda.current_stream())
        return phibar, phibbar[: mesh.nBoundaries], None, None


class _MassFlux(torch.autograd.Function):
    @staticmethod
    def forward(ctx, state, mesh):
        st = state.contiguous()
        mf = torch.zeros(mesh.nFaces, dtype=torch.float64, device=state.device)
        cg.dev_mass_plain(mesh, cg.PREC_F64, st, mf, stream=torch.cuda.current_stream())
        ctx.save_for_backward(st)
        ctx.mesh = mesh
        return mf

    @staticmethod
    def backward(ctx, mbar):
        (st,) = ctx.saved_tensors
        sb = torch.empty_like(st)
        cg.dev_mass_plain_adjoint(ctx.mesh, cg.PREC_F64, st, mbar.contiguous(), sb, stream=torch.cuda.current_stream())
        return sb, None


def gradient(mesh, phi, phiB, sign_mode=cg.SIGN_REFERENCE):
    """GradientPhiGaussDolfyn (nGradient = 1) as a differentiable op."""
    return _Gradient.apply(phi, phiB, mesh, sign_mode)


def mass_flux(mesh, state):
    """Plain face mass flux m_f = rho_f (u_f . S_f) as a differentiable op."""
    return _MassFlux.apply(state, mesh)
