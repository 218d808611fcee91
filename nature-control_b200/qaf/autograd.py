"""torch.autograd wrappers over the discrete adjoint (include/qaf.h, qaf_adjoint_*).

    loss, wT, r1T, r2T = qaf.autograd.rollout(mesh, params, w0, r1_0, r2_0, alpha,
                                              nsteps=2000, checkpoint_every=64, loss_window=100)
    (loss + ...).backward()

Inputs are the initial spectra (reference layout, complex) and the activity
field Ra(x) (real, ny x nx; None: the constant params.alpha). The gradients
follow PyTorch's convention for complex leaves (dL/dRe + i dL/dIm). The
backward pass reruns each checkpoint segment once on the GPU; nothing here
runs on the CPU but the bookkeeping.

`fwd_trans(mesh, phys)` is FwdTrans with its adjoint C2R(W .), so gradients
reach a physical initial Q.
"""
from __future__ import annotations

import torch

from . import Adjoint, Mesh, Params


class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, w0, r1_0, r2_0, alpha, mesh, params, nsteps, checkpoint_every, loss_window):
        adj = Adjoint(mesh, nsteps, checkpoint_every, loss_window)
        p = Params(**{k: getattr(params, k) for k in ("re", "er", "rf", "lam", "alpha", "dt", "q_lin",
                                                        "advect_omega")})
        p.alpha_field = alpha.detach().contiguous() if alpha is not None else None
        loss, (wT, r1T, r2T) = adj.forward(p, w0.detach().contiguous(), r1_0.detach().contiguous(),
                                           r2_0.detach().contiguous(), final_state=True)
        ctx.adj = adj
        ctx.alpha_keep = p.alpha_field
        ctx.has_alpha = alpha is not None
        real = mesh.real_dtype
        return torch.tensor(loss, dtype=real, device=w0.device), wT, r1T, r2T

    @staticmethod
    def backward(ctx, gloss, gwT, gr1T, gr2T):
        adj = ctx.adj
        gl = float(gloss.item()) if gloss is not None else 0.0
        gw, g1, g2, ga = adj.backward((gwT, gr1T, gr2T), grad_loss=gl, want_alpha=ctx.has_alpha)
        return gw, g1, g2, (ga if ctx.has_alpha else None), None, None, None, None, None


def rollout(mesh: Mesh, params: Params, w0, r1_0, r2_0, alpha=None, nsteps: int = 1, checkpoint_every: int = 64,
            loss_window: int = 0):
    """(loss, wT, r1T, r2T) of `nsteps` IF-RK4 steps, differentiable in w0, r1_0, r2_0 and alpha."""
    return _Rollout.apply(w0, r1_0, r2_0, alpha, mesh, params, nsteps, checkpoint_every, loss_window)


class _FwdTrans(torch.autograd.Function):
    @staticmethod
    def forward(ctx, phys, mesh):
        ctx.mesh = mesh
        return mesh.fwd_trans(phys.detach().contiguous())

    @staticmethod
    def backward(ctx, g):
        # adjoint of R2C under the real inner product: C2R(W g), W = 1 on the
        # kx = 0 and kx = nx/2 columns and 1/2 elsewhere; bwd_trans is C2R / (nx ny)
        m = ctx.mesh
        gw = g.detach().clone()
        gw[:, 1:m.nxh - 1] *= 0.5
        gw *= float(m.nx * m.ny)
        return m.bwd_trans(gw.contiguous()), None


def fwd_trans(mesh: Mesh, phys):
    """FwdTrans (R2C, unnormalised) with its adjoint."""
    return _FwdTrans.apply(phys, mesh)
