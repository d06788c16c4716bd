"""torch.autograd.Function for the RPA correlation energy.

The forward pass calls rpa_b200_ec (Pi(u) on the tensor cores, FP64 log-det)
and keeps only its inputs; the backward pass calls rpa_b200_ec_grad, which
recomputes Pi(u) per frequency instead of storing all of them and applies
((1+Pi)^{-1} - 1) to R by FP64 triangular solves.  Gradients flow to R
((NQ, nov) column-major view) and to the occupied / virtual orbital energies.
"""
from __future__ import annotations

import torch


class RPAEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, R, eps_o, eps_v, freqs, weights, handle, prec, alpha):
        ec, _ = handle.ec_rpa(R.detach(), eps_o.detach(), eps_v.detach(), freqs, weights, alpha=alpha, prec=prec)
        ctx.save_for_backward(R.detach(), eps_o.detach(), eps_v.detach(), freqs, weights)
        ctx.handle, ctx.prec, ctx.alpha = handle, prec, alpha
        return torch.tensor(ec, dtype=torch.float64, device=R.device)

    @staticmethod
    def backward(ctx, grad):
        R, eo, ev, fr, w = ctx.saved_tensors
        dR = torch.empty((R.shape[1], R.shape[0]), dtype=torch.float64, device=R.device).T
        dO = torch.empty_like(eo)
        dV = torch.empty_like(ev)
        ctx.handle.ec_grad(R, eo, ev, fr, w, alpha=ctx.alpha, prec=ctx.prec, out=(dR, dO, dV))
        return grad * dR, grad * dO, grad * dV, None, None, None, None, None


def rpa_energy(R, eps_o, eps_v, freqs, weights, handle, prec="split", alpha=4.0):
    """Differentiable E_c(R, eps_o, eps_v); R is an (NQ, nov) column-major CUDA tensor."""
    return RPAEnergy.apply(R, eps_o, eps_v, freqs, weights, handle, prec, alpha)
