"""torch.autograd.Function wrappers of the band and eps_M stages.

The forward passes run the library's FP64 GPU path (pmx_band, pmx_chi_epsm)
at the parameter values given; the backward passes call the hand-written
adjoint over the C-ABI (pmx_band_vjp, pmx_epsm_vjp). Parameters are the
problem's form factors and SOC parameters in the order of
pmx_problem_params (Problem.params()); a linear map `J` (full = J @ theta)
ties a smaller set of free parameters to them, e.g. one form factor shared by
every atom of a shell.

    theta = torch.tensor(..., dtype=torch.float64, requires_grad=True)
    E = band(theta, prob_band, ctx, J)            # [nq, nband], eV
    eps = eps_m(theta, prob_chi, ctx, J)          # [nq, nfreq] complex
    loss = ((E - E_target) ** 2).sum() + ((eps.imag - t) ** 2).sum()
    loss.backward()                               # theta.grad
"""
from __future__ import annotations

import numpy as np
import torch

from . import _capi as C


def _full(theta: torch.Tensor, J) -> np.ndarray:
    th = theta.detach().cpu().numpy().astype(np.float64)
    return th if J is None else np.asarray(J, np.float64) @ th


def _reduce(g: np.ndarray, J) -> np.ndarray:
    return g if J is None else np.asarray(J, np.float64).T @ g


class _Band(torch.autograd.Function):
    @staticmethod
    def forward(fctx, theta, prob, ctx, J):
        full = _full(theta, J)
        prob.set_params(full)
        E = ctx.band(prob)
        fctx.prob, fctx.ctx, fctx.J, fctx.full = prob, ctx, J, full
        return torch.from_numpy(E)

    @staticmethod
    def backward(fctx, gE):
        fctx.prob.set_params(fctx.full)
        g = fctx.ctx.band_vjp(fctx.prob, gE.detach().cpu().numpy().astype(np.float64))
        return torch.from_numpy(_reduce(g, fctx.J)), None, None, None


class _EpsM(torch.autograd.Function):
    @staticmethod
    def forward(fctx, theta, prob, ctx, J):
        full = _full(theta, J)
        prob.set_params(full)
        re, im, eps = ctx.chi_epsm(prob, C.SWITCH_EPSLL, C.PREC_FP64)
        fctx.prob, fctx.ctx, fctx.J, fctx.full = prob, ctx, J, full
        fctx.chi = (re, im)
        return torch.from_numpy(eps)

    @staticmethod
    def backward(fctx, geps):
        # torch's gradient of a complex output is dL/dRe + i dL/dIm, the
        # convention of pmx_epsm_vjp
        fctx.prob.set_params(fctx.full)
        g = fctx.ctx.epsm_vjp(fctx.prob, geps.detach().cpu().numpy(), chi=fctx.chi)
        return torch.from_numpy(_reduce(g, fctx.J)), None, None, None


def band(theta: torch.Tensor, prob: C.Problem, ctx: C.Context, J=None) -> torch.Tensor:
    """Band energies [nq, nband] (eV) of a -switch band problem at theta."""
    return _Band.apply(theta, prob, ctx, J)


def eps_m(theta: torch.Tensor, prob: C.Problem, ctx: C.Context, J=None) -> torch.Tensor:
    """eps_M [nq, nfreq] (complex) of a -switch epsLL problem at theta."""
    return _EpsM.apply(theta, prob, ctx, J)
