"""The hand-written adjoint (pmx_band_vjp, pmx_epsm_vjp) against the
tangent-mode oracle (FP64 reference gradient) and against central finite
differences of the library's own forward path."""
import numpy as np
import pytest

import pmx_oracle as O
import pmx_oracle_grad as OG
from test_oracle_grad import grad_case

pytestmark = pytest.mark.gpu


def _band_args(args):
    """The band variant of a grad_case argv: the q list becomes a 4-point path."""
    out, skip = [], 0
    for i, a in enumerate(args):
        if skip:
            skip -= 1
            continue
        if a in ("-switch", "-qvec", "-kpoint", "-kpointfile"):
            skip = 1
            continue
        out.append(a)
    return out + ["-switch", "band", "-qvec", "0,0,0,0.25,0.1,0,0.5,0.5,0.5,1,0,0"]


@pytest.mark.parametrize("soc", [True, False])
def test_band_vjp_vs_oracle(ctx, tmp_path, soc):
    import picomax_b200 as pm
    args, cr, mat, G, _, _, _, _, o = grad_case(tmp_path, soc=soc)
    bargs = _band_args(args)
    prob = pm.Problem(bargs)
    Q = prob.qpoints()
    E, dE = OG.band_tangent(cr, mat, G, Q, o["nband"], o["nvalence"])
    assert np.max(np.abs(ctx.band(prob) - E)) < 1e-9
    rng = np.random.default_rng(7)
    g = rng.standard_normal(E.shape)
    # equal weights inside degenerate sets (the derivative of a single member
    # of a degenerate set depends on the basis)
    for iq in range(len(Q)):
        lab = OG._clusters(E[iq])
        for c in np.unique(lab):
            g[iq, lab == c] = g[iq, lab == c].mean()
    ref = np.einsum("pqn,qn->p", dE, g)
    got = ctx.band_vjp(prob, g)
    assert np.max(np.abs(got - ref)) < 1e-9 * np.max(np.abs(ref))
    prob.close()


@pytest.mark.parametrize("soc,kk,delta", [(True, 1, 0), (True, 0, 1), (False, 1, 0)])
def test_epsm_vjp_vs_oracle(ctx, tmp_path, soc, kk, delta):
    import picomax_b200 as pm
    dfreq = 0.1 if kk else 0.015
    args, cr, mat, G, hkl, K, KW, Q, o = grad_case(tmp_path, soc=soc, kk=kk, delta=delta, dfreq=dfreq)
    o["kk"], o["delta"] = kk, delta
    _, _, em, dem = OG.chi_ll_epsm(cr, mat, G, hkl, K, KW, Q, **o)
    prob = pm.Problem(args)
    re, im, em_gpu = ctx.chi_epsm(prob, pm.SWITCH_EPSLL, pm.PREC_FP64)
    assert np.max(np.abs(em_gpu - em)) < 1e-9 * np.max(np.abs(em))
    rng = np.random.default_rng(11)
    gbar = rng.standard_normal(em.shape) + 1j * rng.standard_normal(em.shape)
    ref = np.einsum("pqf,qf->p", dem, gbar.conj()).real
    got = ctx.epsm_vjp(prob, gbar)
    got2 = ctx.epsm_vjp(prob, gbar, chi=(re, im))
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(got - ref)) < 1e-8 * scale
    assert np.max(np.abs(got2 - got)) < 1e-12 * scale
    prob.close()


def test_epsm_vjp_vs_gpu_finite_differences(ctx, tmp_path):
    """dL/dp of L = sum_w c_w Im eps_M(w) by the adjoint against central
    differences (h = 1e-7 Ry) of the library's FP64 forward path."""
    import picomax_b200 as pm
    args, *_ = grad_case(tmp_path)
    prob = pm.Problem(args)
    th = prob.params()
    rng = np.random.default_rng(5)
    c = rng.standard_normal(prob.info.nfreq)

    def loss(theta):
        prob.set_params(theta)
        return float(np.sum(c * ctx.chi_epsm(prob, pm.SWITCH_EPSLL, pm.PREC_FP64)[2][0].imag))

    prob.set_params(th)
    got = ctx.epsm_vjp(prob, (1j * c)[None, :])
    h = 1e-7  # the lambda_S direction is curved enough that h = 1e-6 leaves ~5e-6 truncation error
    fd = np.zeros(len(th))
    for p in range(len(th)):
        tp, tm = th.copy(), th.copy()
        tp[p] += h
        tm[p] -= h
        fd[p] = (loss(tp) - loss(tm)) / (2 * h)
    prob.set_params(th)
    assert np.max(np.abs(got - fd)) < 1e-6 * np.max(np.abs(fd))
    prob.close()


def test_torch_autograd_wrappers(ctx, tmp_path):
    """picomax_b200.autograd: backward of a loss through band() and eps_m()
    with a parameter map equals J^T of the C-ABI vector-Jacobian products."""
    import torch
    import picomax_b200 as pm
    from picomax_b200.autograd import band, eps_m
    args, *_ = grad_case(tmp_path)
    pe, pb = pm.Problem(args), pm.Problem(_band_args(args))
    full0 = pe.params()
    J = np.eye(len(full0))[:, :6] * 0.5  # ties the first 6 parameters, zeroes the rest
    th = torch.tensor(np.linalg.lstsq(J, full0, rcond=None)[0], dtype=torch.float64, requires_grad=True)
    E = band(th, pb, ctx, J)
    eps = eps_m(th, pe, ctx, J)
    L = (E ** 2).sum() + (eps.imag ** 2).sum()
    L.backward()
    full = J @ th.detach().numpy()
    pb.set_params(full)
    pe.set_params(full)
    Eh = ctx.band(pb)
    _, _, em = ctx.chi_epsm(pe, pm.SWITCH_EPSLL, pm.PREC_FP64)
    ref = J.T @ (ctx.band_vjp(pb, 2 * Eh) + ctx.epsm_vjp(pe, 2j * em.imag))
    assert np.max(np.abs(th.grad.numpy() - ref)) < 1e-10 * np.max(np.abs(ref))
    pe.close()
    pb.close()
