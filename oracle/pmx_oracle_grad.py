"""Tangent-mode (forward) derivatives of the band energies and of eps_M with
respect to the form factors and SOC parameters. TEST INFRASTRUCTURE ONLY:
used by tests/ to check the library's hand-written adjoint, never by the
picomax_b200 product path.

The reference has no gradients, so nothing here is pinned by reference
output directly. Instead:
  * H(k) is affine in the parameters; affine_parts() returns the constant
    part and dH/dp, and tests check T + sum_p theta_p dH/dp against the pinned
    restatement pmx_oracle.hamiltonian (src/pmx_epm.cpp:56-203);
  * chi_ll_epsm() restates the (L, L) block of chi_LL (src/pmx_chi_copy.cpp:
    320-676) and eps_M with numpy arrays; tests check it against
    pmx_oracle.chi(mode="epsLL");
  * the tangents propagate dH/dp forward through full eigendecompositions
    (numpy.linalg.eigh): d lambda_n = z_n^H A z_n, dz_n = sum_m z_m
    (z_m^H A z_n) / (lambda_n - lambda_m) over non-degenerate m; tests check
    them against central finite differences of the forward functions.
The library computes the same gradients in reverse mode (a vector-Jacobian
product), so the two share no intermediate quantity.

Parameter order (as pmx_problem_params): vg[atom][shell], then lambda_S
(uniform value, or one per -us_so key ascending), then one lambda_A per
-ua_so key ascending.
"""
from __future__ import annotations

import copy
import math

import numpy as np

import pmx_oracle as O

PI = O.PI
SX = np.array([[0, 1], [1, 0]], complex)
SY = np.array([[0, -1j], [1j, 0]], complex)
SZ = np.array([[1, 0], [0, -1]], complex)


def param_vector(mat: O.Material) -> np.ndarray:
    v = [x for row in np.asarray(mat.vg) for x in row]
    if mat.uniform_us is not None:
        v.append(mat.uniform_us)
    else:
        v += [mat.us[k] for k in sorted(mat.us)]
    v += [mat.ua[k] for k in sorted(mat.ua)]
    return np.array(v, float)


def with_params(mat: O.Material, v) -> O.Material:
    m = copy.deepcopy(mat)
    v = list(np.asarray(v, float))
    vg = np.array(m.vg, float)
    na, nv = vg.shape
    m.vg = np.array(v[:na * nv]).reshape(na, nv)
    i = na * nv
    if m.uniform_us is not None:
        m.uniform_us = v[i]
        i += 1
    else:
        for k in sorted(m.us):
            m.us[k] = v[i]
            i += 1
    for k in sorted(m.ua):
        m.ua[k] = v[i]
        i += 1
    return m


def _key_index(m: dict, q2: float) -> int:
    """Index (ascending keys) of the entry soc_form_factor returns, or -1."""
    keys = sorted(m)
    if abs(q2) < 1e-2:
        return keys.index(0.0) if 0.0 in m else -1
    if not keys:
        return -1
    d = [abs(q2 - k) for k in keys]
    i = int(np.argmin(d))
    return i if d[i] < 1e-2 else -1


def affine_parts(cr: O.Crystal, mat: O.Material, G, k):
    """(T, [dH/dp]) with H = T + sum_p theta_p dH/dp (spinor, full Hermitian)."""
    G = np.asarray(G, float)
    n = len(G)
    KG = G + np.asarray(k, float)
    kin = O.KCON * (2.0 * PI / cr.a) ** 2
    I2 = np.eye(2)
    T = np.kron(np.diag(kin * (KG ** 2).sum(1)), I2).astype(complex)
    dG = G[:, None, :] - G[None, :, :]
    g2 = (dG ** 2).sum(-1)
    off = ~np.eye(n, dtype=bool)
    nv = len(mat.g2)
    shell = np.full((n, n), -1)
    for s in reversed(range(nv)):
        shell[np.abs(g2 - mat.g2[s]) < 1e-2] = s
    shell[~(g2 < mat.g2max)] = -1
    shell[~off] = -1
    natom = len(cr.atoms)
    parts = []
    for a in range(natom):
        ph = np.exp(-1j * 2.0 * PI * (dG @ cr.atoms[a]))
        for s in range(nv):
            parts.append(np.kron(np.where(shell == s, ph, 0) * O.RY2EV / natom, I2))
    # SOC: block (i, j) = i VSO(G_j - G_i) ((k+G_j) x (k+G_i)) . sigma
    q = -dG
    phq = 2.0 * PI * (q @ cr.atoms.T)  # [i, j, atom]
    cs, sn = np.cos(phq).mean(-1), np.sin(phq).mean(-1)
    s = np.cross(KG[None, :, :], KG[:, None, :])  # [i, j] = KG_j x KG_i
    sig = s[..., 0, None, None] * SX + s[..., 1, None, None] * SY + s[..., 2, None, None] * SZ  # [i, j, 2, 2]

    def soc_matrix(coef):
        M = np.zeros((2 * n, 2 * n), complex)
        blk = 1j * coef[..., None, None] * sig
        blk[~off] = 0
        for a_ in range(2):
            for b_ in range(2):
                M[a_::2, b_::2] = blk[..., a_, b_]
        return M

    kidx = np.vectorize(lambda x, which: _key_index(mat.us if which == 0 else mat.ua, x))
    if mat.uniform_us is not None:
        parts.append(soc_matrix(O.RY2EV * cs))
    else:
        ku = kidx(g2, 0)
        for i, _ in enumerate(sorted(mat.us)):
            parts.append(soc_matrix(np.where(ku == i, O.RY2EV * cs, 0.0)))
    ka = kidx(g2, 1)
    for i, _ in enumerate(sorted(mat.ua)):
        parts.append(soc_matrix(np.where(ka == i, 1j * O.RY2EV * sn, 0.0)))
    return T, parts


def hamiltonian(cr, mat, G, k):
    T, parts = affine_parts(cr, mat, G, k)
    th = param_vector(mat)
    return T + sum(t * A for t, A in zip(th, parts))


def _clusters(w, tol=1e-8):
    lab = np.zeros(len(w), int)
    for i in range(1, len(w)):
        lab[i] = lab[i - 1] + (1 if w[i] - w[i - 1] > tol else 0)
    return lab


def band_tangent(cr, mat, G, Q, nband, nvalence, refpoint=(0, 0, 0)):
    """(eband [nq][nband], d eband/dp [P][nq][nband]); inside a degenerate set
    the derivative is the set's mean (what central differences of the sorted
    eigenvalues give)."""
    def eig_d(k, nkeep):
        T, parts = affine_parts(cr, mat, G, k)
        H = T + sum(t * A for t, A in zip(param_vector(mat), parts))
        w, Z = np.linalg.eigh(H)
        lab = _clusters(w)
        d = []
        for A in parts:
            hf = np.real(np.einsum("ij,ik,kj->j", Z.conj(), A, Z))
            for c in np.unique(lab):
                sel = lab == c
                hf[sel] = hf[sel].mean()
            d.append(hf)
        return w, np.array(d)
    wr, dr = eig_d(refpoint, nvalence + 1)
    nh = len(wr)
    if 0 < nvalence < nh:
        off, doff = (wr[nvalence - 1] + wr[nvalence]) / 2, (dr[:, nvalence - 1] + dr[:, nvalence]) / 2
    else:
        off, doff = 0.0, np.zeros(len(dr))
    E = np.zeros((len(Q), nband))
    dE = np.zeros((len(dr), len(Q), nband))
    for iq, k in enumerate(Q):
        w, d = eig_d(k, nband)
        m = min(nband, len(w))
        E[iq, :m] = w[:m] - off
        dE[:, iq, :m] = d[:, :m] - doff[:, None]
    return E, dE


def _delta_and_deriv(model, eps, x):
    d = O.delta_fn(model, eps, x)
    if model == 0:
        dd = -x / (eps * eps) * d
    elif model == 1:
        dd = -2.0 * x * eps / (PI * (eps * eps + x * x) ** 2)
    elif model == 2:
        dd = np.where(np.abs(x) < 0.5 * eps, -4.0 / (eps * eps) * np.sign(x), 0.0)
    else:
        dd = np.zeros_like(x)
    return d, dd


def chi_ll_epsm(cr, mat, G, hkl, K, KW, Q, *, neps, nband, nvalence, nfreq, dfreq, epsilon, delta, kk,
                refpoint=(0, 0, 0), tangents=True, tau=1e-8):
    """(chi_LL re, im [nq][npairs][nf], eps_M [nq][nf], d eps_M/dp [P][nq][nf]).
    With tangents=False the last item is None."""
    G = np.asarray(G, float)
    npw = len(G)
    L = O.loci_table(np.asarray(hkl), neps)
    freq = dfreq * np.arange(nfreq)
    npairs = neps * (neps + 1) // 2
    pm, pn = zip(*[(m, n) for m in range(neps) for n in range(m + 1)])
    pm, pn = np.array(pm), np.array(pn)
    off = O.ref_energy(cr, mat, G, nvalence, refpoint)
    bz, acm = cr.bz_volume, cr.a * O.ANG
    SF_LL = 2.0 * bz * O.E ** 2 / (PI * O.EV * acm)
    th = param_vector(mat)
    P = len(th)
    RE = np.zeros((len(Q), npairs, nfreq))
    IM = np.zeros_like(RE)
    dRE = np.zeros((P,) + RE.shape)
    dIM = np.zeros_like(dRE)

    def solve(k):
        T, parts = affine_parts(cr, mat, G, k)
        H = T + sum(t * A for t, A in zip(th, parts))
        w, Z = np.linalg.eigh(H)
        if not tangents:
            return w, Z, None, None
        gap = w[None, :] - w[:, None]  # [m, n] = w_n - w_m
        F = np.where(np.abs(gap) > tau, 1.0 / np.where(np.abs(gap) > tau, gap, 1.0), 0.0)
        dw, dZ = [], []
        for A in parts:
            C = Z.conj().T @ A @ Z
            dw.append(np.real(np.diag(C)))
            dZ.append(Z @ (C * F))
        return w, Z, np.array(dw), np.array(dZ)

    for iq, q in enumerate(Q):
        q = np.asarray(q, float)
        qg = np.array([np.linalg.norm(q + G[m]) for m in range(neps)])
        s_im = np.zeros((npairs, nfreq))
        s_re = np.zeros_like(s_im)
        p_re = np.zeros_like(s_im)
        p_im = np.zeros_like(s_im)
        ds_im = np.zeros((P, npairs, nfreq))
        ds_re = np.zeros_like(ds_im)
        dp_re = np.zeros_like(ds_im)
        dp_im = np.zeros_like(ds_im)
        for ik, k in enumerate(K):
            wk, Zk, dwk, dZk = solve(k)
            wq, Zq, dwq, dZq = solve(np.asarray(k, float) + q)
            cs = []
            for c in range(nband):
                if wk[nband - 1 - c] - off <= 0:
                    break
                cs.append(nband - 1 - c)
            vs = []
            for v in range(nband):
                if wq[v] - off > 0:
                    break
                vs.append(v)
            if not cs or not vs:
                continue
            cs, vs = np.array(cs), np.array(vs)
            Mt = np.zeros((len(cs), len(vs), neps), complex)
            dMt = np.zeros((P, len(cs), len(vs), neps), complex)
            for m in range(neps):
                act = np.nonzero(L[m] >= 0)[0]
                lp = L[m, act]
                for s in (0, 1):
                    ck = Zk[2 * act + s][:, cs]
                    vq = Zq[2 * lp + s][:, vs]
                    Mt[:, :, m] += ck.conj().T @ vq
                    if tangents:
                        dck = dZk[:, 2 * act + s][:, :, cs]
                        dvq = dZq[:, 2 * lp + s][:, :, vs]
                        dMt[:, :, :, m] += np.einsum("prc,rv->pcv", dck.conj(), vq) + np.einsum(
                            "rc,prv->pcv", ck.conj(), dvq)
            de = wk[cs][:, None] - wq[vs][None, :]
            Ot = Mt[..., pm] * Mt[..., pn].conj()  # [c, v, pair]
            x = de[..., None] - freq  # [c, v, f]
            d, dd = _delta_and_deriv(delta, epsilon, x)
            kw = KW[ik]
            s_im += kw * np.einsum("cvp,cvf->pf", Ot.real, d)
            s_re -= kw * np.einsum("cvp,cvf->pf", Ot.imag, d)
            if kk == 0:
                den = de[..., None] ** 2 - freq ** 2
                g = de[..., None] / den
                p_re += kw * np.einsum("cvp,cvf->pf", Ot.real, g)
                p_im += kw * np.einsum("cvp,cvf->pf", Ot.imag, g)
            if tangents:
                dO = dMt[..., pm] * Mt[..., pn].conj() + Mt[..., pm] * dMt[..., pn].conj()
                dde = dwk[:, cs][:, :, None] - dwq[:, vs][:, None, :]  # [P, c, v]
                ds_im += kw * (np.einsum("Pcvp,cvf->Ppf", dO.real, d) +
                               np.einsum("cvp,cvf,Pcv->Ppf", Ot.real, dd, dde))
                ds_re -= kw * (np.einsum("Pcvp,cvf->Ppf", dO.imag, d) +
                               np.einsum("cvp,cvf,Pcv->Ppf", Ot.imag, dd, dde))
                if kk == 0:
                    gd = -(de[..., None] ** 2 + freq ** 2) / den ** 2
                    dp_re += kw * (np.einsum("Pcvp,cvf->Ppf", dO.real, g) +
                                   np.einsum("cvp,cvf,Pcv->Ppf", Ot.real, gd, dde))
                    dp_im += kw * (np.einsum("Pcvp,cvf->Ppf", dO.imag, g) +
                                   np.einsum("cvp,cvf,Pcv->Ppf", Ot.imag, gd, dde))
        f2 = SF_LL / (qg[pm] * qg[pn])
        f1 = np.zeros((npairs, nfreq))
        f1[:, 1:] = f2[:, None]
        IM[iq] = PI * s_im * f1 + (2.0 * p_im * f2[:, None] if kk == 0 else 0.0)
        RE[iq] = PI * s_re * f1 + (2.0 * p_re * f2[:, None] if kk == 0 else 0.0)
        dIM[:, iq] = PI * ds_im * f1 + (2.0 * dp_im * f2[:, None] if kk == 0 else 0.0)
        dRE[:, iq] = PI * ds_re * f1 + (2.0 * dp_re * f2[:, None] if kk == 0 else 0.0)
        if kk:
            RE[iq], IM[iq] = O.kk_transform(RE[iq], IM[iq], freq, dfreq)
            for p_ in range(P):
                dRE[p_, iq], dIM[p_, iq] = O.kk_transform(dRE[p_, iq], dIM[p_, iq], freq, dfreq)
    # eps_M and its tangent
    epsm = np.zeros((len(Q), nfreq), complex)
    depsm = np.zeros((P, len(Q), nfreq), complex)
    for iq in range(len(Q)):
        for f in range(nfreq):
            e = np.eye(neps, dtype=complex)
            de_ = np.zeros((P, neps, neps), complex)
            x = RE[iq, :, f] + 1j * IM[iq, :, f]
            dx = dRE[:, iq, :, f] + 1j * dIM[:, iq, :, f]
            e[pm, pn] += x
            de_[:, pm, pn] += dx
            od = pm != pn
            e[pn[od], pm[od]] += np.conj(x[od])
            de_[:, pn[od], pm[od]] += np.conj(dx[:, od])
            B = np.linalg.inv(e)
            em = 1.0 / B[0, 0]
            epsm[iq, f] = em
            if tangents:
                depsm[:, iq, f] = em * em * np.einsum("a,pab,b->p", B[0, :], de_, B[:, 0])
    return RE, IM, epsm, (depsm if tangents else None)
