"""CPU restatement (numpy) of the reference's EPM band solve and chi(q, w)
accumulation. TEST INFRASTRUCTURE ONLY: used by tests/, by the smoke check and
by bench.py's CPU baseline, never by the picomax_b200 product path.

Pinned against the reference rebuilt from source (oracle/Makefile ->
oracle/_ref) through the golden fixtures in tests/golden/ (made by
tests/golden/make_golden.py): band energies, epsij and epsLL spectra, with and
without spin-orbit coupling.

Every function cites the reference lines it restates. Where the reference
reads options, this module takes the already-parsed lists (G order, k/q
lists, form factors) so that it exercises only the physics: the integer tables
are checked separately against the reference's own -debug 3 dumps and .gpt.
The Hermitian eigensolve uses numpy.linalg.eigh in place of
Eigen::SelfAdjointEigenSolver (both return ascending eigenvalues).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

PI = 3.14159265358979323846
HBAR = 1.054571817e-27
E = 4.803204712570263e-10
EM = 9.1093837015e-28
EV = 1.602176634e-12
RY2EV = 13.605699169854621
ANG = 1e-8
KCON = 3.809982111485962


@dataclass
class Crystal:
    """Preset of init_crystal (src/pmx_io.cpp:126-209)."""
    name: str
    a: float
    f: float = math.sqrt(8.0 / 3.0)
    u: float = 3.0 / 8.0
    recip: np.ndarray = field(init=False)
    atoms: np.ndarray = field(init=False)
    bz_volume: float = field(init=False)

    def __post_init__(self):
        s3 = math.sqrt(3.0)
        if self.name in ("zb", "rs"):
            self.recip = np.array([[-1, 1, 1], [1, -1, 1], [1, 1, -1]], float)
            self.bz_volume = 4.0
            tau = [[0, 0, 0], [0.25, 0.25, 0.25]] if self.name == "zb" else [[0, 0, 0], [0.5, 0, 0]]
        elif self.name in ("wz", "te"):
            f, u = self.f, self.u
            self.recip = np.array([[1, -1 / s3, 0], [1, 1 / s3, 0], [0, 0, 1.0 / f]], float)
            self.bz_volume = abs(np.dot(np.cross(self.recip[0], self.recip[1]), self.recip[2]))
            if self.name == "wz":
                tau = [[0.5, 0.5 / s3, 0], [0.5, -0.5 / s3, 0.5 * f], [0.5, 0.5 / s3, u * f],
                       [0.5, -0.5 / s3, (0.5 + u) * f]]
            else:
                tau = [[0, 0.5 * s3 * u, -1.0 / 3.0 * f], [1.5 * u, 0, 0], [0, -0.5 * s3 * u, 1.0 / 3.0 * f]]
        else:
            raise ValueError(self.name)
        self.atoms = np.array(tau, float)


@dataclass
class Material:
    """Form factors of init_mater (src/pmx_io.cpp:315-417), Ry."""
    g2: list
    vg: np.ndarray               # [natom][nv]
    us: dict = field(default_factory=dict)
    ua: dict = field(default_factory=dict)
    uniform_us: float | None = None

    @property
    def g2max(self):
        return self.g2[-1] + 1e-2


def soc_form_factor(m: dict, q2: float) -> float:
    """get_soc_form_factor (src/pmx_epm.cpp:22-50)."""
    if abs(q2) < 1e-2:
        return m.get(0.0, 0.0)
    best, key = float("inf"), None
    for k in sorted(m):
        d = abs(q2 - k)
        if d < best:
            best, key = d, k
    return m[key] if key is not None and best < 1e-2 else 0.0


def local_potential(cr: Crystal, mat: Material, dG) -> complex:
    """pseudopotential (src/pmx_epm.cpp:171-203), eV; 0 beyond g2max."""
    g2 = float(np.dot(dG, dG))
    if not g2 < mat.g2max:
        return 0j
    idx = next((k for k, v in enumerate(mat.g2) if abs(v - g2) < 1e-2), None)
    if idx is None:
        return 0j
    v = sum(np.exp(-1j * 2.0 * PI * np.dot(dG, t)) * mat.vg[s][idx] for s, t in enumerate(cr.atoms))
    return v / len(cr.atoms) * RY2EV


def soc_scalar(cr: Crystal, mat: Material, q, uniform_ok=True) -> complex:
    """lambda_S cos_sum + i lambda_A sin_sum of src/pmx_epm.cpp:88-118 (H) and
    src/pmx_chi.cpp:209-232 (current, which ignores -use_uniform_us_so)."""
    q2 = float(np.dot(q, q))
    ls = mat.uniform_us if (uniform_ok and mat.uniform_us is not None) else soc_form_factor(mat.us, q2)
    la = soc_form_factor(mat.ua, q2)
    ph = 2.0 * PI * (cr.atoms @ q)
    return ls * RY2EV * np.cos(ph).mean() + 1j * la * RY2EV * np.sin(ph).mean()


def hamiltonian(cr: Crystal, mat: Material, G: np.ndarray, k) -> np.ndarray:
    """Spinor H(k) of HamiltonianEPM (src/pmx_epm.cpp:56-153), returned as the
    full Hermitian matrix whose lower triangle is the reference's."""
    n = len(G)
    kin = KCON * (2.0 * PI / cr.a) ** 2
    H = np.zeros((2 * n, 2 * n), complex)
    KG = G + np.asarray(k, float)
    sx = np.array([[0, 1], [1, 0]], complex)
    sy = np.array([[0, -1j], [1j, 0]], complex)
    sz = np.array([[1, 0], [0, -1]], complex)
    for i in range(n):
        for j in range(i + 1):
            if i == j:
                h0 = kin * float(np.dot(KG[i], KG[i]))
            else:
                h0 = local_potential(cr, mat, G[i] - G[j])
            blk = h0 * np.eye(2, dtype=complex)
            if i != j:
                vso = soc_scalar(cr, mat, G[j] - G[i])
                if vso != 0:
                    s = 1j * vso * np.cross(KG[j], KG[i])
                    blk = blk + s[0] * sx + s[1] * sy + s[2] * sz
            H[2 * i:2 * i + 2, 2 * j:2 * j + 2] = blk
    low = np.tril(H)
    return low + np.conj(np.tril(H, -1)).T


def ref_energy(cr, mat, G, nvalence: int, refpoint=(0, 0, 0)) -> float:
    """setRefEnergy (src/pmx_epm.cpp:393-428)."""
    w = np.linalg.eigvalsh(hamiltonian(cr, mat, G, refpoint))
    if not (0 < nvalence < len(w)):
        return 0.0
    return (w[nvalence - 1] + w[nvalence]) / 2.0


def band(cr, mat, G, Q, nband: int, nvalence: int, refpoint=(0, 0, 0)) -> np.ndarray:
    """empiricalpseudopotentialmethod (src/pmx_epm.cpp:219-253): [NQ][NBAND] eV."""
    off = ref_energy(cr, mat, G, nvalence, refpoint)
    out = np.zeros((len(Q), nband))
    for q, k in enumerate(Q):
        w = np.linalg.eigvalsh(hamiltonian(cr, mat, G, k))
        m = min(nband, len(w))
        out[q, :m] = w[:m] - off
    return out


def uvec_lt(v) -> np.ndarray:
    """[L, (T+iP)/sqrt2, (T-iP)/sqrt2] of uvec_LT (src/pmx_basis.cpp:798-874)."""
    v = np.asarray(v, float)
    nv = np.linalg.norm(v)
    l = np.array([0, 0, 1.0]) if nv == 0 else v / nv
    if v[1] != 0:
        t = np.array([-v[1], v[0], 0.0])
    elif v[2] != 0:
        t = np.array([v[2], 0.0, -v[0]])
    else:
        t = np.array([0, 1.0, 0])
    t = t / np.linalg.norm(t)
    t = t - np.dot(l, t) * l
    t = t / np.linalg.norm(t)
    p = np.cross(l, t)
    p = p / np.linalg.norm(p)
    return np.array([l + 0j, (t + 1j * p) / math.sqrt(2), (t - 1j * p) / math.sqrt(2)])


def soc_current(cr, mat, q) -> np.ndarray:
    """socCurrent (src/pmx_chi.cpp:203-266)."""
    vso = soc_scalar(cr, mat, q, uniform_ok=False)
    I = 1j
    return np.array([I * vso * (q[1] + I * q[2]), I * vso * (q[2] - q[0]), I * vso * (-I * q[0] - q[1])])


def loci_table(hkl: np.ndarray, neps: int) -> np.ndarray:
    """generate_loci (src/pmx_basis.cpp:142-179) by integer hkl identity."""
    where = {tuple(h): i for i, h in enumerate(hkl)}
    L = np.full((neps, len(hkl)), -1, np.int64)
    for m in range(neps):
        for p in range(len(hkl)):
            L[m, p] = where.get(tuple(hkl[p] + hkl[m]), -1)
    return L


def delta_fn(model: int, eps: float, x):
    """diracdelta_* (src/pmx_chi.cpp:90-164): 0 gauss, 1 lorentz, 2 triangle, 3 rect."""
    x = np.asarray(x, float)
    if model == 0:
        return np.exp(-0.5 * x * x / (eps * eps)) / (eps * math.sqrt(2.0 * PI))
    if model == 1:
        return eps / PI / (eps ** 2 + x ** 2)
    if model == 2:
        return np.where(np.abs(x) < 0.5 * eps, 4.0 / eps * (0.5 - np.abs(x) / eps), 0.0)
    return np.where(np.abs(x) < 0.5 * eps, 1.0 / eps, 0.0)


def kk_transform(re: np.ndarray, im: np.ndarray, freq: np.ndarray, dw: float):
    """kramerskronigtransform (src/pmx_chi.cpp:272-309), on the last axis."""
    w = np.asarray(freq, float)
    with np.errstate(divide="ignore", invalid="ignore"):
        K = w[None, :] / (w[None, :] ** 2 - w[:, None] ** 2)  # K[f, s]
    np.fill_diagonal(K, 0.0)
    ds = dw * 2.0 / PI
    return re + ds * (im @ K.T), im + ds * (re @ K.T)


def _eig_k(cr, mat, G, k):
    w, v = np.linalg.eigh(hamiltonian(cr, mat, G, k))
    return w, v


def chi(cr: Crystal, mat: Material, G, hkl, K, KW, Q, *, mode: str, neps: int, nband: int,
        nvalence: int, nfreq: int, dfreq: float, epsilon: float, delta: int, kk: int,
        refpoint=(0, 0, 0)):
    """chi_tensor (mode 'epsij', src/pmx_chi.cpp:319-713) or chi_LL (mode
    'epsLL', src/pmx_chi_copy.cpp:320-676). Returns (re, im) each
    [3, 3, NQ, npairs, NFREQ] in .dat order."""
    G = np.asarray(G, float)
    npw = len(G)
    L = loci_table(np.asarray(hkl), neps)
    off = ref_energy(cr, mat, G, nvalence, refpoint)
    freq = dfreq * np.arange(nfreq)
    npairs = neps * (neps + 1) // 2
    RE = np.zeros((3, 3, len(Q), npairs, nfreq))
    IM = np.zeros_like(RE)
    bz, acm = cr.bz_volume, cr.a * ANG
    SF = 4.0 * bz * PI ** 5 * HBAR ** 4 * E ** 2 / (EV ** 3 * EM ** 2 * acm ** 5)
    SF_LL = 2.0 * bz * E ** 2 / (PI * EV * acm)
    SF_TT = 32.0 * bz * PI ** 3 * HBAR ** 4 * E ** 2 / (EV ** 3 * EM ** 2 * acm ** 5)
    SF_LT = 8.0 * bz * PI * HBAR ** 2 * E ** 2 / (EV ** 2 * EM * acm ** 3)
    # conduction states at k (top of the NBAND window down while E > 0)
    kst = []
    for k in K:
        w, v = _eig_k(cr, mat, G, k)
        ec = []
        for c in range(nband):
            e = w[nband - 1 - c] - off
            if e <= 0:
                break
            ec.append(e)
        kst.append((np.array(ec), v[:, [nband - 1 - c for c in range(len(ec))]]))
    W_g = max(1, int(6.0 * epsilon / dfreq))
    W_l = max(1, int(50.0 * epsilon / dfreq))
    Wh = W_l if delta == 1 else W_g
    for iq, q in enumerate(Q):
        q = np.asarray(q, float)
        U = [uvec_lt(q + G[m]) for m in range(neps)]
        qgn = [np.linalg.norm(q + G[m]) for m in range(neps)]
        vs = [soc_current(cr, mat, G[m]) for m in range(neps)]
        trans = []  # (kw, dE, M[ch][3][neps])
        for ik, k in enumerate(K):
            w, v = _eig_k(cr, mat, G, np.asarray(k) + q)
            ev = []
            for vv in range(nband):
                e = w[vv] - off
                if e > 0:
                    break
                ev.append(e)
            ec, cvec = kst[ik]
            for c in range(len(ec)):
                cu, cd = cvec[0::2, c], cvec[1::2, c]
                for vv in range(len(ev)):
                    vu, vd = v[0::2, vv], v[1::2, vv]
                    if mode == "epsij":
                        M = np.zeros((4, 3, neps), complex)
                    else:
                        M = np.zeros((1, 3, neps), complex)
                    for m in range(neps):
                        act = np.nonzero(L[m] >= 0)[0]
                        lp = L[m, act]
                        orbv = G[act] + np.asarray(k) + q / 2 + G[m] / 2
                        for i in range(3):
                            orb = orbv @ np.conj(U[m][i])
                            s = np.dot(np.conj(U[m][i]), vs[m])
                            uu = np.conj(cu[act]) * vu[lp]
                            dd = np.conj(cd[act]) * vd[lp]
                            if mode == "epsij":
                                M[0, i, m] = np.sum(uu * orb)
                                M[1, i, m] = np.sum(dd * orb)
                                M[2, i, m] = np.sum(np.conj(cu[act]) * vd[lp] * s)
                                M[3, i, m] = np.sum(np.conj(cd[act]) * vu[lp] * s)
                            elif i == 0:
                                M[0, i, m] = np.sum(uu + dd)
                            else:
                                M[0, i, m] = np.sum((uu + dd) * (orb + s))
                    trans.append((KW[ik], ec[c] - ev[vv], M))
        for i in range(3):
            for j in range(3):
                pidx = 0
                for m in range(neps):
                    for n in range(m + 1):
                        s_im = np.zeros(nfreq)
                        s_re = np.zeros(nfreq)
                        p_re = np.zeros(nfreq)
                        p_im = np.zeros(nfreq)
                        for kw, de, M in trans:
                            if mode == "epsij":
                                up_i, dn_i, ud_i, du_i = M[:, i, m]
                                up_j, dn_j, ud_j, du_j = np.conj(M[:, j, n])
                                t = up_i * up_j + dn_i * dn_j - ud_i * ud_j - du_i * du_j
                                reO = t.real + (up_i * dn_j + dn_i * up_j - du_i * ud_j - ud_i * du_j).real
                                imO = t.imag
                                f0 = int((de - freq[0]) / dfreq)
                                lo, hi = max(0, f0 - Wh), min(nfreq - 1, f0 + Wh)
                                if lo > hi:
                                    continue
                                d = delta_fn(delta, epsilon, de - freq[lo:hi + 1])
                                s_im[lo:hi + 1] += kw * reO * d
                                s_re[lo:hi + 1] -= kw * imO * d
                            else:
                                O = M[0, i, m] * np.conj(M[0, j, n])
                                d = delta_fn(delta, epsilon, de - freq)
                                s_im += kw * O.real * d
                                s_re -= kw * O.imag * d
                                if kk == 0:
                                    den = de * de - freq * freq
                                    if i == 0 and j == 0:
                                        g = de / den
                                    elif i == 0 or j == 0:
                                        g = 1.0 / den
                                    else:
                                        g = 1.0 / de / den
                                    p_re += kw * O.real * g
                                    p_im += kw * O.imag * g
                        if mode == "epsij":
                            inv = np.zeros(nfreq)
                            inv[1:] = 1.0 / freq[1:] ** 2
                            IM[i, j, iq, pidx] = SF * (s_im * inv)
                            RE[i, j, iq, pidx] = SF * (s_re * inv)
                        else:
                            f1 = np.zeros(nfreq)
                            if i == 0 and j == 0:
                                f1[1:] = SF_LL / (qgn[m] * qgn[n])
                                f2 = SF_LL / (qgn[m] * qgn[n])
                            elif i == 0:
                                f1[1:] = SF_LT / (qgn[m] * freq[1:])
                                f2 = SF_LT / qgn[m]
                            elif j == 0:
                                f1[1:] = SF_LT / qgn[n]
                                f2 = SF_LT / qgn[n]
                            else:
                                f1[1:] = SF_TT / freq[1:] ** 2
                                f2 = SF_TT
                            IM[i, j, iq, pidx] = PI * s_im * f1 + (2.0 * p_im * f2 if kk == 0 else 0.0)
                            RE[i, j, iq, pidx] = PI * s_re * f1 + (2.0 * p_re * f2 if kk == 0 else 0.0)
                        pidx += 1
        if kk:
            RE[:, :, iq], IM[:, :, iq] = kk_transform(RE[:, :, iq], IM[:, :, iq], freq, dfreq)
    return RE, IM


def chi_xyz(cr: Crystal, mat: Material, G, hkl, K, KW, Q, *, neps: int, nband: int, nvalence: int, nfreq: int,
            dfreq: float, epsilon: float, delta: int, kk: int, refpoint=(0, 0, 0)):
    """chi_xyz (src/pmx_chi_copy.cpp:1070-1303, switch epsxyz): Cartesian
    current-current tensor. Valence states at k (counted up while E - E_ref
    <= 0), conduction states at k+q (counted down from the top of the NBAND
    window while E - E_ref > 0); the overlap multiplies the first NPW
    components of the spinor eigenvectors (the reference's
    eigenvectors().col(v)(p), p < NPW) with the orbital current
    e_i . (G_p + k + q/2 + G_m/2); SCALEFACTOR of the TT block, PV term
    1 / dE / (dE^2 - w^2) when kk = 0. Because component p is paired with plane
    wave loci[m][p], the result depends on the full G order: G must be the
    reference's (pmx_problem_gvectors), not gvectors() of this module.
    Returns (re, im) [3, 3, NQ, npairs, NFREQ]."""
    G = np.asarray(G, float)
    npw = len(G)
    L = loci_table(np.asarray(hkl), neps)
    off = ref_energy(cr, mat, G, nvalence, refpoint)
    freq = dfreq * np.arange(nfreq)
    npairs = neps * (neps + 1) // 2
    RE = np.zeros((3, 3, len(Q), npairs, nfreq))
    IM = np.zeros_like(RE)
    acm = cr.a * ANG
    SF = 32.0 * cr.bz_volume * PI ** 3 * HBAR ** 4 * E ** 2 / (EV ** 3 * EM ** 2 * acm ** 5)
    kst = []
    for k in K:
        w, v = _eig_k(cr, mat, G, k)
        ev = []
        for vv in range(nband):
            e = w[vv] - off
            if e > 0:
                break
            ev.append(e)
        kst.append((np.array(ev), v[:npw, :len(ev)]))
    for iq, q in enumerate(Q):
        q = np.asarray(q, float)
        trans = []  # (kw, dE, oint[3][neps])
        for ik, k in enumerate(K):
            w, v = _eig_k(cr, mat, G, np.asarray(k) + q)
            ec = []
            for c in range(nband):
                e = w[nband - 1 - c] - off
                if e <= 0:
                    break
                ec.append(e)
            cq = v[:npw, [nband - 1 - c for c in range(len(ec))]]
            evk, ck = kst[ik]
            for vv in range(len(evk)):
                for c in range(len(ec)):
                    O = np.zeros((3, neps), complex)
                    for m in range(neps):
                        act = np.nonzero(L[m] >= 0)[0]
                        orbv = G[act] + np.asarray(k) + q / 2 + G[m] / 2
                        prod = np.conj(ck[act, vv]) * cq[L[m, act], c]
                        for i in range(3):
                            O[i, m] = np.sum(prod * orbv[:, i])
                    trans.append((KW[ik], ec[c] - evk[vv], O))
        for i in range(3):
            for j in range(3):
                pidx = 0
                for m in range(neps):
                    for n in range(m + 1):
                        s_im = np.zeros(nfreq)
                        s_re = np.zeros(nfreq)
                        p_re = np.zeros(nfreq)
                        p_im = np.zeros(nfreq)
                        for kw, de, O in trans:
                            o = O[i, m] * np.conj(O[j, n])
                            d = delta_fn(delta, epsilon, de - freq)
                            s_im += kw * o.real * d
                            s_re -= kw * o.imag * d
                            if kk == 0:
                                g = 1.0 / de / (de * de - freq * freq)
                                p_re += kw * o.real * g
                                p_im += kw * o.imag * g
                        inv = np.zeros(nfreq)
                        inv[1:] = 1.0 / freq[1:] ** 2
                        IM[i, j, iq, pidx] = SF * (PI * s_im * inv + 2.0 * p_im)
                        RE[i, j, iq, pidx] = SF * (PI * s_re * inv + 2.0 * p_re)
                        pidx += 1
        if kk:
            RE[:, :, iq], IM[:, :, iq] = kk_transform(RE[:, :, iq], IM[:, :, iq], freq, dfreq)
    return RE, IM


def eps_macroscopic(chi_ll_re: np.ndarray, chi_ll_im: np.ndarray, neps: int) -> np.ndarray:
    """eps_M(w) = 1 / [eps^-1]_00 with eps_mn = delta_mn + chi^LL_mn, Hermitian
    fill of the stored n <= m half (include/matlab_wrapper/+picomax/+eps/
    macroscopic.m:13-29, :79). chi_ll_* are [npairs, nf]; returns [nf] complex."""
    nf = chi_ll_re.shape[-1]
    out = np.zeros(nf, complex)
    for f in range(nf):
        e = np.eye(neps, dtype=complex)
        p = 0
        for m in range(neps):
            for n in range(m + 1):
                val = chi_ll_re[p, f] + 1j * chi_ll_im[p, f]
                e[m, n] += val
                if m != n:
                    e[n, m] += np.conj(val)
                p += 1
        out[f] = 1.0 / np.linalg.inv(e)[0, 0]
    return out


def loss_function(epsm: np.ndarray) -> np.ndarray:
    """EELS loss -Im(1 / eps_M) of eps_M (macroscopic.m:79 gives eps_M; the
    loss is its standard use, the reference's C++ has no counterpart)."""
    return -np.imag(1.0 / np.asarray(epsm, complex))


def plasmon_peak(loss: np.ndarray, dfreq: float, fmin: int = 0):
    """(energy, height) of the largest loss at frequency index >= fmin (lowest
    index on ties), refined by the vertex of the parabola through the peak and
    its two neighbours when they bracket a strict maximum."""
    L = np.asarray(loss, float)
    i = fmin + int(np.argmax(L[fmin:]))
    w, h = i * dfreq, L[i]
    if 0 < i < len(L) - 1:
        ym, y0, yp = L[i - 1], L[i], L[i + 1]
        den = ym - 2.0 * y0 + yp
        if den < 0:
            t = 0.5 * (ym - yp) / den
            w, h = (i + t) * dfreq, y0 - 0.25 * (ym - yp) * t
    return w, h


# ------------------------------------------------------- symmetry of k grids
def point_group_ops(cr: Crystal, species, time_reversal: bool = True) -> np.ndarray:
    """Operations M (integer, reciprocal basis: hkl' = M hkl) of the crystal's
    point group found by mapping atoms: a lattice operation R = B M B^-1
    (|M_ij| <= 1, R orthogonal) is kept when some translation t sends every
    atom tau_s to an atom of the same species modulo the lattice. With time
    reversal -M is added for every M. Restated independently of the library's
    search, which tests the form-factor tables instead (equal results for
    Hamiltonians without spin-orbit coupling). Returns [nops, 3, 3], sorted."""
    Bm = cr.recip.T                       # columns b_j
    Bi = np.linalg.inv(Bm)
    atoms = np.asarray(cr.atoms, float)
    species = list(species)
    out = []
    vals = (-1, 0, 1)
    for code in range(3 ** 9):
        M = np.array([vals[(code // 3 ** e) % 3] for e in range(9)], float).reshape(3, 3)
        R = Bm @ M @ Bi
        if not np.allclose(R.T @ R, np.eye(3), atol=1e-9):
            continue
        found = False
        for j in range(len(atoms)):
            t = atoms[j] - R @ atoms[0]
            ok = True
            for s_ in range(len(atoms)):
                img = R @ atoms[s_] + t
                hit = False
                for s2 in range(len(atoms)):
                    if species[s2] != species[s_]:
                        continue
                    frac = (img - atoms[s2]) @ cr.recip.T   # coordinates along a_i (a_i . b_j = delta_ij)
                    if np.allclose(frac, np.round(frac), atol=1e-9):
                        hit = True
                        break
                if not hit:
                    ok = False
                    break
            if ok:
                found = True
                break
        if found:
            out.append(M.astype(int))
    if time_reversal:
        out = out + [-m for m in out]
    uniq = sorted({tuple(m.ravel()) for m in out})
    return np.array(uniq, int).reshape(-1, 3, 3)


def ibz_reduce(ops, n):
    """Irreducible points of the Gamma-centred grid k = sum_j i_j / n_j b_j
    under the operations `ops` ([nops, 3, 3] integer, a group that maps the
    grid onto itself): each point's representative is the smallest linear
    index i0 + n0 (i1 + n1 i2) of its orbit. Returns (idx [nirr, 3] in index
    order, orbit sizes [nirr])."""
    n = np.asarray(n, np.int64)
    N = int(n.prod())
    L = np.arange(N, dtype=np.int64)
    i = np.stack([L % n[0], (L // n[0]) % n[1], L // (n[0] * n[1])])
    rep = L.copy()
    for M in np.asarray(ops, np.int64):
        j = np.mod(M @ i, n[:, None])
        rep = np.minimum(rep, j[0] + n[0] * (j[1] + n[1] * j[2]))
    w = np.bincount(rep, minlength=N)
    reps = np.nonzero(rep == L)[0]
    idx = np.stack([reps % n[0], (reps // n[0]) % n[1], reps // (n[0] * n[1])], 1)
    return idx.astype(np.int32), w[reps].astype(np.int32)


# ----------------------------------------------------------------- inputs
def gvectors(cr: Crystal, gcut: float, first=None):
    """G list of generate_gpt (src/pmx_basis.cpp:29-81): every integer
    combination with |G| <= gcut + 1e-6, by increasing |G|. The reference's
    order inside a shell comes from std::sort; `first` (an [n,3] array, e.g.
    the reference's .gpt) pins the order of the leading entries, which is all
    the chi layout depends on."""
    imax = int(math.ceil(gcut))
    r = np.arange(-imax, imax + 1)
    hkl = np.array(np.meshgrid(r, r, r, indexing="ij")).reshape(3, -1).T
    G = hkl @ cr.recip
    nrm = np.linalg.norm(G, axis=1)
    keep = nrm <= gcut + 1e-6
    hkl, G, nrm = hkl[keep], G[keep], nrm[keep]
    order = np.argsort(nrm, kind="stable")
    hkl, G = hkl[order], G[order]
    if first is not None:
        first = np.asarray(first, float).reshape(-1, 3)
        idx = [int(np.argmin(np.linalg.norm(G - g, axis=1))) for g in first]
        rest = [i for i in range(len(G)) if i not in set(idx)]
        hkl, G = hkl[idx + rest], G[idx + rest]
    return G, hkl


def from_args(args):
    """Crystal, Material and the numeric options of a picomax argv (the subset
    of inputProcess/init_crystal/init_mater, src/pmx_io.cpp:108-503, that the
    chi and band stages consume)."""
    a = list(args)

    def val(flag, default=None):
        return a[a.index(flag) + 1] if flag in a else default

    cr = Crystal(val("-crystal"), float(val("-a")), float(val("-f", math.sqrt(8.0 / 3.0))),
                 float(val("-u", 3.0 / 8.0)))
    natom = len(cr.atoms)
    vals = [float(x) for x in val("-vg").split(",")]
    nv = len(vals) // (natom + 1)
    vg = np.array(vals[nv:]).reshape(natom, nv)
    mat = Material(g2=vals[:nv], vg=vg)
    if "-use_uniform_us_so" in a:
        mat.uniform_us = float(val("-uniform_us_so_val", 0.0))
    elif "-us_so" in a:
        mat.us = {float(p.split(":")[0]): float(p.split(":")[1]) for p in val("-us_so").split(",")}
    if "-ua_so_val_g0" in a:
        mat.ua[0.0] = float(val("-ua_so_val_g0"))
    if "-ua_so" in a:
        mat.ua.update({float(p.split(":")[0]): float(p.split(":")[1]) for p in val("-ua_so").split(",")})
    encut = float(val("-encut", 200))
    gcut = float(val("-gcut", math.sqrt(encut * (cr.a / 2.0 / PI) ** 2 / KCON)))
    opts = dict(neps=int(val("-neps", 1)), nband=int(val("-nband", 8)), nvalence=int(val("-nvalence", 4)),
                nfreq=int(val("-nfreq", 1)), dfreq=float(val("-dfreq", 0.0)), epsilon=float(val("-epsilon", 0.1)),
                delta=int(val("-delta", 0)), kk=int(val("-kk", 0)))
    return cr, mat, gcut, opts
