"""Pins the tangent-mode gradient oracle (oracle/pmx_oracle_grad.py): its
affine H(k) and chi_LL / eps_M restatements against the pinned oracle, and its
tangents against central finite differences of its own forward functions."""
import numpy as np
import pytest

import pmx_oracle as O
import pmx_oracle_grad as OG

K3 = np.array([[0.2, 0.35, 0.1], [0.3, -0.2, 0.1], [0.0, 0.25, -0.15], [0.45, 0.1, 0.2]])


def grad_case(tmp_path, *, soc=True, kk=1, delta=0, neps=5, nfreq=120, dfreq=0.1, extra=()):
    """A small zinc-blende problem (N_G 27): argv, oracle inputs, options."""
    import picomax_b200 as pm
    from picomax_b200.kgrid import write_kfile
    from picomax_b200.workloads import gaas_form_factors
    vg, socargs = gaas_form_factors()
    if not soc:
        socargs = []
    kf = str(tmp_path / "k.txt")
    write_kfile(kf, K3, np.ones(len(K3)))
    args = ["-switch", "epsLL", "-crystal", "zb", "-a", "5.65", "-vg", vg, "-encut", "40", "-kpoint", "0",
            "-kpointfile", kf, "-qvec", "0.01,0,0", "-neps", str(neps), "-nband", "16", "-nvalence", "8",
            "-nfreq", str(nfreq), "-dfreq", str(dfreq), "-delta", str(delta), "-epsilon", "0.2", "-kk", str(kk),
            ] + socargs + list(extra)
    cr, mat, gcut, o = O.from_args(args)
    prob = pm.Problem(args)
    G, hkl = prob.gvectors()
    K, KW = prob.kpoints()
    Q = prob.qpoints()
    prob.close()
    return args, cr, mat, G, hkl, K, KW, Q, o


@pytest.mark.parametrize("soc", [True, False])
def test_affine_parts_match_hamiltonian(tmp_path, soc):
    extra = () if soc else ("-us_so", "3:0.004,11:0.002", "-ua_so", "4:0.001")
    _, cr, mat, G, _, _, _, _, _ = grad_case(tmp_path, soc=soc, extra=extra)
    for k in ([0.1, 0.2, 0.3], [0.0, 0.0, 0.0]):
        H0 = O.hamiltonian(cr, mat, G, k)
        H1 = OG.hamiltonian(cr, mat, G, k)
        assert np.max(np.abs(H1 - H0)) < 1e-12 * np.max(np.abs(H0))
    # the parameter vector round-trips and matches the library's order
    import picomax_b200 as pm
    args, *_ = grad_case(tmp_path, soc=soc, extra=extra)
    p = pm.Problem(args)
    assert np.allclose(p.params(), OG.param_vector(mat), rtol=0, atol=1e-12)
    v = p.params() * 1.5
    p.set_params(v)
    assert np.array_equal(p.params(), v)
    p.close()


@pytest.mark.parametrize("kk,delta", [(1, 0), (0, 1)])
def test_chi_ll_restatement(tmp_path, kk, delta):
    _, cr, mat, G, hkl, K, KW, Q, o = grad_case(tmp_path, kk=kk, delta=delta)
    o["kk"], o["delta"] = kk, delta
    re, im = O.chi(cr, mat, G, hkl, K, KW, Q, mode="epsLL", **o)
    RE, IM, em, _ = OG.chi_ll_epsm(cr, mat, G, hkl, K, KW, Q, tangents=False, **o)
    scale = max(np.abs(re[0, 0]).max(), np.abs(im[0, 0]).max())
    assert np.max(np.abs(RE - re[0, 0])) < 1e-9 * scale
    assert np.max(np.abs(IM - im[0, 0])) < 1e-9 * scale
    ref = O.eps_macroscopic(re[0, 0, 0], im[0, 0, 0], o["neps"])
    assert np.max(np.abs(em[0] - ref)) < 1e-10 * np.max(np.abs(ref))


def test_band_tangent_vs_fd(tmp_path):
    _, cr, mat, G, _, _, _, _, o = grad_case(tmp_path)
    Q = np.array([[0, 0, 0], [0.25, 0.1, 0.0], [0.5, 0.5, 0.5], [1.0, 0.0, 0.0]])
    E, dE = OG.band_tangent(cr, mat, G, Q, 16, 8)
    th = OG.param_vector(mat)
    h = 1e-6
    for p in range(len(th)):
        tp, tm = th.copy(), th.copy()
        tp[p] += h
        tm[p] -= h
        Ep = O.band(cr, OG.with_params(mat, tp), G, Q, 16, 8)
        Em = O.band(cr, OG.with_params(mat, tm), G, Q, 16, 8)
        fd = (Ep - Em) / (2 * h)
        assert np.max(np.abs(fd - dE[p])) < 1e-6 * max(np.max(np.abs(fd)), 1.0)


@pytest.mark.parametrize("kk,delta", [(1, 0), (0, 1)])
def test_epsm_tangent_vs_fd(tmp_path, kk, delta):
    """Central differences against the tangent; they converge as h^2 (checked
    down to h = 1e-8 Ry). The k-points avoid the near-Gamma region, where
    spin-split pairs only ~0.1 meV apart make the eigenvector terms strongly
    curved; the principal-value case (kk 0) stays below the lowest
    transition, where de / (de^2 - w^2) is smooth. The Gaussian case
    (0.2 eV on 4 k-points) is the more curved one, hence its smaller step."""
    dfreq = 0.1 if kk else 0.015
    _, cr, mat, G, hkl, K, KW, Q, o = grad_case(tmp_path, kk=kk, delta=delta, dfreq=dfreq)
    o["kk"], o["delta"] = kk, delta
    _, _, em, dem = OG.chi_ll_epsm(cr, mat, G, hkl, K, KW, Q, **o)
    th = OG.param_vector(mat)
    h = 1e-7 if kk else 1e-6
    scale = np.max(np.abs(dem))
    for p in range(len(th)):
        tp, tm = th.copy(), th.copy()
        tp[p] += h
        tm[p] -= h
        ep = OG.chi_ll_epsm(cr, OG.with_params(mat, tp), G, hkl, K, KW, Q, tangents=False, **o)[2]
        emn = OG.chi_ll_epsm(cr, OG.with_params(mat, tm), G, hkl, K, KW, Q, tangents=False, **o)[2]
        fd = (ep - emn) / (2 * h)
        assert np.max(np.abs(fd - dem[p])) < 2e-6 * max(np.max(np.abs(fd)), 1e-3 * scale)
