"""Merged multi-crystal launches (pmx_band_batch, pmx_chi_batch) against the
per-problem entry points on crystals of uneven size, with and without SOC."""
import numpy as np
import pytest

from conftest import golden_args, load_golden

pytestmark = pytest.mark.gpu


def _band_problems():
    import picomax_b200 as pm
    from picomax_b200.workloads import gaas_form_factors, workload, wz_form_factors
    import tempfile
    vg, soc = gaas_form_factors()
    tmp = tempfile.mkdtemp()
    si, _, _ = workload("si_band", tmp)
    gaas = ["-switch", "band", "-crystal", "zb", "-a", "5.65", "-vg", vg, "-encut", "80", "-nband", "16",
            "-nvalence", "8", "-qpath", "G,X,L", "-qnum", "7,5"] + soc
    wz = ["-switch", "band", "-crystal", "wz", "-a", "3.19", "-f", "1.626", "-u", "0.375", "-vg", wz_form_factors(),
          "-encut", "150", "-nband", "20", "-nvalence", "16", "-qvec", "0,0,0,0.2,0.1,0,0.3,0,0.2"]
    return [pm.Problem(a) for a in (si, gaas, wz)]


def test_band_batch_matches_single(ctx):
    probs = _band_problems()
    assert len({p.info.npw for p in probs}) == 3
    got = ctx.band_batch(probs)
    for p, g in zip(probs, got):
        assert np.max(np.abs(g - ctx.band(p))) < 1e-9
        p.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_chi_batch_matches_single(ctx, tmp_path, precision):
    import picomax_b200 as pm
    names = ["si_epsLL", "gaas_soc_epsij", "wz_epsij_rect"]
    probs, sws = [], []
    for nm in names:
        (tmp_path / nm).mkdir(exist_ok=True)
        args = golden_args(load_golden(nm), tmp_path / nm)
        probs.append(pm.Problem(args))
        sws.append(pm.SWITCH_EPSLL if "epsLL" in args else pm.SWITCH_EPSIJ)
    for sw in (pm.SWITCH_EPSIJ, pm.SWITCH_EPSLL):
        sel = [p for p, s in zip(probs, sws) if s == sw]
        got = ctx.chi_batch(sel, sw, precision)
        for p, (re, im) in zip(sel, got):
            r0, i0 = ctx.chi(p, sw, precision)
            scale = max(np.abs(r0).max(), np.abs(i0).max())
            tol = 1e-9 if precision == 0 else 1e-5
            assert np.max(np.abs(re - r0)) < tol * scale
            assert np.max(np.abs(im - i0)) < tol * scale
    for p in probs:
        p.close()


def test_epsm_only_outputs(ctx, tmp_path):
    """eps_M without the chi copy-out (re/im NULL): the same eps_M as with it,
    per problem and merged; NULL re with non-NULL im is rejected."""
    import ctypes
    import picomax_b200 as pm
    probs = []
    for nm in ("si_epsLL", "gaas_soc_epsLL_pv"):
        (tmp_path / nm).mkdir(exist_ok=True)
        probs.append(pm.Problem(golden_args(load_golden(nm), tmp_path / nm)))
    for precision in (0, 1):
        full = ctx.chi_batch(probs, pm.SWITCH_EPSLL, precision, epsm=True)
        only = ctx.chi_batch(probs, pm.SWITCH_EPSLL, precision, epsm=True, chi=False)
        for p, (re, im, e_full), (r2, i2, e_only) in zip(probs, full, only):
            assert r2 is None and i2 is None
            assert np.array_equal(e_full, e_only)
            _, _, e1 = ctx.chi_epsm(p, pm.SWITCH_EPSLL, precision, chi=False)
            assert np.array_equal(e1, ctx.chi_epsm(p, pm.SWITCH_EPSLL, precision)[2])
    im = np.zeros(probs[0].info.chi_values)
    eps = np.zeros((probs[0].info.nq, probs[0].info.nfreq, 2))
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    st = ctx._lib.pmx_chi_epsm(ctx.handle, probs[0].handle, pm.SWITCH_EPSLL, 0, None, dp(im), dp(eps))
    assert st == pm.PMX_ERR_INVALID
    for p in probs:
        p.close()


def test_band_batch_large_spin_orbit_sizes(ctx):
    """Spin-orbit H of n = 2 N_G around 900 next to a small crystal in one
    merged call: chunks of the two-stage solver beyond shared memory (V and Y
    in global memory) inside the captured graph, against the per-problem call
    and the oracle's spectrum."""
    import picomax_b200 as pm
    import pmx_oracle as O
    from picomax_b200.workloads import gaas_form_factors
    vg, soc = gaas_form_factors()
    rng = np.random.default_rng(23)
    K = rng.uniform(-0.5, 0.5, (3, 3))
    qv = ",".join(f"{x:.6f}" for x in K.ravel())
    big = ["-switch", "band", "-crystal", "zb", "-a", "5.65", "-vg", vg, "-encut", "275", "-qvec", qv,
           "-nband", "24", "-nvalence", "8"] + soc
    small = ["-switch", "band", "-crystal", "zb", "-a", "5.65", "-vg", vg, "-encut", "60", "-qvec", qv,
             "-nband", "16", "-nvalence", "8"] + soc
    probs = [pm.Problem(big), pm.Problem(small)]
    assert 2 * probs[0].info.npw > 832, probs[0].info.npw
    got = ctx.band_batch(probs)
    for p, g in zip(probs, got):
        assert np.max(np.abs(g - ctx.band(p))) < 1e-9
    cr, mat, gcut, o = O.from_args(big)
    G, _ = probs[0].gvectors()
    ref = O.band(cr, mat, G, probs[0].qpoints(), 24, 8)
    assert np.max(np.abs(got[0] - ref)) < 1e-9
    for p in probs:
        p.close()
