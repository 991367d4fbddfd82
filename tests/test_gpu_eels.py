"""EELS loss function -Im(1/eps_M) and plasmon peaks (pmx_eels) against the
numpy restatement: on eps_M of the reference's own chi_LL spectrum (golden
fixture), and as a plasmon dispersion along a q line against the oracle's
chi_LL. Tolerances: loss 1e-12 of its maximum; peak energies 1e-9 eV on the
same eps_M, 1e-5 eV against the oracle's spectra (chi agrees to 1e-8)."""
import os

import numpy as np
import pytest

from conftest import golden_args, load_golden

import picomax_b200 as pm
import pmx_oracle as O

pytestmark = pytest.mark.gpu


def test_eels_on_reference_chi(ctx, tmp_path):
    g = load_golden("si_epsLL")
    p = pm.Problem(golden_args(g, tmp_path))
    neps, nf, dfreq = p.info.neps, p.info.nfreq, p.info.dfreq
    npairs = neps * (neps + 1) // 2
    n = g["dat"].size // 2
    re = g["dat"][:n].reshape(3, 3, 1, npairs, nf)[0, 0]
    im = g["dat"][n:].reshape(3, 3, 1, npairs, nf)[0, 0]
    epsm = O.eps_macroscopic(re[0], im[0], neps)[None]
    loss, peak = ctx.eels(epsm, dfreq, wmin=1.0)
    ref = O.loss_function(epsm)
    assert np.abs(loss - ref).max() <= 1e-12 * np.abs(ref).max()
    w, h = O.plasmon_peak(ref[0], dfreq, int(np.ceil(1.0 / dfreq - 1e-9)))
    assert abs(peak[0, 0] - w) < 1e-9 and abs(peak[0, 1] - h) <= 1e-12 * abs(h)
    p.close()


def test_plasmon_dispersion_vs_oracle(ctx, tmp_path):
    from picomax_b200.kgrid import gamma_grid, write_kfile
    K, W = gamma_grid("zb", 3, 3, 3)
    kf = os.path.join(str(tmp_path), "k.txt")
    write_kfile(kf, K, W)
    qs = np.array([[0.05, 0, 0], [0.1, 0, 0], [0.15, 0, 0], [0.2, 0, 0]])
    args = ("-switch epsLL -crystal zb -a 5.43 -vg 3,4,8,11,-0.21,0,0.04,0.08,-0.21,0,0.04,0.08 -encut 60 "
            "-nband 16 -nvalence 8 -neps 3 -nfreq 300 -dfreq 0.1 -delta 0 -epsilon 0.5 -kk 1 -kpoint 0").split()
    args += ["-kpointfile", kf, "-qvec", ",".join(f"{x:.6f}" for x in qs.ravel())]
    p = pm.Problem(args)
    nf, dfreq, neps = p.info.nfreq, p.info.dfreq, p.info.neps
    re, im, epsm = ctx.chi_epsm(p, pm.SWITCH_EPSLL, pm.PREC_FP64)
    loss, peak = ctx.eels(epsm, dfreq, wmin=5.0)
    assert peak.shape == (4, 2) and np.all(peak[:, 0] > 5.0)
    # the same eps_M on the host: loss and peaks of the restatement
    ref_loss = O.loss_function(epsm)
    assert np.abs(loss - ref_loss).max() <= 1e-12 * np.abs(ref_loss).max()
    # chi_LL of the oracle for the four q: its eps_M and plasmon peaks
    cr, mat, gcut, o = O.from_args(args)
    G, hkl = p.gvectors()  # the reference's G order (bit-exact in the library): fixes the local-field set
    ore, oim = O.chi(cr, mat, G, hkl, K, np.ones(len(K)) / len(K), qs, mode="epsLL", **o)
    npairs = neps * (neps + 1) // 2
    for iq in range(4):
        e = O.eps_macroscopic(ore[0, 0, iq], oim[0, 0, iq], neps)
        w, h = O.plasmon_peak(O.loss_function(e), dfreq, 50)
        assert abs(peak[iq, 0] - w) < 1e-5, (iq, peak[iq], w)
    p.close()
