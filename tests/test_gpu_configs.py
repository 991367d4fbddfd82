"""CUDA path against the reference at the benchmark configurations' own shapes.

Each fixture (tests/golden/cfg*.npz, made by tests/golden/make_golden.py from
the reference rebuilt from source) keeps a configuration's encut / N_G, NEPS,
frequency grid, broadening, SOC and preset, on a subset of its own k grid:

* cfg1_si_epsLL   Si epsLL, N_G 113, NEPS 15, 1000 w, Gaussian, 32 k
* cfg2_gaas_epsij GaAs + SOC epsij, n 274, NEPS 27, 2000 w, Lorentzian, 128 k
                  (more than 2048 transitions per 256-wide frequency tile:
                  the mixed path flushes its FP32 accumulator into FP64)
* cfg3_wz_epsLL   wurtzite epsLL, N_G 401, NEPS 59, 2000 w, Gaussian, 4 k
* cfg5_te_band    trigonal Te + SOC (n 570), 121-point band path
* cfg5_te_epsLL   trigonal Te + SOC epsLL, NEPS 15, 1000 w, 16 k

Large spectra are stored reduced: every row at a stride of frequencies, the
first three pair rows at every frequency, every row's sum over frequencies,
and max |value|. Tolerances: FP64 1e-8 of max |value| (band 1e-9 eV); mixed
1e-4 of max |value|; row sums at the same relative bound times the number of
frequencies.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_args, load_golden

import picomax_b200 as pm

pytestmark = pytest.mark.gpu

CHI = ["cfg1_si_epsLL", "cfg2_gaas_epsij", "cfg3_wz_epsLL", "cfg5_te_epsLL"]


def _have(name):
    return os.path.exists(os.path.join(GOLDEN, name + ".npz"))


def _switch(args):
    name = args[args.index("-switch") + 1]
    return {"epsij": pm.SWITCH_EPSIJ, "epsLL": pm.SWITCH_EPSLL, "epsxyz": pm.SWITCH_EPSXYZ}[name]


def _compare(g, re, im, tol):
    dat = np.concatenate([re.ravel(), im.ravel()])
    assert dat.size == int(g["dat_size"])
    head = g["dat_head"]
    rows = dat.reshape(head.shape[0], -1, head.shape[2])
    scale = float(g["dat_absmax"])
    nf = rows.shape[2]
    err_f = np.abs(rows[:, :, g["fsel"]] - g["dat_fsel"]).max() / scale
    err_h = np.abs(rows[:, :3, :] - head).max() / scale
    err_s = np.abs(rows.sum(axis=2) - g["dat_rowsum"]).max() / (scale * nf)
    assert abs(np.abs(dat).max() - scale) <= tol * scale
    return max(err_f, err_h, err_s)


@pytest.mark.parametrize("name", CHI)
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_config_chi_vs_reference(ctx, name, precision, tmp_path):
    if not _have(name):
        pytest.skip(f"fixture {name} not generated")
    g = load_golden(name)
    args = golden_args(g, tmp_path)
    p = pm.Problem(args)
    prec = pm.PREC_FP64 if precision == "fp64" else pm.PREC_MIXED
    re, im = ctx.chi(p, _switch(args), prec)
    tol = 1e-8 if precision == "fp64" else 1e-4
    err = _compare(g, re, im, tol)
    assert err <= tol, (name, precision, err)
    p.close()


def test_config_te_band_vs_reference(ctx, tmp_path):
    if not _have("cfg5_te_band"):
        pytest.skip("fixture cfg5_te_band not generated")
    g = load_golden("cfg5_te_band")
    p = pm.Problem(golden_args(g, tmp_path))
    eb = ctx.band(p)
    assert np.max(np.abs(eb.ravel() - g["dat"])) < 1e-9
    p.close()
