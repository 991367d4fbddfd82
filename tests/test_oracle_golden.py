"""Pins the numpy restatement (oracle/pmx_oracle.py) against the reference
rebuilt from source, through the golden fixtures."""
import numpy as np
import pytest

from conftest import arg_value, load_golden

import pmx_oracle as O


def _args(g):
    return [str(x) for x in g["argv"]]


def test_oracle_band_si():
    g = load_golden("si_band")
    args = _args(g)
    cr, mat, gcut, o = O.from_args(args)
    G, _ = O.gvectors(cr, gcut)
    assert len(G) == 113
    import picomax_b200 as pm
    Q = pm.Problem(args).qpoints()
    eb = O.band(cr, mat, G, Q, o["nband"], o["nvalence"])
    ref = g["dat"].reshape(len(Q), o["nband"])
    assert np.max(np.abs(eb - ref)) < 1e-9


def test_oracle_band_gaas_soc():
    g = load_golden("gaas_soc_band")
    args = _args(g)
    cr, mat, gcut, o = O.from_args(args)
    G, _ = O.gvectors(cr, gcut)
    import picomax_b200 as pm
    Q = pm.Problem(args).qpoints()
    eb = O.band(cr, mat, G, Q, o["nband"], o["nvalence"])
    assert np.max(np.abs(eb - g["dat"].reshape(eb.shape))) < 1e-9


@pytest.mark.parametrize("name", ["si_epsij", "gaas_soc_epsij", "si_epsLL", "gaas_soc_epsLL_pv", "wz_epsij_rect"])
def test_oracle_chi(name):
    g = load_golden(name)
    args = _args(g)
    cr, mat, gcut, o = O.from_args(args)
    G, hkl = O.gvectors(cr, gcut, first=g["gpt"])
    q = np.array([float(x) for x in arg_value(args, "-qvec").split(",")]).reshape(-1, 3)
    K = g["kpts"]
    KW = np.ones(len(K)) / len(K)
    mode = "epsLL" if "epsLL" in args else "epsij"
    re, im = O.chi(cr, mat, G, hkl, K, KW, q, mode=mode, **o)
    n = re.size
    ref_re, ref_im = g["dat"][:n].reshape(re.shape), g["dat"][n:].reshape(re.shape)
    scale = max(np.abs(ref_re).max(), np.abs(ref_im).max())
    assert np.max(np.abs(re - ref_re)) < 1e-8 * scale
    assert np.max(np.abs(im - ref_im)) < 1e-8 * scale


@pytest.mark.parametrize("name", ["gaas_soc_epsxyz", "gaas_soc_epsxyz_pv"])
def test_oracle_chi_xyz(name, tmp_path):
    """chi_xyz pairs eigenvector component p with plane wave loci[m][p], so it
    depends on the full G order: the oracle gets the reference's order from the
    host tables (bit-exact against the reference's -debug 3 dumps)."""
    from conftest import golden_args
    import picomax_b200 as pm
    g = load_golden(name)
    args = golden_args(g, tmp_path)
    cr, mat, gcut, o = O.from_args(args)
    p = pm.Problem(args)
    G, hkl = p.gvectors()
    K, KW = p.kpoints()
    Q = p.qpoints()
    p.close()
    re, im = O.chi_xyz(cr, mat, G, hkl, K, KW, Q, **o)
    n = re.size
    ref_re, ref_im = g["dat"][:n].reshape(re.shape), g["dat"][n:].reshape(re.shape)
    scale = max(np.abs(ref_re).max(), np.abs(ref_im).max())
    assert np.max(np.abs(re - ref_re)) < 1e-8 * scale
    assert np.max(np.abs(im - ref_im)) < 1e-8 * scale
