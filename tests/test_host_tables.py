"""Host-side tables against the reference: G order, k/q lists (the -debug 3
dumps of the reference rebuilt from source) and the .gpt bytes."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_args, load_golden

import picomax_b200 as pm


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "dumps", "*.txt"))),
                         ids=lambda p: os.path.basename(p)[:-4])
def test_debug3_dump_identical(path):
    with open(path) as fh:
        argv = fh.readline().split()
        ref = fh.read()
    p = pm.Problem(argv + ["-debug", "3"])
    mine = p.dump()
    mine = mine[mine.index("planewave energy cutoff"):]
    assert mine.splitlines() == ref.splitlines()


@pytest.mark.parametrize("name", ["si_epsij", "gaas_soc_epsij", "si_epsLL", "wz_epsij_rect"])
def test_gpt_bytes(name, tmp_path):
    g = load_golden(name)
    args = golden_args(g, tmp_path)
    p = pm.Problem(args)
    G, _ = p.gvectors()
    assert np.array_equal(G[: p.info.neps].ravel(), g["gpt"])  # bit-exact doubles


def test_loci_is_lattice_sum():
    p = pm.Problem("-crystal wz -a 3.19 -f 1.626 -u 0.375 -vg 1,2,3,4,5,6,7,8,9,10 -encut 150 -neps 20".split())
    G, H = p.gvectors()
    L = p.loci()
    where = {tuple(h): i for i, h in enumerate(H)}
    for m in range(p.info.neps):
        for q in range(p.info.npw):
            assert L[m, q] == where.get(tuple(H[q] + H[m]), -1)
    assert np.array_equal(L[0], np.arange(p.info.npw))


def test_si_plane_wave_count():
    # N_G = 113 for Si at any encut in [102.1, 122.4) eV
    for enc in ("102.2", "110", "122.3"):
        p = pm.Problem(["-crystal", "zb", "-a", "5.43", "-encut", enc, "-vg", "3,0.1,0.1"])
        assert p.info.npw == 113


def test_soc_flag():
    base = "-crystal zb -a 5.65 -encut 60 -vg 3,4,8,11,-0.2,0,0.04,0.08,-0.1,0,0.02,0.04".split()
    assert pm.Problem(base).info.soc == 0
    assert pm.Problem(base + ["-use_uniform_us_so", "-uniform_us_so_val", "0.01"]).info.soc == 1
    assert pm.Problem(base + ["-ua_so", "3:0.01"]).info.soc == 1


def test_bad_options_rejected():
    with pytest.raises(pm.PicomaxError):
        pm.Problem("-crystal zb -encut 100".split())          # missing -a (reference: abort)
    with pytest.raises(pm.PicomaxError):
        pm.Problem("-crystal zb -a 5.43 -vg 3,4,5,6".split())  # -vg arity (reference: abort)
    with pytest.raises(pm.PicomaxError):
        pm.Problem("-crystal zb -a 5.43 -qvec 0,0".split())   # -qvec arity (reference: abort)
    with pytest.raises(pm.PicomaxError):
        pm.Problem("-crystal zb -a 5.43 -qpath G,X".split())  # -qpath without -qnum
