"""Failure paths on the GPU, without faulting it: every one returns a status.

* mixed contraction: a short wait limit plus a test hook that withholds one
  mbarrier arrival make the control warp's bounded wait run out; the call
  returns PMX_ERR_TIMEOUT (the CTAs drain their copies and MMAs, free their
  tensor memory and return) and the context computes correctly afterwards;
* eigensolver: a bisection capped at one round reports non-convergence
  (PMX_ERR_NOCONV, the reference's abort() at src/pmx_epm.cpp:233);
* two-stage eigensolver: a test hook makes the bulge chase's second sweep wait
  for progress that never comes; with a short limit the bounded wait gives up
  and the call returns PMX_ERR_TIMEOUT, and the context solves correctly
  afterwards;
* non-finite form factors give non-finite eigenvalues: PMX_ERR_NOCONV;
* the CLI exits non-zero when it cannot write its output.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import golden_args, load_golden

import picomax_b200 as pm

pytestmark = pytest.mark.gpu


def test_mixed_wait_timeout_returns_status(tmp_path):
    g = load_golden("si_epsLL")
    p = pm.Problem(golden_args(g, tmp_path))
    c = pm.Context(0)
    c.set_wait_limit(1_000_000)  # 1 ms
    c.set_fault(1)
    with pytest.raises(pm.PicomaxError) as e:
        c.chi(p, pm.SWITCH_EPSLL, pm.PREC_MIXED)
    assert e.value.status == pm.PMX_ERR_TIMEOUT
    c.set_fault(0)
    c.set_wait_limit(0)
    re, im = c.chi(p, pm.SWITCH_EPSLL, pm.PREC_MIXED)
    n = re.size
    scale = np.abs(g["dat"]).max()
    assert max(np.abs(re - g["dat"][:n]).max(), np.abs(im - g["dat"][n:]).max()) <= 1e-4 * scale
    c.close()
    p.close()


@pytest.mark.parametrize("name", ["si_band", "gaas_soc_band"])
def test_bisection_cap_returns_noconv(name, tmp_path):
    g = load_golden(name)
    p = pm.Problem(golden_args(g, tmp_path))
    c = pm.Context(0)
    c.set_fault(2)
    with pytest.raises(pm.PicomaxError) as e:
        c.band(p)
    assert e.value.status == pm.PMX_ERR_NOCONV
    c.set_fault(0)
    assert np.max(np.abs(c.band(p).ravel() - g["dat"])) < 1e-9
    c.close()
    p.close()


def test_bulge_chase_wait_timeout_returns_status():
    rng = np.random.default_rng(5)
    n, b, nev = 274, 4, 17
    A = rng.standard_normal((b, n, n)) + 1j * rng.standard_normal((b, n, n))
    A = (A + A.conj().transpose(0, 2, 1)) / 2
    c = pm.Context(0)
    c.set_schedule(0)  # the two-stage solver
    c.set_wait_limit(1_000_000)  # 1 ms
    c.set_fault(3)
    with pytest.raises(pm.PicomaxError) as e:
        c.heev(A, nev)
    assert e.value.status == pm.PMX_ERR_TIMEOUT
    c.set_fault(0)
    c.set_wait_limit(0)
    w, _ = c.heev(A, nev)
    for i in range(b):
        assert np.abs(w[i] - np.linalg.eigvalsh(A[i])[:nev]).max() < 1e-10 * np.abs(A[i]).max() * n
    c.close()


def test_nonfinite_form_factor_returns_noconv():
    args = ("-switch band -crystal zb -a 5.43 -vg 3,4,8,11,nan,0,0.04,0.08,-0.21,0,0.04,0.08 -encut 60 "
            "-nband 8 -nvalence 4 -qpath G,X -qnum 4").split()
    p = pm.Problem(args)
    c = pm.Context(0)
    with pytest.raises(pm.PicomaxError) as e:
        c.band(p)
    assert e.value.status == pm.PMX_ERR_NOCONV
    c.close()
    p.close()


def test_cli_unwritable_wdir_exits_nonzero(tmp_path):
    g = load_golden("si_band")
    args = golden_args(g, tmp_path)
    wdir = os.path.join(str(tmp_path), "missing", "dir")
    r = subprocess.run([pm.CLI_PATH] + args + ["-wdir", wdir, "-outputfile", "out"], capture_output=True, text=True)
    assert r.returncode != 0
    assert "cannot write" in (r.stdout + r.stderr)
