"""Host-side failure paths (no GPU): malformed k-point files are rejected by
the problem parser with PMX_ERR_INVALID instead of the reference's silent
zero-weight points (import_kpt, src/pmx_basis.cpp:200-245)."""
import os

import numpy as np
import pytest

import picomax_b200 as pm
from picomax_b200.kgrid import write_kfile

BASE = ("-switch epsLL -crystal zb -a 5.43 -vg 3,4,8,11,-0.21,0,0.04,0.08,-0.21,0,0.04,0.08 -encut 60 "
        "-nband 8 -nvalence 4 -neps 2 -nfreq 20 -dfreq 0.5 -qvec 0.01,0,0 -kpoint 0").split()


def _problem(kf):
    return pm.Problem(BASE + ["-kpointfile", kf])


def test_kfile_accepted(tmp_path):
    kf = os.path.join(str(tmp_path), "k.txt")
    write_kfile(kf, np.array([[0.1, 0.2, 0.3], [0.0, 0.0, 0.5]]), np.ones(2))
    p = _problem(kf)
    K, W = p.kpoints()
    assert K.shape == (2, 3) and np.allclose(W, 0.5)
    p.close()


@pytest.mark.parametrize("text", [
    "4\n3\n0.1 0.2 0.3 1\n0.0 0.0 0.5 1\n",       # declares 3 points, lists 2
    "4\n2\n0.1 0.2 0.3 1\n0.0 zero 0.5 1\n",      # a point that does not parse
    "0\n1\n0.1 0.2 0.3 1\n",                      # zero total (the weights divide by it)
    "4\n",                                        # no listed count
])
def test_malformed_kfile_rejected(tmp_path, text):
    kf = os.path.join(str(tmp_path), "k.txt")
    with open(kf, "w") as fh:
        fh.write(text)
    with pytest.raises(pm.PicomaxError) as e:
        _problem(kf)
    assert e.value.status == pm.PMX_ERR_INVALID


def test_missing_kfile_rejected(tmp_path):
    with pytest.raises(pm.PicomaxError) as e:
        _problem(os.path.join(str(tmp_path), "absent.txt"))
    assert e.value.status == pm.PMX_ERR_INVALID
