"""The autotuner's choices leave the results unchanged: eigensolver schedules
(tests/test_gpu_parity.py) and the FP64 overlap kernel's tile shapes, timed on
the first overlap launch of a shape over at least 148 k-points."""
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["si_epsLL", "gaas_epsij_6"])
def test_overlap_tile_autotune_same_chi(name):
    import picomax_b200 as pm
    from picomax_b200.workloads import workload
    tmp = tempfile.mkdtemp()
    argv, _, _ = workload(name, tmp)
    p = pm.Problem(argv)
    assert p.info.nk >= 148
    sw = pm.SWITCH_EPSLL if "epsLL" in name else pm.SWITCH_EPSIJ
    # one eigensolver schedule in both contexts, so that only the overlap
    # tiles are tuned
    tuned = pm.Context(0)
    tuned.set_schedule(0)
    r1, i1 = tuned.chi(p, sw, pm.PREC_FP64)
    tun = tuned.tuning()["overlap"]
    assert len(tun) == 1 and len(tun[0]["tiles"]) > 1, tun
    assert [tun[0]["cchunk"], tun[0]["vchunk"]] in tun[0]["tiles"]
    r2, i2 = tuned.chi(p, sw, pm.PREC_FP64)  # the cached choice
    plain = pm.Context(0)
    plain.set_schedule(0)
    plain.set_autotune(False)
    r0, i0 = plain.chi(p, sw, pm.PREC_FP64)
    assert plain.tuning()["overlap"] == []
    for a in (r1, r2):
        assert np.array_equal(a, r0)
    for a in (i1, i2):
        assert np.array_equal(a, i0)
    tuned.close()
    plain.close()
    p.close()
