"""Host-side helpers of bench.py: the profiled DRAM bytes behind
roofline.traffic, and the sizing of the timed sample of the reference CPU
build (a first run on one k-point per core, then scaled in multiples of the
core count towards the target time)."""
import os
import tempfile

import pytest

import bench
from picomax_b200.kgrid import make_kfile
from picomax_b200.workloads import workload

REF_LL = os.path.join(bench.ROOT, "oracle", "_ref", "picomax_ref_ll")


def test_profiled_heev_bytes():
    v = bench.profiled_heev_bytes(274)
    assert v is not None and 1e5 < v < 1e9  # DRAM bytes per 274 x 274 matrix of the committed capture
    assert bench.profiled_heev_bytes(123) is None


@pytest.mark.skipif(not os.path.exists(REF_LL), reason="oracle/_ref not built")
def test_reference_sample_plan():
    d = tempfile.mkdtemp()
    argv, _, _ = workload("si_epsLL", d)
    kf = os.path.join(d, "k4.txt")
    nk = make_kfile(kf, "zb", 4, 4, 4)
    argv = list(argv)
    argv[argv.index("-kpointfile") + 1] = kf
    lines = open(kf).read().splitlines()
    assert int(lines[1]) == nk
    env = dict(os.environ, OMP_NUM_THREADS="2")
    kdep, kk, wall = bench._ref_run(REF_LL, argv, lines, 2, d, env)
    assert kdep > 0 and kk >= 0 and wall >= kdep
    # a target far above one core-batch: the sample grows in multiples of the cores
    sample, first = bench._ref_plan(REF_LL, argv, lines, d, env, 2, target_s=50 * kdep + 1.0)
    assert first is None and (sample % 2 == 0 or sample == nk) and 2 < sample <= nk
    # a target below one core-batch: the first run is the sample
    sample, first = bench._ref_plan(REF_LL, argv, lines, d, env, 2, target_s=0.0)
    assert sample == 2 and first is not None and first[0] > 0
