"""Overlaps of the mixed path on the tensor cores (overlap_tc.cu: tcgen05
kind::tf32, split TF32 operands, FP32 results) against the FP64 overlaps and
the reference:

* |M|^2 of the tensor-core overlaps against the FP64 ones (overlap mode 2
  computes both): max error <= 1e-5 of max |M|^2 (FP32 accumulation in
  tensor memory over the stacked K of real and imaginary parts) for epsLL and
  epsij, with and without spin-orbit coupling (four channels), epsxyz, and
  the config-2 shape;
* the mixed chi with tensor-core overlaps (mode 3) against the mixed chi with
  FP64 overlaps (mode 0) and, where the fixture holds the full spectrum,
  against the reference at 1e-4 (the same bound as with FP64 overlaps); the
  default (mode 1) equals mode 3 without spin-orbit coupling and mode 0 with
  it;
* a wait that runs out (test hook 4: the first chunk's MMAs are never
  committed) returns PMX_ERR_TIMEOUT and leaves the context usable.
"""
import numpy as np
import pytest

from conftest import golden_args, load_golden

import picomax_b200 as pm

pytestmark = pytest.mark.gpu

CASES = ["si_epsLL", "gaas_soc_epsij", "wz_epsij_rect", "gaas_soc_epsxyz", "cfg2_gaas_epsij"]


@pytest.fixture(scope="module")
def ctx():
    c = pm.Context(0)
    yield c
    c.close()


def _switch(args):
    return {"epsij": pm.SWITCH_EPSIJ, "epsLL": pm.SWITCH_EPSLL, "epsxyz": pm.SWITCH_EPSXYZ}[args[args.index("-switch") + 1]]


@pytest.mark.parametrize("name", CASES)
def test_tensor_core_overlaps(ctx, tmp_path, name):
    g = load_golden(name)
    args = golden_args(g, tmp_path)
    p = pm.Problem(args)
    sw = _switch(args)
    ctx.set_overlap_mode(2)
    re2, im2 = ctx.chi(p, sw, pm.PREC_MIXED)
    err, mx = ctx.overlap_error()
    print(name, "|M|^2 err rel", err / mx)
    assert mx > 0 and err <= 1e-5 * mx, (err, mx)
    ctx.set_overlap_mode(0)
    re0, im0 = ctx.chi(p, sw, pm.PREC_MIXED)
    ctx.set_overlap_mode(3)
    re1, im1 = ctx.chi(p, sw, pm.PREC_MIXED)
    ctx.set_overlap_mode(1)
    red, imd = ctx.chi(p, sw, pm.PREC_MIXED)
    scale = max(np.abs(re0).max(), np.abs(im0).max())
    assert np.array_equal(re1, re2) and np.array_equal(im1, im2)
    if p.info.soc:
        assert np.array_equal(red, re0) and np.array_equal(imd, im0)
    else:
        assert np.array_equal(red, re1) and np.array_equal(imd, im1)
    d = max(np.abs(re1 - re0).max(), np.abs(im1 - im0).max()) / scale
    print(name, "chi mode1 vs mode0 rel", d)
    assert d <= 2e-5
    if "dat" in g:
        n = re1.size
        ref = g["dat"]
        rs = np.abs(ref).max()
        assert max(np.abs(re1 - ref[:n]).max(), np.abs(im1 - ref[n:]).max()) <= 1e-4 * rs
    p.close()


def test_tensor_core_overlap_wait_timeout(ctx, tmp_path):
    g = load_golden("gaas_soc_epsij")
    p = pm.Problem(golden_args(g, tmp_path))
    ctx.set_overlap_mode(3)
    ctx.set_wait_limit(1_000_000)  # 1 ms
    ctx.set_fault(4)
    with pytest.raises(pm.PicomaxError) as e:
        ctx.chi(p, pm.SWITCH_EPSIJ, pm.PREC_MIXED)
    assert e.value.status == pm.PMX_ERR_TIMEOUT
    ctx.set_fault(0)
    ctx.set_wait_limit(0)
    re, im = ctx.chi(p, pm.SWITCH_EPSIJ, pm.PREC_MIXED)
    ctx.set_overlap_mode(1)
    n = re.size
    scale = np.abs(g["dat"]).max()
    assert max(np.abs(re - g["dat"][:n]).max(), np.abs(im - g["dat"][n:]).max()) <= 1e-4 * scale
    p.close()
