"""k-sharded chi on the GPU (picomax_b200/sharded.py): the spectra of the
k-point shards, each computed by the library on its own k-file, sum to the
spectrum of the whole list (FP64 path, 1e-12 of max |chi|); the sharded
helper on one rank returns the whole spectrum. The shards run one after the
other on one GPU (nothing waits on another rank here)."""
import numpy as np
import pytest

from conftest import golden_args, load_golden

import picomax_b200 as pm
from picomax_b200.sharded import chi_sharded, shard_argv

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,world", [("gaas_soc_epsij", 2), ("si_epsLL", 3), ("gaas_soc_epsLL_pv", 2)])
def test_shards_sum_to_whole(ctx, tmp_path, name, world):
    g = load_golden(name)
    args = golden_args(g, tmp_path)
    sw = pm.SWITCH_EPSIJ if "epsij" in args else pm.SWITCH_EPSLL
    p = pm.Problem(args)
    re0, im0 = ctx.chi(p, sw, pm.PREC_FP64)
    re = np.zeros_like(re0)
    im = np.zeros_like(im0)
    for r in range(world):
        sargv, k0, k1 = shard_argv(args, str(tmp_path), world, r)
        ps = pm.Problem(sargv)
        a, b = ctx.chi(ps, sw, pm.PREC_FP64)
        re += a
        im += b
        ps.close()
    scale = max(np.abs(re0).max(), np.abs(im0).max())
    assert np.abs(re - re0).max() <= 1e-12 * scale
    assert np.abs(im - im0).max() <= 1e-12 * scale
    p.close()


def test_chi_sharded_single_rank(ctx, tmp_path):
    g = load_golden("gaas_soc_epsij")
    args = golden_args(g, tmp_path)
    re, im = chi_sharded(ctx, args, pm.SWITCH_EPSIJ, pm.PREC_FP64)
    n = re.numel()
    scale = np.abs(g["dat"]).max()
    assert np.abs(re.cpu().numpy() - g["dat"][:n]).max() <= 1e-8 * scale
    assert np.abs(im.cpu().numpy() - g["dat"][n:]).max() <= 1e-8 * scale
