"""Symmetry reduction of Gamma-centred k grids on the device
(pmx_kgrid_reduce) against the oracle's reduction (oracle/pmx_oracle.py
ibz_reduce) under the same operations, bit-exact: representatives (the
smallest linear index of each orbit, in index order) and orbit sizes. Grids
whose axes differ keep the operations that map the grid onto itself. The
k file written from the reduction reads back with weights summing to one.
"""
import os

import numpy as np
import pytest

import pmx_oracle as O
import picomax_b200 as pm
from picomax_b200.kgrid import ibz_grid, write_kfile

from test_kgrid_symmetry import GAAS, SI, SOC, _hex

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = pm.Context(0)
    yield c
    c.close()


def _compatible(ops, n):
    keep = [m for m in ops if all(m[a, b] == 0 or n[a] == n[b] for a in range(3) for b in range(3))]
    return np.array(keep)


CASES = [
    (GAAS, (8, 8, 8), pm.KGRID_TIME_REVERSAL),
    (GAAS, (16, 16, 16), pm.KGRID_TIME_REVERSAL),
    (GAAS + SOC, (12, 12, 12), 0),
    (SI, (10, 10, 10), pm.KGRID_TIME_REVERSAL),
    (GAAS, (8, 8, 4), pm.KGRID_TIME_REVERSAL),
    (GAAS + " -qvec 0.01,0,0", (8, 8, 8), pm.KGRID_TIME_REVERSAL | pm.KGRID_LITTLE_GROUP_Q),
    ("wz", (6, 6, 4), pm.KGRID_TIME_REVERSAL),
    ("te", (5, 5, 4), pm.KGRID_TIME_REVERSAL),
]


@pytest.mark.parametrize("args,n,flags", CASES)
def test_device_reduction_matches_oracle(ctx, args, n, flags):
    if args in ("wz", "te"):
        args, _ = _hex(args)
    p = pm.Problem(args.split())
    ops = _compatible(p.symmetry_ops(flags).astype(np.int64), n)
    ridx, rw = O.ibz_reduce(ops, n)
    idx, w = ctx.kgrid_reduce(p, n, flags)
    assert np.array_equal(idx, ridx) and np.array_equal(w, rw)
    assert w.sum() == np.prod(n)
    p.close()


def test_ibz_kfile_reads_back(ctx, tmp_path):
    p = pm.Problem(GAAS.split())
    K, W, N = ibz_grid(ctx, p, "zb", 8, 8, 8)
    assert len(K) == 29 and W.sum() == N == 512
    path = os.path.join(str(tmp_path), "ibz.txt")
    write_kfile(path, K, W, N)
    q = pm.Problem(GAAS.split() + ["-kpoint", "0", "-kpointfile", path])
    K2, W2 = q.kpoints()
    assert np.allclose(K2, K) and abs(W2.sum() - 1.0) < 1e-12
    p.close()
    q.close()
