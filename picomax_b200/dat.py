"""Readers of the reference's binary outputs (src/pmx_io.cpp:704-826).

* band .dat: float64 [NQ][NBAND], eV.
* chi .dat:  Re block then Im block, each float64 [3][3][NQ][m][n<=m][NFREQ].
* .gpt:      float64 [NEPS][3], units 2 pi / a.
"""
from __future__ import annotations

import numpy as np


def read_band(path: str, nq: int, nband: int) -> np.ndarray:
    return np.fromfile(path, np.float64).reshape(nq, nband)


def read_chi(path: str, nq: int, neps: int, nfreq: int):
    """Returns (re, im) each [3, 3, nq, npairs, nfreq], pair(m, n) = m(m+1)/2 + n."""
    npairs = neps * (neps + 1) // 2
    raw = np.fromfile(path, np.float64)
    blk = 9 * nq * npairs * nfreq
    if raw.size != 2 * blk:
        raise ValueError(f"{path}: {raw.size} values, expected {2 * blk}")
    shape = (3, 3, nq, npairs, nfreq)
    return raw[:blk].reshape(shape), raw[blk:].reshape(shape)


def read_gpt(path: str) -> np.ndarray:
    return np.fromfile(path, np.float64).reshape(-1, 3)


def unpack_pairs(block: np.ndarray, neps: int) -> np.ndarray:
    """[..., npairs, nf] lower-triangle storage -> [..., neps, neps, nf] with
    n > m entries filled as NaN."""
    out = np.full(block.shape[:-2] + (neps, neps, block.shape[-1]), np.nan)
    p = 0
    for m in range(neps):
        for n in range(m + 1):
            out[..., m, n, :] = block[..., p, :]
            p += 1
    return out
