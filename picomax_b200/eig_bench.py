"""Batched Hermitian eigensolve of random matrices through pmx_heev_batched.

python -m picomax_b200.eig_bench [--n 274] [--batch 296] [--nev 17] [--schedule 0] [--reps 3]

Prints the device time of each call (CUDA events around the eigensolver
launches) and the largest eigenvalue error of the first matrix against
numpy. Schedule 0 is the two-stage solver for the sizes it covers (matrices
beyond the shared-memory-resident kernel, padded size <= 800); 1.. are the
one-stage schedules; -1 lets the autotuner choose (it runs on batches of at
least 148 matrices).
"""
from __future__ import annotations

import argparse

import numpy as np

from ._capi import Context


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=274)
    ap.add_argument("--batch", type=int, default=296)
    ap.add_argument("--nev", type=int, default=17)
    ap.add_argument("--schedule", type=int, default=0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    rng = np.random.default_rng(a.seed)
    A = rng.standard_normal((a.batch, a.n, a.n)) + 1j * rng.standard_normal((a.batch, a.n, a.n))
    A = (A + A.conj().transpose(0, 2, 1)) / 2
    ctx = Context(0)
    ctx.set_schedule(a.schedule)
    last = 0.0
    for r in range(a.reps):
        w, _ = ctx.heev(A, a.nev)
        ms, _ = ctx.kernel_time("heev")
        print(f"call {r}: {ms - last:.3f} ms device time for {a.batch} matrices of n = {a.n}")
        last = ms
    err = np.abs(w[0] - np.linalg.eigvalsh(A[0])[:a.nev]).max()
    print(f"max eigenvalue error of matrix 0 vs numpy: {err:.3e}")
    ctx.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
