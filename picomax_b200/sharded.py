"""One chi(q, w) spectrum over several GPUs: the k-points are partitioned.

chi is a weighted sum over k-points, and every later step on the path is
linear in that sum: the scale factors, the principal-value term of -kk 0
and the Kramers-Kronig transform (which adds the transform of each part,
computed from the values before it, src/pmx_chi.cpp:272-309). So rank r
runs the ordinary pipeline (eigensolves, overlaps, contraction, scaling,
KK) on its own contiguous block of the k-point list, keeping the full grid's
weight normaliser (the first line of the kpointfile, import_kpt,
src/pmx_basis.cpp:200-245), and one all-reduce (sum) of the two spectra
gives the whole chi on every rank. eps_M, which is not linear in chi, is
formed after the reduction.

The reference has no multi-GPU path (README.md:420 lists it as future work).
"""
from __future__ import annotations

import os
import tempfile

import numpy as np


def k_partition(nk: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous block [k0, k1) of rank `rank` out of `world` (sizes differ by
    at most one point; ranks beyond nk get an empty block)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank outside the world")
    base, extra = divmod(nk, world)
    k0 = rank * base + min(rank, extra)
    return k0, k0 + base + (1 if rank < extra else 0)


def read_kfile(path: str):
    """(total count, K [n, 3], raw weights [n]) of a kpointfile."""
    rows = []
    with open(path) as fh:
        lines = [ln for ln in fh.read().splitlines() if ln.strip() and not ln.startswith("#")]
    total, listed = int(lines[0].split()[0]), int(lines[1].split()[0])
    for ln in lines[2:2 + listed]:
        rows.append([float(x) for x in ln.split()[:4]])
    a = np.asarray(rows, np.float64).reshape(-1, 4)
    return total, a[:, :3], a[:, 3]


def write_shard(path: str, total: int, K, W) -> None:
    """A kpointfile listing K with raw weights W under the full grid's total."""
    with open(path, "w") as fh:
        fh.write(f"{total}\n{len(K)}\n")
        for k, w in zip(np.asarray(K), np.asarray(W)):
            fh.write(f"{float(k[0])!r} {float(k[1])!r} {float(k[2])!r} {float(w)!r}\n")


def shard_argv(argv, workdir: str, world: int, rank: int):
    """argv of rank `rank`'s shard: the same options with a kpointfile that
    lists only its block of the original file's points. Returns (argv, k0, k1)."""
    argv = [str(a) for a in argv]
    if "-kpointfile" not in argv:
        raise ValueError("k-point sharding needs -kpoint 0 -kpointfile")
    i = argv.index("-kpointfile") + 1
    total, K, W = read_kfile(argv[i])
    k0, k1 = k_partition(len(K), world, rank)
    path = os.path.join(workdir, f"kshard_{rank}_of_{world}.txt")
    write_shard(path, total, K[k0:k1], W[k0:k1])
    out = list(argv)
    out[i] = path
    return out, k0, k1


def chi_sharded(ctx, argv, switch: int, precision: int, group=None):
    """chi of the whole k list on every rank of `group` (torch.distributed,
    NCCL on the GPUs): each rank computes its block with pmx_chi_device on its
    own device, then the spectra are summed with one all-reduce each.
    Returns (re, im) device tensors in .dat order."""
    import torch
    import torch.distributed as dist

    from ._capi import Problem

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    dev = torch.cuda.current_device()
    with tempfile.TemporaryDirectory() as tmp:
        sargv, k0, k1 = shard_argv(argv, tmp, world, rank)
        prob = Problem(sargv)
        re = torch.zeros(prob.info.chi_values, dtype=torch.float64, device=f"cuda:{dev}")
        im = torch.zeros_like(re)
        if k1 > k0:
            ctx.chi_device(prob, switch, precision, re.data_ptr(), im.data_ptr())
        prob.close()
    torch.cuda.synchronize()
    if world > 1:
        dist.all_reduce(re, op=dist.ReduceOp.SUM, group=group)
        dist.all_reduce(im, op=dist.ReduceOp.SUM, group=group)
    return re, im
