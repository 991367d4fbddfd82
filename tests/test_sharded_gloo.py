"""k-sharded chi across ranks (picomax_b200/sharded.py), world size 2 over
gloo on the CPU: each rank computes chi of its block of k-points (the numpy
oracle stands in for the device part), one all-reduce sums the spectra, and
the sum equals chi of the whole k list (scale factors, the principal-value
term and the Kramers-Kronig transform are linear in the k-sum). The same
partition and the same k-file shards drive the GPU path."""
import os
import socket

import numpy as np
import pytest

from conftest import arg_value, load_golden

import pmx_oracle as O
from picomax_b200.sharded import k_partition, read_kfile, shard_argv, write_shard

CASES = ["si_epsLL", "gaas_soc_epsLL_pv"]


def _oracle_chi(g, K, KW):
    args = [str(x) for x in g["argv"]]
    cr, mat, gcut, o = O.from_args(args)
    G, hkl = O.gvectors(cr, gcut, first=g["gpt"])
    q = np.array([float(x) for x in arg_value(args, "-qvec").split(",")]).reshape(-1, 3)
    mode = "epsLL" if "epsLL" in args else "epsij"
    return O.chi(cr, mat, G, hkl, K, KW, q, mode=mode, **o)


def _rank(rank, world, port, name, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = load_golden(name)
        K = g["kpts"]
        k0, k1 = k_partition(len(K), world, rank)
        re, im = _oracle_chi(g, K[k0:k1], np.ones(k1 - k0) / len(K))
        t = torch.from_numpy(np.concatenate([re.ravel(), im.ravel()]))
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        if rank == 0:
            out.put(t.numpy())
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("name", CASES)
def test_k_sharded_allreduce_gloo(name):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, name, q)) for r in range(2)]
    for p in procs:
        p.start()
    summed = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = load_golden(name)
    K = g["kpts"]
    re, im = _oracle_chi(g, K, np.ones(len(K)) / len(K))
    full = np.concatenate([re.ravel(), im.ravel()])
    scale = np.abs(full).max()
    assert np.abs(summed - full).max() <= 1e-12 * scale
    assert np.abs(summed - g["dat"]).max() <= 1e-8 * scale


def test_k_partition_covers_once():
    for nk in (0, 1, 7, 27, 4096):
        for world in (1, 2, 3, 8):
            blocks = [k_partition(nk, world, r) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == nk
            assert all(b[1] == c[0] for b, c in zip(blocks, blocks[1:]))
            assert max(b[1] - b[0] for b in blocks) - min(b[1] - b[0] for b in blocks) <= 1


def test_shard_kfiles_keep_the_grid_normaliser(tmp_path):
    K = np.random.default_rng(0).uniform(-0.5, 0.5, (10, 3))
    W = np.arange(1, 11, dtype=float)
    src = os.path.join(str(tmp_path), "k.txt")
    write_shard(src, 64, K, W)
    argv = ["-switch", "epsLL", "-kpoint", "0", "-kpointfile", src]
    got = []
    for r in range(3):
        a, k0, k1 = shard_argv(argv, str(tmp_path), 3, r)
        total, Ks, Ws = read_kfile(a[a.index("-kpointfile") + 1])
        assert total == 64 and np.array_equal(Ks, K[k0:k1]) and np.array_equal(Ws, W[k0:k1])
        got.append(Ks)
    assert np.array_equal(np.concatenate(got), K)
