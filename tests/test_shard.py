"""Weak-scaling shard logic on CPU: world_size-2 gloo ranks, each testing a
contiguous k-mer range with the oracle as the per-shard computation; the
all-gathered, merged result must equal one run over the whole batch."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from supergwas_b200 import api, shard, synth

HIT = api.HIT_DTYPE


def _oracle_hits(X, n, U, y, thr, log10_thresh):
    from oracle import oracle as O
    st = O.cols_stats(X, n, U, y, thr)
    idx = np.nonzero(st["tested"] & (st["pval"] <= 10.0 ** -log10_thresh))[0]
    h = np.zeros(idx.size, HIT)
    h["kmer"] = idx
    h["effect"] = st["effect"][idx]
    h["pval"] = st["pval"][idx]
    h["chisq"] = st["chisq"][idx]
    return st["n_tested"], h


def _worker(rank, world, port, X, n, U, y, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    s, e = shard.shard_range(X.shape[0], rank, world)
    nt, h = _oracle_hits(X[s:e], n, U, y, 0.0, 2.0)
    parts = [None] * world
    dist.all_gather_object(parts, (s, nt, h))
    if rank == 0:
        q.put(shard.merge(parts))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def test_shard_ranges_cover():
    for m in (0, 1, 7, 128, 1001):
        for w in (1, 2, 3, 8):
            rs = [shard.shard_range(m, r, w) for r in range(w)]
            assert rs[0][0] == 0 and rs[-1][1] == m
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            assert max(e - s for s, e in rs) - min(e - s for s, e in rs) <= 1


def test_two_rank_gloo_merge_equals_single_run():
    ds = synth.simulate(n=120, m=3001, S=3, r=3, n_causal=5, missing=0.0, seed=21)
    X = ds.packed_overlap()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, X, ds.n, ds.U, ds.y, q)) for r in range(2)]
    for p in procs:
        p.start()
    total, hits = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    nt, h = _oracle_hits(X, ds.n, ds.U, ds.y, 0.0, 2.0)
    assert total == nt
    assert np.array_equal(hits["kmer"], h["kmer"])
    assert np.array_equal(hits["chisq"], h["chisq"])
