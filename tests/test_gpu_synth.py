"""The seeded device generator of bench batches (lib/libkgwas_bench.so).

Each row is a function of (seed, row index) only, so the streaming workload
can regenerate any 16 GB chunk of its 625 GB batch on its own: a chunk
generated by itself equals the same rows of a longer generation.  The rows
follow the Balding-Nichols model (ancestral frequency Beta(0.5, 0.5), mean
0.5; subpopulations differentiated at F = 0.1), and padding bits are zero.
"""
import numpy as np
import pytest

from supergwas_b200 import synth

pytestmark = pytest.mark.gpu


def _gen(n, m, S, seed, first=0):
    import torch
    from supergwas_b200 import synth_gpu
    out = torch.empty((m, synth.words_per_kmer(n)), dtype=torch.int64, device="cuda")
    synth_gpu.synth_rows(out, n, S, seed, first=first)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint64)


def test_chunks_regenerate_alone(built):
    n, S = 5000, 12
    whole = _gen(n, 3000, S, 47)
    assert np.array_equal(whole, _gen(n, 3000, S, 47))          # deterministic
    part = _gen(n, 1000, S, 47, first=1500)                       # a chunk on its own
    assert np.array_equal(part, whole[1500:2500])
    assert not np.array_equal(_gen(n, 1000, S, 48, first=1500), part)  # another seed, other rows


def test_model_statistics(built):
    n, S, m = 1200, 6, 20000
    X = synth.unpack_rows(_gen(n, m, S, 5), n).astype(np.float64)
    packed = _gen(n, m, S, 5)
    # padding bits past n are zero
    assert np.all(synth.unpack_rows(packed, synth.words_per_kmer(n) * 64)[:, n:] == 0)
    f = X.mean(axis=1)                       # per-k-mer frequency ~ Beta(0.5, 0.5): mean 0.5, variance 1/8
    assert abs(f.mean() - 0.5) < 0.02
    assert abs(f.var() - 0.125) < 0.015
    # per-subpopulation frequencies spread around the k-mer's: F_ST near 0.1
    pop = (np.arange(n) * S) // n
    fs = np.stack([X[:, pop == s].mean(axis=1) for s in range(S)], axis=1)
    pbar = fs.mean(axis=1)
    keep = (pbar > 0.1) & (pbar < 0.9)
    fst = (fs[keep].var(axis=1) / (pbar[keep] * (1 - pbar[keep]))).mean()
    assert 0.06 < fst < 0.14, fst
