"""Many phenotypes in one launch (kg_set_phenotypes / kg_launch_multi_device)
against the FP64 oracle run phenotype by phenotype, and against the
single-phenotype C ABI.

Each phenotype has its own missing samples (so its own overlap n, U and y'),
rows hold every sample of the batch, and the batch is split into shards of
uneven length whose tested counts must match the oracle's per shard.
"""
import numpy as np
import pytest

from oracle import oracle as O
from supergwas_b200 import api, synth

pytestmark = pytest.mark.gpu


def make_batch(n_all, m, n_pheno, r_list, seed, wpk=None):
    rng = np.random.default_rng(seed)
    base = synth.simulate(n=n_all, m=m, S=6, r=2, n_causal=0, missing=0.0, seed=seed)
    packed = base.packed_all
    if wpk and packed.shape[1] < wpk:
        packed = np.concatenate([packed, np.zeros((m, wpk - packed.shape[1]), np.uint64)], axis=1)
    X = synth.unpack_rows(base.packed_all, n_all)
    phenos = []
    for p in range(n_pheno):
        miss = rng.uniform(0.0, 0.3)
        keep = np.sort(rng.choice(n_all, size=n_all - int(miss * n_all), replace=False))
        r = r_list[p % len(r_list)]
        sk = rng.choice(m, size=min(m, 5000), replace=False)
        U, Ph = synth.structure_basis(X[sk][:, keep].T, r)
        causal = rng.choice(m, size=5, replace=False)
        y = rng.standard_normal(5) @ X[causal][:, keep].astype(float) + rng.standard_normal(keep.size)
        if Ph.shape[1]:
            y += 0.5 * Ph[:, -1]
        phenos.append((U, y, keep))
    return packed, phenos


def oracle_pheno(packed_all, n_all, U, y, keep, thr):
    return O.cols_stats(synth.select_samples(packed_all, n_all, keep), keep.size, U, y, thr)


KERNEL_NAME = {"mpb": "image resident (mpb)", "mpb2": "SM pair, cta_group::2 (mpb2)", "mp": "image streamed (mp)"}


@pytest.mark.parametrize("kernel", ["mpb", "mpb2", "mp"])
@pytest.mark.parametrize("case", [(1000, 6000, 5, (16,), 16), (2000, 3000, 9, (20, 4), 32),
                                  (300, 2500, 7, (3, 6), 16), (1000, 7001, 5, (20, 18), 16)],
                         ids=["n1000_r16", "n2000_r20", "n300_r3", "n1000_r20"])
def test_multi_matches_oracle(built, case, kernel, monkeypatch):
    """Every many-phenotype kernel: one phenotype group's limb image resident
    in shared memory (kernel_mpb.cu), two phenotypes per M = 256 MMA on a
    pair of SMs (kernel_mpb2.cu, where one phenotype fills a group), and the
    image streamed from L2 per 128 samples (kernel_mp.cu)."""
    monkeypatch.setenv("KG_MP_KERNEL", kernel)
    n_all, m, npheno, rl, wpk = case
    packed, phenos = make_batch(n_all, m, npheno, rl, seed=n_all + m, wpk=wpk)
    shards = np.array([0, 7, m // 3, m // 3 + 1, m - 5], dtype=np.uint64)
    with api.Kgwas(corr_threshold=0.0, log10_thresh=0.0) as g:     # every tested k-mer is a row
        g.set_phenotypes(phenos, n_all)
        tested, hits = g.run_multi_host(packed, shards)
        used = g.multi_shape()["kernel"]
    if kernel == "mpb2" and used != KERNEL_NAME["mpb2"]:
        pytest.skip("these phenotypes share an MMA group on one SM (the pair kernel needs NP >= 48 and PPG = 1)")
    assert used == KERNEL_NAME[kernel]
    bounds = list(shards.astype(int)) + [m]
    for p, (U, y, keep) in enumerate(phenos):
        o = oracle_pheno(packed[:, :synth.words_per_kmer(n_all)], n_all, U, y, keep, 0.0)
        for si in range(len(shards)):
            assert tested[si, p] == int(o["tested"][bounds[si]:bounds[si + 1]].sum()), (p, si)
        h = hits[hits["pheno"] == p]
        exp = np.nonzero(o["tested"])[0]
        assert np.array_equal(h["kmer"].astype(np.int64), exp), p
        ml = np.abs(O.mlog10p(h["chisq"]) - o["mlog10p"][exp])
        assert ml.max() <= 1e-6, (p, ml.max())
        shard_of = np.searchsorted(shards.astype(np.int64), exp, side="right") - 1
        assert np.array_equal(h["shard"], shard_of)


def test_multi_matches_single_phenotype_api(built):
    n_all, m = 1000, 20000
    packed, phenos = make_batch(n_all, m, 3, (16,), seed=77)
    with api.Kgwas(corr_threshold=0.2, log10_thresh=1.5) as g:
        g.set_phenotypes(phenos, n_all)
        tested, hits = g.run_multi_host(packed)
    for p, (U, y, keep) in enumerate(phenos):
        with api.Kgwas(corr_threshold=0.2, log10_thresh=1.5) as s:
            s.set_structure(U, y, keep, n_all)
            r = s.run_host(packed)
        assert tested[0, p] == r.n_tested
        h = hits[hits["pheno"] == p]
        assert np.array_equal(h["kmer"], r.hits["kmer"])
        assert np.allclose(h["chisq"], r.hits["chisq"], rtol=1e-12, atol=0)


@pytest.mark.parametrize("r", [16, 20])
def test_multi_graph_replay(built, r):
    """Repeated device launches with the same rows replay a captured CUDA
    graph (r = 20: the SM-pair kernel's cluster launch inside the graph)."""
    import torch
    n_all, m = 1000, 30000
    packed, phenos = make_batch(n_all, m, 4, (r,), seed=5)
    dx = torch.from_numpy(packed.view(np.int64)).cuda()
    st = torch.cuda.current_stream().cuda_stream
    outs = []
    with api.Kgwas(corr_threshold=0.0, log10_thresh=2.0) as g:
        g.set_phenotypes(phenos, n_all)
        for _ in range(4):
            g.launch_multi_device(dx.data_ptr(), m, packed.shape[1], None, st)
            outs.append(g.fetch_multi())
    for t, h in outs[1:]:
        assert np.array_equal(t, outs[0][0])
        assert np.array_equal(h, outs[0][1])


def test_multi_streamed_chunks_match_single_chunk(built, monkeypatch):
    """Host rows streamed in many chunks through two device buffers give the
    same counts and rows as one chunk (shard boundaries inside chunks)."""
    n_all, m = 1000, 40000
    packed, phenos = make_batch(n_all, m, 3, (8,), seed=19)
    shards = np.array([0, 1000, 13333, 27001], dtype=np.uint64)
    with api.Kgwas(corr_threshold=0.0, log10_thresh=1.0) as g:
        g.set_phenotypes(phenos, n_all)
        t1, h1 = g.run_multi_host(packed, shards)
        monkeypatch.setenv("KG_CHUNK_MB", "1")      # 128-byte rows: 8192 k-mers per chunk
        t2, h2 = g.run_multi_host(packed, shards)
    assert np.array_equal(t1, t2)
    assert np.array_equal(h1, h2)


def test_multi_kernels_bit_identical(built, monkeypatch):
    """The three many-phenotype kernels give the same counts and the same
    rows bit for bit (same limb image, same exact integer sums), also with
    several L2 blocks per launch and a partial last block and pair-tile."""
    n_all, m = 2000, 50000
    packed, phenos = make_batch(n_all, m, 7, (20, 9), seed=23, wpk=32)
    shards = np.array([0, 4096, 30001], dtype=np.uint64)
    out = {}
    for kernel, bt in (("mpb", None), ("mpb", "2"), ("mpb2", None), ("mpb2", "3"), ("mp", None)):
        monkeypatch.setenv("KG_MP_KERNEL", kernel)
        monkeypatch.delenv("KG_MP_BT", raising=False)
        if bt:
            monkeypatch.setenv("KG_MP_BT", bt)
        with api.Kgwas(corr_threshold=0.0, log10_thresh=1.0) as g:
            g.set_phenotypes(phenos, n_all)
            out[(kernel, bt)] = g.run_multi_host(packed, shards)
            assert g.multi_shape()["kernel"] == KERNEL_NAME[kernel]
    t0, h0 = out[("mp", None)]
    for key in (("mpb", None), ("mpb", "2"), ("mpb2", None), ("mpb2", "3")):
        t, h = out[key]
        assert np.array_equal(t, t0), key
        assert np.array_equal(h, h0), key


def test_multi_autotuner_picks_a_measured_shape(built):
    """Without a kernel request the autotuner times the candidate shapes and
    keeps one; the result equals the streamed kernel's."""
    import os
    n_all, m = 2000, 60000
    packed, phenos = make_batch(n_all, m, 4, (20,), seed=29, wpk=32)
    assert "KG_MP_KERNEL" not in os.environ
    with api.Kgwas(corr_threshold=0.0, log10_thresh=1.0) as g:
        g.set_phenotypes(phenos, n_all)
        t1, h1 = g.run_multi_host(packed)
        shape = g.multi_shape()
    assert shape["kernel"] in KERNEL_NAME.values() and shape["bt"] >= 1
    os.environ["KG_MP_KERNEL"] = "mp"
    try:
        with api.Kgwas(corr_threshold=0.0, log10_thresh=1.0) as g:
            g.set_phenotypes(phenos, n_all)
            t2, h2 = g.run_multi_host(packed)
    finally:
        del os.environ["KG_MP_KERNEL"]
    assert np.array_equal(t1, t2)
    assert np.array_equal(h1, h2)
