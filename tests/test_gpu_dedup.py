"""Runs of equal adjacent rows (kg_run_host): batches sorted by bit pattern
(src/convert_matrix.cpp:366-368) repeat rows; one row per run is tested on the
device and the result must equal the test of every row: the same .count
value (each tested run counts once per row) and the same emitted rows, bit
for bit, in row order."""
import numpy as np
import pytest

from oracle import oracle as O
from supergwas_b200 import api, synth

pytestmark = pytest.mark.gpu


def _distinct(X):
    """X without rows equal to their predecessor."""
    return X[np.r_[True, np.any(X[1:] != X[:-1], axis=1)]]


def _runs(X, seed, long_row=None, long_run=0):
    """X with row u repeated 1..6 times (row long_row `long_run` times more)."""
    rng = np.random.default_rng(seed)
    reps = rng.integers(1, 7, size=X.shape[0])
    if long_row is not None:
        reps[long_row] += long_run
    return np.repeat(X, reps, axis=0), reps


def _expand(hits, reps):
    """Hits of the distinct rows, repeated for every copy, in row order."""
    first = np.concatenate([[0], np.cumsum(reps)[:-1]])
    k = hits["kmer"].astype(np.int64)
    out = np.repeat(hits, reps[k])
    if hits.shape[0]:
        out["kmer"] = np.concatenate([first[i] + np.arange(reps[i]) for i in k])
    return out


@pytest.mark.parametrize("prec", ["split", "fp64"])
@pytest.mark.parametrize("thr", [0.0, 0.2])
def test_runs_match_every_row(built, monkeypatch, prec, thr):
    ds = synth.simulate(n=300, m=20000, S=5, r=6, n_causal=20, missing=0.0, seed=7)
    X = _distinct(ds.packed_overlap())
    with api.Kgwas(precision=prec, corr_threshold=thr, log10_thresh=2.0) as g:
        g.set_structure(ds.U, ds.y)
        base = g.run_host(X, stats=True)
        assert base.hits.shape[0] > 0
        # one hit row repeated 70000 more times
        X2, reps = _runs(X, 3, int(base.hits["kmer"][0]), 70000)
        got = g.run_host(X2)
        assert g.last_unique_rows() == X.shape[0]
        monkeypatch.setenv("KG_DEDUP", "0")
        every = g.run_host(X2)
        assert g.last_unique_rows() == 0
    # the .count value: each tested distinct row once per copy
    assert got.n_tested == int((base.stats["tested"].astype(np.int64) * reps).sum()) == every.n_tested
    exp = _expand(base.hits, reps)
    assert np.array_equal(got.hits, exp)
    assert np.array_equal(every.hits, exp)
    assert got.hits.shape[0] > 70000


def test_runs_against_oracle(built):
    """A fixture-sized batch with runs, through the oracle on the expanded rows."""
    ds = synth.simulate(n=200, m=3000, S=4, r=5, n_causal=10, missing=0.0, seed=11)
    X2, _ = _runs(_distinct(ds.packed_overlap()), 5)
    o = O.cols_stats(X2, ds.n, ds.U, ds.y, 0.2)
    with api.Kgwas(corr_threshold=0.2, log10_thresh=2.0) as g:
        g.set_structure(ds.U, ds.y)
        res = g.run_host(X2)
        assert 0 < g.last_unique_rows() < X2.shape[0]
    assert res.n_tested == o["n_tested"]
    exp = set(np.nonzero(o["tested"] & (o["pval"] <= 1e-2))[0].tolist())
    near = set(np.nonzero(np.abs(o["mlog10p"] - 2.0) <= 1e-6)[0].tolist())
    assert not ((exp ^ set(res.hits["kmer"].tolist())) - near)


def test_no_runs_no_scan(built):
    """Rows without repeats are tested as they are."""
    ds = synth.simulate(n=300, m=20000, S=5, r=6, n_causal=20, missing=0.0, seed=7)
    with api.Kgwas(log10_thresh=2.0) as g:
        g.set_structure(ds.U, ds.y)
        g.run_host(ds.packed_overlap())
        assert g.last_unique_rows() == 0


@pytest.mark.parametrize("kernel", ["stationary", "streamed"])
def test_multi_runs_match_every_row(built, monkeypatch, kernel):
    """kg_run_multi_host with runs: per-(shard, phenotype) counts and rows as
    for every row; a shard start also starts a run, so a run of equal rows
    that crosses a shard boundary is counted in both shards."""
    from test_gpu_multi import make_batch
    if kernel == "streamed":
        monkeypatch.setenv("KG_MP_STREAMED", "1")
    n_all, m = 1000, 6000
    packed, phenos = make_batch(n_all, m, 5, (16, 4), seed=91, wpk=16)
    packed = _distinct(packed)
    X2, reps = _runs(packed, 13, 17, 5000)
    m2 = X2.shape[0]
    # shard starts in the middle of runs, at a run start, and an empty shard
    first = np.concatenate([[0], np.cumsum(reps)[:-1]])
    shards = np.array([0, first[17] + 100, first[40], first[40], m2 - 3], dtype=np.uint64)
    with api.Kgwas(corr_threshold=0.2, log10_thresh=1.0) as g:
        g.set_phenotypes(phenos, n_all)
        t_runs, h_runs = g.run_multi_host(X2, shards)
        assert 0 < g.last_unique_rows() < m2
        monkeypatch.setenv("KG_DEDUP", "0")
        t_all, h_all = g.run_multi_host(X2, shards)
        assert g.last_unique_rows() == 0
    assert np.array_equal(t_runs, t_all)
    assert np.array_equal(h_runs, h_all)
    assert h_runs.shape[0] > 0
