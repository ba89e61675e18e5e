"""GPU parity: the C ABI (both arithmetic forms) against the FP64 oracle.

Tolerances (the bar the split-precision form is built to):
  * integer outputs (tested flag, .count, emitted k-mer set): identical, except
    k-mers whose |cor| lies within 1e-9 (relative) of CORR_THRESHOLD;
  * -log10 p: absolute error <= 1e-6 (split) / 1e-9 (fp64), every k-mer;
  * chi-square: relative error <= 1e-6 at the 99th percentile and for every
    k-mer with chi2 >= 1e-3 (split); <= 1e-9 everywhere (fp64).  Below that the
    relative error of any finite-precision x.y' is unbounded (chi2 -> 0).
"""
import numpy as np
import pytest

import helpers as H
from oracle import oracle as O
from supergwas_b200 import api, synth

pytestmark = pytest.mark.gpu

TOL = {"split": dict(ml=1e-6, rel99=1e-6, relmax=1e-6, relfloor=1e-3),
       "fp64": dict(ml=1e-9, rel99=1e-9, relmax=1e-9, relfloor=0.0)}


def check_against_oracle(res, o, prec, thr, log10_thresh=6.0):
    st = res.stats
    tol = TOL[prec]
    band = np.abs(np.abs(o["cor"]) - thr) <= 1e-9 * max(thr, 1e-3)
    same = (st["tested"] == o["tested"]) | band
    assert same.all(), np.nonzero(~same)[0][:10]
    assert abs(res.n_tested - o["n_tested"]) <= int(band.sum())
    msk = st["tested"] & o["tested"]
    if msk.any():
        T0, T1 = o["chisq"][msk], st["chisq"][msk]
        rel = np.abs(T1 - T0) / np.maximum(T0, 1e-300)
        assert np.percentile(rel, 99) <= tol["rel99"]
        big = T0 >= tol["relfloor"]
        if big.any():
            assert rel[big].max() <= tol["relmax"], rel[big].max()
        ml = np.abs(st["mlog10p"][msk] - o["mlog10p"][msk])
        assert ml.max() <= tol["ml"], ml.max()
        e0, e1 = o["effect"][msk], st["effect"][msk]
        # effect = xyM/(xxM yyM): relative error follows xyM's (absolute floor for xyM ~ 0)
        assert np.all(np.abs(e1 - e0) <= 1e-6 * np.abs(e0) + 1e-9 * np.abs(e0).max())
    # emitted rows == oracle's p <= 10^-log10 set (outside the band)
    p_thr = 10.0 ** (-log10_thresh)
    exp = set(np.nonzero(o["tested"] & (o["pval"] <= p_thr))[0].tolist())
    got = set(res.hits["kmer"].tolist())
    ml_cut = np.abs(o["mlog10p"] - log10_thresh) <= 1e-6
    diff = (exp ^ got) - set(np.nonzero(band | ml_cut)[0].tolist())
    assert not diff, sorted(diff)[:10]
    assert np.all(np.diff(res.hits["kmer"].astype(np.int64)) > 0)


@pytest.mark.parametrize("prec", ["split", "fp64"])
@pytest.mark.parametrize("name", H.FIXTURES)
def test_fixture_parity(built, prec, name):
    fx = H.load_fixture(name)
    n = int(fx["idxs"].shape[0])
    for thr in (0.0, 0.2):
        o = O.cols_stats(fx["packed"], n, fx["U"], fx["y"], thr)
        with api.Kgwas(precision=prec, corr_threshold=thr, log10_thresh=2.0) as g:
            yy = g.set_structure(fx["U"], fx["y"])
            assert abs(yy - o["yyM"]) <= 1e-12 * max(1.0, abs(o["yyM"])) + 1e-13
            res = g.run_host(fx["packed"], stats=True)
        check_against_oracle(res, o, prec, thr, 2.0)


SHAPES = [  # (n, m, r)  -- ragged n and m around the 64-bit word, 128-k-mer tile and 256-sample chunk
    (1, 50, 0), (2, 300, 1), (63, 129, 2), (64, 128, 3), (65, 127, 3), (127, 1000, 4),
    (128, 1, 4), (129, 257, 5), (255, 3000, 6), (256, 2049, 8), (257, 999, 8), (1000, 5000, 16),
    (2000, 3000, 20), (700, 777, 32),
]


@pytest.mark.parametrize("prec", ["split", "fp64"])
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "n%d_m%d_r%d" % s)
def test_shapes(built, prec, shape):
    n, m, r = shape
    S = max(1, min(5, n // 2))
    ds = synth.simulate(n=n, m=m, S=S, r=min(r, max(n - 1, 0)) if n > 1 else 0, n_causal=min(3, m),
                        missing=0.0, seed=100 + n + m)
    X = ds.packed_overlap()
    U = ds.U if r > 0 and n > 1 else np.zeros((ds.n, 0))
    o = O.cols_stats(X, ds.n, U, ds.y, 0.0)
    with api.Kgwas(precision=prec, corr_threshold=0.0, log10_thresh=1.0) as g:
        g.set_structure(U, ds.y)
        res = g.run_host(X, stats=True)
    check_against_oracle(res, o, prec, 0.0, 1.0)


def test_empty_input(built):
    with api.Kgwas() as g:
        g.set_structure(np.ones((10, 1)) / np.sqrt(10), np.arange(10.0))
        res = g.run_host(np.zeros((0, 2), np.uint64))
    assert res.n_tested == 0 and res.hits.shape == (0,)


def test_padding_bits_ignored(built):
    """Bits at sample positions >= n must not change anything."""
    ds = synth.simulate(n=100, m=2000, S=4, r=4, n_causal=5, missing=0.0, seed=9)
    X = ds.packed_overlap()
    Xg = X.copy()
    Xg[:, 1] |= np.uint64(0xFFFFFFF000000000)   # samples 100..127
    for prec in ("split", "fp64"):
        with api.Kgwas(precision=prec, corr_threshold=0.0, log10_thresh=0.5) as g:
            g.set_structure(ds.U, ds.y)
            a = g.run_host(X, stats=True)
            b = g.run_host(Xg, stats=True)
        assert a.n_tested == b.n_tested
        assert np.array_equal(a.hits, b.hits)


def test_device_launch_matches_host_run(built):
    import torch
    ds = synth.simulate(n=1000, m=20000, S=8, r=16, n_causal=20, missing=0.05, seed=4)
    X = ds.packed_overlap()
    with api.Kgwas(corr_threshold=0.0, log10_thresh=2.0) as g:
        g.set_structure(ds.U, ds.y)
        a = g.run_host(X, stats=True)
        dx = torch.from_numpy(X.view(np.int64)).cuda()
        st = torch.cuda.current_stream().cuda_stream
        g.launch_device(dx.data_ptr(), X.shape[0], X.shape[1], st, stats=True)
        b = g.fetch(stats=True)
        assert g.last_launch_count() == 2     # association kernel + FP64 refinement
    assert a.n_tested == b.n_tested
    assert np.array_equal(a.hits, b.hits)
    for k in ("tested", "chisq", "pval", "effect"):
        assert np.array_equal(a.stats[k], b.stats[k])


def test_chunked_host_run_is_identical(built, monkeypatch):
    ds = synth.simulate(n=300, m=50000, S=5, r=6, n_causal=20, missing=0.0, seed=5)
    X = ds.packed_overlap()
    with api.Kgwas(corr_threshold=0.0, log10_thresh=1.5) as g:
        g.set_structure(ds.U, ds.y)
        a = g.run_host(X, stats=True)
        monkeypatch.setenv("KG_CHUNK_MB", "1")   # 48-byte rows: 3 chunks, 2 buffers in flight
        b = g.run_host(X, stats=True)
        assert g.last_launch_count() == 3 * 2  # per chunk: association kernel + FP64 refinement
    assert a.n_tested == b.n_tested
    assert np.array_equal(a.hits, b.hits)
    assert np.array_equal(a.stats["chisq"], b.stats["chisq"])


def test_hit_buffer_growth(built):
    """More rows than the initial device hit buffer (65536): re-run with a larger one."""
    ds = synth.simulate(n=64, m=150000, S=2, r=2, n_causal=0, missing=0.0, seed=6)
    X = ds.packed_overlap()
    o = O.cols_stats(X, ds.n, ds.U, ds.y, 0.0)
    with api.Kgwas(corr_threshold=0.0, log10_thresh=0.0) as g:
        g.set_structure(ds.U, ds.y)
        res = g.run_host(X)
    assert res.hits.shape[0] == o["n_tested"] > 65536


def test_errors_are_codes_not_crashes(built):
    with api.Kgwas() as g:
        with pytest.raises(api.KgError) as e:
            g.run_host(np.zeros((4, 2), np.uint64))
        assert e.value.code == 4                      # structure not set
        g.set_structure(np.ones((200, 1)) / np.sqrt(200), np.arange(200.0))
        with pytest.raises(api.KgError) as e:
            g.run_host(np.zeros((4, 3), np.uint64))   # odd words_per_kmer
        assert e.value.code == 1
        with pytest.raises(api.KgError) as e:
            g.run_host(np.zeros((4, 2), np.uint64))   # 128 bits < n = 200
        assert e.value.code == 1
        with pytest.raises(api.KgError):
            g.set_structure(np.full((10, 1), np.nan), np.arange(10.0))


KERNEL_SHAPES = [(1000, 20000, 16, 16), (950, 3001, 10, 16), (1500, 7000, 20, 32), (64, 4000, 4, 16),
                 (300, 129, 6, 16), (1024, 1, 16, 16)]


@pytest.mark.parametrize("shape", KERNEL_SHAPES, ids=lambda s: "n%d_m%d_r%d_w%d" % s)
def test_tensor_kernels_bit_identical(built, shape, monkeypatch):
    """The TMEM-A and smem-A kernels compute the same exact int32 limb sums
    and the same epilogue: their statistics must agree bit for bit, and both
    must meet the oracle tolerances.  Rows are padded to `wpk` words so small
    n also reaches the TMEM-A kernel."""
    n, m, r, wpk = shape
    ds = synth.simulate(n=n, m=m, S=4, r=r, n_causal=min(5, m), missing=0.05, seed=7 + n)
    X = ds.packed_overlap()
    if X.shape[1] < wpk:
        X = np.concatenate([X, np.zeros((m, wpk - X.shape[1]), np.uint64)], axis=1)
    o = O.cols_stats(X, ds.n, ds.U, ds.y, 0.0)
    out = {}
    for kern in ("ts", "ss"):
        monkeypatch.setenv("KG_KERNEL", kern)
        with api.Kgwas(corr_threshold=0.0, log10_thresh=1.0) as g:
            g.set_structure(ds.U, ds.y)
            out[kern] = g.run_host(X, stats=True)
            assert g.last_kernel() == kern
        check_against_oracle(out[kern], o, "split", 0.0, 1.0)
    for f in ("tested", "chisq", "pval", "effect", "mlog10p", "xxM", "xyM", "cor"):
        assert np.array_equal(out["ts"].stats[f], out["ss"].stats[f]), f
    assert np.array_equal(out["ts"].hits, out["ss"].hits)


def test_sample_positions(built):
    """Rows holding every sample of the batch, phenotype on a subset
    (kg_set_structure_ex) == rows repacked to the overlap."""
    ds = synth.simulate(n=1000, m=10000, S=8, r=16, n_causal=10, missing=0.2, seed=12)
    Xo = ds.packed_overlap()
    o = O.cols_stats(Xo, ds.n, ds.U, ds.y, 0.0)
    for prec in ("split", "fp64"):
        with api.Kgwas(precision=prec, corr_threshold=0.0, log10_thresh=1.0) as g:
            g.set_structure(ds.U, ds.y, ds.idxs, ds.n_all)
            res = g.run_host(ds.packed_all, stats=True)
        check_against_oracle(res, o, prec, 0.0, 1.0)


def test_stats_off_gives_same_hits(built):
    """Without per-k-mer outputs the epilogue skips log/erfc for k-mers that
    cannot reach the emit cut; the emitted rows must not change."""
    ds = synth.simulate(n=1000, m=50000, S=8, r=16, n_causal=30, missing=0.05, seed=13)
    X = ds.packed_overlap()
    for lt in (0.0, 1.3, 4.0, 8.0):
        with api.Kgwas(corr_threshold=0.0, log10_thresh=lt) as g:
            g.set_structure(ds.U, ds.y)
            a = g.run_host(X, stats=True)
            b = g.run_host(X)
        assert a.n_tested == b.n_tested
        assert np.array_equal(a.hits, b.hits)
