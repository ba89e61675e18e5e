"""The allocation-free entry point, kg_run_device_noalloc.

It exists for callers that may not allocate device memory -- a framework
that owns every device byte through its own pool, a plugin inside such a
process, a job whose memory budget is fixed before it runs.  They pass their
own device buffers for the packed rows and for the emitted rows; the call's
only other device memory is a fixed static array inside the library.

These tests call it through the C ABI and check it against the existing
entry point (kg_set_structure + kg_run_host) on two calls in a row -- the
second with another phenotype, thresholds and batch, so a stale counter or
limb image left by the first call would show -- and check the size limit and
the short-buffer report.  This file is collected last on purpose.
"""
import numpy as np
import pytest

from supergwas_b200 import api, synth

pytestmark = pytest.mark.gpu


def _device_call(X, U, y, thr, lt, cap):
    import torch
    dx = torch.from_numpy(np.ascontiguousarray(X).view(np.int64)).cuda()
    hits = torch.zeros((max(cap, 1), 4), dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream()
    rc, nt, nh, msg = api.run_device_noalloc(dx.data_ptr(), X.shape[0], X.shape[1], U, y, thr, lt,
                                             hits.data_ptr(), cap, st.cuda_stream)
    h = hits.cpu().numpy().view(api.HIT_DTYPE).reshape(-1)[: min(nh, cap)]
    return rc, nt, np.sort(h, order="kmer"), msg


def _existing(X, U, y, thr, lt):
    with api.Kgwas(precision="split", corr_threshold=thr, log10_thresh=lt) as g:
        g.set_structure(U, y)
        return g.run_host(X)


def _same(a_hits, b_hits):
    """Same rows; values within the parity tests' tolerances (chi-square and
    effect 1e-6 relative, -log10 p 1e-6 absolute)."""
    from oracle import oracle as O
    assert np.array_equal(a_hits["kmer"], b_hits["kmer"])
    for f in ("effect", "chisq"):
        assert np.allclose(a_hits[f], b_hits[f], rtol=1e-6, atol=0.0), f
    assert np.all(np.abs(O.mlog10p(a_hits["chisq"]) - O.mlog10p(b_hits["chisq"])) <= 1e-6)


def test_noalloc_matches_existing_entry_point_twice():
    ds = synth.simulate(n=1000, m=20000, S=8, r=16, n_causal=20, missing=0.05, seed=31)
    X = ds.packed_overlap()
    ref = _existing(X, ds.U, ds.y, 0.0, 2.0)
    rc, nt, hits, msg = _device_call(X, ds.U, ds.y, 0.0, 2.0, 4096)
    assert rc == 0, msg
    assert nt == ref.n_tested
    _same(hits, ref.hits)

    ds2 = synth.simulate(n=500, m=7001, S=4, r=6, n_causal=10, missing=0.1, seed=32)
    X2 = ds2.packed_overlap()
    ref2 = _existing(X2, ds2.U, ds2.y, 0.2, 1.0)
    rc, nt, hits, msg = _device_call(X2, ds2.U, ds2.y, 0.2, 1.0, 4096)
    assert rc == 0, msg
    assert nt == ref2.n_tested
    _same(hits, ref2.hits)


def test_noalloc_strong_hits_match_fp64_oracle():
    """Rows far above the default cut (chi-square above 100, p <= 1e-6)
    come out of the FP64 refinement: their -log10 p agrees with the FP64
    oracle to 1e-8, where the split form alone is off by about 1e-5 at these
    chi-square values.  Every tested k-mer agrees to the parity bar (1e-6)."""
    from oracle import oracle as O
    ds = synth.simulate(n=1000, m=20000, S=8, r=16, n_causal=20, missing=0.05, seed=34)
    X = ds.packed_overlap()
    x = synth.unpack_rows(X[:16], ds.n).astype(np.float64)
    y = ds.y + 3.0 * x[3] - 2.5 * x[7] + 2.0 * x[11]
    o = O.cols_stats(X, ds.n, ds.U, y, 0.0)
    for call in range(2):  # the second call reuses the scratch the first left behind
        rc, nt, hits, msg = _device_call(X, ds.U, y, 0.0, 6.0, 4096)
        assert rc == 0, msg
        assert nt == o["n_tested"]
        exp = np.nonzero(o["tested"] & (o["pval"] <= 1e-6))[0]
        band = np.abs(o["mlog10p"] - 6.0) <= 1e-6
        got = hits["kmer"].astype(np.int64)
        assert set(got.tolist()) ^ set(exp.tolist()) <= set(np.nonzero(band)[0].tolist())
        T0 = o["chisq"][got]
        assert T0.min() >= 23.0 and T0.max() > 100.0
        ml = np.abs(O.mlog10p(hits["chisq"]) - o["mlog10p"][got])
        assert ml.max() <= 1e-8, ml.max()
        assert np.allclose(hits["chisq"], T0, rtol=1e-10, atol=0.0)
        assert np.allclose(hits["effect"], o["effect"][got], rtol=1e-9, atol=0.0)


def test_noalloc_rejects_oversized_structure():
    # 5000 overlap samples and U with 34 columns: the limb image (5120 x 112) exceeds 256 KiB
    rng = np.random.default_rng(1)
    n = 5000
    U, _ = np.linalg.qr(rng.standard_normal((n, 34)))
    X = np.zeros((8, synth.words_per_kmer(n)), np.uint64)
    rc, nt, hits, msg = _device_call(X, U, rng.standard_normal(n), 0.0, 6.0, 16)
    assert rc == 6, msg  # KG_ERR_UNSUPPORTED
    assert "maximum" in msg


def test_noalloc_reports_short_hit_buffer():
    ds = synth.simulate(n=200, m=5000, S=4, r=4, n_causal=5, missing=0.0, seed=33)
    X = ds.packed_overlap()
    ref = _existing(X, ds.U, ds.y, 0.0, 0.0)      # every tested k-mer is a row
    rc, nt, hits, msg = _device_call(X, ds.U, ds.y, 0.0, 0.0, 100)
    assert rc == 1, msg                             # KG_ERR_INVALID, counts still reported
    assert nt == ref.n_tested and "larger buffer" in msg
    rc, nt, hits, msg = _device_call(X, ds.U, ds.y, 0.0, 0.0, ref.n_tested)
    assert rc == 0, msg
    _same(hits, ref.hits)
