"""kg_reserve_host: the host pipeline's buffers allocated ahead of kg_run_host.

bin/kgwas reserves them on the thread that creates the context while it still
reads the column files; the run that follows must give the same rows and
counts as a run that allocates them itself, also when the reservation was
made for a smaller or a larger batch (the buffers grow, or are reused).
"""
import numpy as np
import pytest

from oracle import oracle as O
from supergwas_b200 import api, synth
from test_gpu_parity import check_against_oracle

pytestmark = pytest.mark.gpu


def test_reserved_buffers_give_the_same_run(built, monkeypatch):
    monkeypatch.setenv("KG_CHUNK_MB", "2")  # several chunks per run
    ds = synth.simulate(n=1000, m=60_000, S=8, r=16, n_causal=20, missing=0.05, seed=73)
    X = ds.packed_overlap()
    m, wpk = X.shape
    o = O.cols_stats(X, ds.n, ds.U, ds.y, 0.0)
    with api.Kgwas(precision="split", corr_threshold=0.0, log10_thresh=2.0) as g:
        g.set_structure(ds.U, ds.y)
        ref = g.run_host(X, stats=True)
    check_against_oracle(ref, o, "split", 0.0, 2.0)
    for reserve_rows in (m, 1000, 4 * m):
        with api.Kgwas(precision="split", corr_threshold=0.0, log10_thresh=2.0) as g:
            g.reserve_host(reserve_rows, wpk)  # before the structure, as bin/kgwas does
            g.set_structure(ds.U, ds.y)
            res = g.run_host(X)
            assert res.n_tested == ref.n_tested
            assert np.array_equal(res.hits, ref.hits)


def test_reserve_rejects_an_empty_batch(built):
    with api.Kgwas() as g:
        with pytest.raises(api.KgError):
            g.reserve_host(0, 16)
