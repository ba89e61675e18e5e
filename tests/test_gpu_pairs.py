"""GPU parity of the 2-D pair test (kg_pairs_run_host, bin/kgwas_2d).

Against the FP64 pair oracle (oracle/kgwas_oracle.c, kgo_pairs) and the
reference kgwas_2d's own outputs (tests/golden/pairs/).  Tolerances:
  * pair set and order: identical, except pairs whose p lies within 1e-9
    (relative) of the cut;
  * -log10 p: absolute error <= 1e-6 for every returned pair; chi-square
    relative error <= 1e-6 for chi-square >= 1e-3 (split form; pairs with
    chi-square >= 12 are recomputed in FP64 and agree to 1e-9);
  * against the reference's files: FP32 resolution (test_pairs_golden.py).
"""
import json
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import oracle as O
from supergwas_b200 import api, build, synth
from test_pairs_golden import FX, PAIR_REL, compare_pairs, load_pairs_fixture, log10_of, parse_pairs, task_range

pytestmark = pytest.mark.gpu


def pair_dataset(n, N, r, seed):
    ds = synth.simulate(n=n, m=N, S=4, r=r, n_causal=0, missing=0.0, seed=seed)
    X = ds.packed_overlap()
    x = synth.unpack_rows(X, ds.n).astype(float)
    rng = np.random.default_rng(seed)
    y = 2.0 * x[3] * x[7] + 1.0 * x[11] * x[13] + rng.standard_normal(ds.n)
    return X, ds.n, ds.U, y


def check(res, n_eval, st, thr, r0, r1):
    N = st["pval"].shape[0]
    ev = st["evaluated"].copy()
    ev[:r0] = False
    ev[r1:] = False
    assert n_eval == int(ev.sum())
    p_thr = 10.0 ** (-thr)
    exp = ev & (st["pval"] <= p_thr)
    got = np.zeros_like(exp)
    got[res["a"].astype(np.int64), res["b"].astype(np.int64)] = True
    diff = np.argwhere(got != exp)
    for i, j in diff:
        assert abs(st["pval"][i, j] - p_thr) <= 1e-9 * p_thr, (i, j)
    order = np.lexsort((res["b"], res["a"]))
    assert np.array_equal(order, np.arange(res.shape[0]))
    a, b = res["a"].astype(np.int64), res["b"].astype(np.int64)
    assert np.all(a < b)
    T0, T1 = st["chisq"][a, b], res["chisq"]
    ml = np.abs(O.mlog10p(T1) - st["mlog10p"][a, b])
    assert ml.max(initial=0) <= 1e-6, ml.max()
    big = T0 >= 1e-3
    rel = np.abs(T1 - T0) / np.maximum(T0, 1e-300)
    assert rel[big].max(initial=0) <= 1e-6, rel[big].max()
    ref = T0 >= 12.0
    assert rel[ref].max(initial=0) <= 1e-9, rel[ref].max()
    assert np.all(np.abs(res["effect"][ref] - st["effect"][a[ref], b[ref]]) <=
                  1e-9 * np.abs(st["effect"][a[ref], b[ref]]) + 1e-15)


@pytest.mark.parametrize("case", [(1000, 300, 16, 1), (200, 257, 5, 2), (61, 130, 3, 3), (2000, 160, 20, 4),
                                  (130, 129, 0, 5)],
                         ids=["n1000_N300_r16", "n200_N257_r5", "n61_N130_r3", "n2000_N160_r20", "n130_N129_r0"])
def test_pairs_match_oracle(built, case):
    n, N, r, seed = case
    X, n, U, y = pair_dataset(n, N, r, seed)
    st = O.pairs_stats(X, n, U, y)
    for thr in (0.0, 2.0):
        with api.Kgwas(log10_thresh=thr) as g:
            g.set_structure(U, y)
            res, n_eval = g.run_pairs_host(X)
        check(res, n_eval, st, thr, 0, N)


def test_pairs_row_ranges_partition_the_pairs(built):
    X, n, U, y = pair_dataset(300, 333, 6, 9)
    st = O.pairs_stats(X, n, U, y)
    N = X.shape[0]
    parts = []
    with api.Kgwas(log10_thresh=1.0) as g:
        g.set_structure(U, y)
        full, ne = g.run_pairs_host(X)
        for r0, r1 in ((0, 100), (100, 101), (101, 250), (250, N)):
            res, n_eval = g.run_pairs_host(X, r0, r1)
            check(res, n_eval, st, 1.0, r0, r1)
            parts.append(res)
        empty, n0 = g.run_pairs_host(X, N - 1, N)    # the last row has no j > i
    assert np.array_equal(np.concatenate(parts), full)
    assert empty.shape[0] == 0 and n0 == 0


def test_pairs_cli_matches_reference(built):
    fx = load_pairs_fixture()
    meta = json.load(open(os.path.join(FX, "meta.json")))
    N = fx["X"].shape[0]
    st = O.pairs_stats(fx["X"], fx["n"], fx["U"], fx["y"])
    work = tempfile.mkdtemp()
    try:
        ubin = os.path.join(work, "U2D.bin")
        synth.write_ubin(ubin, fx["U"])
        exe = os.path.join(build.BIN_DIR, "kgwas_2d")
        for v in meta["variants"]:
            out = os.path.join(work, "out_" + v["name"])
            r = subprocess.run([exe, os.path.join(FX, "samples.txt"), os.path.join(FX, "phenotype.txt"), ubin,
                                os.path.join(FX, "index"), out, *v["args"]], capture_output=True, text=True,
                               env=dict(os.environ, BLAS_THREADS="4", EMIT_THREADS="4"))
            assert r.returncode == 0, r.stderr[-2000:]
            t, nt, r0, r1 = task_range(v, N)
            tag = "ref_" + v["name"]
            suffix = f".part_{t}.tsv" if nt > 1 else ".tsv"
            if r0 >= N:
                assert not os.path.exists(out + suffix) and not os.path.exists(out + ".kmers")
                continue
            compare_pairs(parse_pairs(out + suffix), parse_pairs(os.path.join(FX, tag + suffix)), st,
                          log10_of(v), PAIR_REL)
            if t == 0:
                assert open(out + ".kmers").read() == open(os.path.join(FX, tag + ".kmers")).read()
            else:
                assert not os.path.exists(out + ".kmers")
    finally:
        shutil.rmtree(work)
