"""Pin the pair-test oracle to the reference's kgwas_2d (CPU only).

tests/golden/pairs/ holds a sharded index built by the reference's
build_index and the outputs of the reference's kgwas_2d on it
(src/kgwas_2d.cpp).  The reference evaluates x12.y and U^T x12 in FP32
(src/kgwas_2d.cpp:306-312), the oracle in long double, so:
  * the k-mer list (.kmers) is identical: index reader, canonical order,
    dropped bitstrings;
  * the pair rows are the same set in the same order, except pairs whose p
    lies within FP32 resolution of the cut;
  * effect and p agree to FP32 resolution (measured <= 2e-5 relative).
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
FX = os.path.join(HERE, "golden", "pairs")
PAIR_REL = 1e-3       # FP32 x12.y and U^T x12 in the reference


def load_pairs_fixture():
    z = np.load(os.path.join(FX, "inputs.npz"))
    K, kmers, bits = O.read_index_bits(os.path.join(FX, "index"))
    idxs = z["idxs"]
    n = idxs.shape[0]
    X, keep = O.pair_matrix(bits, idxs, n)
    return dict(U=z["U"], y=z["y"], idxs=idxs, n=n, X=X, kmers=[kmers[j] for j in keep])


def parse_pairs(path):
    rows = []
    for line in open(path).read().splitlines():
        a, b, e, p = line.split("\t")
        rows.append((int(a), int(b), float(e), float(p)))
    return rows


def log10_of(v):
    a = v["args"]
    return float(a[0]) if a and not a[0].startswith("-") else 6.0


def task_range(v, N):
    a = v["args"]
    nt = int(a[a.index("--num-tasks") + 1]) if "--num-tasks" in a else 1
    t = int(a[a.index("--task-id") + 1]) if "--task-id" in a else 0
    per = (N + nt - 1) // nt
    return t, nt, t * per, min(t * per + per, N)


def expected_pairs(st, thr, r0, r1):
    N = st["pval"].shape[0]
    p_thr = 10.0 ** (-thr)
    ii, jj = np.nonzero(st["evaluated"] & (st["pval"] <= p_thr))
    sel = (ii >= r0) & (ii < r1)
    return [(int(i), int(j), st["effect"][i, j], st["pval"][i, j]) for i, j in zip(ii[sel], jj[sel])]


def compare_pairs(got, ref, st, thr, rel):
    """Same (i, j) rows in the same order, except pairs whose p is within
    `rel` of the cut; matching rows agree to `rel`."""
    p_thr = 10.0 ** (-thr)
    g = {(a, b): (e, p) for a, b, e, p in got}
    r = {(a, b): (e, p) for a, b, e, p in ref}
    for k in set(g) ^ set(r):
        p = st["pval"][k]
        assert abs(p - p_thr) <= rel * p_thr, (k, p, p_thr)
    assert [x[:2] for x in got if x[:2] in r] == [x[:2] for x in ref if x[:2] in g]
    for k in set(g) & set(r):
        (e0, p0), (e1, p1) = r[k], g[k]
        assert abs(e1 - e0) <= rel * abs(e0) + 1e-9, (k, e0, e1)
        assert abs(p1 - p0) <= rel * p0 + 1e-300, (k, p0, p1)


def test_pairs_oracle_matches_reference():
    fx = load_pairs_fixture()
    meta = json.load(open(os.path.join(FX, "meta.json")))
    N = fx["X"].shape[0]
    st = O.pairs_stats(fx["X"], fx["n"], fx["U"], fx["y"])
    for v in meta["variants"]:
        tag = "ref_" + v["name"]
        assert open(os.path.join(FX, tag + ".rc")).read().strip() == "0"
        t, nt, r0, r1 = task_range(v, N)
        path = os.path.join(FX, tag + (f".part_{t}.tsv" if nt > 1 else ".tsv"))
        if r0 >= N:
            assert not os.path.exists(path)          # "no rows to process": no files at all
            assert not os.path.exists(os.path.join(FX, tag + ".kmers"))
            continue
        ref = parse_pairs(path)
        got = expected_pairs(st, log10_of(v), r0, r1)
        compare_pairs(got, ref, st, log10_of(v), PAIR_REL)
        kf = os.path.join(FX, tag + ".kmers")
        if t == 0:
            assert open(kf).read().splitlines() == fx["kmers"]
        else:
            assert not os.path.exists(kf)


def test_pairs_row_text_format():
    assert O.pair_rows([(2, 9, -0.00897499034, 1.193936660e-03)]) == "2\t9\t-0.00897499034\t1.193936660e-03\n"
    assert O.pair_rows([(0, 1, 1.5e-7, 2e-300)]) == "0\t1\t1.5e-07\t2.000000000e-300\n"
