"""Pin the FP64 oracle to the reference's own outputs (CPU only).

The golden files under tests/golden/ were produced by running the
reference kgwas binary (COLS mode, FP32 linear algebra, src/kgwas.cpp:138-166;
ROWS mode, FP64, src/kgwas.cpp:455-476).  The oracle must reproduce:
  * the .count value and the emitted k-mer rows, in order, exactly, except for
    k-mers inside the tolerance band of the pre-filter or emit cut;
  * ROWS-mode floats to the reference's 6-significant-digit print precision
    (values at a rounding boundary may differ by one unit in the last digit);
  * COLS-mode floats to the reference's FP32 resolution.
"""
import os

import numpy as np
import pytest

import helpers as H
from oracle import oracle as O

ROWS_REL = 1.1e-5    # 6 printed significant digits: one unit in the last digit is <= 1e-5 relative
COLS_REL = 1e-2      # reference COLS computes xxM/xyM in FP32 (measured <= 6.5e-3 on these fixtures)


def _thr(variant):
    return float(variant.get("env", {}).get("CORR_THRESHOLD", "0.2"))


def _log10(variant):
    a = variant["args"]
    return float(a[0]) if a and not a[0].startswith("--") else 6.0


def _log10_2d(variant):
    a = variant["args"]
    if "--log10-thresh-2d" in a:
        return float(a[a.index("--log10-thresh-2d") + 1])
    return 15.0


def _oracle_text(fx, st, variant):
    n = fx["packed"].shape[0] and int(fx["idxs"].shape[0])
    from supergwas_b200 import synth
    X = synth.unpack_rows(fx["packed"], n)

    def bits_of(j):
        return "".join("1" if b else "0" for b in X[j])
    return O.emit_rows(fx["kmers"], st, _log10(variant), _log10_2d(variant), bits_of)


@pytest.mark.parametrize("name", H.FIXTURES)
def test_oracle_matches_reference(name):
    fx = H.load_fixture(name)
    mt = H.meta(name)
    n = int(fx["idxs"].shape[0])
    for v in mt["variants"]:
        thr = _thr(v)
        st = O.cols_stats(fx["packed"], n, fx["U"], fx["y"], thr)
        band = H.band_kmers(st, thr, _log10(v))
        one, two = _oracle_text(fx, st, v)
        got1 = [l.split("\t") for l in one.splitlines()]
        got2 = [l.split("\t") for l in two.splitlines()] if two is not None else None
        for mode, tol in (("rows", ROWS_REL), ("cols", COLS_REL)):
            cnt = open(H.ref_file(name, mode, v["name"], ".tsv.count")).read()
            exp = O.count_line("batch_000.tsv", st["n_tested"])
            if not band:
                assert cnt == exp, (name, v["name"], mode)
            ref1 = H.parse_rows(H.ref_file(name, mode, v["name"], ".tsv"))
            H.compare_rows(got1, ref1, fx["kmers"], band, tol)
            ref2 = H.parse_rows(H.ref_file(name, mode, v["name"], ".2d.tsv"))
            if got2 is None:
                assert ref2 is None
            else:
                H.compare_rows(got2, ref2, fx["kmers"], band, tol)


def test_yspan_emits_p_one():
    fx = H.load_fixture("yspan")
    st = O.cols_stats(fx["packed"], int(fx["idxs"].shape[0]), fx["U"], fx["y"], 0.0)
    assert st["yyM"] < 1e-12
    assert np.all(st["pval"][st["tested"]] == 1.0)
    assert np.all(st["effect"] == 0.0)


def test_edge_constant_columns_not_tested():
    fx = H.load_fixture("edge")
    st = O.cols_stats(fx["packed"], int(fx["idxs"].shape[0]), fx["U"], fx["y"], 0.0)
    # k-mers 5..8 are constant on the phenotyped samples (all-0 / all-1)
    assert not st["tested"][5:9].any()


@pytest.mark.slow
def test_oracle_matches_reference_cfg1():
    """Config 1 (n=200, m=1e6, r=5+1): full reference parity of the oracle."""
    ds = H.load_cfg1()
    X = ds.packed_overlap()
    mt = H.meta("cfg1")
    for v in mt["variants"]:
        thr = _thr(v)
        st = O.cols_stats(X, ds.n, ds.U, ds.y, thr)
        band = H.band_kmers(st, thr, _log10(v))
        fx = {"packed": X, "idxs": ds.idxs, "kmers": ds.kmers}
        one, two = _oracle_text(fx, st, v)
        got1 = [l.split("\t") for l in one.splitlines()]
        got2 = [l.split("\t") for l in two.splitlines()]
        for mode, tol in (("rows", ROWS_REL), ("cols", COLS_REL)):
            cnt = open(H.ref_file("cfg1", mode, v["name"], ".tsv.count")).read().split("\t")
            assert abs(int(cnt[1]) - st["n_tested"]) <= len(band)
            ref1 = H.parse_rows(H.ref_file("cfg1", mode, v["name"], ".tsv"))
            H.compare_rows(got1, ref1, ds.kmers, band, tol)
            ref2 = H.parse_rows(H.ref_file("cfg1", mode, v["name"], ".2d.tsv"))
            H.compare_rows(got2, ref2, ds.kmers, band, tol)
