"""The kgwas program against the reference's own output files.

Integer parity (row set, row order, k-mer strings, .2d bitstrings, .count)
is exact outside the tolerance band of the pre-filter and emit cuts; floats
agree to the reference's print precision (ROWS mode, FP64) or its FP32
resolution (COLS mode).
"""
import os
import tempfile

import pytest

import helpers as H
from oracle import oracle as O
from test_oracle_golden import COLS_REL, ROWS_REL, _log10, _thr

pytestmark = pytest.mark.gpu


def _check_outputs(out, name, mode, variant, kmers, band):
    tol = ROWS_REL if mode == "rows" else COLS_REL
    got = open(out + ".count").read()
    ref = open(H.ref_file(name, mode, variant["name"], ".tsv.count")).read()
    if band:
        assert abs(int(got.split("\t")[1]) - int(ref.split("\t")[1])) <= len(band)
        assert got.split("\t")[0] == ref.split("\t")[0]
    else:
        assert got == ref
    H.compare_rows(H.parse_rows(out), H.parse_rows(H.ref_file(name, mode, variant["name"], ".tsv")),
                   kmers, band, tol)
    ref2 = H.parse_rows(H.ref_file(name, mode, variant["name"], ".2d.tsv"))
    got2 = H.parse_rows(O.path_2d(out))
    assert (ref2 is None) == (got2 is None)
    if ref2 is not None:
        H.compare_rows(got2, ref2, kmers, band, tol)


@pytest.mark.parametrize("prec", ["split", "fp64"])
@pytest.mark.parametrize("name", H.FIXTURES)
def test_cli_matches_reference(built, name, prec):
    fx = H.load_fixture(name)
    n = int(fx["idxs"].shape[0])
    work = tempfile.mkdtemp()
    paths, rows = H.materialise(name, work)
    for v in H.meta(name)["variants"]:
        st = O.cols_stats(fx["packed"], n, fx["U"], fx["y"], _thr(v))
        band = H.band_kmers(st, _thr(v), _log10(v))
        for mode, inp in (("cols", paths["batch"]), ("rows", rows)):
            out = os.path.join(work, f"{mode}_{v['name']}", "batch_000.tsv")
            os.makedirs(os.path.dirname(out))
            env = dict(v.get("env", {}))
            env["KGWAS_PRECISION"] = prec
            r = H.run_cli([paths["samples"], paths["pheno"], inp, paths["ubin"], out, *v["args"],
                           "--mode", mode], env)
            assert r.returncode == 0, r.stderr[-2000:]
            _check_outputs(out, name, mode, v, fx["kmers"], band)


@pytest.mark.slow
def test_cli_matches_reference_cfg1(built):
    """Config 1: n=200 (190 phenotyped), m=1e6, r=5+1, auto-detected COLS mode and gz ROWS input."""
    ds = H.load_cfg1()
    X = ds.packed_overlap()
    work = tempfile.mkdtemp()
    paths, rows = H.materialise_cfg1(work)
    for v in H.meta("cfg1")["variants"]:
        st = O.cols_stats(X, ds.n, ds.U, ds.y, _thr(v))
        band = H.band_kmers(st, _thr(v), _log10(v))
        for mode, inp in (("cols", paths["batch"]), ("rows", rows)):
            out = os.path.join(work, f"{mode}_{v['name']}", "batch_000.tsv")
            os.makedirs(os.path.dirname(out))
            r = H.run_cli([paths["samples"], paths["pheno"], inp, paths["ubin"], out, *v["args"]],
                          v.get("env", {}))
            assert r.returncode == 0, r.stderr[-2000:]
            _check_outputs(out, "cfg1", mode, v, ds.kmers, band)


@pytest.mark.parametrize("name", ["small", "edge"])
def test_kbits_sidecar_reuse(built, name):
    """KGWAS_KBITS=1: the first run writes the packed rows next to the batch,
    later runs read them back instead of the column files.  Every run, the
    one that writes the sidecar and those that read it, must give the
    reference's own files for the fixture (src/kgwas.cpp:225-304)."""
    import glob
    import shutil
    fx = H.load_fixture(name)
    n = int(fx["idxs"].shape[0])
    work = tempfile.mkdtemp()
    paths, _ = H.materialise(name, work)
    variants = H.meta(name)["variants"]
    for i, v in enumerate([variants[0]] + variants):
        st = O.cols_stats(fx["packed"], n, fx["U"], fx["y"], _thr(v))
        band = H.band_kmers(st, _thr(v), _log10(v))
        out = os.path.join(work, f"run{i}", "batch_000.tsv")
        os.makedirs(os.path.dirname(out))
        env = dict(v.get("env", {}), KGWAS_KBITS="1")
        r = H.run_cli([paths["samples"], paths["pheno"], paths["batch"], paths["ubin"], out, *v["args"],
                       "--mode", "cols"], env)
        assert r.returncode == 0, r.stderr[-2000:]
        if i == 0:
            assert len(glob.glob(os.path.join(paths["batch"], "*.kbits"))) == 1
            # the sidecar stands in for the columns: blank every column (same
            # length, so N is still inferred), which would change the output
            # if the columns were read again
            for f in glob.glob(os.path.join(paths["batch"], "bits", "col_*.txt")):
                length = len(open(f).readline().rstrip("\n"))
                with open(f, "w") as fh:
                    fh.write("0" * length + "\n")
        else:
            assert "packed rows from" in r.stderr
        _check_outputs(out, name, "cols", v, fx["kmers"], band)
    shutil.rmtree(work)


def _build_index_like(tsv, out, shards):
    """The index that build_index makes of one kgwas output file: the staged
    reference build_index when present, else the library's writer (pinned to
    build_index's own files by the CPU suite)."""
    if os.access(os.path.join(O.REF_DIR, "build_index"), os.X_OK):
        r = O.run_reference_tool("build_index", [tsv, out, "--shards", str(shards)])
        assert r.returncode == 0, r.stderr[-2000:]
    else:
        assert H.index_check_lib().index_from_tsv(tsv.encode(), out.encode(), shards) == 0


@pytest.mark.parametrize("mode", ["cols", "rows"])
def test_index_out_matches_build_index(built, mode):
    """--index-out / --index-2d-out write the .tsv and .2d rows as sharded
    k-mer indexes: the same files (index.meta, shard_*.umap/.bits/.bloom) that
    the reference build_index writes from the .tsv and the .2d.tsv
    (src/build_index.cpp), here on GPU-emitted rows."""
    import shutil
    work = tempfile.mkdtemp()
    paths, rows = H.materialise("small", work)
    out = os.path.join(work, "run", "batch_000.tsv")
    os.makedirs(os.path.dirname(out))
    idx1, idx2 = os.path.join(work, "idx1"), os.path.join(work, "idx2")
    inp = paths["batch"] if mode == "cols" else rows
    r = H.run_cli([paths["samples"], paths["pheno"], inp, paths["ubin"], out, "0", "--log10-thresh-2d", "1",
                   "--mode", mode, "--index-out", idx1, "--index-2d-out", idx2], {"CORR_THRESHOLD": "0"})
    assert r.returncode == 0, r.stderr[-2000:]
    two = O.path_2d(out)
    assert len(H.parse_rows(out)) > 1000 and len(H.parse_rows(two)) > 100
    _build_index_like(out, os.path.join(work, "ref1"), 16)
    _build_index_like(two, os.path.join(work, "ref2"), 4)
    H.same_dir_files(idx1, os.path.join(work, "ref1"))
    H.same_dir_files(idx2, os.path.join(work, "ref2"))
    shutil.rmtree(work)


def test_rows_batches_give_the_same_files(built):
    """ROWS mode in batches of 37 rows (each next batch read while the current
    one is tested) writes the same .tsv, .2d.tsv and .count as one batch."""
    import shutil
    work = tempfile.mkdtemp()
    paths, rows = H.materialise("small", work)
    outs = []
    for tag, env in (("one", {}), ("many", {"KGWAS_ROWS_BATCH": "37"})):
        out = os.path.join(work, tag, "batch_000.tsv")
        os.makedirs(os.path.dirname(out))
        r = H.run_cli([paths["samples"], paths["pheno"], rows, paths["ubin"], out, "0", "--log10-thresh-2d", "1",
                       "--mode", "rows"], dict(env, CORR_THRESHOLD="0"))
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append([open(f, "rb").read() for f in (out, O.path_2d(out), out + ".count")])
    assert outs[0] == outs[1]
    assert outs[0][0].count(b"\n") > 100
    shutil.rmtree(work)

