"""Shared helpers of the test suite: golden fixtures, output parsing, CLI runs."""
from __future__ import annotations

import gzip
import json
import os
import shutil
import subprocess
import tempfile

import numpy as np

from supergwas_b200 import build, synth
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = ("small", "edge", "yspan")


def meta(name):
    return json.load(open(os.path.join(GOLDEN, name, "meta.json")))


def load_fixture(name):
    """Inputs of a committed fixture: dict with packed_all, n_all, y, idxs, U, kmers."""
    d = os.path.join(GOLDEN, name)
    z = np.load(os.path.join(d, "inputs.npz"))
    out = {k: z[k] for k in z.files}
    out["n_all"] = int(out["n_all"])
    out["kmers"] = open(os.path.join(d, "kmers.txt")).read().splitlines()
    out["packed"] = synth.select_samples(out["packed_all"], out["n_all"], out["idxs"])
    return out


_CFG1 = None


def load_cfg1():
    """Config-1 dataset regenerated from its seed (checked against the committed SHA-256)."""
    global _CFG1
    if _CFG1 is None:
        import hashlib
        mt = meta("cfg1")
        ds = synth.simulate(**mt["generator"])
        h = hashlib.sha256(np.ascontiguousarray(ds.packed_all).tobytes()).hexdigest()
        assert h == mt["sha256_packed_all"], "synthetic generator drifted from the golden inputs"
        _CFG1 = ds
    return _CFG1


def materialise(name, work):
    """Reference-format inputs of a fixture under `work`; returns (paths, rows_file)."""
    d = os.path.join(GOLDEN, name)
    mt = meta(name)
    fx = load_fixture(name)
    os.makedirs(work, exist_ok=True)
    paths = dict(samples=os.path.join(work, "samples.txt"), pheno=os.path.join(work, "phenotype.txt"),
                 ubin=os.path.join(work, "U.bin"), batch=os.path.join(work, "batch_000"))
    shutil.copy(os.path.join(d, "samples.txt"), paths["samples"])
    shutil.copy(os.path.join(d, "phenotype.txt"), paths["pheno"])
    synth.write_ubin(paths["ubin"], fx["U"])
    synth.write_batch(paths["batch"], fx["packed_all"], fx["n_all"], fx["kmers"],
                      gz_columns=mt.get("gz_columns", []), kmers_plain_gz=mt.get("kmers_plain_gz", False))
    rows = os.path.join(work, "rows.tsv")
    synth.write_rows_file(rows, fx["packed_all"], fx["n_all"], fx["kmers"])
    return paths, rows


def materialise_cfg1(work):
    ds = load_cfg1()
    paths = synth.write_dataset(work, ds)
    rows = os.path.join(work, "rows.tsv.gz")
    synth.write_rows_file(rows, ds.packed_all, ds.n_all, ds.kmers)
    return paths, rows


def parse_rows(path):
    """Rows of a .tsv (3 columns) or .2d.tsv (4 columns) output."""
    rows = []
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            p = line.rstrip("\n").split("\t")
            rows.append(p)
    return rows


def ref_file(name, mode, variant, ext):
    return os.path.join(GOLDEN, name, f"ref_{mode}_{variant}{ext}")


def run_cli(args, env_extra=None, timeout=600):
    env = dict(os.environ)
    if env_extra:
        env.update({k: str(v) for k, v in env_extra.items()})
    return subprocess.run([build.CLI, *map(str, args)], env=env, capture_output=True, text=True,
                          timeout=timeout)


def band_kmers(stats, corr_thr, log10_thresh, n_tol=1e-5, p_tol=5e-3):
    """Indices whose integer outcome may legitimately differ from an FP32 reference:
    |cor| within n_tol (relative) of the pre-filter cut, or -log10 p within p_tol of the emit cut."""
    cor = np.abs(stats["cor"])
    near_gate = np.abs(cor - corr_thr) <= n_tol * max(corr_thr, 1e-3)
    ml = stats["mlog10p"]
    near_emit = stats["tested"] & (np.abs(ml - log10_thresh) <= p_tol)
    return set(np.nonzero(near_gate | near_emit)[0].tolist())


def compare_rows(got_rows, ref_rows, kmers, band, rel_tol, abs_floor=1e-300):
    """Integer parity (k-mer set and order) outside `band`, floats within rel_tol."""
    idx_of = {}
    for i, k in enumerate(kmers):
        idx_of.setdefault(k, i)
    g = [r for r in got_rows if idx_of[r[0]] not in band]
    f = [r for r in ref_rows if idx_of[r[0]] not in band]
    assert [r[0] for r in g] == [r[0] for r in f], "row set / order differs outside the tolerance band"
    for a, b in zip(g, f):
        assert a[1:-2] == b[1:-2]  # bitstring column of .2d rows
        for x, y in zip(map(float, a[-2:]), map(float, b[-2:])):
            assert abs(x - y) <= rel_tol * max(abs(y), abs(x)) + abs_floor, (a, b)
    return len(g)


def index_check_lib():
    """tests/native/index_check.cpp with the library's index writer
    (supergwas_b200/csrc/kgwas_io.cpp), built with g++ on first use:
    ``index_from_tsv(tsv, dir, M)`` writes the sharded index of a .tsv or .2d.tsv."""
    import ctypes
    here = os.path.dirname(os.path.abspath(__file__))
    out = os.path.join(here, "native", "_build", "libindex_check.so")
    src = [os.path.join(here, "native", "index_check.cpp"), os.path.join(build.CSRC, "kgwas_io.cpp")]
    if not os.path.exists(out) or any(os.path.getmtime(s) > os.path.getmtime(out) for s in src):
        os.makedirs(os.path.dirname(out), exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-o", out, *src, "-lz"],
                       check=True)
    return ctypes.CDLL(out)


def same_dir_files(a, b):
    """Both directories hold the same file names with byte-identical contents."""
    assert sorted(os.listdir(a)) == sorted(os.listdir(b))
    for f in os.listdir(b):
        assert open(os.path.join(a, f), "rb").read() == open(os.path.join(b, f), "rb").read(), f

