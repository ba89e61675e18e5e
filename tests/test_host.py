"""CPU-only checks: the C ABI library, host-side algebra, formats and CLI errors."""
import ctypes
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np
import pytest

import helpers as H
from oracle import oracle as O
from supergwas_b200 import api, build, synth

HERE = os.path.dirname(os.path.abspath(__file__))


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_library_exports_every_header_symbol(built):
    L = api.lib()
    syms = api.header_symbols()
    assert len(syms) >= 12
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert api.version().startswith("kgwas-b200")


def test_default_opts_match_reference_defaults(built):
    o = api._Opts()
    api.lib().kg_default_opts(ctypes.byref(o))
    assert o.corr_threshold == 0.2        # src/kgwas.cpp:30
    assert o.log10_thresh == 6.0          # src/kgwas.cpp:28
    assert o.precision == api.PREC["split"]


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU error path")
def test_create_without_gpu_fails_cleanly(built):
    with pytest.raises(api.KgError) as e:
        api.Kgwas()
    assert e.value.code in (2, 6)


def test_pack_roundtrip():
    rng = np.random.default_rng(0)
    for n in (1, 63, 64, 65, 200, 1000):
        x = (rng.random((37, n)) < 0.4).astype(np.uint8)
        p = synth.pack_rows(x)
        assert p.shape[1] == synth.words_per_kmer(n) and p.shape[1] % 2 == 0
        assert np.array_equal(synth.unpack_rows(p, n), x)


def test_ubin_roundtrip(tmp_path):
    U = np.random.default_rng(1).standard_normal((17, 4))
    synth.write_ubin(tmp_path / "U.bin", U)
    b = (tmp_path / "U.bin").read_bytes()
    assert np.frombuffer(b[:8], np.int32).tolist() == [17, 4]
    assert np.array_equal(synth.read_ubin(tmp_path / "U.bin"), U)


def test_count_and_2d_names():
    assert O.count_line("/a/b/batch_000.tsv", 7) == "batch_000\t7\n"
    assert O.count_line("x.y.tsv", 1) == "x.y\t1\n"
    assert O.path_2d("/a/b.tsv") == "/a/b.2d.tsv"
    assert O.path_2d("noext") == "noext.2d"


# ---------------------------------------------------- host algebra on the CPU

_EMU = None


def emu_lib():
    global _EMU
    if _EMU is None:
        out = os.path.join(HERE, "native", "_build", "libprep_check.so")
        src = [os.path.join(HERE, "native", "prep_check.cpp"),
               os.path.join(build.CSRC, "prep.cpp")]
        if not os.path.exists(out) or any(os.path.getmtime(s) > os.path.getmtime(out) for s in src):
            os.makedirs(os.path.dirname(out), exist_ok=True)
            subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", out, *src], check=True)
        _EMU = ctypes.CDLL(out)
    return _EMU


def emulate(packed, n, U, y, split, lu=3, ly=5, thr=0.0):
    L = emu_lib()
    dp = ctypes.POINTER(ctypes.c_double)
    packed = np.ascontiguousarray(packed)
    m, wpk = packed.shape
    Uc = np.ascontiguousarray(np.asarray(U).T)
    y = np.ascontiguousarray(y, dtype=np.float64)
    f = ("chisq", "effect", "xxM", "xyM", "cor")
    out = {k: np.zeros(m) for k in f}
    t = np.zeros(m, np.uint8)
    yy = ctypes.c_double()
    rc = L.prep_emulate(Uc.ctypes.data_as(dp), n, U.shape[1], y.ctypes.data_as(dp),
                        packed.ctypes.data_as(ctypes.c_void_p), ctypes.c_int64(m), wpk, split, lu, ly,
                        ctypes.c_double(thr), t.ctypes.data_as(ctypes.c_void_p),
                        *[out[k].ctypes.data_as(dp) for k in f], ctypes.byref(yy))
    assert rc == 0
    out["tested"] = t.astype(bool)
    return out


@pytest.mark.parametrize("split", [0, 1])
def test_prep_algebra_matches_oracle(split):
    """prepare()/make_limbs() + the kernels' arithmetic, replayed on the CPU."""
    for (n, m, S, r, seed) in [(200, 20000, 5, 5, 1), (1000, 8000, 8, 16, 2), (61, 3000, 3, 3, 3)]:
        ds = synth.simulate(n=n, m=m, S=S, r=r, n_causal=20, missing=0.05, seed=seed)
        X = ds.packed_overlap()
        o = O.cols_stats(X, ds.n, ds.U, ds.y, 0.0)
        e = emulate(X, ds.n, ds.U, ds.y, split)
        assert np.array_equal(e["tested"], o["tested"])
        msk = o["tested"]
        rel = np.abs(e["chisq"] - o["chisq"]) / np.maximum(o["chisq"], 1e-300)
        ml = np.abs(O.mlog10p(e["chisq"]) - o["mlog10p"])
        if split:
            assert np.percentile(rel[msk], 99) <= 1e-6
            assert ml[msk].max() <= 1e-6
        else:
            assert rel[msk].max() <= 1e-9
            assert ml[msk].max() <= 1e-11


def test_tmem_b_image_matches_unpack():
    """make_b_image_ts lays B out for the A bytes the TMEM kernel's unpack
    forms (two masks per shift, -2 V on the 64 x columns): recombined limb
    sums equal -128 * x . V for every column, with no int32 overflow."""
    L = emu_lib()
    L.ts_image_check.restype = ctypes.c_int64
    dp = ctypes.POINTER(ctypes.c_double)
    for (n, m, S, r, seed) in [(1000, 600, 8, 16, 5), (61, 400, 3, 3, 6), (300, 300, 4, 6, 7)]:
        ds = synth.simulate(n=n, m=m, S=S, r=r, n_causal=10, missing=0.05, seed=seed)
        X = np.ascontiguousarray(ds.packed_overlap())
        Uc = np.ascontiguousarray(np.asarray(ds.U).T)
        y = np.ascontiguousarray(ds.y, dtype=np.float64)
        bad = L.ts_image_check(Uc.ctypes.data_as(dp), ds.n, ds.U.shape[1], y.ctypes.data_as(dp),
                               X.ctypes.data_as(ctypes.c_void_p), ctypes.c_int64(X.shape[0]), X.shape[1])
        assert bad == 0, (n, bad)
    # all-ones rows: largest limb sums
    ds = synth.simulate(n=1000, m=50, S=8, r=16, n_causal=5, missing=0.0, seed=8)
    X = np.full_like(ds.packed_overlap(), np.uint64(0xFFFFFFFFFFFFFFFF))
    Uc = np.ascontiguousarray(np.asarray(ds.U).T)
    y = np.ascontiguousarray(ds.y, dtype=np.float64)
    bad = L.ts_image_check(Uc.ctypes.data_as(dp), ds.n, ds.U.shape[1], y.ctypes.data_as(dp),
                           X.ctypes.data_as(ctypes.c_void_p), ctypes.c_int64(X.shape[0]), X.shape[1])
    assert bad == 0


def test_prep_general_U_without_intercept():
    """U that does not contain the constant vector (no intercept column)."""
    fx = H.load_fixture("edge")
    n = int(fx["idxs"].shape[0])
    o = O.cols_stats(fx["packed"], n, fx["U"], fx["y"], 0.0)
    for split in (0, 1):
        e = emulate(fx["packed"], n, fx["U"], fx["y"], split)
        assert np.array_equal(e["tested"], o["tested"])
        ml = np.abs(O.mlog10p(e["chisq"]) - o["mlog10p"])
        assert ml[o["tested"]].max() <= 1e-6


# ---------------------------------------------------------- CLI error paths

def _fault_cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(H.GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg


def test_cli_errors_match_reference(built):
    """Malformed inputs give the reference's [ERROR] line and exit code 1,
    before any GPU work (src/kgwas_utils.hpp:34-37)."""
    mg = _fault_cases()
    expected = json.load(open(os.path.join(H.GOLDEN, "faults.json")))
    for name, mutate, env in mg.fault_cases():
        work, w = mg.fault_workdir()
        try:
            argv = mutate(w)
            r = H.run_cli(argv, env)
            exp = expected[name]
            assert r.returncode == exp["rc"], (name, r.returncode, r.stderr[-500:])
            assert mg.error_line(r.stderr, work) == exp["error"], (name, r.stderr[-500:])
        finally:
            shutil.rmtree(work)


def test_kgwas_2d_errors_match_reference(built):
    """Malformed kgwas_2d inputs (index directory, shards, bitstrings, U.bin,
    arguments) give the reference kgwas_2d's exit code and last [ERROR] line,
    before any GPU work (src/kgwas_2d.cpp:45-207, src/map_utils.hpp:319-479)."""
    mg = _fault_cases()
    expected = json.load(open(os.path.join(H.GOLDEN, "pair_faults.json")))
    exe = os.path.join(build.BIN_DIR, "kgwas_2d")
    for name, mutate, env in mg.pair_fault_cases():
        work, w = mg.pair_fault_workdir()
        try:
            argv = mutate(w)
            e = dict(os.environ, BLAS_THREADS="1", EMIT_THREADS="1")
            e.update({k: str(v) for k, v in env.items()})
            r = subprocess.run([exe, *argv], capture_output=True, text=True, env=e)
            exp = expected[name]
            assert r.returncode == exp["rc"], (name, r.returncode, r.stderr[-500:])
            assert mg.error_line(r.stderr, work) == exp["error"], (name, r.stderr[-500:])
        finally:
            shutil.rmtree(work)


def test_index_writer_matches_build_index(tmp_path):
    """The index writer of kgwas --index-out / --index-2d-out (kgio::write_index)
    on the rows of a reference .2d.tsv and .tsv gives the files of the
    reference build_index byte for byte:
    index.meta, and per shard the .umap, .bits and .bloom (src/build_index.cpp,
    src/map_utils.hpp:109-160, 331-372, 562-575)."""
    L = H.index_check_lib()
    d = os.path.join(H.GOLDEN, "index")
    got = str(tmp_path / "idx")
    assert L.index_from_tsv(os.path.join(d, "input.2d.tsv").encode(), got.encode(), 4) == 0
    H.same_dir_files(got, os.path.join(d, "ref_index"))
    # the 1-D index of the 3-column .tsv rows: 16 shards, no .bits files
    got = str(tmp_path / "idx1")
    tsv = os.path.join(H.GOLDEN, "small", "ref_cols_all.tsv")
    assert L.index_from_tsv(tsv.encode(), got.encode(), 16) == 0
    H.same_dir_files(got, os.path.join(d, "ref_index_1d"))


def test_index_merge_matches_build_index(built, tmp_path):
    """bin/kgwas_index_merge joins per-batch indexes into the index that
    build_index makes of all the batches' rows: the golden .2d.tsv split into
    three batches, each indexed on its own (2 shards), merged to 4 shards, gives
    the reference build_index's files of the whole .2d.tsv byte for byte."""
    d = os.path.join(H.GOLDEN, "index")
    lines = open(os.path.join(d, "input.2d.tsv")).read().splitlines(keepends=True)
    L = H.index_check_lib()
    parts = []
    for b, chunk in enumerate((lines[:100], lines[100:101], lines[101:])):
        tsv = tmp_path / f"batch_{b:03d}.2d.tsv"
        tsv.write_text("".join(chunk))
        out = str(tmp_path / f"idx_{b}")
        assert L.index_from_tsv(str(tsv).encode(), out.encode(), 2) == 0
        parts.append(out)
    merged = str(tmp_path / "merged")
    r = subprocess.run([build.MERGE, merged, *parts, "--shards", "4"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    H.same_dir_files(merged, os.path.join(d, "ref_index"))
    # a K mismatch or a missing input is an [ERROR] exit
    r = subprocess.run([build.MERGE, str(tmp_path / "bad"), parts[0], str(tmp_path / "none")],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "[ERROR]" in r.stderr


def test_index_out_option_errors(built, tmp_path):
    """The index options are checked before any input or GPU is touched."""
    base = ["s.txt", "p.txt", "in", "U.bin", str(tmp_path / "o.tsv"), "--mode", "cols"]
    for extra, msg in ((["--index-2d-out", "d", "--log10-thresh-2d", "0"], "--index-2d-out needs the .2d rows"),
                       (["--index-out", "d", "--index-shards", "12"], "--index-shards must be a power of 2"),
                       (["--index-2d-shards", "0"], "--index-2d-shards must be a power of 2")):
        r = H.run_cli([*base, *extra])
        assert r.returncode == 1 and msg in r.stderr, (extra, r.stderr)


def _runs_lib():
    out = os.path.join(HERE, "native", "_build", "libruns_check.so")
    src = os.path.join(HERE, "native", "runs_check.cpp")
    deps = [src, build.LIB, os.path.join(build.CSRC, "ctx.hpp")]
    if not os.path.exists(out) or any(os.path.getmtime(d) > os.path.getmtime(out) for d in deps):
        os.makedirs(os.path.dirname(out), exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", out, src, "-I/usr/local/cuda/include",
                        "-L" + build.LIB_DIR, "-lkgwas_cuda", "-Wl,-rpath," + build.LIB_DIR], check=True)
    L = ctypes.CDLL(out)
    vp = ctypes.c_void_p
    L.runs_check.argtypes = [vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, vp, ctypes.c_int, vp, vp, vp]
    L.runs_check.restype = ctypes.c_uint64
    return L


@pytest.mark.parametrize("m,wpk,s0,cnt", [(300_000, 16, 0, 300_000), (300_000, 2, 1234, 200_001),
                                          (5_000, 4, 10, 4000)])
def test_run_finder(built, m, wpk, s0, cnt):
    """The host scan behind runs of equal rows (kgctx::scan_gather): a row
    starts a run at the range start, where it differs from its predecessor,
    and at every bound; each run's first row reaches the device in row order."""
    rng = np.random.default_rng(m + wpk)
    base = rng.integers(0, 2**63, size=(m // 2, wpk), dtype=np.uint64)
    k = base[1::7].shape[0]
    base[0:7 * k:7] = base[1::7]                       # neighbouring runs of the same row merge
    reps = rng.integers(1, 6, size=base.shape[0])
    X = np.ascontiguousarray(np.repeat(base, reps, axis=0)[:m])
    assert X.shape[0] == m >= s0 + cnt
    bounds = np.unique(np.r_[rng.integers(s0, s0 + cnt, size=9), s0 + 5, s0 + cnt + 3]).astype(np.uint64)
    rows = np.arange(s0, s0 + cnt)
    diff = np.r_[True, np.any(X[rows[1:]] != X[rows[1:] - 1], axis=1)]
    start = diff | np.isin(rows, bounds)
    exp_first = rows[start]
    exp_len = np.diff(np.r_[exp_first, s0 + cnt])
    L = _runs_lib()
    first = np.zeros(cnt, np.uint64)
    lens = np.zeros(cnt, np.uint32)
    out = np.zeros((cnt, wpk), np.uint64)
    nu = L.runs_check(X.ctypes.data, ctypes.c_uint64(s0), ctypes.c_uint64(cnt), ctypes.c_uint32(wpk),
                      bounds.ctypes.data, ctypes.c_int(bounds.size), first.ctypes.data, lens.ctypes.data,
                      out.ctypes.data)
    assert nu == exp_first.size
    assert np.array_equal(first[:nu], exp_first)
    assert np.array_equal(lens[:nu], exp_len)
    assert np.array_equal(out[:nu], X[exp_first])


def _rows_lib():
    out = os.path.join(HERE, "native", "_build", "librows_check.so")
    src = [os.path.join(HERE, "native", "rows_check.cpp"), os.path.join(build.CSRC, "kgwas_io.cpp")]
    deps = src + [os.path.join(build.CSRC, "kgwas_io.hpp")]
    if not os.path.exists(out) or any(os.path.getmtime(d) > os.path.getmtime(out) for d in deps):
        os.makedirs(os.path.dirname(out), exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-o", out, *src, "-lz"],
                       check=True)
    L = ctypes.CDLL(out)
    vp = ctypes.c_void_p
    L.rows_parse.argtypes = [ctypes.c_char_p, vp, ctypes.c_int, ctypes.c_int, ctypes.c_ulong, vp, ctypes.c_ulong,
                             vp, ctypes.c_ulong, vp, vp]
    L.rows_parse.restype = ctypes.c_long
    return L


def _rows_expected(lines, idxs, gz):
    """src/kgwas.cpp:435-459 restated: the rows, k-mers and non-empty lines of a ROWS file."""
    n = len(idxs)
    W = synth.words_per_kmer(n)
    kmers, rows, nonempty = [], [], 0
    for ln in lines:
        if gz and ln.endswith("\r"):
            ln = ln[:-1]
        if not ln:
            continue
        nonempty += 1
        t = ln.find("\t")
        if t < 0:
            t = ln.find(" ")
        if t < 0:
            continue
        bits = ln[t + 1:]
        row = np.zeros(W, np.uint64)
        for j, pos in enumerate(idxs):
            assert pos <= len(bits)
            if pos < len(bits) and bits[pos] == "1":
                row[j >> 6] |= np.uint64(1 << (j & 63))
        kmers.append(ln[:t])
        rows.append(row)
    return kmers, np.array(rows, np.uint64).reshape(-1, W), nonempty


@pytest.mark.parametrize("gz", [False, True])
@pytest.mark.parametrize("threads,max_rows", [(1, 10**6), (8, 10**6), (8, 7), (3, 1)])
def test_rows_reader(tmp_path, gz, threads, max_rows):
    """The parallel ROWS reader gives the rows of the line-by-line reading of
    src/kgwas.cpp:435-459: tab or space separators, lines without one skipped,
    empty lines, '\\r' (kept in plain files, dropped before '\\n' in gz
    files), a bitstring one character short reading '\\0', a last line without
    '\\n', in batches of at most max_rows rows."""
    import gzip
    rng = np.random.default_rng(threads * 31 + max_rows + gz)
    n_all = 150
    idxs = sorted(rng.choice(n_all, size=120, replace=False).tolist())
    lines = []
    for i in range(400):
        k = "".join(rng.choice(list("ACGT"), size=31))
        bits = "".join(rng.choice(["0", "1"], size=n_all))
        kind = i % 10
        if kind == 1:
            lines.append("")
        elif kind == 2:
            lines.append(k + " " + bits)
        elif kind == 3:
            lines.append(k + "_noseparator")
        elif kind == 4:
            lines.append(k + "\t" + bits + "\r")
        elif kind == 5:
            lines.append(k + "\t" + bits[: idxs[-1]])      # one short: reads the terminator
        elif kind == 6:
            lines.append(k + "\t" + bits[: idxs[-1]] + "\r")  # the last sample reads the '\\r' (plain)
        else:
            lines.append(k + "\t" + bits)
    text = "\n".join(lines)                                 # no '\\n' after the last line
    path = tmp_path / ("rows.tsv.gz" if gz else "rows.tsv")
    if gz:
        with gzip.open(path, "wb") as f:
            f.write(text.encode())
    else:
        path.write_text(text)
    exp_k, exp_rows, exp_lines = _rows_expected(lines, idxs, gz)
    L = _rows_lib()
    W = synth.words_per_kmer(len(idxs))
    packed = np.zeros(len(lines) * W, np.uint64)
    kbuf = ctypes.create_string_buffer(len(text) + 16)
    nl, nb = ctypes.c_ulong(0), ctypes.c_ulong(0)
    ia = np.array(idxs, np.int32)
    got = L.rows_parse(str(path).encode(), ia.ctypes.data, len(idxs), threads, max_rows, packed.ctypes.data,
                       packed.size, ctypes.addressof(kbuf), len(kbuf), ctypes.byref(nl), ctypes.byref(nb))
    assert got == len(exp_k)
    assert kbuf.value.decode().split("\n")[:-1] == exp_k
    assert np.array_equal(packed[: got * W].reshape(-1, W), exp_rows)
    assert nl.value == exp_lines
    assert nb.value == (got + max_rows - 1) // max_rows if max_rows < got else nb.value == 1


def test_rows_reader_short_bitstring(tmp_path):
    """A bitstring that ends before an overlap sample's position stops the
    program with the first such row's k-mer, in file order."""
    p = tmp_path / "rows.tsv"
    p.write_text("AAA\t0101\nCCC\t01\nGGG\t0\n")
    _rows_lib()  # built here; the child process only loads it
    lib = os.path.join(HERE, "native", "_build", "librows_check.so")
    code = ("import ctypes, numpy as np; L = ctypes.CDLL(%r); vp = ctypes.c_void_p; "
            "L.rows_parse.argtypes = [ctypes.c_char_p, vp, ctypes.c_int, ctypes.c_int, ctypes.c_ulong, vp, "
            "ctypes.c_ulong, vp, ctypes.c_ulong, vp, vp]; "
            "ia = np.array([0, 3], np.int32); b = np.zeros(64, np.uint64); k = ctypes.create_string_buffer(256); "
            "n = ctypes.c_ulong(); m = ctypes.c_ulong(); "
            "L.rows_parse(%r, ia.ctypes.data, 2, 4, 100, b.ctypes.data, 64, ctypes.addressof(k), 256, "
            "ctypes.byref(n), ctypes.byref(m))") % (lib, str(p).encode())
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=HERE)
    assert r.returncode == 1
    assert r.stderr.strip().splitlines()[-1] == "[ERROR] bitstring shorter than the samples list in row: CCC"


@pytest.mark.parametrize("N,n_all,threads", [(1003, 77, 1), (20011, 150, 4), (8, 64, 2)])
def test_column_reader(tmp_path, N, n_all, threads):
    """The COLS reader (kgio::load_matrix_packed) packs sample idxs[k] of the
    batch's column files (src/kgwas_utils.hpp:225-282; some columns gzipped)
    into bit k of each k-mer's row, for k-mer counts and sample counts that
    are not multiples of 8 or 64."""
    out_so = os.path.join(HERE, "native", "_build", "libcols_check.so")
    src = [os.path.join(HERE, "native", "cols_check.cpp"), os.path.join(build.CSRC, "kgwas_io.cpp")]
    if not os.path.exists(out_so) or any(os.path.getmtime(x) > os.path.getmtime(out_so) for x in src):
        os.makedirs(os.path.dirname(out_so), exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-o", out_so, *src, "-lz"],
                       check=True)
    L = ctypes.CDLL(out_so)
    vp = ctypes.c_void_p
    L.cols_read.argtypes = [ctypes.c_char_p, vp, ctypes.c_int, ctypes.c_ulong, ctypes.c_int, vp]
    rng = np.random.default_rng(N + n_all)
    x = (rng.random((N, n_all)) < 0.4).astype(np.uint8)
    packed_all = synth.pack_rows(x)
    kmers = synth.random_kmers(rng, N, 31)
    d = str(tmp_path / "batch_000")
    synth.write_batch(d, packed_all, n_all, kmers, gz_columns=range(0, n_all, 5))
    idxs = np.sort(rng.choice(n_all, size=n_all - n_all // 7, replace=False)).astype(np.int32)
    W = synth.words_per_kmer(idxs.size)
    got = np.zeros((N, W), np.uint64)
    L.cols_read(os.path.join(d, "bits").encode(), idxs.ctypes.data, idxs.size, N, threads, got.ctypes.data)
    exp = synth.select_samples(packed_all, n_all, idxs)
    assert exp.shape == got.shape
    assert np.array_equal(got, exp)

