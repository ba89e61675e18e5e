"""Generate the golden vectors under tests/golden/ by running the reference.

The reference ``kgwas`` binary (staged into oracle/_ref/ by
oracle/stage_ref.sh) is run as a black box on seeded synthetic batches, in
COLS mode (``src/kgwas.cpp:168-307``) and ROWS mode (``src/kgwas.cpp:343-522``).
Its output files (``.tsv``, ``.2d.tsv``, ``.count``) are committed together
with the inputs (or, for the 1M-k-mer case, the generator seed and a SHA-256
of the generated packed matrix), so the GPU box can check parity without the
reference.

Run:  python tests/golden/make_golden.py [fixture ...]
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from supergwas_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

THREADS = {"LOAD_THREADS": 4, "BLAS_THREADS": 4, "EMIT_THREADS": 4}


def sha256_array(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_variants(fx_dir, paths, variants, rows_input):
    os.makedirs(fx_dir, exist_ok=True)
    for v in variants:
        for mode in v.get("modes", ("cols", "rows")):
            out = os.path.join(tempfile.mkdtemp(), "batch_000.tsv")
            inp = paths["batch"] if mode == "cols" else rows_input
            args = [paths["samples"], paths["pheno"], inp, paths["ubin"], out, *v["args"],
                    "--mode", mode]
            env = dict(THREADS)
            env.update(v.get("env", {}))
            r = O.run_reference(args, env)
            tag = f"ref_{mode}_{v['name']}"
            with open(os.path.join(fx_dir, tag + ".rc"), "w") as f:
                f.write(f"{r.returncode}\n")
            if r.returncode != 0:
                with open(os.path.join(fx_dir, tag + ".err"), "w") as f:
                    f.write([l for l in r.stderr.splitlines() if l.startswith("[ERROR]")][-1] + "\n")
                continue
            shutil.copy(out, os.path.join(fx_dir, tag + ".tsv"))
            p2 = O.path_2d(out)
            if os.path.exists(p2):
                shutil.copy(p2, os.path.join(fx_dir, tag + ".2d.tsv"))
            shutil.copy(out + ".count", os.path.join(fx_dir, tag + ".tsv.count"))


def save_inputs(fx_dir, ds, samples_text, pheno_text, extra_meta):
    os.makedirs(fx_dir, exist_ok=True)
    np.savez_compressed(os.path.join(fx_dir, "inputs.npz"), packed_all=ds.packed_all,
                        n_all=np.int64(ds.n_all), y=ds.y, idxs=ds.idxs, U=ds.U)
    with open(os.path.join(fx_dir, "samples.txt"), "w", newline="") as f:
        f.write(samples_text)
    with open(os.path.join(fx_dir, "phenotype.txt"), "w", newline="") as f:
        f.write(pheno_text)
    with open(os.path.join(fx_dir, "kmers.txt"), "w") as f:
        f.write("".join(k + "\n" for k in ds.kmers))
    with open(os.path.join(fx_dir, "meta.json"), "w") as f:
        json.dump(extra_meta, f, indent=1, sort_keys=True)


def materialise(fx_dir, work, meta):
    """Write the reference-format input files of a committed fixture into ``work``."""
    z = np.load(os.path.join(fx_dir, "inputs.npz"))
    n_all = int(z["n_all"])
    kmers = open(os.path.join(fx_dir, "kmers.txt")).read().splitlines()
    os.makedirs(work, exist_ok=True)
    paths = dict(samples=os.path.join(work, "samples.txt"),
                 pheno=os.path.join(work, "phenotype.txt"),
                 ubin=os.path.join(work, "U.bin"), batch=os.path.join(work, "batch_000"))
    shutil.copy(os.path.join(fx_dir, "samples.txt"), paths["samples"])
    shutil.copy(os.path.join(fx_dir, "phenotype.txt"), paths["pheno"])
    synth.write_ubin(paths["ubin"], z["U"])
    synth.write_batch(paths["batch"], z["packed_all"], n_all, kmers,
                      gz_columns=meta.get("gz_columns", []),
                      kmers_plain_gz=meta.get("kmers_plain_gz", False))
    rows = os.path.join(work, "rows.tsv")
    synth.write_rows_file(rows, z["packed_all"], n_all, kmers)
    return paths, rows


VARIANTS_FULL = [
    # every tested k-mer is emitted: full numerical comparison
    {"name": "all", "env": {"CORR_THRESHOLD": "0"}, "args": ["0", "--log10-thresh-2d", "1"]},
    # reference defaults (CORR_THRESHOLD 0.2, log10 6, .2d at 15), with a looser emit cut
    {"name": "default", "env": {}, "args": ["2"]},
]


def fx_small():
    ds = synth.simulate(n=200, m=3000, S=5, r=5, n_causal=20, missing=0.05, seed=7)
    samples_text = "".join(s + "\n" for s in ds.samples)
    pheno_text = "".join(f"{i} {float(v)!r}\n" for i, v in zip(ds.pheno_ids, ds.y))
    meta = {"desc": "n=200 (190 phenotyped), m=3000, S=5, r=5+1, 20 causal, seed 7",
            "variants": VARIANTS_FULL}
    return ds, samples_text, pheno_text, meta


def fx_edge():
    """Edge cases of the reader and of the statistic.

    * samples.txt with CRLF endings, an empty line and a bare "\\r" line
      (src/kgwas_utils.hpp:51-61 keeps it as an empty id);
    * phenotype.txt with a duplicated id (last value wins, :63-70), an id
      absent from samples.txt, and 9 samples without a phenotype, so the
      overlap n=61 is not a multiple of 8;
    * k-mers constant on the overlap but not on all samples, all-0 and all-1;
    * a k-mer equal to the phenotype's sign pattern (strong association);
    * U without a constant column (random orthonormal basis, k=4);
    * some columns gzipped (.txt.gz), kmers.txt.gz stored uncompressed.
    """
    rng = np.random.default_rng(11)
    n_all, m = 70, 700
    S = 3
    pop = (np.arange(n_all) * S) // n_all
    _, ps = synth.draw_frequencies(rng, m, S)
    x = synth.draw_bits(rng, ps, pop)
    miss = np.array([3, 9, 17, 18, 30, 41, 52, 63, 69])
    keep = np.setdiff1d(np.arange(n_all), miss)
    x[5, :] = 0
    x[6, :] = 1
    x[7, :] = 1; x[7, miss[0]] = 0          # constant on the overlap only
    x[8, :] = 0; x[8, miss[1]] = 1
    y = rng.standard_normal(keep.shape[0])
    x[9, keep] = (y > 0).astype(np.uint8)  # strongly associated
    Q, _ = np.linalg.qr(rng.standard_normal((keep.shape[0], 4)))
    kmers = synth.random_kmers(rng, m, 21)
    samples = [f"acc_{i}" for i in range(n_all)]
    lines = []
    for i, s in enumerate(samples):
        lines.append(s + "\r\n")
        if i == 20:
            lines.append("\n")       # skipped
        if i == 40:
            lines.append("\r\n")     # kept as an empty id
    samples_text = "".join(lines)
    # the bare "\r" line adds one sample position after acc_40
    all_ids = [s for s in samples[:41]] + [""] + samples[41:]
    n_file = len(all_ids)
    # rebuild x over the 71 sample positions: position 41 is the empty id
    x71 = np.zeros((m, n_file), np.uint8)
    x71[:, :41] = x[:, :41]
    x71[:, 42:] = x[:, 41:]
    keep71 = np.array([i if i < 41 else i + 1 for i in keep])
    ph = []
    for jj, i in enumerate(keep):
        ph.append(f"{samples[i]}\t{float(y[jj])!r}\n")
        if jj == 10:
            ph.append(f"{samples[i]} 123.5\n")  # overwritten below (last wins)
            ph.append(f"{samples[i]}   {float(y[jj])!r}\n")
    ph.insert(3, "not_a_sample 4.0\n")
    pheno_text = "".join(ph)
    ds = synth.Dataset(n_all=n_file, samples=all_ids, pheno_ids=[samples[i] for i in keep],
                       y=y, idxs=keep71.astype(np.int64), U=Q,
                       packed_all=synth.pack_rows(x71), kmers=kmers)
    meta = {"desc": "edge cases: CRLF/empty ids, duplicate phenotype ids, n=61, constant "
                    "columns on the overlap, r2 near 1, U without intercept, gz columns",
            "gz_columns": [0, 2, 33, 70], "kmers_plain_gz": True,
            "variants": VARIANTS_FULL + [
                {"name": "thr0", "env": {"CORR_THRESHOLD": "0.0"}, "args": ["0"]},
                {"name": "no2d", "env": {"CORR_THRESHOLD": "0.1"},
                 "args": ["1", "--log10-thresh-2d", "0"]}]}
    return ds, samples_text, pheno_text, meta


def fx_yspan():
    """Phenotype inside span(U): yyM ~ 0, so every test returns p = 1."""
    rng = np.random.default_rng(5)
    ds = synth.simulate(n=64, m=400, S=2, r=3, n_causal=0, missing=0.0, seed=5)
    ds.y = 2.5 * ds.U[:, 1] - 0.75 * ds.U[:, 0] + 1e-15 * rng.standard_normal(ds.n)
    samples_text = "".join(s + "\n" for s in ds.samples)
    pheno_text = "".join(f"{i} {float(v)!r}\n" for i, v in zip(ds.pheno_ids, ds.y))
    meta = {"desc": "y in span(U): yyM ~ 0 (warn, p = 1 everywhere)",
            "variants": [{"name": "all", "env": {"CORR_THRESHOLD": "0"}, "args": ["0"]}]}
    return ds, samples_text, pheno_text, meta


CFG1 = dict(n=200, m=1_000_000, S=5, r=5, n_causal=20, missing=0.05, seed=42)


def cfg1_dataset():
    return synth.simulate(**CFG1)


def make_cfg1():
    """Config 1 (n=200, m=1e6, r=5+1): reference outputs only; inputs regenerate from the seed."""
    fx_dir = os.path.join(HERE, "cfg1")
    ds = cfg1_dataset()
    work = tempfile.mkdtemp()
    paths = synth.write_dataset(work, ds)
    rows = os.path.join(work, "rows.tsv")
    synth.write_rows_file(rows, ds.packed_all, ds.n_all, ds.kmers)
    meta = {"desc": "config 1: n=200, S=5, m=1e6, r=5+1, 20 causal, 5% missing, seed 42",
            "generator": CFG1, "sha256_packed_all": sha256_array(ds.packed_all),
            "sha256_y": sha256_array(ds.y), "sha256_U": sha256_array(ds.U),
            "variants": [
                {"name": "default", "env": {}, "args": []},
                {"name": "thr0_l3", "env": {"CORR_THRESHOLD": "0"}, "args": ["3"]}]}
    os.makedirs(fx_dir, exist_ok=True)
    with open(os.path.join(fx_dir, "meta.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    run_variants(fx_dir, paths, meta["variants"], rows)
    shutil.rmtree(work)


def make(name, fn):
    fx_dir = os.path.join(HERE, name)
    ds, samples_text, pheno_text, meta = fn()
    save_inputs(fx_dir, ds, samples_text, pheno_text, meta)
    work = tempfile.mkdtemp()
    paths, rows = materialise(fx_dir, work, meta)
    run_variants(fx_dir, paths, meta["variants"], rows)
    shutil.rmtree(work)


# ------------------------------------------------------------ fault injection

def fault_cases():
    """(name, mutate(work_paths) -> argv tail, env) for malformed inputs.

    Each case runs the reference on a small valid batch with one defect and
    records its exit code and its last ``[ERROR]`` line (paths replaced by
    ``<W>``).  The defects are those the reference's readers check
    (src/kgwas.cpp:67-126, src/kgwas_utils.hpp:34-37,51-332)."""
    import gzip as _gz

    def wr(p, b):
        with open(p, "wb") as f:
            f.write(b)

    def col(w, j):
        return os.path.join(w["batch"], "bits", f"col_{j:06d}.txt")

    cases = []
    cases.append(("usage", lambda w: ["ONLY"], {}))
    cases.append(("bad_log10", lambda w: [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"], "abc"], {}))
    cases.append(("neg_log10", lambda w: [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"], "-1"], {}))
    cases.append(("bad_mode", lambda w: [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"], "--mode", "x"], {}))
    cases.append(("no_input", lambda w: [w["samples"], w["pheno"], w["batch"] + "_nope", w["ubin"], w["out"]], {}))
    cases.append(("no_samples", lambda w: [w["samples"] + ".nope", w["pheno"], w["batch"], w["ubin"], w["out"]], {}))
    cases.append(("no_pheno", lambda w: [w["samples"], w["pheno"] + ".nope", w["batch"], w["ubin"], w["out"]], {}))

    def empty_samples(w):
        wr(w["samples"], b"\n\n")
        return [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"]]
    cases.append(("samples_empty", empty_samples, {}))

    def no_overlap(w):
        wr(w["pheno"], b"zzz 1.0\nyyy 2.0\n")
        return [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"]]
    cases.append(("no_overlap", no_overlap, {}))
    cases.append(("no_ubin", lambda w: [w["samples"], w["pheno"], w["batch"], w["ubin"] + ".nope", w["out"]], {}))

    def short_hdr(w):
        wr(w["ubin"], b"\x01\x00")
        return [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"]]
    cases.append(("ubin_short_header", short_hdr, {}))

    def n_mismatch(w):
        U = synth.read_ubin(w["ubin"])
        synth.write_ubin(w["ubin"], U[:-1])
        return [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"]]
    cases.append(("ubin_n_mismatch", n_mismatch, {}))

    def short_body(w):
        b = open(w["ubin"], "rb").read()
        wr(w["ubin"], b[:-8])
        return [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"]]
    cases.append(("ubin_short_body", short_body, {}))

    def miss_first(w):
        os.remove(col(w, 0))
        return [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"]]
    cases.append(("missing_first_column", miss_first, {"LOAD_THREADS": "1"}))

    def miss_other(w):
        os.remove(col(w, 7))
        return [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"]]
    cases.append(("missing_column", miss_other, {"LOAD_THREADS": "1"}))

    def short_txt(w):
        b = open(col(w, 5), "rb").read()
        wr(col(w, 5), b[:50])
        return [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"]]
    cases.append(("short_txt_column", short_txt, {"LOAD_THREADS": "1"}))

    def short_gz(w):
        b = open(col(w, 5), "rb").read()
        os.remove(col(w, 5))
        with _gz.open(col(w, 5) + ".gz", "wb") as f:
            f.write(b[:50])
        return [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"]]
    cases.append(("short_gz_column", short_gz, {"LOAD_THREADS": "1"}))

    def long_gz(w):
        b = open(col(w, 5), "rb").read()
        os.remove(col(w, 5))
        with _gz.open(col(w, 5) + ".gz", "wb") as f:
            f.write(b[:-1] + b"01\n")
        return [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"]]
    cases.append(("long_gz_column", long_gz, {"LOAD_THREADS": "1"}))

    def kmer_count(w):
        p = os.path.join(w["batch"], "kmers.txt.gz")
        lines = _gz.open(p).read().splitlines(keepends=True)
        with _gz.open(p, "wb") as f:
            f.write(b"".join(lines[:-3]))
        return [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"]]
    cases.append(("kmers_count", kmer_count, {}))

    def kmer_unterminated(w):
        p = os.path.join(w["batch"], "kmers.txt.gz")
        data = _gz.open(p).read()
        with _gz.open(p, "wb") as f:
            f.write(data[:-1])   # last line loses its newline: not counted
        return [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"]]
    cases.append(("kmers_unterminated", kmer_unterminated, {}))

    def no_kmers(w):
        os.remove(os.path.join(w["batch"], "kmers.txt.gz"))
        return [w["samples"], w["pheno"], w["batch"], w["ubin"], w["out"]]
    cases.append(("kmers_missing", no_kmers, {}))
    cases.append(("rows_missing", lambda w: [w["samples"], w["pheno"], w["batch"] + "/nope.tsv", w["ubin"],
                                             w["out"], "--mode", "rows"], {}))

    def rows_n_mismatch(w):
        U = synth.read_ubin(w["ubin"])
        synth.write_ubin(w["ubin"], U[:-1])
        return [w["samples"], w["pheno"], w["rows"], w["ubin"], w["out"], "--mode", "rows"]
    cases.append(("rows_ubin_n_mismatch", rows_n_mismatch, {}))
    return cases


def fault_workdir():
    ds = synth.simulate(n=40, m=300, S=2, r=2, n_causal=0, missing=0.0, seed=3)
    work = tempfile.mkdtemp()
    w = synth.write_dataset(work, ds)
    w["out"] = os.path.join(work, "out.tsv")
    w["rows"] = os.path.join(work, "rows.tsv")
    synth.write_rows_file(w["rows"], ds.packed_all, ds.n_all, ds.kmers)
    return work, w


def error_line(stderr: str, work: str) -> str:
    errs = [l for l in stderr.splitlines() if "[ERROR]" in l]
    if not errs:
        return ""
    return errs[-1][errs[-1].index("[ERROR]"):].replace(work, "<W>")


def make_faults():
    out = {}
    for name, mutate, env in fault_cases():
        work, w = fault_workdir()
        argv = mutate(w)
        e = dict(THREADS)
        e.update(env)
        r = O.run_reference(argv, e)
        out[name] = {"rc": r.returncode, "error": error_line(r.stderr, work)}
        shutil.rmtree(work)
    with open(os.path.join(HERE, "faults.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    return out


FIXTURES = {"small": fx_small, "edge": fx_edge, "yspan": fx_yspan}


# ------------------------------------------------------------ 2-D pair test

PAIR_VARIANTS = [
    {"name": "l0", "args": ["0"]},                                # every scored pair is a row
    {"name": "l2", "args": ["2"]},
    {"name": "task1of3", "args": ["1.5", "--num-tasks", "3", "--task-id", "1"]},
    {"name": "task5of3", "args": ["1.5", "--num-tasks", "3", "--task-id", "5"]},  # no rows
]


def pair_fault_cases():
    """(name, mutate(work) -> argv, env) for malformed inputs of kgwas_2d: the
    checks of parse_args, build_overlap, load_Ubin and load_X_from_index
    (src/kgwas_2d.cpp:45-207, src/map_utils.hpp:319-479)."""
    import struct

    def base(w, *extra):
        return [w["samples"], w["pheno"], w["ubin"], w["index"], w["out"], *extra]

    def shard(w, s, ext):
        return os.path.join(w["index"], f"shard_{s:03d}{ext}")

    def patch(path, off, data):
        b = bytearray(open(path, "rb").read())
        b[off:off + len(data)] = data
        open(path, "wb").write(bytes(b))

    def rewrite_bits(w, fn):
        """fn(bitstring) -> new bitstring (or "") for every record of every shard."""
        meta = open(os.path.join(w["index"], "index.meta")).read()
        M = int([l for l in meta.splitlines() if l.startswith("M=")][0][2:])
        for s_ in range(M):
            p = shard(w, s_, ".bits")
            b = open(p, "rb").read()
            (n,) = struct.unpack_from("<Q", b, 0)
            out, off = [struct.pack("<Q", n)], 8
            for _ in range(n):
                (ln,) = struct.unpack_from("<I", b, off)
                nb = fn(b[off + 4: off + 4 + ln].decode()).encode()
                out.append(struct.pack("<I", len(nb)) + nb)
                off += 4 + ln
            open(p, "wb").write(b"".join(out))

    cases = [("usage", lambda w: ["ONLY"], {})]
    cases.append(("bad_log10", lambda w: base(w, "abc"), {}))
    cases.append(("index_not_dir", lambda w: [w["samples"], w["pheno"], w["ubin"], w["index"] + "_nope", w["out"]], {}))

    def meta_missing(w):
        os.remove(os.path.join(w["index"], "index.meta"))
        return base(w)
    cases.append(("meta_missing", meta_missing, {}))

    def meta_invalid(w):
        open(os.path.join(w["index"], "index.meta"), "w").write("K=0\nM=4\nN=10\n")
        return base(w)
    cases.append(("meta_invalid", meta_invalid, {}))

    def umap_missing(w):
        os.remove(shard(w, 1, ".umap"))
        return base(w)
    cases.append(("umap_missing", umap_missing, {}))

    def bad_magic(w):
        patch(shard(w, 2, ".umap"), 0, b"XMAPd4")
        return base(w)
    cases.append(("bad_magic", bad_magic, {}))

    def k_mismatch(w):
        patch(shard(w, 0, ".umap"), 8, struct.pack("<I", 21))
        return base(w)
    cases.append(("k_mismatch", k_mismatch, {}))

    def bits_missing(w):
        os.remove(shard(w, 3, ".bits"))
        return base(w)
    cases.append(("bits_missing", bits_missing, {}))

    def bits_n_mismatch(w):
        (n,) = struct.unpack_from("<Q", open(shard(w, 1, ".bits"), "rb").read(), 0)
        patch(shard(w, 1, ".bits"), 0, struct.pack("<Q", n + 1))
        return base(w)
    cases.append(("bits_n_mismatch", bits_n_mismatch, {}))

    def no_bitstrings(w):
        rewrite_bits(w, lambda b: "")
        return base(w)
    cases.append(("no_bitstrings", no_bitstrings, {}))

    def all_wrong_length(w):
        rewrite_bits(w, lambda b: b[:20])
        return base(w)
    cases.append(("all_wrong_length", all_wrong_length, {}))

    def one_kmer(w):
        state = {"kept": 0}

        def keep_one(b):
            if b and not state["kept"]:
                state["kept"] = 1
                return b
            return ""
        rewrite_bits(w, keep_one)
        return base(w)
    cases.append(("one_kmer", one_kmer, {}))

    def ubin_n_mismatch(w):
        U = synth.read_ubin(w["ubin"])
        synth.write_ubin(w["ubin"], U[:-1])
        return base(w)
    cases.append(("ubin_n_mismatch", ubin_n_mismatch, {}))
    return cases


def pair_fault_workdir():
    """A writable copy of the pairs fixture: samples, phenotype, U2D.bin, index."""
    work = tempfile.mkdtemp()
    fx = os.path.join(HERE, "pairs")
    w = {"samples": os.path.join(work, "samples.txt"), "pheno": os.path.join(work, "phenotype.txt"),
         "ubin": os.path.join(work, "U2D.bin"), "index": os.path.join(work, "index"),
         "out": os.path.join(work, "out")}
    shutil.copy(os.path.join(fx, "samples.txt"), w["samples"])
    shutil.copy(os.path.join(fx, "phenotype.txt"), w["pheno"])
    shutil.copytree(os.path.join(fx, "index"), w["index"])
    synth.write_ubin(w["ubin"], np.load(os.path.join(fx, "inputs.npz"))["U"])
    return work, w


def make_pair_faults():
    out = {}
    for name, mutate, env in pair_fault_cases():
        work, w = pair_fault_workdir()
        argv = mutate(w)
        e = {"BLAS_THREADS": 1, "EMIT_THREADS": 1}
        e.update(env)
        r = O.run_reference_tool("kgwas_2d", argv, e)
        out[name] = {"rc": r.returncode, "error": error_line(r.stderr, work)}
        shutil.rmtree(work)
    with open(os.path.join(HERE, "pair_faults.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    return out


def make_index():
    """The reference build_index on the small fixture's reference kgwas
    outputs (all rows): the .2d.tsv at 4 shards and the .tsv at the default 16,
    the sharded indexes that kgwas --index-2d-out / --index-out must reproduce
    byte for byte (src/build_index.cpp)."""
    d = os.path.join(HERE, "index")
    os.makedirs(d, exist_ok=True)
    shutil.copy(os.path.join(HERE, "small", "ref_cols_all.2d.tsv"), os.path.join(d, "input.2d.tsv"))
    out = os.path.join(d, "ref_index")
    if os.path.isdir(out):
        shutil.rmtree(out)
    r = O.run_reference_tool("build_index", [os.path.join(d, "input.2d.tsv"), out, "--shards", "4"])
    assert r.returncode == 0, r.stderr
    # the 1-D index of the 3-column .tsv rows, at build_index's default 16 shards
    out = os.path.join(d, "ref_index_1d")
    if os.path.isdir(out):
        shutil.rmtree(out)
    r = O.run_reference_tool("build_index", [os.path.join(HERE, "small", "ref_cols_all.tsv"), out])
    assert r.returncode == 0, r.stderr


def make_pairs():
    """2-D pair test (src/kgwas_2d.cpp): a kgwas-style .2d.tsv of k-mers with
    bitstrings is turned into a sharded index by the reference's build_index
    and tested by the reference's kgwas_2d; inputs (index directory included)
    and outputs are committed.  Edge cases of the index reader: bitstrings of
    the overlap length and of the samples length, bitstrings of another
    length (dropped), rows without a bitstring (not in the test), a k-mer and
    its reverse complement (one canonical entry), an all-zero and an all-one
    row."""
    rng = np.random.default_rng(29)
    n_all, m = 110, 160
    pop = (np.arange(n_all) * 3) // n_all
    _, ps = synth.draw_frequencies(rng, m, 3)
    x = synth.draw_bits(rng, ps, pop)
    x[4, :] = 0
    x[5, :] = 1
    miss = np.sort(rng.choice(n_all, size=7, replace=False))
    keep = np.setdiff1d(np.arange(n_all), miss)
    n = keep.size
    X = x[:, keep].astype(float)
    y = 1.5 * X[10] * X[20] - 1.0 * X[30] * X[40] + rng.standard_normal(n)
    Q, _ = np.linalg.qr(np.column_stack([np.ones(n), X[rng.choice(m, 40)].T @ rng.standard_normal((40, 3))]))
    kmers = synth.random_kmers(rng, m, 31)
    comp = {"A": "T", "C": "G", "G": "C", "T": "A"}
    kmers[7] = "".join(comp[c] for c in reversed(kmers[6]))     # reverse complement of k-mer 6
    samples = [f"s{i:03d}" for i in range(n_all)]
    fx_dir = os.path.join(HERE, "pairs")
    os.makedirs(fx_dir, exist_ok=True)
    with open(os.path.join(fx_dir, "samples.txt"), "w") as f:
        f.write("".join(s + "\n" for s in samples))
    with open(os.path.join(fx_dir, "phenotype.txt"), "w") as f:
        f.write("".join(f"{samples[i]}\t{float(v)!r}\n" for i, v in zip(keep, y)))
    np.savez_compressed(os.path.join(fx_dir, "inputs.npz"), U=Q, y=y, idxs=keep.astype(np.int64),
                        n_all=np.int64(n_all))
    lines = []
    for j in range(m):
        if j in (11, 12):                                       # no bitstring
            lines.append(f"{kmers[j]}\t0.1\t1e-30\n")
            continue
        if j in (13, 14):                                       # wrong length: dropped
            b = "".join("1" if v else "0" for v in x[j, keep[:-3]])
        elif j % 9 == 0:                                        # samples order (length n_all)
            b = "".join("1" if v else "0" for v in x[j])
        else:                                                   # overlap order (length n)
            b = "".join("1" if v else "0" for v in x[j, keep])
        lines.append(f"{kmers[j]}\t{b}\t0.1\t1e-30\n")
    work = tempfile.mkdtemp()
    tsv = os.path.join(work, "hits.2d.tsv")
    with open(tsv, "w") as f:
        f.write("kmer\tbits\teffect\tp_value\n" + "".join(lines))
    idx = os.path.join(fx_dir, "index")
    if os.path.isdir(idx):
        shutil.rmtree(idx)
    r = O.run_reference_tool("build_index", [tsv, idx, "--shards", "4"])
    assert r.returncode == 0, r.stderr
    for f in os.listdir(idx):
        if f.endswith(".bloom"):
            os.remove(os.path.join(idx, f))                     # not read by kgwas_2d
    synth.write_ubin(os.path.join(work, "U2D.bin"), Q)
    meta = {"desc": "2-D pair test: n_all=110 (103 phenotyped), 160 k-mers (2 without bitstrings, 2 with a "
                    "bitstring of another length, one reverse-complement duplicate), r=3+1, two planted pairs",
            "variants": PAIR_VARIANTS}
    with open(os.path.join(fx_dir, "meta.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    for v in PAIR_VARIANTS:
        out = os.path.join(work, "out_" + v["name"])
        r = O.run_reference_tool("kgwas_2d", [os.path.join(fx_dir, "samples.txt"), os.path.join(fx_dir, "phenotype.txt"),
                                              os.path.join(work, "U2D.bin"), idx, out, *v["args"]],
                                 {"BLAS_THREADS": 4, "EMIT_THREADS": 4})
        tag = "ref_" + v["name"]
        with open(os.path.join(fx_dir, tag + ".rc"), "w") as f:
            f.write(f"{r.returncode}\n")
        for ext in (".tsv", ".part_1.tsv", ".part_5.tsv", ".kmers"):
            if os.path.exists(out + ext):
                shutil.copy(out + ext, os.path.join(fx_dir, tag + ext))
    shutil.rmtree(work)

if __name__ == "__main__":
    if not O.ref_available():
        sys.exit("stage the reference first: bash oracle/stage_ref.sh REFERENCE_DIR")
    names = sys.argv[1:] or [*FIXTURES, "cfg1", "faults", "pairs", "pair_faults", "index"]
    for nm in names:
        if nm == "cfg1":
            make_cfg1()
        elif nm == "pairs":
            make_pairs()
        elif nm == "pair_faults":
            make_pair_faults()
        elif nm == "index":
            make_index()
        elif nm == "faults":
            make_faults()
        else:
            make(nm, FIXTURES[nm])
        print("made", nm)
