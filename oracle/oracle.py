"""TEST INFRASTRUCTURE ONLY -- Python face of the FP64 CPU oracle.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, always as the checker.  It loads ``oracle/_build/libkgwas_oracle.so``
(built from ``kgwas_oracle.c`` by ``oracle/Makefile``) and runs the staged
reference binary ``oracle/_ref/kgwas`` as a black box.

Reference behaviour restated here:
  * per-k-mer statistics -- ``kgwas_oracle.c`` (src/kgwas.cpp:44-56,138-218,461-476)
  * output rows and ``.count`` text -- :func:`emit_rows`, following
    src/kgwas.cpp:225-304 (default ``std::ostream`` float formatting, i.e.
    ``%g`` with 6 significant digits; ``.2d`` path insertion; count basename).
  * 2-D pair test -- ``kgwas_oracle.c`` (src/kgwas_2d.cpp:237-331), the
    sharded index reader :func:`read_index_bits` (src/map_utils.hpp:319-479,
    src/kgwas_2d.cpp:80-207) and the pair rows :func:`pair_rows`
    (src/kgwas_2d.cpp:350-367: ``%.9g`` effect, ``%.9e`` p).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libkgwas_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.kgo_cols.restype = ctypes.c_int64
        L.kgo_cols.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                               dp, ctypes.c_int, dp, ctypes.c_double,
                               ctypes.c_void_p, dp, dp, dp, dp, dp, dp, dp]
        L.kgo_yyM.restype = ctypes.c_double
        L.kgo_yyM.argtypes = [ctypes.c_int, dp, ctypes.c_int, dp, dp]
        L.kgo_mlog10p.restype = None
        L.kgo_mlog10p.argtypes = [dp, ctypes.c_int64, dp]
        L.kgo_pairs.restype = ctypes.c_int64
        L.kgo_pairs.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, dp,
                                ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, dp, dp, dp, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def cols_stats(packed: np.ndarray, n: int, U: np.ndarray, y: np.ndarray,
               corr_threshold: float = 0.2) -> dict:
    """Per-k-mer oracle statistics for k-mer-major packed rows over n samples."""
    packed = np.ascontiguousarray(packed, dtype=np.uint64)
    m, wpk = packed.shape
    U = np.asfortranarray(U, dtype=np.float64)
    assert U.shape[0] == n
    k = U.shape[1]
    y = np.ascontiguousarray(y, dtype=np.float64)
    out = {name: np.zeros(m, np.float64) for name in
           ("cor", "xxM", "xyM", "chisq", "pval", "effect", "mlog10p")}
    tested = np.zeros(m, np.uint8)
    Ucol = np.ascontiguousarray(U.T)  # k x n row-major == n x k column-major
    nt = lib().kgo_cols(packed.ctypes.data, m, wpk, n, _dp(Ucol), k, _dp(y),
                        float(corr_threshold), tested.ctypes.data,
                        _dp(out["cor"]), _dp(out["xxM"]), _dp(out["xyM"]),
                        _dp(out["chisq"]), _dp(out["pval"]), _dp(out["effect"]),
                        _dp(out["mlog10p"]))
    out["tested"] = tested.astype(bool)
    out["n_tested"] = int(nt)
    out["yyM"] = yyM(U, y)
    return out


def yyM(U: np.ndarray, y: np.ndarray) -> float:
    U = np.asarray(U, dtype=np.float64)
    Ucol = np.ascontiguousarray(U.T)
    y = np.ascontiguousarray(y, dtype=np.float64)
    return float(lib().kgo_yyM(U.shape[0], _dp(Ucol), U.shape[1], _dp(y),
                               ctypes.POINTER(ctypes.c_double)()))


def mlog10p(T: np.ndarray) -> np.ndarray:
    T = np.ascontiguousarray(T, dtype=np.float64)
    out = np.zeros_like(T)
    lib().kgo_mlog10p(_dp(T), T.shape[0], _dp(out))
    return out


def fmt(v: float) -> str:
    """``std::ostream << double`` with default flags (precision 6, %g)."""
    return "%g" % v


def emit_rows(kmers, stats: dict, log10_thresh: float = 6.0,
              log10_thresh_2d: float = 15.0, bits_of=None):
    """Output text of one batch, following src/kgwas.cpp:225-289.

    Returns (tsv_text, tsv2d_text or None).  ``bits_of(j)`` gives the
    overlap-sample bitstring of k-mer j for ``.2d.tsv`` rows.
    """
    p_thresh = 10.0 ** (-log10_thresh)
    do_2d = log10_thresh_2d > 0.0
    p2 = 10.0 ** (-log10_thresh_2d) if do_2d else 0.0
    one, two = [], []
    idx = np.nonzero(stats["tested"])[0]
    for j in idx:
        p = float(stats["pval"][j])
        if p <= p_thresh:
            e = float(stats["effect"][j])
            one.append(f"{kmers[j]}\t{fmt(e)}\t{fmt(p)}\n")
            if do_2d and p <= p2:
                two.append(f"{kmers[j]}\t{bits_of(j)}\t{fmt(e)}\t{fmt(p)}\n")
    return "".join(one), ("".join(two) if do_2d else None)


def path_2d(out_file: str) -> str:
    """``.2d`` inserted before the last '.' of the path (src/kgwas.cpp:273-278)."""
    dot = out_file.rfind(".")
    return out_file[:dot] + ".2d" + out_file[dot:] if dot >= 0 else out_file + ".2d"


def count_line(out_file: str, n_tested: int) -> str:
    """``.count`` content (src/kgwas.cpp:291-304)."""
    name = out_file
    s = max(name.rfind("/"), name.rfind("\\"))
    if s >= 0:
        name = name[s + 1:]
    d = name.rfind(".")
    if d >= 0:
        name = name[:d]
    return f"{name}\t{n_tested}\n"


# ------------------------------------------------------ reference black box

def ref_available() -> bool:
    return os.access(os.path.join(REF_DIR, "kgwas"), os.X_OK)


def ref_env(extra: dict | None = None) -> dict:
    env = dict(os.environ)
    dirs = [REF_DIR]
    ld = os.path.join(REF_DIR, "libdirs.txt")
    if os.path.exists(ld):
        dirs.append(open(ld).read().strip())
    if env.get("LD_LIBRARY_PATH"):
        dirs.append(env["LD_LIBRARY_PATH"])
    env["LD_LIBRARY_PATH"] = ":".join(dirs)
    if extra:
        env.update({k: str(v) for k, v in extra.items()})
    return env


def run_reference(args, env_extra: dict | None = None, timeout: float = 3600.0):
    """Run the staged reference ``kgwas`` with argv ``args``; returns CompletedProcess."""
    exe = os.path.join(REF_DIR, "kgwas")
    return subprocess.run([exe, *map(str, args)], env=ref_env(env_extra),
                          capture_output=True, text=True, timeout=timeout)


# ------------------------------------------------------------ 2-D pair test

def read_index_bits(index_dir: str):
    """k-mers with bitstrings of a sharded d4 index, sorted by their 2-bit
    encoding (src/kgwas_2d.cpp:93-153): returns (K, kmers, bitstrings)."""
    import struct
    meta = {}
    for line in open(os.path.join(index_dir, "index.meta")):
        if "=" in line:
            k, v = line.strip().split("=", 1)
            meta[k] = int(v)
    K, M = meta["K"], meta["M"]
    ent = []
    for s in range(M):
        ub = open(os.path.join(index_dir, f"shard_{s:03d}.umap"), "rb").read()
        assert ub[:8] == b"UMAPd4\0\0"
        k, n = struct.unpack_from("<IQ", ub, 8)
        assert k == K
        keys = [int.from_bytes(ub[20 + 32 * i: 36 + 32 * i], "little") for i in range(n)]
        order = list(dict.fromkeys(keys))
        bits = {}
        bb = open(os.path.join(index_dir, f"shard_{s:03d}.bits"), "rb").read()
        (bn,) = struct.unpack_from("<Q", bb, 0)
        assert bn == n
        off = 8
        for i in range(n):
            (blen,) = struct.unpack_from("<I", bb, off)
            off += 4
            if blen:
                bits[keys[i]] = bb[off:off + blen].decode()
            off += blen
        ent += [(key, bits[key]) for key in order if key in bits]
    ent.sort()
    dec = "ACGT"
    kmers = ["".join(dec[(key >> (2 * (K - 1 - c))) & 3] for c in range(K)) for key, _ in ent]
    return K, kmers, [b for _, b in ent]


def pair_matrix(bitstrings, idxs, n: int):
    """Packed overlap rows of the index k-mers (src/kgwas_2d.cpp:163-192): a
    bitstring of length n is in overlap order, a longer one (beyond the
    largest overlap position) in samples order, others are dropped.  Returns
    (packed rows, indices of the kept k-mers)."""
    maxidx = int(max(idxs)) if len(idxs) else -1
    rows, keep = [], []
    for j, b in enumerate(bitstrings):
        if len(b) == n:
            rows.append(np.frombuffer(b.encode(), np.uint8) == ord("1"))
        elif maxidx >= 0 and len(b) > maxidx:
            bb = np.frombuffer(b.encode(), np.uint8)
            rows.append(bb[np.asarray(idxs)] == ord("1"))
        else:
            continue
        keep.append(j)
    x = np.array(rows, dtype=np.uint8).reshape(len(rows), n)
    wpk = (n + 63) // 64
    wpk += wpk & 1
    packed = np.zeros((len(rows), wpk), np.uint64)
    for w in range(wpk):
        blk = x[:, 64 * w: 64 * w + 64].astype(np.uint64)
        packed[:, w] = (blk << np.arange(blk.shape[1], dtype=np.uint64)).sum(axis=1, dtype=np.uint64)
    return packed, keep


def pairs_stats(packed: np.ndarray, n: int, U: np.ndarray, y: np.ndarray, row_start: int = 0,
                row_end: int | None = None) -> dict:
    """Dense N x N pair statistics (i < j): evaluated, chisq, pval, effect, mlog10p."""
    packed = np.ascontiguousarray(packed, dtype=np.uint64)
    N, wpk = packed.shape
    row_end = N if row_end is None else row_end
    U = np.ascontiguousarray(np.asarray(U, dtype=np.float64).T)
    y = np.ascontiguousarray(y, dtype=np.float64)
    out = {k: np.zeros((N, N)) for k in ("chisq", "pval", "effect", "mlog10p")}
    out["pval"][:] = 1.0
    ev = np.zeros((N, N), np.uint8)
    lib().kgo_pairs(packed.ctypes.data, N, wpk, n, _dp(U), U.shape[0], _dp(y), row_start, row_end,
                    ev.ctypes.data, _dp(out["chisq"]), _dp(out["pval"]), _dp(out["effect"]), _dp(out["mlog10p"]))
    out["evaluated"] = ev.astype(bool)
    return out


def pair_rows(pairs) -> str:
    """Text of the pair rows: "i<TAB>j<TAB>effect (%.9g)<TAB>p (%.9e)" (src/kgwas_2d.cpp:359-362)."""
    return "".join(f"{int(a)}\t{int(b)}\t{e:.9g}\t{p:.9e}\n" for a, b, e, p in pairs)


def run_reference_tool(tool: str, args, env_extra: dict | None = None, timeout: float = 3600.0):
    """Run a staged reference binary (kgwas_2d, build_index) as a black box."""
    exe = os.path.join(REF_DIR, tool)
    return subprocess.run([exe, *map(str, args)], env=ref_env(env_extra), capture_output=True, text=True,
                          timeout=timeout)

