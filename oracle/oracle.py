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
