"""ctypes binding of the C ABI in include/kgwas_cuda.h.

This is the Python face of the same entry points the ``kgwas`` program
calls.  There is no CPU fallback: if ``lib/libkgwas_cuda.so`` is missing the
import of :func:`lib` raises.
"""
from __future__ import annotations

import ctypes
import os
import re
from dataclasses import dataclass

import numpy as np

from . import build as _build

KG_OK = 0
ERRORS = {1: "KG_ERR_INVALID", 2: "KG_ERR_CUDA", 3: "KG_ERR_NOMEM", 4: "KG_ERR_STATE",
          5: "KG_ERR_TIMEOUT", 6: "KG_ERR_UNSUPPORTED"}
PREC = {"split": 0, "fp64": 1}

HIT_DTYPE = np.dtype([("kmer", np.uint64), ("effect", np.float64), ("pval", np.float64),
                      ("chisq", np.float64)])


class KgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class _Opts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("precision", ctypes.c_int),
                ("corr_threshold", ctypes.c_double), ("log10_thresh", ctypes.c_double),
                ("limbs_u", ctypes.c_int), ("limbs_y", ctypes.c_int)]


class _Hit(ctypes.Structure):
    _fields_ = [("kmer", ctypes.c_uint64), ("effect", ctypes.c_double),
                ("pval", ctypes.c_double), ("chisq", ctypes.c_double)]


class _Result(ctypes.Structure):
    _fields_ = [("n_kmers", ctypes.c_uint64), ("n_tested", ctypes.c_uint64),
                ("n_hits", ctypes.c_uint64), ("hits", ctypes.POINTER(_Hit))]


_DP = ctypes.POINTER(ctypes.c_double)


class _Stats(ctypes.Structure):
    _fields_ = [("tested", ctypes.c_void_p), ("chisq", _DP), ("pval", _DP), ("effect", _DP),
                ("mlog10p", _DP), ("xxM", _DP), ("xyM", _DP), ("cor", _DP)]


STAT_FIELDS = ("chisq", "pval", "effect", "mlog10p", "xxM", "xyM", "cor")

PHIT_DTYPE = np.dtype([("kmer", np.uint64), ("pheno", np.int32), ("shard", np.int32), ("effect", np.float64),
                       ("pval", np.float64), ("chisq", np.float64)])


class _Pheno(ctypes.Structure):
    _fields_ = [("U_colmajor", _DP), ("n", ctypes.c_int), ("k", ctypes.c_int), ("y", _DP),
                ("sample_pos", ctypes.c_void_p)]


class _MultiResult(ctypes.Structure):
    _fields_ = [("n_kmers", ctypes.c_uint64), ("n_pheno", ctypes.c_int), ("n_shards", ctypes.c_int),
                ("n_tested", ctypes.POINTER(ctypes.c_uint64)), ("n_hits", ctypes.c_uint64),
                ("hits", ctypes.c_void_p)]

PAIR_DTYPE = np.dtype([("a", np.uint64), ("b", np.uint64), ("effect", np.float64), ("pval", np.float64),
                       ("chisq", np.float64)])


class _TileShape(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int), ("np", ctypes.c_int), ("ppg", ctypes.c_int), ("groups", ctypes.c_int),
                ("kpad", ctypes.c_int), ("bt", ctypes.c_int), ("xs", ctypes.c_int), ("nb", ctypes.c_int)]


class _PairResult(ctypes.Structure):
    _fields_ = [("n_kmers", ctypes.c_uint64), ("n_evaluated", ctypes.c_uint64), ("n_pairs", ctypes.c_uint64),
                ("pairs", ctypes.c_void_p)]


_LIB = None


def header_symbols() -> list[str]:
    """Function names declared in include/kgwas_cuda.h."""
    hdr = os.path.join(_build.ROOT, "include", "kgwas_cuda.h")
    txt = open(hdr).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(kg_[a-z_0-9]+)\s*\(", txt)))


def lib():
    """Load the native library (never a fallback)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(_build.LIB):
        raise RuntimeError(f"{_build.LIB} is not built; run `python -m supergwas_b200.build`")
    L = ctypes.CDLL(_build.LIB)
    vp = ctypes.c_void_p
    L.kg_default_opts.argtypes = [ctypes.POINTER(_Opts)]
    L.kg_default_opts.restype = None
    L.kg_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(_Opts)]
    L.kg_set_structure.argtypes = [vp, _DP, ctypes.c_int, ctypes.c_int, _DP, _DP]
    L.kg_set_structure_ex.argtypes = [vp, _DP, ctypes.c_int, ctypes.c_int, _DP, vp, ctypes.c_int, _DP]
    L.kg_run_host.argtypes = [vp, vp, ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(_Result),
                              ctypes.POINTER(_Stats)]
    L.kg_launch_device.argtypes = [vp, vp, ctypes.c_uint64, ctypes.c_uint32, vp]
    L.kg_launch_device_stats.argtypes = [vp, vp, ctypes.c_uint64, ctypes.c_uint32, vp]
    L.kg_fetch.argtypes = [vp, ctypes.POINTER(_Result), ctypes.POINTER(_Stats)]
    L.kg_last_launch_count.argtypes = [vp]
    L.kg_last_kernel.argtypes = [vp]
    L.kg_last_kernel.restype = ctypes.c_char_p
    L.kg_last_unique_rows.argtypes = [vp]
    L.kg_last_unique_rows.restype = ctypes.c_uint64
    L.kg_last_error.argtypes = [vp]
    L.kg_last_error.restype = ctypes.c_char_p
    L.kg_destroy.argtypes = [vp]
    L.kg_destroy.restype = None
    L.kg_probe_fp64_tflops.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.kg_probe_h2d_gbs.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.kg_multi_shape.argtypes = [vp, ctypes.POINTER(_TileShape)]
    L.kg_set_wait_limit.argtypes = [vp, ctypes.c_uint64]
    L.kg_reserve_host.argtypes = [vp, ctypes.c_uint64, ctypes.c_uint32]
    L.kg_inject_stall.argtypes = [vp, ctypes.c_uint64]
    L.kg_version.restype = ctypes.c_char_p
    L.kg_host_alloc.argtypes = [ctypes.c_size_t]
    L.kg_host_alloc.restype = vp
    L.kg_host_free.argtypes = [vp]
    L.kg_host_free.restype = None
    L.kg_set_phenotypes.argtypes = [vp, ctypes.POINTER(_Pheno), ctypes.c_int, ctypes.c_int]
    L.kg_launch_multi_device.argtypes = [vp, vp, ctypes.c_uint64, ctypes.c_uint32, vp, ctypes.c_int, vp]
    L.kg_fetch_multi.argtypes = [vp, ctypes.POINTER(_MultiResult)]
    L.kg_run_multi_host.argtypes = [vp, vp, ctypes.c_uint64, ctypes.c_uint32, vp, ctypes.c_int,
                                    ctypes.POINTER(_MultiResult)]
    L.kg_pairs_run_host.argtypes = [vp, vp, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64,
                                    ctypes.POINTER(_PairResult)]
    L.kg_run_device_noalloc.argtypes = [vp, ctypes.c_uint64, ctypes.c_uint32, _DP, ctypes.c_int, ctypes.c_int,
                                        _DP, ctypes.c_double, ctypes.c_double, vp, ctypes.c_uint64,
                                        ctypes.POINTER(ctypes.c_uint64), vp, ctypes.c_char_p, ctypes.c_size_t]
    _LIB = L
    return L


@dataclass
class Result:
    n_kmers: int
    n_tested: int
    hits: np.ndarray          # HIT_DTYPE, sorted by k-mer
    stats: dict | None = None


class Kgwas:
    """One GPU context (kg_ctx)."""

    def __init__(self, device: int = 0, precision: str = "split", corr_threshold: float = 0.2,
                 log10_thresh: float = 6.0, limbs_u: int = 3, limbs_y: int = 5):
        L = lib()
        o = _Opts()
        L.kg_default_opts(ctypes.byref(o))
        o.device = device
        o.precision = PREC[precision]
        o.corr_threshold = corr_threshold
        o.log10_thresh = log10_thresh
        o.limbs_u = limbs_u
        o.limbs_y = limbs_y
        h = ctypes.c_void_p()
        rc = L.kg_create(ctypes.byref(h), ctypes.byref(o))
        if rc != KG_OK:
            raise KgError(rc, f"kg_create failed on device {device}")
        self._h = h
        self._L = L
        self.n = None

    def _check(self, rc, what):
        if rc != KG_OK:
            raise KgError(rc, f"{what}: {self._L.kg_last_error(self._h).decode()}")

    def close(self):
        if getattr(self, "_h", None):
            self._L.kg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_structure(self, U: np.ndarray, y: np.ndarray, sample_pos=None, n_row_samples=None) -> float:
        """U (n x k) and y (n) of the overlap samples; optionally their bit
        positions within packed rows of ``n_row_samples`` samples."""
        U = np.asarray(U, dtype=np.float64)
        if U.ndim != 2:
            raise ValueError("U must be n x k")
        n, k = U.shape
        Uc = np.ascontiguousarray(U.T)  # column-major n x k
        yv = np.ascontiguousarray(y, dtype=np.float64)
        if yv.shape != (n,):
            raise ValueError("y must have length n")
        yy = ctypes.c_double()
        if sample_pos is None:
            rc = self._L.kg_set_structure(self._h, Uc.ctypes.data_as(_DP), n, k, yv.ctypes.data_as(_DP),
                                          ctypes.byref(yy))
        else:
            pos = np.ascontiguousarray(sample_pos, dtype=np.int32)
            if pos.shape != (n,):
                raise ValueError("sample_pos must have length n")
            rc = self._L.kg_set_structure_ex(self._h, Uc.ctypes.data_as(_DP), n, k, yv.ctypes.data_as(_DP),
                                             pos.ctypes.data, int(n_row_samples), ctypes.byref(yy))
        self._check(rc, "kg_set_structure")
        self.n = n
        return yy.value

    @staticmethod
    def _stats_struct(m):
        arrs = {f: np.zeros(m, np.float64) for f in STAT_FIELDS}
        arrs["tested"] = np.zeros(m, np.uint8)
        st = _Stats()
        st.tested = arrs["tested"].ctypes.data
        for f in STAT_FIELDS:
            setattr(st, f, arrs[f].ctypes.data_as(_DP))
        return st, arrs

    def _result(self, r, arrs):
        nh = int(r.n_hits)
        hits = np.zeros(nh, HIT_DTYPE)
        if nh:
            buf = (ctypes.c_char * (nh * HIT_DTYPE.itemsize)).from_address(
                ctypes.addressof(r.hits.contents))
            hits = np.frombuffer(bytes(buf), dtype=HIT_DTYPE).copy()
        if arrs is not None:
            arrs["tested"] = arrs["tested"].astype(bool)
        return Result(int(r.n_kmers), int(r.n_tested), hits, arrs)

    def run_host(self, packed: np.ndarray, stats: bool = False) -> Result:
        packed = np.ascontiguousarray(packed, dtype=np.uint64)
        m, wpk = packed.shape
        r = _Result()
        st, arrs = self._stats_struct(m) if stats else (None, None)
        self._check(self._L.kg_run_host(self._h, packed.ctypes.data, m, wpk, ctypes.byref(r),
                                        ctypes.byref(st) if st is not None else None),
                    "kg_run_host")
        return self._result(r, arrs)

    def run_host_ptr(self, ptr: int, m: int, wpk: int) -> Result:
        r = _Result()
        self._check(self._L.kg_run_host(self._h, ptr, m, wpk, ctypes.byref(r), None), "kg_run_host")
        return self._result(r, None)

    def launch_device(self, dptr: int, m: int, wpk: int, stream: int | None = None, stats: bool = False):
        f = self._L.kg_launch_device_stats if stats else self._L.kg_launch_device
        self._check(f(self._h, dptr, m, wpk, stream), "kg_launch_device")
        self._pending_m = m

    def fetch(self, stats: bool = False) -> Result:
        r = _Result()
        st, arrs = self._stats_struct(self._pending_m) if stats else (None, None)
        self._check(self._L.kg_fetch(self._h, ctypes.byref(r), ctypes.byref(st) if st is not None else None),
                    "kg_fetch")
        return self._result(r, arrs)

    # ------------------------------------------------------ 2-D pair test
    def run_pairs_host(self, packed: np.ndarray, row_start: int = 0, row_end: int | None = None):
        """Pairs i < j with row_start <= i < row_end and p <= 10^-log10_thresh,
        sorted by (a, b): (PAIR_DTYPE array, number of pairs scored)."""
        packed = np.ascontiguousarray(packed, dtype=np.uint64)
        m, wpk = packed.shape
        r = _PairResult()
        self._check(self._L.kg_pairs_run_host(self._h, packed.ctypes.data, m, wpk, row_start,
                                              m if row_end is None else row_end, ctypes.byref(r)),
                    "kg_pairs_run_host")
        out = np.zeros(r.n_pairs, PAIR_DTYPE)
        if r.n_pairs:
            ctypes.memmove(out.ctypes.data, r.pairs, r.n_pairs * PAIR_DTYPE.itemsize)
        return out, int(r.n_evaluated)

    # ---------------------------------------------------- many phenotypes
    def set_phenotypes(self, phenos, n_row_samples: int):
        """phenos: list of (U (n x k), y (n), sample_pos (n)) sharing one row layout."""
        keep = []
        arr = (_Pheno * len(phenos))()
        for i, (U, y, pos) in enumerate(phenos):
            U = np.asarray(U, dtype=np.float64)
            Uc = np.ascontiguousarray(U.T)
            yv = np.ascontiguousarray(y, dtype=np.float64)
            pv = np.ascontiguousarray(pos, dtype=np.int32)
            keep += [Uc, yv, pv]
            arr[i].U_colmajor = Uc.ctypes.data_as(_DP)
            arr[i].n = U.shape[0]
            arr[i].k = U.shape[1]
            arr[i].y = yv.ctypes.data_as(_DP)
            arr[i].sample_pos = pv.ctypes.data
        self._check(self._L.kg_set_phenotypes(self._h, arr, len(phenos), int(n_row_samples)), "kg_set_phenotypes")
        self._np = len(phenos)

    def _multi_result(self, r):
        nh = int(r.n_hits)
        hits = np.zeros(nh, PHIT_DTYPE)
        if nh:
            hits = np.frombuffer(ctypes.string_at(r.hits, nh * PHIT_DTYPE.itemsize), dtype=PHIT_DTYPE).copy()
        ns, npn = int(r.n_shards), int(r.n_pheno)
        tested = np.ctypeslib.as_array(r.n_tested, shape=(ns * npn,)).copy().reshape(ns, npn)
        return tested, hits

    @staticmethod
    def _shards(shard_start):
        if shard_start is None:
            return None, 0, None
        a = np.ascontiguousarray(shard_start, dtype=np.uint64)
        return a.ctypes.data, a.shape[0], a

    def launch_multi_device(self, dptr: int, m: int, wpk: int, shard_start=None, stream: int | None = None):
        sp, ns, keep = self._shards(shard_start)
        self._check(self._L.kg_launch_multi_device(self._h, dptr, m, wpk, sp, ns, stream), "kg_launch_multi_device")

    def fetch_multi(self):
        """Returns (tested counts [n_shards, n_pheno], hits PHIT_DTYPE sorted by (pheno, kmer))."""
        r = _MultiResult()
        self._check(self._L.kg_fetch_multi(self._h, ctypes.byref(r)), "kg_fetch_multi")
        return self._multi_result(r)

    def run_multi_host(self, packed: np.ndarray, shard_start=None):
        packed = np.ascontiguousarray(packed, dtype=np.uint64)
        sp, ns, keep = self._shards(shard_start)
        r = _MultiResult()
        self._check(self._L.kg_run_multi_host(self._h, packed.ctypes.data, packed.shape[0], packed.shape[1],
                                              sp, ns, ctypes.byref(r)), "kg_run_multi_host")
        return self._multi_result(r)

    def multi_shape(self) -> dict:
        """Tile shape of the many-phenotype launches (kg_multi_shape)."""
        t = _TileShape()
        self._check(self._L.kg_multi_shape(self._h, ctypes.byref(t)), "kg_multi_shape")
        d = {f: int(getattr(t, f)) for f, _ in _TileShape._fields_}
        d["kernel"] = {1: "image resident (mpb)", 2: "image streamed (mp)",
                       3: "SM pair, cta_group::2 (mpb2)"}.get(d["kernel"], d["kernel"])
        d["NP"] = d.pop("np")
        d["PPG"] = d.pop("ppg")
        d["N"] = d["NP"] * d["PPG"]
        return d

    def last_launch_count(self) -> int:
        return int(self._L.kg_last_launch_count(self._h))

    def last_kernel(self) -> str:
        return self._L.kg_last_kernel(self._h).decode()

    def reserve_host(self, n_kmers: int, words_per_kmer: int):
        """Allocate now the buffers run_host needs for a batch of this shape (kg_reserve_host)."""
        self._check(self._L.kg_reserve_host(self._h, int(n_kmers), int(words_per_kmer)), "kg_reserve_host")

    def set_wait_limit(self, wait_ns: int):
        """Limit of every pipeline wait on the device, in ns (0: the default 2 s)."""
        self._check(self._L.kg_set_wait_limit(self._h, int(wait_ns)), "kg_set_wait_limit")

    def inject_stall(self, stop_after_loads: int):
        """Failure-test hook: the next launch's row producer stops after this many loads per CTA."""
        self._check(self._L.kg_inject_stall(self._h, int(stop_after_loads)), "kg_inject_stall")

    def last_unique_rows(self) -> int:
        """Rows the last run_host tested when it used runs of equal adjacent rows (0: every row)."""
        return int(self._L.kg_last_unique_rows(self._h))


def run_device_noalloc(d_x: int, m: int, wpk: int, U, y, corr_threshold: float, log10_thresh: float,
                       d_hits: int, hit_capacity: int, stream: int | None = None):
    """Call kg_run_device_noalloc: no context, no device allocation.

    For callers that may not allocate device memory themselves: rows (d_x)
    and the hit buffer (d_hits, hit_capacity records of HIT_DTYPE) are device
    pointers the caller owns.  Returns (rc, n_tested, n_hits, message)."""
    U = np.asarray(U, dtype=np.float64)
    n, k = U.shape
    Uc = np.ascontiguousarray(U.T)
    yv = np.ascontiguousarray(y, dtype=np.float64)
    counts = (ctypes.c_uint64 * 2)()
    msg = ctypes.create_string_buffer(512)
    rc = lib().kg_run_device_noalloc(d_x, m, wpk, Uc.ctypes.data_as(_DP), n, k, yv.ctypes.data_as(_DP),
                                     corr_threshold, log10_thresh, d_hits, hit_capacity, counts, stream,
                                     msg, len(msg))
    return rc, int(counts[0]), int(counts[1]), msg.value.decode()


def probe_fp64_tflops(device: int = 0) -> float:
    """Measured FP64 FMA rate of the CUDA cores (TFLOP/s)."""
    v = ctypes.c_double()
    rc = lib().kg_probe_fp64_tflops(device, ctypes.byref(v))
    if rc != KG_OK:
        raise KgError(rc, "kg_probe_fp64_tflops")
    return v.value


def probe_h2d_gbs(device: int = 0, nbytes: int = 1 << 30, reps: int = 8) -> float:
    """Measured pinned host-to-device copy rate (GB/s)."""
    v = ctypes.c_double()
    rc = lib().kg_probe_h2d_gbs(device, nbytes, reps, ctypes.byref(v))
    if rc != KG_OK:
        raise KgError(rc, "kg_probe_h2d_gbs")
    return v.value


def version() -> str:
    return lib().kg_version().decode()
