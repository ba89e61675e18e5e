"""Seeded synthetic k-mer presence/absence data in the reference's file formats.

The reference pipeline produces its inputs upstream of ``kgwas``:

* ``batch_*/bits/col_%06d.txt`` -- one ASCII line of '0'/'1' per sample, one
  byte per k-mer (written by ``src/convert_matrix.cpp:220-258``);
* ``batch_*/kmers.txt.gz`` -- one k-mer per line (``src/convert_matrix.cpp:209-215``);
* ``U.bin`` -- ``int32 n, int32 k`` then ``n*k`` float64 column-major
  (``src/compute_structure_all.cpp:80-88``), built from a centred k-mer sample
  by eig(XX^T), z-scored PCs and a thin SVD of ``[1, PCs]``
  (``src/compute_structure_all.cpp:150-186``);
* ``samples.txt`` (one id per line) and ``phenotype.txt`` (``id value``).

This module generates the same files from a Balding-Nichols model
(ancestral frequency p ~ Beta(0.5, 0.5), per-subpopulation frequency
p_s ~ Beta(p(1-F)/F, (1-p)(1-F)/F), F = 0.1), plus the packed format this
package computes on: k-mer-major rows of ``words_per_kmer`` little-endian
uint64 words, sample ``i`` in bit ``i % 64`` of word ``i // 64``, padding bits
zero, ``words_per_kmer`` even so that every row starts on a 16-byte boundary.
"""
from __future__ import annotations

import gzip
import os
import struct
from dataclasses import dataclass, field

import numpy as np

F_ST = 0.1


def words_per_kmer(n: int) -> int:
    """uint64 words per packed k-mer row: ceil(n/64) rounded up to even."""
    w = (n + 63) // 64
    return w + (w & 1)


def pack_rows(x: np.ndarray, wpk: int | None = None) -> np.ndarray:
    """Pack a (m, n) 0/1 matrix (k-mer-major) into (m, wpk) uint64 words."""
    x = np.ascontiguousarray(x, dtype=np.uint8)
    m, n = x.shape
    if wpk is None:
        wpk = words_per_kmer(n)
    nb = wpk * 64
    if n < nb:
        x = np.concatenate([x, np.zeros((m, nb - n), np.uint8)], axis=1)
    b = np.packbits(x, axis=1, bitorder="little")  # (m, wpk*8) bytes
    return np.ascontiguousarray(b).view(np.uint64).reshape(m, wpk)


def unpack_rows(packed: np.ndarray, n: int) -> np.ndarray:
    """Inverse of :func:`pack_rows`: (m, wpk) uint64 -> (m, n) uint8."""
    m = packed.shape[0]
    b = np.ascontiguousarray(packed).view(np.uint8).reshape(m, -1)
    return np.unpackbits(b, axis=1, bitorder="little")[:, :n]


def select_samples(packed: np.ndarray, n_all: int, idxs: np.ndarray) -> np.ndarray:
    """Repack rows keeping only the samples ``idxs`` (in that order)."""
    x = unpack_rows(packed, n_all)[:, idxs]
    return pack_rows(x)


def draw_frequencies(rng: np.random.Generator, m: int, S: int, F: float = F_ST):
    p = rng.beta(0.5, 0.5, size=m)
    p = np.clip(p, 1e-9, 1 - 1e-9)
    c = (1.0 - F) / F
    ps = rng.beta((p * c)[:, None], ((1.0 - p) * c)[:, None], size=(m, S))
    return p, ps


def draw_bits(rng: np.random.Generator, ps: np.ndarray, pop: np.ndarray) -> np.ndarray:
    """(m, n) uint8 presence/absence with sample i drawn at ps[:, pop[i]]."""
    m = ps.shape[0]
    n = pop.shape[0]
    u = rng.random((m, n), dtype=np.float32)
    return (u < ps[:, pop].astype(np.float32)).astype(np.uint8)


def structure_basis(Xs: np.ndarray, r: int) -> np.ndarray:
    """U for the 1-D null: orthonormal basis of [1, z-scored top-r PCs].

    Follows ``src/compute_structure_all.cpp:150-186``: centre the
    samples x k-mers matrix by column, eigen-decompose G = X X^T, keep the top
    ``r`` eigenvectors scaled by sqrt(eigenvalue), z-score each PC column
    (sample sd, n-1), prepend a column of ones and take the thin SVD's U.
    """
    X = Xs.astype(np.float64)
    n = X.shape[0]
    if r <= 0 or n < 2:
        return np.full((n, 1), 1.0 / np.sqrt(n)), np.zeros((n, 0))
    X = X - X.mean(axis=0, keepdims=True)
    G = X @ X.T
    evals, evecs = np.linalg.eigh(G)
    Ur = evecs[:, -r:]
    lam = np.maximum(evals[-r:], 0.0)
    Ph = Ur * np.sqrt(lam)[None, :]
    mu = Ph.mean(axis=0, keepdims=True)
    Ph = Ph - mu
    sd = np.sqrt((Ph ** 2).sum(axis=0) / (Ph.shape[0] - 1))
    sd[sd == 0.0] = 1.0
    Ph = Ph / sd[None, :]
    Z = np.concatenate([np.ones((X.shape[0], 1)), Ph], axis=1)
    U, _, _ = np.linalg.svd(Z, full_matrices=False)
    return np.ascontiguousarray(U), Ph


def random_kmers_text(rng: np.random.Generator, m: int, k: int = 31) -> bytes:
    """m random k-mers as the bytes of a kmers.txt file (one per line)."""
    alph = np.frombuffer(b"ACGT", dtype=np.uint8)
    rows = np.empty((m, k + 1), dtype=np.uint8)
    rows[:, :k] = alph[rng.integers(0, 4, size=(m, k), dtype=np.uint8)]
    rows[:, k] = ord("\n")
    return rows.tobytes()


def random_kmers(rng: np.random.Generator, m: int, k: int = 31) -> list[str]:
    alph = np.frombuffer(b"ACGT", dtype=np.uint8)
    codes = rng.integers(0, 4, size=(m, k), dtype=np.uint8)
    arr = alph[codes]
    return [bytes(row).decode() for row in arr]


@dataclass
class Dataset:
    """One synthetic batch and its structure/phenotype inputs."""
    n_all: int
    samples: list
    pheno_ids: list            # overlap ids, in samples order
    y: np.ndarray              # float64, overlap order
    idxs: np.ndarray           # positions of overlap samples in ``samples``
    U: np.ndarray              # (n_ov, k) float64
    packed_all: np.ndarray     # (m, words_per_kmer(n_all)) uint64, all samples
    kmers: list
    causal: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))

    @property
    def n(self) -> int:
        return int(self.idxs.shape[0])

    @property
    def m(self) -> int:
        return int(self.packed_all.shape[0])

    def packed_overlap(self) -> np.ndarray:
        return select_samples(self.packed_all, self.n_all, self.idxs)


def simulate(n: int, m: int, S: int, r: int, n_causal: int, missing: float,
             seed: int, structure_kmers: int = 50_000, kmer_len: int = 31,
             chunk: int = 200_000) -> Dataset:
    """Balding-Nichols batch with n samples in S even subpopulations.

    y = sum of N(0,1) effects of ``n_causal`` random k-mers + 0.5 * PC1 + N(0,1)
    on the phenotyped samples; ``missing`` of the samples get no phenotype.
    """
    rng = np.random.default_rng(seed)
    pop = (np.arange(n) * S) // n
    packed = np.zeros((m, words_per_kmer(n)), dtype=np.uint64)
    for s in range(0, m, chunk):
        e = min(m, s + chunk)
        _, ps = draw_frequencies(rng, e - s, S)
        packed[s:e] = pack_rows(draw_bits(rng, ps, pop))
    samples = [f"S{i:05d}" for i in range(n)]
    n_miss = int(round(missing * n))
    miss = np.sort(rng.choice(n, size=n_miss, replace=False)) if n_miss else np.zeros(0, np.int64)
    keep = np.setdiff1d(np.arange(n), miss)
    sk = min(structure_kmers, m)
    sidx = np.sort(rng.choice(m, size=sk, replace=False))
    Xs = unpack_rows(packed[sidx], n)[:, keep].T  # (n_ov, sk)
    U, Ph = structure_basis(Xs, r)
    causal = np.sort(rng.choice(m, size=n_causal, replace=False)) if n_causal else np.zeros(0, np.int64)
    beta = rng.standard_normal(n_causal)
    g = np.zeros(keep.shape[0])
    if n_causal:
        Xc = unpack_rows(packed[causal], n)[:, keep].astype(np.float64)
        g = beta @ Xc
    pc1 = Ph[:, -1] if Ph.shape[1] else 0.0
    y = g + 0.5 * pc1 + rng.standard_normal(keep.shape[0])
    kmers = random_kmers(rng, m, kmer_len)
    return Dataset(n_all=n, samples=samples, pheno_ids=[samples[i] for i in keep],
                   y=y, idxs=keep.astype(np.int64), U=U, packed_all=packed,
                   kmers=kmers, causal=causal)


# ----------------------------------------------------------------- writers

def write_samples(path: str, samples) -> None:
    with open(path, "w") as f:
        for s in samples:
            f.write(s + "\n")


def write_pheno(path: str, ids, y) -> None:
    with open(path, "w") as f:
        for i, v in zip(ids, y):
            f.write(f"{i} {float(v)!r}\n")


def write_ubin(path: str, U: np.ndarray) -> None:
    U = np.asarray(U, dtype=np.float64)
    n, k = U.shape
    with open(path, "wb") as f:
        f.write(struct.pack("<ii", n, k))
        f.write(np.asfortranarray(U).tobytes(order="F"))


def read_ubin(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        n, k = struct.unpack("<ii", f.read(8))
        return np.frombuffer(f.read(8 * n * k), dtype=np.float64).reshape(k, n).T.copy()


def write_batch(dirpath: str, packed_all: np.ndarray, n_all: int, kmers,
                gz_columns=(), kmers_plain_gz: bool = False) -> None:
    """Write a ``batch_*/`` directory: bits/col_%06d.txt[.gz] and kmers.txt.gz.

    ``gz_columns`` lists sample positions whose column is written gzipped;
    ``kmers`` is a list of strings or the bytes of the k-mer file.
    """
    os.makedirs(os.path.join(dirpath, "bits"), exist_ok=True)
    gzs = set(int(i) for i in gz_columns)
    m = packed_all.shape[0]
    # 64 samples (one packed word) at a time: their m-byte columns as rows
    for w in range((n_all + 63) // 64):
        bits = np.unpackbits(np.ascontiguousarray(packed_all[:, w]).view(np.uint8).reshape(m, 8), axis=1,
                             bitorder="little")  # (m, 64)
        cols = np.ascontiguousarray(bits.T) + np.uint8(ord("0"))
        for t in range(min(64, n_all - 64 * w)):
            j = 64 * w + t
            line = cols[t].tobytes() + b"\n"
            p = os.path.join(dirpath, "bits", f"col_{j:06d}.txt")
            if j in gzs:
                with gzip.open(p + ".gz", "wb", compresslevel=1) as f:
                    f.write(line)
            else:
                with open(p, "wb") as f:
                    f.write(line)
    data = kmers if isinstance(kmers, (bytes, bytearray)) else "".join(k + "\n" for k in kmers).encode()
    kp = os.path.join(dirpath, "kmers.txt.gz")
    if kmers_plain_gz:
        with open(kp, "wb") as f:  # zlib's gzopen reads plain files transparently
            f.write(data)
    else:
        with gzip.open(kp, "wb", compresslevel=1) as f:
            f.write(data)


def write_rows_file(path: str, packed_all: np.ndarray, n_all: int, kmers) -> None:
    """ROWS-mode input: ``kmer\\tbitstring`` lines (``src/kgwas.cpp:443-452``)."""
    x = unpack_rows(packed_all, n_all)
    op = gzip.open if path.endswith(".gz") else open
    with op(path, "wb") as f:
        for i, k in enumerate(kmers):
            f.write(k.encode() + b"\t" + (x[i] + ord("0")).astype(np.uint8).tobytes() + b"\n")


def write_dataset(root: str, ds: Dataset, batch: str = "batch_000", **kw) -> dict:
    os.makedirs(root, exist_ok=True)
    paths = dict(samples=os.path.join(root, "samples.txt"),
                 pheno=os.path.join(root, "phenotype.txt"),
                 ubin=os.path.join(root, "U.bin"),
                 batch=os.path.join(root, batch))
    write_samples(paths["samples"], ds.samples)
    write_pheno(paths["pheno"], ds.pheno_ids, ds.y)
    write_ubin(paths["ubin"], ds.U)
    write_batch(paths["batch"], ds.packed_all, ds.n_all, ds.kmers, **kw)
    return paths
