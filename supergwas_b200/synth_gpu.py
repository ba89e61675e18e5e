"""Device-side generator of large seeded synthetic batches (bench workloads).

Same Balding-Nichols model as :mod:`supergwas_b200.synth` (ancestral
p ~ Beta(0.5, 0.5), per-subpopulation p_s ~ Beta(p(1-F)/F, (1-p)(1-F)/F),
F = 0.1, x ~ Bernoulli(p_s)), written straight into the packed k-mer-major
layout in device memory, chunk by chunk, each chunk from its own seeded
generator.  The structure matrix U and the phenotype y are then built on the
host from a 50,000-k-mer sample and the causal k-mers, exactly as in
:func:`supergwas_b200.synth.simulate`.
"""
from __future__ import annotations

import os

import numpy as np
import torch

from . import synth


def gen_packed(n: int, m: int, S: int, seed: int, device: str = "cuda", chunk: int = 1 << 20,
               out: torch.Tensor | None = None) -> torch.Tensor:
    """(m, words_per_kmer(n)) int64 tensor of packed rows on `device`."""
    W = synth.words_per_kmer(n)
    if out is None:
        out = torch.empty((m, W), dtype=torch.int64, device=device)
    pop = torch.as_tensor((np.arange(n) * S) // n, device=device)
    weights = (2 ** torch.arange(8, device=device, dtype=torch.int32)).to(torch.uint8)
    c = (1.0 - synth.F_ST) / synth.F_ST
    for s in range(0, m, chunk):
        e = min(m, s + chunk)
        cm = e - s
        g = torch.Generator(device=device)
        g.manual_seed(int(seed) * 1_000_003 + s // chunk)
        u = torch.rand(cm, generator=g, device=device, dtype=torch.float64)
        p = torch.sin(0.5 * torch.pi * u) ** 2            # Beta(0.5, 0.5) (arcsine law)
        p = p.clamp(1e-6, 1 - 1e-6)
        a = (p * c).unsqueeze(1).expand(cm, S)
        b = ((1 - p) * c).unsqueeze(1).expand(cm, S)
        ga = torch._standard_gamma(a.contiguous(), generator=g)
        gb = torch._standard_gamma(b.contiguous(), generator=g)
        ps = torch.nan_to_num(ga / (ga + gb), nan=0.5).to(torch.float32)
        probs = ps[:, pop]                                   # (cm, n)
        bits = torch.rand(cm, n, generator=g, device=device, dtype=torch.float32) < probs
        del probs
        if W * 64 > n:
            bits = torch.cat([bits, torch.zeros(cm, W * 64 - n, dtype=torch.bool, device=device)], 1)
        by = (bits.view(cm, W * 8, 8).to(torch.uint8) * weights).sum(-1, dtype=torch.int32).to(torch.uint8)
        out[s:e] = by.view(torch.int64).view(cm, W)
        del bits, by
    return out


_SYNTH = None


def synth_rows(out: torch.Tensor, n: int, S: int, seed: int, first: int = 0, stream=None) -> torch.Tensor:
    """Rows first .. first + out.shape[0] - 1 of a seeded batch from the CUDA
    generator (lib/libkgwas_bench.so): the same Balding-Nichols model, each
    row a function of (seed, row index) only, so a chunk of any batch can be
    regenerated on its own.  ``out`` is an (m, words_per_kmer(n)) int64 tensor
    on the device; the kernel runs on ``stream`` (default: the current one)."""
    import ctypes
    from . import build
    global _SYNTH
    if _SYNTH is None:
        if not os.path.exists(build.BENCH_LIB):
            raise RuntimeError(f"{build.BENCH_LIB} is not built; run `python -m supergwas_b200.build`")
        _SYNTH = ctypes.CDLL(build.BENCH_LIB)
        _SYNTH.kg_synth_rows.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p]
    st = stream if stream is not None else torch.cuda.current_stream()
    rc = _SYNTH.kg_synth_rows(out.data_ptr(), out.shape[0], n, out.shape[1], S, first, seed, st.cuda_stream)
    if rc != 0:
        raise RuntimeError(f"kg_synth_rows failed ({rc})")
    return out


def structure_and_phenotype(packed_dev: torch.Tensor, n: int, r: int, n_causal: int, missing: float,
                            seed: int, structure_kmers: int = 50_000):
    """U (overlap x (r+1)), y and overlap indices for a device-resident batch."""
    rng = np.random.default_rng(seed)
    m = packed_dev.shape[0]
    n_miss = int(round(missing * n))
    miss = np.sort(rng.choice(n, size=n_miss, replace=False)) if n_miss else np.zeros(0, np.int64)
    keep = np.setdiff1d(np.arange(n), miss)
    sk = min(structure_kmers, m)
    sidx = np.sort(rng.choice(m, size=sk, replace=False))
    rows = packed_dev[torch.as_tensor(sidx, device=packed_dev.device)].cpu().numpy().view(np.uint64)
    Xs = synth.unpack_rows(rows, n)[:, keep].T
    U, Ph = synth.structure_basis(Xs, r)
    causal = np.sort(rng.choice(m, size=n_causal, replace=False))
    beta = rng.standard_normal(n_causal)
    crow = packed_dev[torch.as_tensor(causal, device=packed_dev.device)].cpu().numpy().view(np.uint64)
    g = beta @ synth.unpack_rows(crow, n)[:, keep].astype(np.float64)
    pc1 = Ph[:, -1] if Ph.shape[1] else 0.0
    y = g + 0.5 * pc1 + rng.standard_normal(keep.shape[0])
    return U, y, keep, causal


def batched_phenotypes(packed_dev: torch.Tensor, n: int, n_pheno: int, r: int, seed: int,
                       missing_max: float = 0.3, structure_kmers: int = 20_000, n_causal: int = 50):
    """Phenotypes for one batch, each with its own missing samples.

    Phenotype p drops a uniform(0, missing_max) fraction of the n samples, and
    gets its own U (intercept + top r z-scored PCs of a centred k-mer sample
    restricted to its overlap, as synth.structure_basis) and its own
    y = causal effects + 0.5 PC1 + N(0, 1).  Returns [(U, y, keep)].
    """
    rng = np.random.default_rng(seed)
    m = packed_dev.shape[0]
    dev = packed_dev.device
    sk = min(structure_kmers, m)
    sidx = np.sort(rng.choice(m, size=sk, replace=False))
    rows = packed_dev[torch.as_tensor(sidx, device=dev)].cpu().numpy().view(np.uint64)
    Xs_all = torch.as_tensor(synth.unpack_rows(rows, n), device=dev, dtype=torch.float64)  # (sk, n)
    out = []
    for p in range(n_pheno):
        miss = rng.uniform(0.0, missing_max)
        keep = np.sort(rng.choice(n, size=n - int(round(miss * n)), replace=False))
        X = Xs_all[:, torch.as_tensor(keep, device=dev)].T  # (n_p, sk)
        X = X - X.mean(dim=0, keepdim=True)
        evals, evecs = torch.linalg.eigh(X @ X.T)
        Ph = (evecs[:, -r:] * torch.sqrt(torch.clamp(evals[-r:], min=0.0))).cpu().numpy()
        Ph = Ph - Ph.mean(axis=0, keepdims=True)
        sd = np.sqrt((Ph ** 2).sum(axis=0) / (Ph.shape[0] - 1))
        sd[sd == 0.0] = 1.0
        Ph = Ph / sd
        Z = np.concatenate([np.ones((keep.size, 1)), Ph], axis=1)
        U, _, _ = np.linalg.svd(Z, full_matrices=False)
        causal = np.sort(rng.choice(m, size=n_causal, replace=False))
        crow = packed_dev[torch.as_tensor(causal, device=dev)].cpu().numpy().view(np.uint64)
        g = rng.standard_normal(n_causal) @ synth.unpack_rows(crow, n)[:, keep].astype(np.float64)
        y = g + 0.5 * Ph[:, -1] + rng.standard_normal(keep.size)
        out.append((np.ascontiguousarray(U), y, keep))
    return out


def lognormal_shards(m: int, lo: int, hi: int, seed: int) -> np.ndarray:
    """Start offsets of shards of lognormal length clipped to [lo, hi] covering m k-mers."""
    rng = np.random.default_rng(seed)
    starts, s = [], 0
    mu = np.log(np.sqrt(lo * hi))
    while s < m:
        starts.append(s)
        s += int(np.clip(rng.lognormal(mu, 0.8), lo, hi))
    return np.asarray(starts, dtype=np.uint64)
