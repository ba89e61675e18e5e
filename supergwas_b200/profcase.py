"""A small, self-contained launch sequence for profilers.

  python -m supergwas_b200.profcase [--kmers M] [--n N] [--r R]
         [--kernel ts|ss|fp64|multi|pairs] [--launches L] [--pheno P]

Generates a seeded batch on the device (same model as bench.py), sets the
structure (or P phenotypes for ``multi``), and runs the association kernel L
times so that `ncu -k regex:<kernel>` can capture a few launches of a batch
larger than L2 without the rest of the bench.  ``pairs`` tests every pair of
the first --kmers rows (use a few thousand).
"""
from __future__ import annotations

import argparse
import os
import time


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kmers", type=int, default=4_000_000)
    ap.add_argument("--n", type=int, default=1000)
    ap.add_argument("--r", type=int, default=16)
    ap.add_argument("--kernel", default="ts", choices=["ts", "ss", "fp64", "multi", "pairs"])
    ap.add_argument("--launches", type=int, default=3)
    ap.add_argument("--pheno", type=int, default=16)
    a = ap.parse_args()
    import numpy as np
    import torch
    from . import api, build, synth_gpu
    build.build_all()
    if a.kernel in ("ts", "ss"):
        os.environ["KG_KERNEL"] = a.kernel
    X = synth_gpu.gen_packed(a.n, a.kmers, 8, 44)
    wpk = X.shape[1]
    st = torch.cuda.Stream()  # a real stream handle (NULL would select the context's own stream)
    times = []
    if a.kernel == "multi":
        phenos = synth_gpu.batched_phenotypes(X, a.n, a.pheno, a.r, 46)
        g = api.Kgwas(precision="split", corr_threshold=0.0, log10_thresh=6.0)
        g.set_phenotypes(phenos, a.n)
        for _ in range(2):  # autotuner, graph capture
            g.launch_multi_device(X.data_ptr(), a.kmers, wpk, None, st.cuda_stream)
            g.fetch_multi()
        for _ in range(a.launches):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            g.launch_multi_device(X.data_ptr(), a.kmers, wpk, None, st.cuda_stream)
            e1.record(st)
            tested, hits = g.fetch_multi()
            times.append(e0.elapsed_time(e1))
        desc = f"tests={int(tested.sum())} hits={hits.shape[0]}"
        units = a.kmers * a.pheno
    elif a.kernel == "pairs":
        U, y, keep, _ = synth_gpu.structure_and_phenotype(X, a.n, a.r, 50, 0.0, 44)
        Xh = X.cpu().numpy().view(np.uint64)
        g = api.Kgwas(precision="split", log10_thresh=6.0)
        g.set_structure(U, y)
        g.run_pairs_host(Xh)
        for _ in range(a.launches):
            t0 = time.perf_counter()
            res, n_eval = g.run_pairs_host(Xh)
            times.append(1e3 * (time.perf_counter() - t0))
        desc = f"pairs_scored={n_eval} emitted={res.shape[0]}"
        units = a.kmers * (a.kmers - 1) // 2
    else:
        U, y, keep, _ = synth_gpu.structure_and_phenotype(X, a.n, a.r, 50, 0.05, 44)
        g = api.Kgwas(precision="fp64" if a.kernel == "fp64" else "split", corr_threshold=0.0, log10_thresh=6.0)
        g.set_structure(U, y, keep, a.n)
        g.launch_device(X.data_ptr(), a.kmers, wpk, st.cuda_stream)  # warm-up
        g.fetch()
        torch.cuda.synchronize()
        for _ in range(a.launches):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            g.launch_device(X.data_ptr(), a.kmers, wpk, st.cuda_stream)
            e1.record(st)
            r = g.fetch()
            times.append(e0.elapsed_time(e1))
        desc = f"kernel={g.last_kernel()} tested={r.n_tested} hits={r.hits.shape[0]}"
        units = a.kmers
    times.sort()
    med = times[len(times) // 2]
    print(f"{a.kernel} kmers={a.kmers} {desc} ms_per_launch={med:.3f} units_per_s={units / med * 1e3:.4g}")
    g.close()


if __name__ == "__main__":
    main()
