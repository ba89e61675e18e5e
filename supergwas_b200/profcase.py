"""A small, self-contained launch sequence for profilers.

  python -m supergwas_b200.profcase [--kmers M] [--n N] [--r R] [--kernel ts|ss|fp64] [--launches L]

Generates a seeded batch on the device (same model as bench.py), sets the
structure, and runs the association kernel L times through kg_launch_device
so that `ncu -k regex:<kernel>` can capture a few launches of a batch larger
than L2 without the rest of the bench.
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
    ap.add_argument("--kernel", default="ts", choices=["ts", "ss", "fp64"])
    ap.add_argument("--launches", type=int, default=3)
    a = ap.parse_args()
    import torch
    from . import api, build, synth_gpu
    build.build_all()
    if a.kernel in ("ts", "ss"):
        os.environ["KG_KERNEL"] = a.kernel
    X = synth_gpu.gen_packed(a.n, a.kmers, 8, 44)
    U, y, keep, _ = synth_gpu.structure_and_phenotype(X, a.n, a.r, 50, 0.05, 44)
    wpk = X.shape[1]
    g = api.Kgwas(precision="fp64" if a.kernel == "fp64" else "split", corr_threshold=0.0, log10_thresh=6.0)
    g.set_structure(U, y, keep, a.n)
    st = torch.cuda.Stream()  # a real stream handle (NULL would select the context's own stream)
    g.launch_device(X.data_ptr(), a.kmers, wpk, st.cuda_stream)  # warm-up
    g.fetch()
    torch.cuda.synchronize()
    times = []
    for _ in range(a.launches):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        g.launch_device(X.data_ptr(), a.kmers, wpk, st.cuda_stream)
        e1.record(st)
        r = g.fetch()
        times.append(e0.elapsed_time(e1))
    times.sort()
    med = times[len(times) // 2]
    print(f"kernel={g.last_kernel()} kmers={a.kmers} tested={r.n_tested} hits={r.hits.shape[0]} "
          f"device_ms_per_launch={med:.3f} kmers_per_s={a.kmers / med * 1e3:.4g}")
    g.close()


if __name__ == "__main__":
    main()
