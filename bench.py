"""Throughput of the B200 k-mer association test.

Workload (default): n=1,000 samples (8 subpopulations, 5% without phenotype),
m=200,000,000 k-mers packed 1 bit/sample (16 uint64 words = 128 B per k-mer,
25.6 GB resident in HBM), U = intercept + 16 PCs, one phenotype with 50 causal
k-mers, CORR_THRESHOLD=0 (every non-constant k-mer is tested).  Seeded
synthetic data, generated on the device.

A step = one pass of the association test over the whole batch: pre-filter,
U^T x and x.y' contraction, chi-square and p, hit compaction, count.
``value`` times the split-precision tensor-core kernel with the batch resident
in HBM; ``e2e`` times kg_run_host from pinned host memory (host-to-device
copies inside the timed region); ``fp64_form`` is the plain FP64 CUDA-core
kernel on the same batch.  The batch (25.6 GB) is far larger than L2 (126 MB),
so no L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(n=1000, m=200_000_000, S=8, r=16, n_causal=50, missing=0.05, seed=44)
METRIC = "k-mer tests/s (split-precision tcgen05 kernel, n=1000, r=16+1, batch resident in HBM)"


def rank_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


# DRAM bytes (read + write) per k-mer of ts_kernel<64,1> on the bench workload
# (n=1000, 128-byte rows, r=16+1): dram__bytes_read.sum + dram__bytes_write.sum
# of one ncu capture of a 4M-k-mer launch (512 MB of rows, > L2) divided by the
# k-mers it processed; the traffic grows in proportion to the k-mers, so a full
# launch moves this many bytes per k-mer.  Capture and command:
# profiles/ts_kernel_n1000_r16.md.
TS_DRAM_BYTES_PER_KMER = 129.2


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.out = tempfile.NamedTemporaryFile("w+", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.dev)], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.proc or not self.out:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.out.flush()
        rows = [l.split(", ") for l in open(self.out.name).read().strip().splitlines() if l.count(",") >= 8]
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        sm = [float(r[1]) for r in rows]
        mx = max(float(r[2]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        pw = [float(r[3]) for r in rows]
        load = [s for s, w in zip(sm, pw) if w > 200.0] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows), "power_w_median": statistics.median(pw), "power_w_max": max(pw)}


# ------------------------------------------------------------ CPU baseline

def reference_binary():
    exe = os.path.join(ROOT, "oracle", "_ref", "kgwas")
    return exe if os.access(exe, os.X_OK) else None


def cpu_reference_run(n, m_sample, r, seed, threads, workdir, S=None):
    """Run the reference kgwas (COLS mode) on an m_sample-k-mer batch; returns (tests, seconds)."""
    from supergwas_b200 import synth
    from oracle import oracle as O
    ds = synth.simulate(n=n, m=m_sample, S=S or WORKLOAD["S"], r=r, n_causal=min(50, m_sample),
                        missing=WORKLOAD["missing"], seed=seed, structure_kmers=min(50_000, m_sample))
    paths = synth.write_dataset(workdir, ds)
    out = os.path.join(workdir, "out", "batch_000.tsv")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    env = {"CORR_THRESHOLD": "0", "LOAD_THREADS": threads, "BLAS_THREADS": threads, "EMIT_THREADS": threads}
    t0 = time.perf_counter()
    res = O.run_reference([paths["samples"], paths["pheno"], paths["batch"], paths["ubin"], out, "6"], env)
    dt = time.perf_counter() - t0
    if res.returncode != 0:
        raise RuntimeError(res.stderr[-500:])
    tested = int(open(out + ".count").read().split("\t")[1])
    return tested, dt, paths


def cpu_port_run(n, m_sample, r, seed):
    """The oracle (single-thread C port) on an m_sample-k-mer batch."""
    from supergwas_b200 import synth
    from oracle import oracle as O
    ds = synth.simulate(n=n, m=m_sample, S=WORKLOAD["S"], r=r, n_causal=min(50, m_sample),
                        missing=WORKLOAD["missing"], seed=seed, structure_kmers=min(50_000, m_sample))
    X = ds.packed_overlap()
    t0 = time.perf_counter()
    st = O.cols_stats(X, ds.n, ds.U, ds.y, 0.0)
    return st["n_tested"], time.perf_counter() - t0


def cpu_baseline(n, r, seed, sample_kmers):
    threads = os.cpu_count() or 1
    if reference_binary():
        with tempfile.TemporaryDirectory() as d:
            tested, dt, _ = cpu_reference_run(n, sample_kmers, r, seed, threads, d)
        return {"value": tested / dt, "unit": "k-mer tests/s", "cores": threads, "kind": "reference",
                "sample": f"reference kgwas --mode cols (shipped binary), n={n}, r={r}+1, "
                          f"{sample_kmers} k-mers, CORR_THRESHOLD=0, wall clock incl. its file load"}
    m = max(1000, sample_kmers // 20)
    tested, dt = cpu_port_run(n, m, r, seed)
    return {"value": tested / dt, "unit": "k-mer tests/s", "cores": 1, "kind": "port",
            "sample": f"FP64 C oracle, n={n}, r={r}+1, {m} k-mers, CORR_THRESHOLD=0"}


def run_reference_arm(args):
    """The reference's own CPU implementation on this box's host cores: one
    batch of ``--ref-kmers`` k-mers of the bench workload, run W + K times."""
    rank, world, _ = rank_env()
    if rank != 0:
        return
    W = WORKLOAD
    threads = os.cpu_count() or 1
    m_sample = args.ref_kmers
    vals = []
    kind = "reference" if reference_binary() else "port"
    with tempfile.TemporaryDirectory() as d:
        if kind == "reference":
            from oracle import oracle as O
            tested, dt, paths = cpu_reference_run(W["n"], m_sample, W["r"], W["seed"], threads, d)
            env = {"CORR_THRESHOLD": "0", "LOAD_THREADS": threads, "BLAS_THREADS": threads,
                   "EMIT_THREADS": threads}
            out = os.path.join(d, "out", "batch_000.tsv")
            for i in range(args.warmup + args.steps):
                t0 = time.perf_counter()
                res = O.run_reference([paths["samples"], paths["pheno"], paths["batch"], paths["ubin"], out,
                                       "6"], env)
                dt = time.perf_counter() - t0
                if res.returncode != 0:
                    raise RuntimeError(res.stderr[-500:])
                if i >= args.warmup:
                    vals.append((int(open(out + ".count").read().split("\t")[1]), dt))
        else:
            for i in range(args.warmup + args.steps):
                tested, dt = cpu_port_run(W["n"], max(1000, m_sample // 20), W["r"], W["seed"])
                if i >= args.warmup:
                    vals.append((tested, dt))
    tests = sum(t for t, _ in vals)
    secs = sum(s for _, s in vals)
    v = tests / secs
    ms = m_sample if kind == "reference" else max(1000, m_sample // 20)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "k-mer tests/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / len(vals),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (reference COLS mode)" if kind == "reference" else "f64",
            "data": "synthetic",
            "config": {"workload": f"n={W['n']} (5% unphenotyped), r={W['r']}+1, 1 phenotype, "
                                   f"CORR_THRESHOLD=0; each step one {ms}-k-mer batch of that workload",
                       "parallelism": "host cores"},
            "cpu_baseline": {"value": v, "unit": "k-mer tests/s", "cores": threads if kind == "reference" else 1,
                             "kind": kind,
                             "sample": (f"shipped reference kgwas --mode cols on {ms} k-mers per step, wall "
                                        "clock of the process (file load included)") if kind == "reference"
                             else f"FP64 C oracle on {ms} k-mers per step"},
            "e2e": {"value": v, "unit": "k-mer tests/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- GPU arm

def accuracy_report(X_dev, m_sub, wpk, U, y, keep, n_all):
    """Split form vs the FP64 oracle on the first m_sub k-mers: chi2 rel / -log10 p abs errors."""
    from oracle import oracle as O
    from supergwas_b200 import api, synth
    Xh = X_dev[:m_sub].cpu().numpy().view(np.uint64)
    Xo = synth.select_samples(Xh, n_all, keep)
    o = O.cols_stats(Xo, len(keep), U, y, 0.0)
    with api.Kgwas(precision="split", corr_threshold=0.0, log10_thresh=6.0) as g:
        g.set_structure(U, y, keep, n_all)
        res = g.run_host(Xh, stats=True)
    st = res.stats
    msk = st["tested"] & o["tested"]
    T0, T1 = o["chisq"][msk], st["chisq"][msk]
    rel = np.abs(T1 - T0) / np.maximum(T0, 1e-300)
    ml = np.abs(st["mlog10p"][msk] - o["mlog10p"][msk])
    return {"kmers_checked": int(m_sub), "tested_identical": bool(np.array_equal(st["tested"], o["tested"])),
            "chisq_rel_max": float(rel.max()), "chisq_rel_p99": float(np.percentile(rel, 99)),
            "chisq_rel_max_T_ge_1e-3": float(rel[T0 >= 1e-3].max()),
            "mlog10p_abs_max": float(ml.max()), "mlog10p_abs_p99": float(np.percentile(ml, 99)),
            "reference": "FP64 C oracle (long-double accumulation)"}


def time_device(g, X, m, wpk, steps, warmup, stream):
    import torch
    launches = 0
    for _ in range(warmup):
        g.launch_device(X.data_ptr(), m, wpk, stream.cuda_stream)
        g.fetch()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    tested = 0
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        for i in range(steps):
            g.launch_device(X.data_ptr(), m, wpk, stream.cuda_stream)
            launches += g.last_launch_count()
            ev[i + 1].record(stream)
    torch.cuda.synchronize()
    res = g.fetch()
    tested = res.n_tested
    per = [ev[i].elapsed_time(ev[i + 1]) for i in range(steps)]
    return tested, per, launches


def run_ours(args):
    import torch
    import torch.distributed as dist
    from supergwas_b200 import api, build, synth_gpu
    rank, world, local = rank_env()
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    build.build_all()
    W = dict(WORKLOAD)
    if args.kmers:
        W["m"] = args.kmers
    n, m, r = W["n"], W["m"], W["r"]
    wpk = (n + 63) // 64
    wpk += wpk & 1
    t_gen = time.perf_counter()
    X = synth_gpu.gen_packed(n, m, W["S"], W["seed"] + 1000 * rank)
    U, y, keep, causal = synth_gpu.structure_and_phenotype(X, n, r, W["n_causal"], W["missing"],
                                                           W["seed"] + 1000 * rank)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen
    stream = torch.cuda.Stream()
    hbm, bf16, peak_src = measured_peaks()

    g = api.Kgwas(device=local, precision="split", corr_threshold=0.0, log10_thresh=6.0)
    g.set_structure(U, y, keep, n)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as ck:
        tested, per, launches = time_device(g, X, m, wpk, args.steps, args.warmup, stream)
        if world > 1:
            dist.barrier()
    clocks = ck.summary()
    t_split = sum(per) / 1e3

    # plain FP64 form on the same batch
    f = api.Kgwas(device=local, precision="fp64", corr_threshold=0.0, log10_thresh=6.0)
    f.set_structure(U, y, keep, n)
    fsteps = max(1, min(args.steps, 3))
    ftested, fper, _ = time_device(f, X, m, wpk, fsteps, 1, stream)
    t_fp64 = sum(fper) / fsteps / 1e3

    # end to end through kg_run_host from pinned host memory
    m_e2e = min(m, args.e2e_kmers) if args.e2e_kmers else m
    hbuf = api.lib().kg_host_alloc(m_e2e * wpk * 8)
    if not hbuf:
        raise RuntimeError("kg_host_alloc failed")
    import ctypes
    hview = (ctypes.c_char * (m_e2e * wpk * 8)).from_address(hbuf)
    ht = torch.frombuffer(hview, dtype=torch.int64).view(m_e2e, wpk)
    ht.copy_(X[:m_e2e])
    torch.cuda.synchronize()
    e2e_steps = max(1, min(args.steps, 5))
    g.run_host_ptr(hbuf, m_e2e, wpk)  # warm-up (allocates chunk buffers)
    t0 = time.perf_counter()
    e2e_tested = 0
    for _ in range(e2e_steps):
        rr = g.run_host_ptr(hbuf, m_e2e, wpk)
        e2e_tested += rr.n_tested
    t_e2e = (time.perf_counter() - t0) / e2e_steps
    d2h = 3 * 8 + rr.hits.shape[0] * 32
    api.lib().kg_host_free(hbuf)

    # the programs on files at a pipeline-sized batch (rank 0)
    leg_files = None
    if rank == 0 and args.files_kmers and not args.no_legs:
        leg_files = files_cols_leg(X[:min(m, args.files_kmers)].cpu().numpy().view(np.uint64), n, U, y, keep, local)

    # measured peaks of the FP64 form and of the host link
    fp64_peak = api.probe_fp64_tflops(local)
    h2d_peak = api.probe_h2d_gbs(local, 1 << 30, 8)
    # plain FP64 form at n=1000, m=5e7, r=10+1
    leg_fp64 = None if args.no_legs else fp64_config2_leg(X, local, rank, 3, 3, fp64_peak)
    acc = accuracy_report(X, min(m, args.acc_kmers), wpk, U, y, keep, n) if rank == 0 else None
    # batched 64 phenotypes (n=2000, m=1e8, r=20+1) on a batch of its own
    del X
    torch.cuda.empty_cache()
    leg_batched = None if args.no_legs else batched_leg(local, rank, 0, 3, 3, args.acc_kmers // 4)

    # max over ranks of device time; sum of tests
    if world > 1:
        tt = torch.tensor([t_split, float(tested)], dtype=torch.float64, device="cuda")
        mx = tt.clone()
        dist.all_reduce(mx[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(tt[1:], op=dist.ReduceOp.SUM)
        t_split_all = float(mx[0])
        tested_all = float(tt[1])
    else:
        t_split_all = t_split
        tested_all = float(tested)

    if rank == 0:
        value = tested_all * args.steps / t_split_all
        t_launch = t_split / args.steps
        alg_bytes = m * ((n + 7) // 8)          # packed x, 1 bit per sample (algorithmic)
        achieved = alg_bytes / t_launch / 1e9
        traffic_pk = TS_DRAM_BYTES_PER_KMER if (n, r) == (1000, 16) else None
        N = 64
        kpad = ((n + 255) // 256) * 256
        tops = 2.0 * m * kpad * N / t_launch / 1e12
        sm_mhz = clocks.get("sm_mhz") or 0.0
        n_sm = torch.cuda.get_device_properties(local).multi_processor_count
        hw_peak = 16384.0 * n_sm * sm_mhz * 1e6 / 1e12 if sm_mhz else None
        cpu = cpu_baseline(n, r, W["seed"], args.cpu_kmers) if not args.no_cpu else None
        line = {
            "metric": METRIC, "value": value, "unit": "k-mer tests/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_split_all / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "i8 limbs -> i32 TMEM, f64 epilogue",
            "data": "synthetic (seeded Balding-Nichols, generated on device)",
            "config": {"workload": f"n={n} (5% unphenotyped), m={m} k-mers per GPU, r={r}+1, 1 phenotype, "
                                   f"CORR_THRESHOLD=0", "kmers_per_gpu": m, "bytes_per_kmer": wpk * 8,
                       "l2": "inputs (%.1f GB) >> L2; no flush needed" % (m * wpk * 8 / 1e9),
                       "parallelism": f"weak: {world} GPU(s), independent k-mer shards"},
            "tests_per_step": tested_all,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "peak_source": peak_src,
                         "traffic": (traffic_pk * m if traffic_pk else None),
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "tensor": {"achieved_tops_int8": tops, "peak_tops_int8": 2 * bf16,
                                    "frac": tops / (2 * bf16),
                                    "peak_note": "2x measured bf16 burst (int8 MMA issues at twice the bf16 rate)",
                                    # 16384 int8 ops per SM-cycle at the median SM clock of the timed
                                    # region (an N=64 MMA issues at that rate: --workload mma-rate)
                                    "hw_peak_tops_int8_at_clock": hw_peak,
                                    "frac_of_hw_peak": tops / hw_peak if hw_peak else None,
                                    "useful_columns": "54 of N=64 (count, 5 y' limbs, 16 x 3 U limbs)"}},
            "fp64_form": {"value": ftested / t_fp64, "unit": "k-mer tests/s", "ms_per_step": 1e3 * t_fp64,
                          "split_speedup": value / world / (ftested / t_fp64),
                          "fp64_tflops": 2.0 * m * (((n + 127) // 128) * 128) * 20 / t_fp64 / 1e12,
                          "fp64_frac": 2.0 * m * (((n + 127) // 128) * 128) * 20 / t_fp64 / 1e12 / fp64_peak},
            "fp64_config2": leg_fp64,
            "files_cols": leg_files,
            "batched": leg_batched,
            "peaks": {"hbm_gbs": hbm, "hbm_source": peak_src, "bf16_tflops": bf16,
                      "fp64_tflops": fp64_peak, "fp64_source": "measured (kg_probe_fp64_tflops)",
                      "h2d_gbs": h2d_peak, "h2d_source": "measured (kg_probe_h2d_gbs, 8 x 1 GiB pinned)"},
            "accuracy_vs_fp64_oracle": acc,
            "e2e": {"value": e2e_tested / e2e_steps / t_e2e * world, "unit": "k-mer tests/s",
                    "h2d_bytes_per_step": m_e2e * wpk * 8, "d2h_bytes_per_step": d2h,
                    "kmers_per_step": m_e2e, "api": "kg_run_host (pinned host buffer)",
                    "h2d_gbs": m_e2e * wpk * 8 / t_e2e / 1e9,
                    "link_frac": m_e2e * wpk * 8 / t_e2e / 1e9 / h2d_peak if h2d_peak else None},
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "gen_seconds": t_gen,
        }
        print(json.dumps(line), flush=True)
    g.close()
    f.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


BATCHED = dict(n=2000, m=100_000_000, S=8, r=20, n_pheno=64, seed=46, shard_lo=1_000_000, shard_hi=20_000_000)


def batched_leg(local, rank, m, steps, warmup, acc_kmers):
    """Batched multi-phenotype workload (n=2000, r=20+1, 64 phenotypes with
    their own missing masks, lognormal shards): one fused launch per step over
    every phenotype and every shard, replayed from a captured CUDA graph.
    Returns the leg's figures (dict)."""
    import torch
    from supergwas_b200 import api, synth_gpu, synth
    from oracle import oracle as O
    W = dict(BATCHED)
    if m:
        W["m"] = m
    n, m, r, npn = W["n"], W["m"], W["r"], W["n_pheno"]
    wpk = synth.words_per_kmer(n)
    t_gen = time.perf_counter()
    X = synth_gpu.gen_packed(n, m, W["S"], W["seed"] + 1000 * rank)
    phenos = synth_gpu.batched_phenotypes(X, n, npn, r, W["seed"] + 1000 * rank)
    shards = synth_gpu.lognormal_shards(m, W["shard_lo"], W["shard_hi"], W["seed"])
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen
    st = torch.cuda.Stream()
    g = api.Kgwas(device=local, precision="split", corr_threshold=0.0, log10_thresh=6.0)
    g.set_phenotypes(phenos, n)
    for _ in range(warmup):  # first: autotuner; second: graph capture
        g.launch_multi_device(X.data_ptr(), m, wpk, shards, st.cuda_stream)
        tested, hits = g.fetch_multi()
    shape = g.multi_shape()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    launches = 0
    with Clocks(local) as ck:
        ev[0].record(st)
        for i in range(steps):
            g.launch_multi_device(X.data_ptr(), m, wpk, shards, st.cuda_stream)
            launches += g.last_launch_count()
            ev[i + 1].record(st)
        torch.cuda.synchronize()
    tested, hits = g.fetch_multi()
    g.close()
    t = sum(ev[i].elapsed_time(ev[i + 1]) for i in range(steps)) / 1e3
    tests = float(tested.sum())
    value = tests * steps / t
    # accuracy per phenotype on a sample: every tested k-mer emitted, vs the FP64 oracle
    m_acc = min(m, acc_kmers)
    acc = []
    with api.Kgwas(device=local, precision="split", corr_threshold=0.0, log10_thresh=0.0) as ga:
        ga.set_phenotypes(phenos, n)
        ga.launch_multi_device(X.data_ptr(), m_acc, wpk, None, st.cuda_stream)
        _, ah = ga.fetch_multi()
    Xh = X[:m_acc].cpu().numpy().view(np.uint64)
    del X
    torch.cuda.empty_cache()
    for p in range(0, npn, max(1, npn // 8)):
        U, y, keep = phenos[p]
        o = O.cols_stats(synth.select_samples(Xh, n, keep), keep.size, U, y, 0.0)
        h = ah[ah["pheno"] == p]
        exp = np.nonzero(o["tested"])[0]
        same = np.array_equal(h["kmer"].astype(np.int64), exp)
        ml = np.abs(O.mlog10p(h["chisq"]) - o["mlog10p"][exp]) if same else np.array([np.inf])
        T0, T1 = (o["chisq"][exp], h["chisq"]) if same else (np.ones(1), np.full(1, np.inf))
        rel = np.abs(T1 - T0) / np.maximum(T0, 1e-300)
        acc.append({"pheno": p, "n": int(keep.size), "kmers_checked": int(m_acc), "tested_identical": bool(same),
                    "mlog10p_abs_max": float(ml.max()), "chisq_rel_p99": float(np.percentile(rel, 99)),
                    "chisq_rel_max_T_ge_1e-3": float(rel[T0 >= 1e-3].max()) if (T0 >= 1e-3).any() else 0.0})
    hbm, bf16, peak_src = measured_peaks()
    ops = 2.0 * m * shape["kpad"] * shape["NP"] * npn   # int8 ops executed (padded columns included)
    tops = ops / (t / steps) / 1e12
    return {"metric": "k-mer tests/s (batched: 64 phenotypes x 1e8 k-mers, n=2000, r=20+1, one fused launch)",
            "value": value, "unit": "k-mer tests/s", "steps": steps, "warmup": warmup,
            "ms_per_step": 1e3 * t / steps, "tests_per_step": tests, "gpu_launches": launches,
            "config": {"workload": f"batched: n={n}, m={m}, r={r}+1, {npn} phenotypes (0-30% missing each), "
                                   f"{len(shards)} lognormal shards of {W['shard_lo']}-{W['shard_hi']} k-mers, "
                                   "CORR_THRESHOLD=0",
                       "l2": "inputs (%.1f GB) >> L2; no flush needed" % (m * wpk * 8 / 1e9)},
            "tile_shape": shape,
            "roofline": {"bound": "tensor", "achieved": tops, "peak": 2 * bf16, "unit": "TOP/s int8",
                         "frac": tops / (2 * bf16), "peak_source": peak_src + " (2x bf16 burst)",
                         "ops_per_launch": ops, "traffic": None},
            "accuracy_vs_fp64_oracle": acc, "clocks": ck.summary(), "gen_seconds": t_gen}


def run_batched(args):
    import torch
    from supergwas_b200 import build
    rank, world, local = rank_env()
    torch.cuda.set_device(local)
    build.build_all()
    leg = batched_leg(local, rank, args.kmers, args.steps, args.warmup, args.acc_kmers // 4)
    line = dict(leg)
    line.update({"n_gpus": world, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                 "dtype": "i8 limbs -> i32 TMEM, f64 epilogue", "data": "synthetic (seeded, generated on device)"})
    line["config"]["parallelism"] = f"weak: {world} GPU(s)"
    if rank == 0:
        print(json.dumps(line), flush=True)


FP64_CFG2 = dict(n=1000, m=50_000_000, r=10, n_causal=50, missing=0.05, seed=45)


def fp64_config2_leg(X, local, rank, steps, warmup, fp64_peak):
    """Plain FP64 form at n=1000, m=5e7, r=10+1 (50 causal k-mers): the first
    5e7 rows of the device batch (same generator, 8 subpopulations) with a
    structure of 10 PCs and its own phenotype.  HBM GB/s of the packed rows
    and FP64 TFLOP/s against the measured DFMA peak."""
    import torch
    from supergwas_b200 import api, synth_gpu
    C = FP64_CFG2
    n, m, r = C["n"], min(C["m"], X.shape[0]), C["r"]
    wpk = X.shape[1]
    Xc = X[:m]
    U, y, keep, _ = synth_gpu.structure_and_phenotype(Xc, n, r, C["n_causal"], C["missing"], C["seed"] + 1000 * rank)
    st = torch.cuda.Stream()
    with api.Kgwas(device=local, precision="fp64", corr_threshold=0.0, log10_thresh=6.0) as f:
        f.set_structure(U, y, keep, n)
        tested, per, launches = time_device(f, Xc, m, wpk, steps, warmup, st)
    t = sum(per) / steps / 1e3
    cm = 16                       # FP64 columns [count, d_0..d_10, d_y] padded to the kernel's 16
    kpad = ((n + 127) // 128) * 128
    flops = 2.0 * m * kpad * cm   # one FMA per (sample, column) per k-mer, padding included
    alg_bytes = m * ((n + 7) // 8)
    return {"value": tested / t, "unit": "k-mer tests/s", "ms_per_step": 1e3 * t, "steps": steps,
            "warmup": warmup, "gpu_launches": launches,
            "config": {"workload": f"fp64 form: n={n} (5% unphenotyped), m={m}, r={r}+1, 1 phenotype "
                                   f"({C['n_causal']} causal), CORR_THRESHOLD=0"},
            "hbm_gbs": alg_bytes / t / 1e9,
            "fp64": {"achieved_tflops": flops / t / 1e12, "peak_tflops": fp64_peak,
                     "frac": (flops / t / 1e12 / fp64_peak) if fp64_peak else None,
                     "peak_source": "measured (kg_probe_fp64_tflops: DFMA chains on every SM)"}}


STREAMING = dict(n=5000, S=12, r=32, n_pheno=8, seed=47, m_total=1_000_000_000, chunk_bytes=16_000_000_000,
                 chunks=8, fp64_kmers=2_000_000, acc_kmers=20_000, cpu_kmers=200_000)


def run_streaming(args):
    """Large streaming workload (n=5000 in 12 subpopulations, r=32+1, 8
    phenotypes with their own missing masks, m=1e9 k-mers = 625 GB of packed
    rows).  The rows live in pinned host memory in 16 GB chunks and stream
    through kg_run_multi_host (chunked host-to-device copies overlapped with
    the fused kernels).  625 GB does not fit host memory, so each chunk is
    regenerated from its own seed while the previous one is tested: the
    device generator writes chunk c+1 and copies it into the other pinned
    buffer (device-to-host, the other direction of the link) while chunk c
    streams in.  --steps chunks are timed (the per-chunk rate is steady; the
    line extrapolates the whole 1e9).  Also: the plain FP64 form on a
    device-resident sample of every phenotype, the split form's accuracy
    against the FP64 oracle, and the reference kgwas on a slice."""
    import threading
    import torch
    from supergwas_b200 import api, build, synth_gpu, synth
    from oracle import oracle as O
    rank, world, local = rank_env()
    torch.cuda.set_device(local)
    build.build_all()
    W = dict(STREAMING)
    n, S, r, npn, seed = W["n"], W["S"], W["r"], W["n_pheno"], W["seed"] + 1000 * rank
    wpk = synth.words_per_kmer(n)
    row = wpk * 8
    per = args.kmers or int(W["chunk_bytes"] // row)          # 25,000,000 rows = 16 GB at n=5000
    nchunks = max(1, args.steps)
    t_gen = time.perf_counter()
    dgen = torch.empty((per, wpk), dtype=torch.int64, device="cuda")
    hbuf = [torch.empty((per, wpk), dtype=torch.int64, pin_memory=True) for _ in range(2)]
    gs = torch.cuda.Stream()
    gen_s = []

    def produce(c, b):
        t = time.perf_counter()
        synth_gpu.synth_rows(dgen, n, S, seed, first=c * per, stream=gs)
        with torch.cuda.stream(gs):
            hbuf[b].copy_(dgen, non_blocking=True)
        gs.synchronize()
        gen_s.append(time.perf_counter() - t)

    produce(0, 0)
    phenos = synth_gpu.batched_phenotypes(dgen, n, npn, r, seed, structure_kmers=20_000)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen
    h2d_peak = api.probe_h2d_gbs(local, 1 << 30, 8)
    g = api.Kgwas(device=local, precision="split", corr_threshold=0.0, log10_thresh=6.0)
    g.set_phenotypes(phenos, n)
    view = [h.numpy().view(np.uint64) for h in hbuf]
    warm = min(per, 2_000_000)
    for _ in range(max(1, args.warmup)):
        g.run_multi_host(view[0][:warm])
    shape = g.multi_shape()
    chunk_s, tests = [], 0.0
    hits_total = 0
    with Clocks(local) as ck:
        t0 = time.perf_counter()
        for c in range(nchunks):
            th = None
            if c + 1 < nchunks:
                th = threading.Thread(target=produce, args=(c + 1, (c + 1) % 2))
                th.start()
            tc = time.perf_counter()
            tested, hits = g.run_multi_host(view[c % 2])
            chunk_s.append(time.perf_counter() - tc)
            tests += float(tested.sum())
            hits_total += int(hits.shape[0])
            if th is not None:
                th.join()
        t = time.perf_counter() - t0
    launches = g.last_launch_count()
    value = tests / t
    kmers_per_s = nchunks * per / t
    # accuracy of the split form on a sample of the last chunk, every phenotype, vs the FP64 oracle
    m_acc = min(per, W["acc_kmers"])
    Xh = view[(nchunks - 1) % 2][:m_acc].copy()
    with api.Kgwas(device=local, precision="split", corr_threshold=0.0, log10_thresh=0.0) as ga:
        ga.set_phenotypes(phenos, n)
        _, ah = ga.run_multi_host(Xh)
    acc = []
    for p in range(npn):
        U, y, keep = phenos[p]
        o = O.cols_stats(synth.select_samples(Xh, n, keep), keep.size, U, y, 0.0)
        h = ah[ah["pheno"] == p]
        exp = np.nonzero(o["tested"])[0]
        same = np.array_equal(h["kmer"].astype(np.int64), exp)
        ml = np.abs(O.mlog10p(h["chisq"]) - o["mlog10p"][exp]) if same else np.array([np.inf])
        T0, T1 = (o["chisq"][exp], h["chisq"]) if same else (np.ones(1), np.full(1, np.inf))
        rel = np.abs(T1 - T0) / np.maximum(T0, 1e-300)
        acc.append({"pheno": p, "n": int(keep.size), "tested_identical": bool(same),
                    "mlog10p_abs_max": float(ml.max()), "chisq_rel_p99": float(np.percentile(rel, 99))})
    # plain FP64 form, every phenotype, on a device-resident sample (the last chunk's rows)
    m64 = min(per, W["fp64_kmers"])
    dgen[:m64].copy_(hbuf[(nchunks - 1) % 2][:m64])
    st = torch.cuda.Stream()
    f_tests, f_t = 0.0, 0.0
    for U, y, keep in phenos:
        with api.Kgwas(device=local, precision="fp64", corr_threshold=0.0, log10_thresh=6.0) as f:
            f.set_structure(U, y, keep, n)
            tt, per_ms, _ = time_device(f, dgen[:m64], m64, wpk, 2, 1, st)
        f_tests += tt
        f_t += sum(per_ms) / len(per_ms) / 1e3
    fp64_value = f_tests / f_t
    # the reference kgwas (one phenotype per process, as the pipeline runs it) on a slice
    cpu = None
    if not args.no_cpu and reference_binary() and rank == 0:
        threads = os.cpu_count() or 1
        with tempfile.TemporaryDirectory() as d:
            tested_ref, dt, _ = cpu_reference_run(n, W["cpu_kmers"], r, W["seed"], threads, d, S=S)
        cpu = {"value": tested_ref / dt, "unit": "k-mer tests/s", "cores": threads, "kind": "reference",
               "sample": f"reference kgwas --mode cols, one phenotype, n={n}, r={r}+1, {W['cpu_kmers']} k-mers, "
                         "CORR_THRESHOLD=0, wall clock incl. its file load; a test is one (k-mer, phenotype), so "
                         "the rate carries over to 8 phenotypes run as 8 processes"}
    h2d_gbs = nchunks * per * row / sum(chunk_s) / 1e9
    line = {"metric": "k-mer tests/s (streaming from pinned host: 8 phenotypes, n=5000, r=32+1, 16 GB chunks)",
            "value": value, "unit": "k-mer tests/s", "n_gpus": world, "steps": nchunks, "warmup": args.warmup,
            "ms_per_step": 1e3 * t / nchunks, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "i8 limbs -> i32 TMEM, f64 epilogue",
            "data": "synthetic (seeded Balding-Nichols, each chunk regenerated on the device from its seed)",
            "config": {"workload": f"streaming: n={n} ({S} subpopulations), m=1e9 k-mers as {W['m_total'] // per} "
                                   f"chunks of {per} ({per * row / 1e9:.1f} GB) in pinned host memory, r={r}+1, "
                                   f"{npn} phenotypes (0-30% missing each), CORR_THRESHOLD=0; {nchunks} chunks timed",
                       "parallelism": f"weak: {world} GPU(s)"},
            "tile_shape": shape,
            "e2e": {"value": value, "unit": "k-mer tests/s", "h2d_bytes_per_step": per * row,
                    "d2h_bytes_per_step": hits_total * 40 // nchunks + npn * 8, "api": "kg_run_multi_host"},
            "roofline": {"bound": "host link", "achieved": h2d_gbs, "peak": h2d_peak, "unit": "GB/s",
                         "frac": h2d_gbs / h2d_peak if h2d_peak else None,
                         "peak_source": "measured (kg_probe_h2d_gbs, 8 x 1 GiB pinned)", "traffic": None},
            "kmers_per_s": kmers_per_s, "full_1e9_seconds_extrapolated": W["m_total"] / kmers_per_s,
            "chunk_seconds": chunk_s, "regen_seconds": gen_s[1:],
            # the last chunk streams while no regeneration shares the link: the
            # rate of kg_run_multi_host itself on 16 GB of pinned host rows
            "last_chunk_alone": {"seconds": chunk_s[-1], "h2d_gbs": per * row / chunk_s[-1] / 1e9,
                                 "link_frac": per * row / chunk_s[-1] / 1e9 / h2d_peak if h2d_peak else None,
                                 "tests_per_s": tests / nchunks / chunk_s[-1]},
            "fp64_form": {"value": fp64_value, "unit": "k-mer tests/s",
                          "sample": f"{m64} device-resident k-mers x {npn} phenotypes",
                          "split_speedup": value / world / fp64_value},
            "accuracy_vs_fp64_oracle": acc, "cpu_baseline": cpu,
            "gpu_launches": launches, "clocks": ck.summary(), "gen_seconds": t_gen}
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.close()


SORTED = dict(n=1000, m=50_000_000, S=8, r=16, n_causal=50, missing=0.05, seed=49, mean_run=5)


def run_sorted(args):
    """End to end (kg_run_host) on a batch sorted by bit pattern, as real
    batches are (src/convert_matrix.cpp:366-368): each distinct row repeated
    1..9 times (mean 5).  From pageable host memory (how the kgwas program
    passes its rows) the rows are staged through pinned buffers anyway, and
    the runs of equal rows are found during that pass: one row per run is
    copied and tested.  Also timed: the same rows testing every row, and from
    pinned memory (copied by DMA without a host pass; runs only on request)."""
    import ctypes
    import torch
    from supergwas_b200 import api, build, synth_gpu
    rank, world, local = rank_env()
    torch.cuda.set_device(local)
    build.build_all()
    W = dict(SORTED)
    if args.kmers:
        W["m"] = args.kmers
    n, m, r, mr = W["n"], W["m"], W["r"], W["mean_run"]
    wpk = (n + 63) // 64
    wpk += wpk & 1
    t_gen = time.perf_counter()
    gen = torch.Generator(device="cuda").manual_seed(W["seed"] + 1000 * rank)
    reps = torch.randint(1, 2 * mr, (int(1.2 * m / mr) + 64,), device="cuda", generator=gen)
    cum = reps.cumsum(0)
    d = int((cum < m).sum()) + 1
    reps = reps[:d].clone()
    reps[-1] -= int(cum[d - 1]) - m
    Xd = synth_gpu.gen_packed(n, d, W["S"], W["seed"] + 1000 * rank)
    U, y, keep, _ = synth_gpu.structure_and_phenotype(Xd, n, r, W["n_causal"], W["missing"], W["seed"] + 1000 * rank)
    nbytes = m * wpk * 8
    pageable = np.empty((m, wpk), dtype=np.uint64)
    torch.from_numpy(pageable.view(np.int64)).copy_(torch.repeat_interleave(Xd, reps, dim=0))
    hbuf = api.lib().kg_host_alloc(nbytes)
    if not hbuf:
        raise RuntimeError("kg_host_alloc failed")
    pinned = np.ctypeslib.as_array((ctypes.c_uint64 * (m * wpk)).from_address(hbuf)).reshape(m, wpk)
    pinned[:] = pageable
    del Xd
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen
    g = api.Kgwas(device=local, precision="split", corr_threshold=0.0, log10_thresh=6.0)
    g.set_structure(U, y, keep, n)

    def timed(buf, steps, dedup=None):
        if dedup is not None:
            os.environ["KG_DEDUP"] = dedup
        try:
            for _ in range(args.warmup):
                g.run_host(buf)
            t0 = time.perf_counter()
            tests = 0
            for _ in range(steps):
                res = g.run_host(buf)
                tests += res.n_tested
            return tests / (time.perf_counter() - t0), res, g.last_unique_rows()
        finally:
            os.environ.pop("KG_DEDUP", None)

    with Clocks(local) as ck:
        t0 = time.perf_counter()
        value, res, unique = timed(pageable, args.steps)
        t = time.perf_counter() - t0
    launches = g.last_launch_count()
    short = max(1, min(args.steps, 3))
    v_page_all, r1, _ = timed(pageable, short, "0")
    v_pin_all, r2, _ = timed(pinned, short, "0")
    v_pin_runs, r3, _ = timed(pinned, short, "1")
    for rr in (r1, r2, r3):
        assert rr.n_tested == res.n_tested and np.array_equal(rr.hits, res.hits)
    line = {"metric": "k-mer tests/s end to end (kg_run_host, pageable host rows) on a batch sorted by bit pattern",
            "value": value, "unit": "k-mer tests/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "i8 limbs -> i32 TMEM, f64 epilogue", "data": "synthetic (seeded, generated on device)",
            "config": {"workload": f"sorted: n={n} (5% unphenotyped), {m} k-mers per step from {d} distinct rows "
                                   f"(runs of 1..9, mean {mr}), r={r}+1, 1 phenotype, CORR_THRESHOLD=0",
                       "parallelism": f"weak: {world} GPU(s)"},
            "e2e": {"value": value, "unit": "k-mer tests/s", "h2d_bytes_per_step": unique * wpk * 8 + unique * 4,
                    "d2h_bytes_per_step": 3 * 8 + int(res.hits.shape[0]) * 32},
            "rows_tested_per_step": unique,
            "pageable_every_row": v_page_all, "pinned_every_row": v_pin_all, "pinned_runs": v_pin_runs,
            "host_threads": os.cpu_count(),
            "gpu_launches": launches, "clocks": ck.summary(), "gen_seconds": t_gen}
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.close()
    api.lib().kg_host_free(hbuf)


FILES = dict(n=1000, m=1_000_000, r=16, seed=50)


def files_cols_leg(Xh, n, U, y, keep, local, seed=51):
    """The drop-in comparison at a pipeline-sized batch: the rows Xh (all n
    samples) written as one batch_*/ directory (n column files and a
    kmers.txt.gz of random 31-mers) with samples.txt, phenotype.txt (the
    phenotyped samples) and U.bin, then the reference's kgwas and bin/kgwas
    in COLS mode on the same files (CORR_THRESHOLD=0, files in the page
    cache, all host threads for both).  Wall clock of each process; bin/kgwas
    runs twice and the second run counts (the first loads the CUDA libraries
    from disk)."""
    from supergwas_b200 import build, synth
    from oracle import oracle as O
    m = Xh.shape[0]
    threads = os.cpu_count() or 1
    env = {"CORR_THRESHOLD": "0", "LOAD_THREADS": str(threads), "BLAS_THREADS": str(threads),
           "EMIT_THREADS": str(threads), "KGWAS_DEVICE": str(local)}
    rng = np.random.default_rng(seed)
    with tempfile.TemporaryDirectory() as d:
        t_w = time.perf_counter()
        samples = [f"S{i:05d}" for i in range(n)]
        paths = dict(samples=os.path.join(d, "samples.txt"), pheno=os.path.join(d, "phenotype.txt"),
                     ubin=os.path.join(d, "U.bin"), batch=os.path.join(d, "batch_000"))
        synth.write_samples(paths["samples"], samples)
        synth.write_pheno(paths["pheno"], [samples[i] for i in keep], y)
        synth.write_ubin(paths["ubin"], U)
        synth.write_batch(paths["batch"], Xh, n, synth.random_kmers_text(rng, m))
        t_w = time.perf_counter() - t_w
        args = [paths["samples"], paths["pheno"], paths["batch"], paths["ubin"]]

        def run(tag, reference):
            out = os.path.join(d, tag, "batch_000.tsv")
            os.makedirs(os.path.dirname(out), exist_ok=True)
            t0 = time.perf_counter()
            if reference:
                r = O.run_reference([*args, out, "6", "--mode", "cols"], env)
            else:
                r = subprocess.run([build.CLI, *args, out, "6", "--mode", "cols"], env=dict(os.environ, **env),
                                   capture_output=True, text=True)
            dt = time.perf_counter() - t0
            if r.returncode != 0:
                raise RuntimeError(f"{tag}: {r.stderr[-500:]}")
            return open(out + ".count").read(), dt, r.stderr

        run("warm", False)
        c_ours, s_ours, err_ours = run("ours", False)
        c_ref, s_ref, _ = run("ref", True) if reference_binary() else (None, None, None)
    tested = int(c_ours.split("\t")[1])
    # the program's own milestones ("[TIME] <what> <seconds> s", from its start)
    marks = {}
    for line in (err_ours or "").splitlines():
        if line.startswith("[TIME] ") and line.endswith(" s"):
            what, _, sec = line[7:-2].rpartition(" ")
            try:
                marks[what] = float(sec)
            except ValueError:
                pass
    return {"kmers": m, "ours_seconds": s_ours, "ours_tests_per_s": tested / s_ours, "ours_milestones_s": marks,
            "reference_seconds": s_ref, "reference_tests_per_s": tested / s_ref if s_ref else None,
            "speedup": s_ref / s_ours if s_ref else None, "count_lines_identical": c_ours == c_ref,
            "write_seconds": t_w, "threads": threads,
            "workload": f"first {m} k-mers of the bench batch as pipeline files: {n} column files, kmers.txt.gz, "
                        "COLS mode, CORR_THRESHOLD=0, files in the page cache"}


def run_files(args):
    """End to end through the programs, as the pipeline calls them: the
    reference's kgwas and this package's bin/kgwas on the same files of one
    batch (n=1000, r=16+1, 1M k-mers, CORR_THRESHOLD=0, files in the page
    cache): COLS mode on the batch_*/ column files (first read, then with the
    packed .kbits sidecar) and ROWS mode on a kmer<TAB>bitstring file.  Wall
    clock of each process, one run each (a run is seconds long)."""
    import subprocess
    from supergwas_b200 import build, synth
    from oracle import oracle as O
    rank, world, local = rank_env()
    if rank != 0:
        return
    build.build_all()
    F = dict(FILES)
    if args.kmers:
        F["m"] = args.kmers
    n, m, r = F["n"], F["m"], F["r"]
    threads = os.cpu_count() or 1
    env = {"CORR_THRESHOLD": "0", "LOAD_THREADS": str(threads), "BLAS_THREADS": str(threads),
           "EMIT_THREADS": str(threads), "KGWAS_DEVICE": str(local)}
    t_gen = time.perf_counter()
    with tempfile.TemporaryDirectory() as d:
        ds = synth.simulate(n=n, m=m, S=WORKLOAD["S"], r=r, n_causal=50, missing=WORKLOAD["missing"],
                            seed=F["seed"], structure_kmers=min(50_000, m))
        paths = synth.write_dataset(d, ds)
        rows = os.path.join(d, "rows.tsv")
        synth.write_rows_file(rows, ds.packed_all, ds.n_all, ds.kmers)
        for root, _, files in os.walk(d):  # into the page cache
            for f in files:
                with open(os.path.join(root, f), "rb") as fh:
                    while fh.read(1 << 24):
                        pass
        t_gen = time.perf_counter() - t_gen

        def run(exe_args, extra, tag, reference=False):
            out = os.path.join(d, tag, "batch_000.tsv")
            os.makedirs(os.path.dirname(out), exist_ok=True)
            e = dict(env, **extra)
            t0 = time.perf_counter()
            if reference:
                res = O.run_reference([*exe_args[:4], out, "6", *exe_args[4:]], e)
            else:
                res = subprocess.run([build.CLI, *exe_args[:4], out, "6", *exe_args[4:]],
                                     env=dict(os.environ, **e), capture_output=True, text=True)
            dt = time.perf_counter() - t0
            if res.returncode != 0:
                raise RuntimeError(f"{tag}: {res.stderr[-500:]}")
            count = open(out + ".count").read()
            nrows = sum(1 for _ in open(out))
            phases[tag] = [ln for ln in res.stderr.splitlines() if ln.startswith("[TIME]")]
            return int(count.split("\t")[1]), dt, count, nrows

        phases = {}
        base = [paths["samples"], paths["pheno"]]
        cols = [*base, paths["batch"], paths["ubin"], "--mode", "cols"]
        rowsa = [*base, rows, paths["ubin"], "--mode", "rows"]
        run(cols, {}, "warm")  # GPU context and library load once
        t_c, s_c, c_c, h_c = run(cols, {}, "cols")
        run(cols, {"KGWAS_KBITS": "1"}, "kb_write")
        t_k, s_k, c_k, h_k = run(cols, {"KGWAS_KBITS": "1"}, "kb_read")
        t_r, s_r, c_r, h_r = run(rowsa, {}, "rows")
        t_rc, s_rc, c_rc, h_rc = run(cols, {}, "ref_cols", reference=True)
        t_rr, s_rr, c_rr, h_rr = run(rowsa, {}, "ref_rows", reference=True)
    same = c_c == c_k == c_rc and c_r == c_rr
    line = {"metric": "k-mer tests/s end to end through the kgwas program (files in, files out)",
            "value": t_c / s_c, "unit": "k-mer tests/s", "n_gpus": 1, "steps": 1, "warmup": 1,
            "ms_per_step": 1e3 * s_c, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "i8 limbs -> i32 TMEM, f64 epilogue", "data": "synthetic (seeded), written as pipeline files",
            "config": {"workload": f"files: n={n} (5% unphenotyped), {m} k-mers in one batch_*/ directory "
                                   f"({n} column files) and one ROWS file, r={r}+1, CORR_THRESHOLD=0, "
                                   f"files in the page cache, {threads} host threads for both programs",
                       "parallelism": "1 GPU + host threads"},
            "e2e": {"value": t_c / s_c, "unit": "k-mer tests/s", "h2d_bytes_per_step": m * 128,
                    "d2h_bytes_per_step": None},
            "cols_seconds": s_c, "cols_kbits_seconds": s_k, "rows_seconds": s_r,
            "cols_kbits": t_k / s_k, "rows": t_r / s_r,
            "reference_cols": t_rc / s_rc, "reference_cols_seconds": s_rc,
            "reference_rows": t_rr / s_rr, "reference_rows_seconds": s_rr,
            "count_lines_identical": same, "emitted_rows": {"cols": h_c, "reference_cols": h_rc, "rows": h_r,
                                                            "reference_rows": h_rr},
            "phases": {k: v for k, v in phases.items() if k in ("cols", "kb_read", "rows")},
            "gpu_launches": None, "gen_seconds": t_gen}
    print(json.dumps(line), flush=True)


PAIRS = dict(n=1000, N=50_000, S=8, r=16, seed=48, cpu_N=3000)


def reference_pairs_run(X, n, U, y, N_cpu, threads, workdir):
    """The reference kgwas_2d on the first N_cpu k-mers: index built by the
    reference's build_index from a .2d.tsv of bitstrings; returns (pairs scored
    by the oracle's rules, seconds of the kgwas_2d process)."""
    from supergwas_b200 import synth
    from oracle import oracle as O
    rng = np.random.default_rng(7)
    kmers = synth.random_kmers(rng, N_cpu, 31)
    x = synth.unpack_rows(X[:N_cpu], n)
    tsv = os.path.join(workdir, "hits.2d.tsv")
    with open(tsv, "w") as f:
        for j in range(N_cpu):
            f.write(kmers[j] + "\t" + "".join("1" if v else "0" for v in x[j]) + "\t0\t1\n")
    idx = os.path.join(workdir, "index")
    r = O.run_reference_tool("build_index", [tsv, idx, "--shards", "4"])
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-500:])
    ids = [f"s{i}" for i in range(n)]
    synth.write_samples(os.path.join(workdir, "samples.txt"), ids)
    synth.write_pheno(os.path.join(workdir, "pheno.txt"), ids, y)
    synth.write_ubin(os.path.join(workdir, "U.bin"), U)
    t0 = time.perf_counter()
    r = O.run_reference_tool("kgwas_2d", [os.path.join(workdir, "samples.txt"), os.path.join(workdir, "pheno.txt"),
                                          os.path.join(workdir, "U.bin"), idx, os.path.join(workdir, "out"), "6"],
                             {"BLAS_THREADS": threads, "EMIT_THREADS": threads})
    dt = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-500:])
    return N_cpu * (N_cpu - 1) // 2, dt


def run_pairs(args):
    """2-D pair test (kgwas_2d): every pair of N k-mers, n=1000, r=16+1,
    through kg_pairs_run_host (rows from host memory, pairs back sorted)."""
    import torch
    from supergwas_b200 import api, build, synth_gpu
    rank, world, local = rank_env()
    torch.cuda.set_device(local)
    build.build_all()
    W = dict(PAIRS)
    if args.kmers:
        W["N"] = args.kmers
    n, N, r = W["n"], W["N"], W["r"]
    Xd = synth_gpu.gen_packed(n, N, W["S"], W["seed"] + 1000 * rank)
    U, _, keep, _ = synth_gpu.structure_and_phenotype(Xd, n, r, 1, 0.0, W["seed"])
    X = Xd.cpu().numpy().view(np.uint64)
    from supergwas_b200 import synth
    x = synth.unpack_rows(X[:64], n).astype(np.float64)
    rng = np.random.default_rng(W["seed"])
    y = 1.5 * x[3] * x[17] - 1.0 * x[5] * x[9] + rng.standard_normal(n)
    g = api.Kgwas(device=local, log10_thresh=6.0)
    g.set_structure(U, y)
    for _ in range(args.warmup):
        res, n_eval = g.run_pairs_host(X)
    torch.cuda.synchronize()
    times = []
    with Clocks(local) as ck:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            res, n_eval = g.run_pairs_host(X)
            times.append(time.perf_counter() - t0)
    t = sum(times) / len(times)
    value = n_eval / t * world
    hbm, bf16, peak_src = measured_peaks()
    kpad = ((n + 255) // 256) * 256
    ops = 2.0 * kpad * 64 * (N * (N - 1) / 2)
    cpu = None
    if not args.no_cpu and reference_binary() and rank == 0:
        threads = os.cpu_count() or 1
        with tempfile.TemporaryDirectory() as d:
            npairs, dt = reference_pairs_run(X, n, U, y, W["cpu_N"], threads, d)
        cpu = {"value": npairs / dt, "unit": "pair tests/s", "cores": threads, "kind": "reference",
               "sample": f"reference kgwas_2d on {W['cpu_N']} k-mers ({npairs} pairs), n={n}, r={r}+1, "
                         "wall clock incl. its index load"}
    line = {"metric": f"pair tests/s (2-D pair test, n={n}, r={r}+1, {N} k-mers)", "value": value,
            "unit": "pair tests/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "i8 limbs -> i32 TMEM, f64 epilogue", "data": "synthetic (seeded, generated on device)",
            "config": {"workload": f"pairs: n={n}, N={N} k-mers ({N * (N - 1) // 2} pairs), r={r}+1, "
                                   "log10_thresh=6", "parallelism": f"weak: {world} GPU(s)"},
            "pairs_scored": n_eval, "pairs_emitted": int(res.shape[0]),
            "roofline": {"bound": "tensor", "achieved": ops / t / 1e12, "peak": 2 * bf16, "unit": "TOP/s int8",
                         "frac": ops / t / 1e12 / (2 * bf16), "peak_source": peak_src + " (2x bf16 burst)",
                         "traffic": None},
            "e2e": {"value": value, "unit": "pair tests/s", "h2d_bytes_per_step": int(X.nbytes),
                    "d2h_bytes_per_step": int(res.shape[0]) * 40 + 32, "api": "kg_pairs_run_host"},
            "gpu_launches": 2 * args.steps, "clocks": ck.summary(), "cpu_baseline": cpu}
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.close()


def run_profile(args):
    """A short launch sequence for profilers, no timing rules: a seeded batch
    of --kmers rows generated on the device, the structure (or --pheno
    phenotypes for ``multi``), then --launches launches of the chosen kernel
    on its own stream, so that `ncu -k regex:<kernel> -s 1 -c 1..3` captures a
    few launches of a batch larger than L2 without the rest of the bench.
    ``pairs`` tests every pair of the first --kmers rows (a few thousand)."""
    import torch
    from supergwas_b200 import api, build, synth_gpu
    rank, world, local = rank_env()
    torch.cuda.set_device(local)
    build.build_all()
    kern = args.kernel
    if kern in ("ts", "ss"):
        os.environ["KG_KERNEL"] = kern
    n, r, m = args.n, args.r, args.kmers or 4_000_000
    X = synth_gpu.gen_packed(n, m, 8, 44)
    wpk = X.shape[1]
    st = torch.cuda.Stream()  # a real stream handle (NULL would select the context's own stream)
    times = []
    if kern == "multi":
        phenos = synth_gpu.batched_phenotypes(X, n, args.pheno, r, 46)
        g = api.Kgwas(device=local, precision="split", corr_threshold=0.0, log10_thresh=6.0)
        g.set_phenotypes(phenos, n)
        for _ in range(2):  # autotuner, graph capture
            g.launch_multi_device(X.data_ptr(), m, wpk, None, st.cuda_stream)
            g.fetch_multi()
        for _ in range(args.launches):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            g.launch_multi_device(X.data_ptr(), m, wpk, None, st.cuda_stream)
            e1.record(st)
            tested, hits = g.fetch_multi()
            times.append(e0.elapsed_time(e1))
        desc = f"shape={g.multi_shape()} tests={int(tested.sum())} hits={hits.shape[0]}"
        units = m * args.pheno
    elif kern == "pairs":
        U, y, keep, _ = synth_gpu.structure_and_phenotype(X, n, r, 50, 0.0, 44)
        Xh = X.cpu().numpy().view(np.uint64)
        g = api.Kgwas(device=local, precision="split", log10_thresh=6.0)
        g.set_structure(U, y)
        g.run_pairs_host(Xh)
        for _ in range(args.launches):
            t0 = time.perf_counter()
            res, n_eval = g.run_pairs_host(Xh)
            times.append(1e3 * (time.perf_counter() - t0))
        desc = f"pairs_scored={n_eval} emitted={res.shape[0]}"
        units = m * (m - 1) // 2
    else:
        U, y, keep, _ = synth_gpu.structure_and_phenotype(X, n, r, 50, 0.05, 44)
        g = api.Kgwas(device=local, precision="fp64" if kern == "fp64" else "split", corr_threshold=0.0,
                      log10_thresh=6.0)
        g.set_structure(U, y, keep, n)
        g.launch_device(X.data_ptr(), m, wpk, st.cuda_stream)  # warm-up
        g.fetch()
        torch.cuda.synchronize()
        for _ in range(args.launches):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            g.launch_device(X.data_ptr(), m, wpk, st.cuda_stream)
            e1.record(st)
            res = g.fetch()
            times.append(e0.elapsed_time(e1))
        desc = f"kernel={g.last_kernel()} tested={res.n_tested} hits={res.hits.shape[0]}"
        units = m
    times.sort()
    med = times[len(times) // 2]
    print(f"profile {kern} n={n} r={r} kmers={m} {desc} ms_per_launch={med:.3f} units_per_s={units / med * 1e3:.4g}",
          flush=True)
    g.close()


def run_mma_rate(args):
    """Back-to-back tcgen05.mma kind::i8 rates per SM (libkgwas_bench.so):
    the ceiling of the association kernels' contractions.  One JSON line; the
    rows give cycles per MMA of one issuing stream and int8 MACs per SM-cycle
    against the 8192 of the hardware."""
    import ctypes
    import torch
    from supergwas_b200 import build
    rank, world, local = rank_env()
    torch.cuda.set_device(local)
    build.build_all()
    L = ctypes.CDLL(build.BENCH_LIB)
    L.kg_bench_mma_rate.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_ulonglong)]
    names = {0: "one CTA per SM", 1: "two CTAs per SM", 2: "CTA pair, cta_group::2 (M=256)",
             3: "one CTA per SM, 4 warps storing to TMEM (one wait per store)",
             4: "one CTA per SM, 4 warps loading from TMEM",
             5: "one CTA per SM, 4 warps storing to TMEM (4 stores per wait)",
             6: "no MMAs, 4 warps storing to TMEM (4 stores per wait)",
             7: "one CTA per SM, 4 warps reading shared memory", 8: "no MMAs, 4 warps reading shared memory",
             9: "one issuer walking A slots and the B image, a commit every 16 MMAs",
             10: "one issuer walking A slots and the B image, a commit every 4 MMAs",
             11: "ring of 3 A slots: 16 MMAs per use, waits for the commit of the slot's previous use",
             12: "ring of 2 A slots: 16 MMAs per use, waits for the commit of the slot's previous use",
             13: "ring of 3 A slots, the wait spinning on mbarrier.test_wait",
             14: "ring of 3 A slots, the wait on try_wait with a suspend-time hint",
             15: "ring of 3 A slots, the wait on try_wait without a hint, clock every 1024 tests",
             16: "ring of 3 A slots, the wait spinning on test_wait, bounded by a count (no clock)",
             17: "ring of 3 A slots, the wait on try_wait, bounded by the SM cycle counter",
             18: "one A slot: waits for its own last commit before each use of 16 MMAs",
             19: "ring of 3 A slots, a helper warp waiting for the commits and freeing the slots",
             20: "ring of 3 A slots, unrolled uses with compile-time offsets after a tcgen05 fence",
             21: "no ring: unrolled uses, a try_wait that succeeds at once before each",
             22: "no ring: unrolled uses, two clock reads before each",
             23: "one slot of 16 MMAs, each use after the last one's commit",
             24: "one slot of 1 MMA, each use after the last one's commit",
             25: "commits alone, each after the last one's arrival",
             26: "ring of 3 slots of 16 MMAs, freed through a helper warp",
             27: "ring of 6 slots of 8 MMAs (384 columns)",
             28: "ring of 7 slots of 8 MMAs (448 columns)",
             29: "ring of 7 slots of 8 MMAs, freed through a helper warp",
             30: "ring of 3 slots of 16 MMAs (384 columns)",
             31: "ring of 3 slots of 16 MMAs, no tcgen05 fence after the wait",
             32: "one slot of 16 MMAs, no tcgen05 fence after the wait",
             33: "ring of 3 slots of 16 MMAs, try_wait with a suspend-time hint",
             34: "ring of 3 slots of 16 MMAs, the next slot waited for before the commit",
             35: "ring of 2 slots of 16 MMAs, the next slot waited for before the commit",
             36: "ring of 6 slots of 8 MMAs, the next slot waited for before the commit",
             37: "ring of 3 slots of 16 MMAs, 7 other warps spinning on try_wait",
             38: "ring of 3 slots of 16 MMAs, 7 other warps on try_wait with a suspend-time hint",
             39: "ring of 3 slots of 16 MMAs, 7 other warps sleeping 128 ns between tries",
             40: "kernel-shaped ring (576 threads, issuer warp 17, warp-wide waits)",
             41: "kernel-shaped ring, two accumulators alternating by tile",
             42: "kernel-shaped ring, two accumulators with the epilogue hand-off",
             43: "kernel-shaped ring, slots freed through a group of four warps",
             44: "kernel-shaped ring, accumulator and slot hand-offs",
             45: "as 44, one thread waiting at the top of each use",
             46: "as 45, the accumulator waited for one use earlier",
             47: "as 44, one thread waiting for the next use's barriers after 8 of 16 MMAs",
             48: "as 44, one thread testing after 8 of 16 MMAs, waiting after the commits only on a miss",
             49: "as 43, one thread waiting at the top of each use",
             50: "as 43, one thread waiting after 8 of 16 MMAs",
             51: "as 44, eight other warps doing integer work (2 chains)",
             52: "as 47, eight other warps doing integer work (2 chains)",
             53: "as 44, eight other warps doing integer work (4 chains)",
             54: "as 47, eight other warps doing integer work (4 chains)",
             55: "as 44 with two issuers taking alternate tiles",
             56: "as 55, eight other warps doing integer work (2 chains)",
             57: "as 55, eight other warps doing integer work (4 chains)",
             58: "two issuers, private rings of 3 slots of 8 MMAs",
             59: "two issuers, private rings of 2 slots of 8 MMAs",
             60: "two issuers, private rings of 1 slot of 16 MMAs",
             61: "as 55, eight other warps running FP64 multiply-add chains",
             62: "as 44, eight other warps running FP64 multiply-add chains"}
    table = [(0, 32, 1), (0, 64, 1), (0, 80, 1), (0, 128, 1), (0, 160, 1), (0, 256, 1), (0, 32, 2), (0, 64, 2),
             (0, 64, 4), (1, 64, 1), (2, 64, 1), (2, 128, 1), (2, 160, 1), (2, 256, 1), (3, 64, 1), (3, 128, 1),
             (4, 64, 1), (4, 128, 1), (5, 64, 1), (6, 64, 1), (7, 64, 1), (8, 64, 1), (7, 128, 1),
             (9, 64, 1), (10, 64, 1), (11, 64, 1), (12, 64, 1), (9, 80, 1), (11, 80, 1), (11, 128, 1),
             (13, 64, 1), (14, 64, 1), (15, 64, 1), (13, 80, 1), (14, 80, 1), (16, 64, 1), (17, 64, 1),
             (16, 128, 1), (17, 128, 1), (18, 64, 1), (18, 128, 1), (19, 64, 1), (19, 128, 1),
             (20, 64, 1), (21, 64, 1), (22, 64, 1), (23, 64, 1), (24, 64, 1), (25, 64, 1), (26, 64, 1),
             (27, 64, 1), (28, 64, 1), (29, 64, 1), (30, 64, 1), (31, 64, 1), (32, 64, 1), (33, 64, 1),
             (34, 64, 1), (35, 64, 1), (36, 64, 1), (37, 64, 1), (38, 64, 1), (39, 64, 1),
             (40, 64, 1), (41, 64, 1), (42, 64, 1), (43, 64, 1), (44, 64, 1), (45, 64, 1), (46, 64, 1),
             (47, 64, 1), (48, 64, 1), (49, 64, 1), (50, 64, 1), (51, 64, 1), (52, 64, 1), (53, 64, 1),
             (54, 64, 1), (55, 64, 1), (56, 64, 1), (57, 64, 1), (58, 64, 1), (59, 64, 1), (60, 64, 1), (61, 64, 1),
             (62, 64, 1)]
    rows = []
    for kind, N, iss in table:
        cyc, side, err = ctypes.c_double(), ctypes.c_double(), ctypes.c_ulonglong()
        rc = L.kg_bench_mma_rate(kind, N, iss, ctypes.byref(cyc), ctypes.byref(side), ctypes.byref(err))
        if rc != 0:
            rows.append({"setup": names[kind], "N": N, "issuers": iss, "rc": rc})
            continue
        M = 256 if kind == 2 else 128
        streams = iss * (2 if kind == 1 else 1)
        per_sm_macs = 128.0 * N * 32 * streams / cyc.value if cyc.value else None  # 128 rows per SM
        row = {"setup": names[kind], "M": M, "N": N, "issuers": iss,
               "cycles_per_mma": cyc.value if cyc.value else None, "int8_macs_per_sm_cycle": per_sm_macs,
               "frac_of_8192": per_sm_macs / 8192.0 if per_sm_macs else None, "wait_errors": err.value}
        if 11 <= kind <= 22 and side.value:
            row["issuer_wait_cycles_avg"] = side.value
        if kind >= 23:
            row["cycles_per_use"] = side.value
        if 3 <= kind <= 8:
            row["side_cycles_per_tmem_op"] = side.value
            if kind in (3, 5, 6):  # 4 warps x 4 KB per store: bytes written per SM-cycle
                row["tmem_store_bytes_per_sm_cycle"] = 4 * 4096 / side.value
            if kind in (7, 8):     # 4 warps x 512 B per ld.shared.v4
                row["smem_read_bytes_per_sm_cycle"] = 4 * 512 / side.value
        rows.append(row)
    # timeline of one issuer on a ring of A slots: how long a use takes to
    # issue (queue back-pressure) and how long the wait for its slot takes
    L.kg_bench_mma_timeline.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong)]
    timelines = []
    forms = {0: "with a disable-output-lane mask", 1: "no mask", 2: "no mask, constant accumulate predicate"}
    for nsl, form in ((1, 0), (2, 0), (3, 0), (1, 1), (3, 1), (1, 2), (3, 2), (4, 0)):
        buf = (ctypes.c_ulonglong * (3 * 256))()
        rc = L.kg_bench_mma_timeline(nsl, form, buf)
        if rc != 0:
            timelines.append({"slots": nsl, "form": form, "rc": rc})
            continue
        t = [buf[i] for i in range(3 * 256)]
        nuse = 4096 // 48 if nsl == 4 else 256
        uses = range(4 if nsl == 4 else 16, nuse)  # steady state
        wait = [t[3 * u + 1] - t[3 * u] for u in uses]
        issue = [t[3 * u + 2] - t[3 * u + 1] for u in uses]
        period = (t[3 * (nuse - 1) + 2] - t[3 * uses[0] + 2]) / (nuse - 1 - uses[0])
        timelines.append({"slots": 1 if nsl == 4 else nsl, "mmas_per_use": 48 if nsl == 4 else 16,
                          "form": forms[form], "cycles_per_use": period,
                          "wait_cycles_avg": sum(wait) / len(wait), "wait_cycles_max": max(wait),
                          "issue_cycles_avg": sum(issue) / len(issue), "issue_cycles_max": max(issue),
                          "first_uses": [[t[3 * u], t[3 * u + 1], t[3 * u + 2]] for u in range(8)]})
    if rank == 0:
        print(json.dumps({"metric": "tcgen05.mma kind::i8 rate per SM (4096 back-to-back MMAs, K=32)",
                          "unit": "int8 MACs per SM-cycle", "rows": rows, "ring_timelines": timelines}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--kmers", type=int, default=0, help="k-mers per GPU (default 2e8)")
    ap.add_argument("--e2e-kmers", type=int, default=50_000_000,
                    help="k-mers per step of the end-to-end leg (pinned host batch; 0 = all)")
    ap.add_argument("--acc-kmers", type=int, default=200_000)
    ap.add_argument("--cpu-kmers", type=int, default=1_000_000)
    ap.add_argument("--ref-kmers", type=int, default=500_000)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--files-kmers", type=int, default=4_000_000,
                    help="k-mers of the pipeline-files leg of the default workload (0 = skip)")
    ap.add_argument("--no-legs", action="store_true",
                    help="default workload only: skip the FP64 n=1000/r=10 and the batched 64-phenotype legs")
    ap.add_argument("--workload", default="precision",
                    choices=["precision", "batched", "streaming", "pairs", "sorted", "files", "profile", "mma-rate"],
                    help="precision: the default single-phenotype workload; batched: 64 phenotypes; "
                         "streaming: 8 phenotypes at n=5000 from pinned host memory; pairs: the 2-D pair test; "
                         "sorted: end to end on a batch with runs of equal rows; "
                         "files: the kgwas program against the reference's on the same files; "
                         "profile: a few launches of one kernel for ncu (--kernel, --launches, --n, --r, --pheno); "
                         "mma-rate: tcgen05 MMA rates per SM")
    ap.add_argument("--kernel", default="ts", choices=["ts", "ss", "fp64", "multi", "pairs"])
    ap.add_argument("--launches", type=int, default=3)
    ap.add_argument("--n", type=int, default=1000, help="samples (profile workload)")
    ap.add_argument("--r", type=int, default=16, help="PCs (profile workload)")
    ap.add_argument("--pheno", type=int, default=16, help="phenotypes (profile workload, multi)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours" and not os.environ.get("KG_BENCH_ALLOW_SHORT"):
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "streaming":
        run_streaming(args)
    elif args.workload == "pairs":
        run_pairs(args)
    elif args.workload == "sorted":
        run_sorted(args)
    elif args.workload == "files":
        run_files(args)
    elif args.workload == "profile":
        run_profile(args)
    elif args.workload == "mma-rate":
        run_mma_rate(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
