#!/usr/bin/env python
"""Benchmark of the TEEbench equi-join hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload rho_c2|rho_c2_sel50|rsm_c2|lrn_c3_z1|radix_c3_z1|...]

One step = one full join (histogram, partitioning passes, build/probe) of a
device-resident synthetic |R| = 2^27, |S| = 2^30 uniform foreign-key workload,
count only (the headline configuration).  On N > 1 GPUs (torchrun) the same
join is spread over the ranks: each holds 1/N of R and S, splits its rows by
key hash, an NCCL all-to-all exchanges the pieces, every rank joins its share
and the counts are all-reduced (strong scaling).  Prints ONE JSON line on
rank 0.

* value      whole-job input M tuples/s = (|R| + |S|) * K / max-over-ranks
             device time (CUDA events on the join stream);
* e2e        the same metric through the drop-in RHO(table_t*, table_t*, int)
             with pinned host buffers: H2D of R and S, the join and the result
             read-back inside each timed step;
* roofline   the dominant kernel (the partitioning scatter) against the
             measured HBM copy bandwidth, from per-phase CUDA events recorded
             by the library on the join stream during the timed steps;
* learned_vs_radix  LRN against RHO with and without its skew split on the
             skewed configuration (2^26 / 2^29 Zipf z = 1), same process,
             clocks sampled;
* cpu_baseline  the reference's own RHO (oracle/_ref, built from the
             reference sources) on this host's cores, on the workload's own
             rows, at the physical and at the logical core count.

--impl reference times that reference RHO on the host cores (all logical
CPUs) on the same configuration, inputs from the reference's own generators;
rank 0 only.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GiB = 1 << 30
WORKLOADS = {
    # name: (algo, log2 |R|, log2 |S|, S generator, selectivity / zipf)
    "rho_c2": ("RHO", 27, 30, "fk", 100),
    "rho_c2_sel50": ("RHO", 27, 30, "fk", 50),
    "rht_c2": ("RHT", 27, 30, "fk", 100),
    "rsm_c2": ("RSM", 27, 30, "fk", 100),
    "psm_c2": ("PSM", 27, 30, "fk", 100),
    "radix_c3_z1": ("RHO", 26, 29, "zipf", 1.0),
    "plain_c3_z1": ("RHO", 26, 29, "zipf", 1.0, {"skew_split": 0}),
    "lrn_c3_z1": ("LRN", 26, 29, "zipf", 1.0),
    "radix_c3_z15": ("RHO", 26, 29, "zipf", 1.5),
    "plain_c3_z15": ("RHO", 26, 29, "zipf", 1.5, {"skew_split": 0}),
    "lrn_c3_z15": ("LRN", 26, 29, "zipf", 1.5),
    "rho_c1": ("RHO", 21, 21, "fk", 100),
    # the headline join spread over the ranks (key-hash split, all-to-all); the
    # default workload takes this path whenever more than one GPU runs
    "rho_c2_sharded": ("RHO", 27, 30, "fk", 100, {"sharded": 1}),
    # 2^28 / 2^31 Zipf z = 1.0, materialised (2^31 output rows, 25.8 GB)
    "lrn_c5_mat": ("LRN", 28, 31, "zipf", 1.0, {"materialize": 1}),
    "radix_c5_mat": ("RHO", 28, 31, "zipf", 1.0, {"materialize": 1}),
}


def wl_spec(wl):
    """(algo, log2 |R|, log2 |S|, S kind, selectivity or z, config overrides)."""
    w = WORKLOADS[wl]
    return tuple(w[:5]) + (dict(w[5]) if len(w) > 5 else {},)


# Batched workload (4096 joins): |R_i| = round(2^U), U ~ Uniform[lo, hi];
# |S_i| = k |R_i|, k ~ UniformInt[1, 16]; R_i a seeded permutation of
# 1..|R_i|; S_i uniform foreign keys, or Zipf z = 1.0 over R_i's keys for a
# seeded 20% of the joins.
BATCH_WORKLOADS = {
    # name: (joins, log2 |R| low, log2 |R| high, Zipf fraction)
    "batch_c4": (4096, 10, 20, 0.2),
}


def batch_sizes(njoins, lo, hi, zipf_frac, seed=4):
    rs = np.random.RandomState(seed)
    nR = np.round(2.0 ** rs.uniform(lo, hi, njoins)).astype(np.int64)
    k = rs.randint(1, 17, njoins)
    zipf = rs.random_sample(njoins) < zipf_frac
    return nR, nR * k, zipf


def make_batch_device(torch, tbg, njoins, lo, hi, zipf_frac, seed=4, stream=0):
    """Generates the batched workload on the device (the library's seeded
    generators) in one buffer.  Returns (buffer, [(dR, nR, dS, nS)], zipf)."""
    nR, nS, zipf = batch_sizes(njoins, lo, hi, zipf_frac, seed)
    total = int(nR.sum() + nS.sum())
    buf = torch.empty(max(total, 1), dtype=torch.int64, device="cuda")
    base = buf.data_ptr()
    joins, off = [], 0
    for i in range(njoins):
        pR = base + 8 * off
        off += int(nR[i])
        pS = base + 8 * off
        off += int(nS[i])
        tbg.gen_pk(pR, int(nR[i]), 1000 + 2 * i + seed * 100003, stream)
        if zipf[i]:
            tbg.gen_zipf(pS, int(nS[i]), int(nR[i]), 1.0, 0, 1001 + 2 * i + seed * 100003, stream)
        else:
            tbg.gen_fk(pS, int(nS[i]), int(nR[i]), 1001 + 2 * i + seed * 100003, stream)
        joins.append((pR, int(nR[i]), pS, int(nS[i])))
    return buf, joins, zipf


def max_over_ranks(x, dist, device):
    """The job's time: the largest of the ranks' device times (every rank
    calls it with its own x; with one process it returns x)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_rows(n, world, rank):
    """[lo, hi): the rows rank owns when n rows are split evenly over world."""
    base, rem = divmod(n, world)
    lo = rank * base + min(rank, rem)
    return lo, lo + base + (1 if rank < rem else 0)


def job_mtuples(world, rows_per_rank, steps, seconds):
    """Whole-job throughput under weak scaling: every rank joins its own
    rows_per_rank input rows per step."""
    return world * rows_per_rank * steps / seconds / 1e6


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index, interval_ms=50):
        self.idx = gpu_index
        self.interval_ms = interval_ms
        self.samples = []
        self._proc = None
        self._th = None

    def _read(self):
        for line in self._proc.stdout:
            line = line.strip()
            if line:
                self.samples.append([x.strip() for x in line.split(",")])

    def __enter__(self):
        # one nvidia-smi child streaming a line every interval_ms
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", str(self.interval_ms)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._th = threading.Thread(target=self._read, daemon=True)
            self._th.start()
            # the timed region starts once nvidia-smi streams (at most 3 s)
            t0 = time.time()
            while not self.samples and time.time() - t0 < 3.0 and self._proc.poll() is None:
                time.sleep(0.01)
        except OSError:
            self._proc = None
        return self

    def __exit__(self, *a):
        if self._proc is not None:
            self._proc.terminate()  # our own child, by its handle
            try:
                self._proc.wait(timeout=10)
            except subprocess.TimeoutExpired:
                self._proc.kill()
            self._th.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 5 + i and s[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


# --------------------------------------------------------------------- CPU
def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def host_cpu():
    """lscpu model, physical cores and logical CPUs this process may use."""
    info = {"model": None, "physical_cores": None, "logical_cpus": host_threads()}
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=30).stdout
        kv = {}
        for line in out.splitlines():
            if ":" in line:
                k, v = line.split(":", 1)
                kv[k.strip()] = v.strip()
        info["model"] = kv.get("Model name")
        cps, sockets = int(kv.get("Core(s) per socket", "0")), int(kv.get("Socket(s)", "0"))
        tpc = int(kv.get("Thread(s) per core", "1") or 1)
        phys = cps * sockets
        if phys:  # cores whose threads this process may use
            info["physical_cores"] = max(1, min(phys, info["logical_cpus"] // max(tpc, 1)))
    except (OSError, ValueError, subprocess.SubprocessError):
        pass
    if not info["physical_cores"]:
        info["physical_cores"] = info["logical_cpus"]
    return info


def reference_inputs(wl, nR, nS, zipf_sample):
    """Inputs of the reference arm, made by the reference's own generators
    (oracle/_ref, App/Lib/generator.cpp): R = create_relation_pk(|R|) with
    seed 11111, S = create_relation_fk(|S|, maxid) or create_relation_fk_sel
    with seed 22222 (native.cpp:63-64, :113), payloads = row index.  Zipf S
    is drawn by inverse CDF over R's keys (rank = key) on a bounded sample
    of zipf_sample rows: the reference's own Zipf generator needs minutes at
    these sizes.  Returns (R, S, description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    _, _, _, kind, param, _ = wl_spec(wl)
    O.ref_seed(11111)
    R = O.ref_gen("pk", nR)
    R["payload"] = np.arange(nR, dtype=np.uint32)
    if kind == "fk":
        O.ref_seed(22222)
        if int(param) == 100:
            S = O.ref_gen("fk", nS, nR)
            how = f"create_relation_fk(|S|={nS}, maxid={nR})"
        else:
            maxid = nR * 100 // int(param)
            S = O.ref_gen("fk_sel", nS, maxid)
            how = f"create_relation_fk_sel(|S|={nS}, maxid={maxid})"
    else:
        n = min(nS, zipf_sample)
        rng = np.random.default_rng(22222)
        w = 1.0 / np.arange(1, nR + 1, dtype=np.float64) ** float(param)
        cdf = np.cumsum(w)
        cdf /= cdf[-1]
        S = np.zeros(n, dtype=R.dtype)
        S["key"] = (np.searchsorted(cdf, rng.random(n)) + 1).astype(np.uint32)
        how = f"Zipf z={param} over R's keys by inverse CDF, a sample of {n} rows"
    S["payload"] = np.arange(len(S), dtype=np.uint32)
    return R, S, f"create_relation_pk(|R|={nR}) + " + how + " (the reference's generators, seeds 11111 / 22222)"


def cpu_reference_run(R, S, algo, steps, warmup, threads, materialize=False):
    """Times the reference's own join (oracle/_ref) on the host: warm-up
    calls, then `steps` calls; each call joins fresh private copies of R and
    S (the reference clobbers its inputs), timed by its own Total Runtime.
    Returns the median seconds per join, every timing and the last count."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    times, count = [], None
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        c, _, rt_us = O.ref_join(algo, R, S, nthreads=threads, materialize=materialize)
        wall = time.perf_counter() - t0
        if i >= warmup:
            times.append(rt_us * 1e-6 if rt_us and rt_us > 0 else wall)
        count = c
    return statistics.median(times), times, count


def reference_available():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O.ref() is not None


def cpu_baseline_leg(R, S, algo, materialize, reps=3):
    """The reference's join on this host's cores at the physical core count
    and at the logical CPU count, median of `reps` calls each (plus one
    warm-up).  R and S are the workload's own rows (or a stated sample)."""
    cpu = host_cpu()
    runs = {}
    for label, th in (("physical", cpu["physical_cores"]), ("logical", cpu["logical_cpus"])):
        if label == "logical" and th == cpu["physical_cores"] and "physical" in runs:
            runs[label] = dict(runs["physical"])
            continue
        t, ts, c = cpu_reference_run(R, S, algo, reps, 1, th, materialize)
        runs[label] = {"threads": th, "median_s": t, "runs_s": ts, "count": c,
                       "Mtuples_s": (len(R) + len(S)) / t / 1e6}
    best = max(runs.values(), key=lambda r: r["Mtuples_s"])
    return best, runs, cpu


def reference_main(args, metric, base_config, world, mat, scaling="weak"):
    """The reference arm: the reference's own join (oracle/_ref, compiled from
    its sources) timed on this host's cores, all logical CPUs, on the
    workload's configuration; `warmup` untimed calls, then `steps` timed ones
    (each on fresh copies of R and S), the median of its Total Runtime."""
    if not reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libtbref.so not built"}))
        return 0
    algo = wl_spec(args.workload)[0]
    ref_algo = algo if algo in ("RHO", "RHT", "RSM", "PSM") else "RHO"
    nR, nS = base_config["nR"], base_config["nS"]
    t0 = time.perf_counter()
    R, S, how = reference_inputs(args.workload, nR, nS, 1 << 27)
    if mat and len(S) > (1 << 26):  # one malloc'd list node per output row: keep it bounded
        S = S[: 1 << 26].copy()
        how += f"; materialising: the first {len(S)} S rows"
    gen_s = time.perf_counter() - t0
    cpu = host_cpu()
    threads = cpu["logical_cpus"]
    steps, warm = max(1, args.steps), max(0, args.warmup)
    t, ts, count = cpu_reference_run(R, S, ref_algo, steps, warm, threads, mat)
    value = (len(R) + len(S)) / t / 1e6
    sample = (f"reference {ref_algo}{'_mat' if mat else ''} (oracle/_ref, built from the reference's sources) on "
              f"|R|={len(R)}, |S|={len(S)}: {how}; {threads} threads (all logical CPUs of "
              f"{cpu['model']}, {cpu['physical_cores']} physical cores); median of {steps} calls after {warm} "
              f"warm-up calls, its own Total Runtime (us)")
    config = dict(base_config)
    if len(S) != nS:
        config["sampled_nS"] = len(S)
    line = {"impl": "reference", "metric": metric, "value": value, "unit": "Mtuples/s", "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": scaling, "vs_baseline": None, "dtype": "u32", "data": "synthetic", "config": config,
            "matches": int(count),
            "cpu_baseline": {"value": value, "unit": "Mtuples/s", "cores": threads, "kind": "reference",
                             "sample": sample, "host": cpu, "runs_ms": [x * 1e3 for x in ts],
                             "input_generation_s": gen_s},
            "e2e": {"value": value, "unit": "Mtuples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------------- GPU
# Learned vs radix partitioning on the skewed configuration: |R| = 2^26
# unique keys, |S| = 2^29 Zipf over R's keys, hot keys at small ranks (rank =
# key) or scattered over the key range by a seeded permutation.
LVR_CASES = [("z1", 1.0, 0), ("z1_scattered", 1.0, 1)]
LVR_VARIANTS = [("lrn", "LRN", {}), ("rho_skew_split", "RHO", {}), ("rho_plain", "RHO", {"skew_split": 0})]


def learned_vs_radix(tbg, torch, dev, stream, steps, warmup, lr=26, ls=29, cases=LVR_CASES):
    """Times LRN, RHO with its S-side skew split (the library default) and RHO
    without it (the reference's behaviour) on the same device-resident
    inputs, CUDA events on the join stream, the clock sampler running."""
    sh = stream.cuda_stream
    nR, nS = 1 << lr, 1 << ls
    tR = torch.empty(nR, dtype=torch.int64, device=dev)
    tS = torch.empty(nS, dtype=torch.int64, device=dev)
    pR, pS = tR.data_ptr(), tS.data_ptr()
    tbg.gen_pk(pR, nR, 11111, sh)
    out = {"workload": f"|R|=2^{lr} unique keys, |S|=2^{ls} Zipf over R's keys (rank = key, or ranks scattered "
                       f"over the keys by a seeded permutation), count only",
           "steps": steps, "warmup": warmup, "timing": "CUDA events around the timed joins on their stream",
           "cases": {}}
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    for label, z, scatter in cases:
        tbg.gen_zipf(pS, nS, nR, z, scatter, 22222, sh)
        stream.synchronize()
        entry = {"z": z, "scattered": bool(scatter)}
        with ClockSampler(dev.index) as clk:
            for name, algo, over in LVR_VARIANTS:
                cfg = tbg.config(algo, **over)
                for _ in range(warmup):
                    _, m, st = tbg.join_device(cfg, pR, nR, pS, nS, stream=sh)
                torch.cuda.synchronize()
                ev0.record(stream)
                for _ in range(steps):
                    _, m, st = tbg.join_device(cfg, pR, nR, pS, nS, stream=sh)
                ev1.record(stream)
                torch.cuda.synchronize()
                ms = ev0.elapsed_time(ev1) / steps
                part_rows = nS - int(st.heavy_rows_S)
                mean_s = part_rows / st.partitions if st.partitions else 0.0
                entry[name] = {"ms": ms, "Mtuples_s": (nR + nS) / ms / 1e3, "matches": int(m),
                               "radix_bits": st.radix_bits, "max_part_S": int(st.max_part_S),
                               "mean_part_S": mean_s,
                               "max_over_mean_S": int(st.max_part_S) / mean_s if mean_s else None,
                               "used_fallback": st.used_fallback, "heavy_keys": int(st.heavy_keys),
                               "heavy_rows_S": int(st.heavy_rows_S), "train_steps": st.train_steps,
                               "train_loss": st.train_loss}
        entry["clocks"] = clk.summary()
        counts = {entry[n]["matches"] for n, _, _ in LVR_VARIANTS}
        entry["identical_counts"] = len(counts) == 1 and counts == {nS}
        entry["lrn_speedup_vs_plain"] = entry["rho_plain"]["ms"] / entry["lrn"]["ms"]
        entry["lrn_speedup_vs_skew_split"] = entry["rho_skew_split"]["ms"] / entry["lrn"]["ms"]
        out["cases"][label] = entry
    del tR, tS
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rho_c2", choices=sorted(WORKLOADS) + sorted(BATCH_WORKLOADS))
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-pageable-e2e", action="store_true",
                    help="skip the drop-in's end-to-end run on pageable host memory")
    ap.add_argument("--no-learned-block", action="store_true",
                    help="skip the learned-vs-radix comparison the headline line carries")
    ap.add_argument("--cpu-sample-log2", type=int, default=30, help="S rows (log2) of the CPU baseline's sample")
    # smaller cases of the same workload (profiling captures); never the reported configuration
    ap.add_argument("--log2-r", type=int, default=None)
    ap.add_argument("--log2-s", type=int, default=None)
    ap.add_argument("--joins", type=int, default=None)
    ap.add_argument("--log2-lo", type=int, default=None)
    ap.add_argument("--log2-hi", type=int, default=None)
    ap.add_argument("--no-autotune", action="store_true", help="batch: built-in heuristic plan")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload in BATCH_WORKLOADS:
        return batch_main(args, rank, world, local)
    if wl_spec(args.workload)[5].get("sharded") or (args.workload == "rho_c2" and world > 1):
        # the headline join on several GPUs: one join spread over the ranks
        return sharded_main(args, rank, world, local)
    algo, lr, ls, kind, param, over = wl_spec(args.workload)
    lr = args.log2_r if args.log2_r is not None else lr
    ls = args.log2_s if args.log2_s is not None else ls
    nR, nS = 1 << lr, 1 << ls
    mat = bool(over.get("materialize"))
    workload_name = f"{algo} |R|=2^{lr} |S|=2^{ls} " + (
        f"uniform FK {param}% selectivity" if kind == "fk" else f"Zipf z={param}") + (
        ", materialised (key, R payload, S payload) rows" if mat else ", count only") + (
        "".join(f", {k}={v}" for k, v in over.items() if k != "materialize"))
    metric = ("input Mtuples/s (|R|+|S|)/t, " + ("materialising" if mat else "count-only") +
              " equi-join, bit-exact")

    base_config = {"workload": workload_name, "global_batch": world * (nR + nS), "nR": nR, "nS": nS}
    # the headline is one join (spread over the ranks when N > 1); the other
    # workloads run one independent join per rank
    scaling = "strong" if args.workload == "rho_c2" else "weak"
    if args.impl == "reference":
        if rank != 0:
            return 0
        return reference_main(args, metric, base_config, world, mat, scaling=scaling)

    import torch
    import torch.distributed as dist
    tbg = importlib.import_module("tee-bench_b200")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:  # the rank's GPU is current before NCCL binds to it
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300), device_id=dev)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream

    # device-resident inputs (generated on the GPU; S differs per rank)
    tR = torch.empty(nR, dtype=torch.int64, device=dev)
    tS = torch.empty(nS, dtype=torch.int64, device=dev)
    pR, pS = tR.data_ptr(), tS.data_ptr()
    with torch.cuda.stream(stream):
        tbg.gen_pk(pR, nR, 11111, sh)
        if kind == "fk":
            tbg.gen_fk(pS, nS, nR * 100 // int(param), 22222 + rank, sh)
        else:
            tbg.gen_zipf(pS, nS, nR, float(param), 0, 22222 + rank, sh)
    stream.synchronize()
    host_rows = None  # the workload's rows for the CPU baseline (rank 0, one GPU)
    if rank == 0 and world == 1 and not args.no_cpu_baseline and reference_available():
        nS_cpu = min(nS, 1 << (26 if mat else args.cpu_sample_log2))
        host_rows = (host_copy_rows(tR, nR), host_copy_rows(tS, nS_cpu), nS)

    cfg = tbg.config(algo, **over)
    cfg.timing = 1
    expect = None
    if kind == "fk" or kind == "zipf":
        expect = nS * nR // (nR * 100 // int(param)) if kind == "fk" else nS
    pO, cap = 0, 0
    if mat:  # every S key is one of R's unique keys: exactly |S| output rows
        cap = nS
        tO = torch.empty(3 * cap, dtype=torch.int32, device=dev)
        pO = tO.data_ptr()
    # warm-up
    for _ in range(args.warmup):
        _, m, st = tbg.join_device(cfg, pR, nR, pS, nS, pO, cap, stream=sh)
    if expect is not None and m != expect:
        raise SystemExit(f"wrong match count {m} != {expect}")

    # timed region: K joins back to back on the stream, events around them
    phase = {"ms_hist": 0.0, "ms_pass1": 0.0, "ms_pass2": 0.0, "ms_join": 0.0, "ms_learn": 0.0}
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = tbg.kernel_launches()
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            _, m, st = tbg.join_device(cfg, pR, nR, pS, nS, pO, cap, stream=sh)
            for k in phase:
                phase[k] += getattr(st, k)
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = tbg.kernel_launches() - l0
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms, dist, dev)
    if world > 1:
        dist.barrier()
    value = job_mtuples(world, nR + nS, args.steps, ms / 1e3)

    # e2e through the drop-in entry point with pinned host buffers
    e2e = None
    if args.e2e_steps > 0 and mat:
        # the drop-in would build 2^31 list nodes on the host; the device API
        # with every step's inputs copied in and its rows copied out stands in
        hR = torch.empty(nR, dtype=torch.int64, pin_memory=True)
        hS = torch.empty(nS, dtype=torch.int64, pin_memory=True)
        hO = torch.empty(3 * cap, dtype=torch.int32, pin_memory=True)
        hR.copy_(tR)
        hS.copy_(tS)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.e2e_steps):
            with torch.cuda.stream(stream):
                tR.copy_(hR, non_blocking=True)
                tS.copy_(hS, non_blocking=True)
            _, cnt, _ = tbg.join_device(cfg, pR, nR, pS, nS, pO, cap, stream=sh)
            with torch.cuda.stream(stream):
                hO[: 3 * cnt].copy_(tO[: 3 * cnt], non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        el = e0.elapsed_time(e1) / 1e3
        el = max_over_ranks(el, dist, dev)
        e2e = {"value": job_mtuples(world, nR + nS, args.e2e_steps, el), "unit": "Mtuples/s",
               "h2d_bytes_per_step": (nR + nS) * 8, "d2h_bytes_per_step": int(cnt) * 12,
               "api": "tbg_join_device(materialize) with R, S copied from and the rows copied to pinned host "
                      "memory each step",
               "count": int(cnt)}
        del hR, hS, hO
    elif args.e2e_steps > 0:
        hR = torch.empty(nR, dtype=torch.int64, pin_memory=True)
        hS = torch.empty(nS, dtype=torch.int64, pin_memory=True)
        hR.copy_(tR)
        hS.copy_(tS)
        del tR, tS
        torch.cuda.empty_cache()
        import ctypes as C
        tabR = tbg.Table(C.cast(hR.data_ptr(), C.POINTER(tbg.Row)), nR, 0, 0)
        tabS = tbg.Table(C.cast(hS.data_ptr(), C.POINTER(tbg.Row)), nS, 0, 0)
        fn = getattr(tbg.lib(), algo)
        res = fn(C.byref(tabR), C.byref(tabS), 1)  # warm-up (allocations)
        tbg.lib().tbg_result_free(res)
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            res = fn(C.byref(tabR), C.byref(tabS), 1)
            cnt = res.contents.totalresults
            tbg.lib().tbg_result_free(res)
        el = max_over_ranks(time.perf_counter() - t0, dist, dev)
        h2d, d2h = tbg.last_transfer_bytes()
        e2e = {"value": job_mtuples(world, nR + nS, args.e2e_steps, el), "unit": "Mtuples/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "api": f"{algo}(table_t*, table_t*, int) drop-in, pinned host buffers",
               "count": int(cnt)}
        if not args.no_pageable_e2e:
            # the same call on ordinary (pageable) host memory, as the
            # reference's driver allocates its tables (generator.cpp:22)
            pR = np.empty(nR, dtype=np.int64)
            pS = np.empty(nS, dtype=np.int64)
            pR[:] = hR.numpy()
            pS[:] = hS.numpy()
            del hR, hS
            tabR = tbg.Table(C.cast(pR.ctypes.data, C.POINTER(tbg.Row)), nR, 0, 0)
            tabS = tbg.Table(C.cast(pS.ctypes.data, C.POINTER(tbg.Row)), nS, 0, 0)
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            for _ in range(args.e2e_steps):
                res = fn(C.byref(tabR), C.byref(tabS), 1)
                cntp = res.contents.totalresults
                tbg.lib().tbg_result_free(res)
            el = max_over_ranks(time.perf_counter() - t0, dist, dev)
            e2e["pageable"] = {"value": job_mtuples(world, nR + nS, args.e2e_steps, el), "unit": "Mtuples/s",
                               "api": f"{algo}(table_t*, table_t*, int) drop-in, pageable (malloc'd) host buffers",
                               "count": int(cntp)}
            del pR, pS

    peak, peak_kind = read_peaks()
    # algorithmic bytes: histogram reads 8 B/row; each partitioning pass
    # reads and writes 8 B/row; build/probe reads 8 B/row
    rows = nR + nS
    K = args.steps
    passes = st.passes or 2
    pipe_ms = ms / K
    peak_source = (f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                   else "fallback 6650 GB/s")
    if algo in ("RHO", "RHT") and not mat:
        scat_ms = (phase["ms_pass1"] + phase["ms_pass2"]) / K
        scat_bytes = 16 * rows * passes
        achieved = scat_bytes / (scat_ms / 1e3) / 1e9 if scat_ms > 0 else None
        traffic, traffic_source = None, None
        tp = os.path.join(ROOT, "profiles", "ncu_traffic.json")
        geom = (f"B{st.radix_bits}_{st.radix_bits // 2}+{st.radix_bits - st.radix_bits // 2}" if passes == 2
                else f"B{st.radix_bits}")
        if os.path.exists(tp):
            with open(tp) as f:
                tt = json.load(f)
            k = tt.get("k_part_pass", {}).get(geom)
            if k:  # DRAM bytes per row moved at this radix geometry, from one ncu capture
                traffic = k["dram_bytes_per_row"] * rows * passes
                traffic_source = f"profiles/ncu_traffic.json [{geom}]: {k['source']}"
        total_bytes = (8 + 16 * passes + 8) * rows
        roofline = {"bound": "hbm",
                    "kernel": f"k_part_pass1 + k_part_pass2 ({passes} partitioning passes over R and S, "
                              f"{2 * passes} launches per join)",
                    "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak if achieved else None, "traffic": traffic,
                    "traffic_source": traffic_source or f"no ncu capture at radix geometry {geom}",
                    "peak_source": peak_source,
                    "algorithmic_bytes_per_row_per_pass": 16,
                    "timing": "library CUDA events on the join stream around each pass, summed over "
                              "the timed steps",
                    "pipeline": {"bytes_per_row": 8 + 16 * passes + 8,
                                 "achieved_gbs": total_bytes / (pipe_ms / 1e3) / 1e9,
                                 "frac": total_bytes / (pipe_ms / 1e3) / 1e9 / peak}}
    else:
        # whole join: LRN's learning and bypass run on two streams and PSM's
        # sort passes are not radix passes, so the pipeline is the unit
        if algo == "PSM" and st.partitions:
            # MSD sort: R's key range, histogram (it checks S's keys against
            # R's range), radix passes by the top bits, one bucket-sort pass
            # (its re-reads of a bucket come from L2), merge
            sp = st.passes
            alg = 8 * nR + (8 + 16 * sp + 8) * rows
            model = (f"PSM (MSD sort): R's key range 8 B per R row + histogram 8 + {sp - 1} radix passes x 16 + "
                     f"bucket sort 16 + merge read 8 B/row")
        elif algo == "PSM":
            sp = st.passes or 4  # key-range read, per pass histogram read + scatter, merge read
            alg = (8 + 24 * sp + 8) * rows
            model = f"PSM: key range 8 + {sp} LSD passes x (histogram 8 + scatter 16) + merge read 8 B/row"
        else:
            heavy = int(st.heavy_rows_S) if algo == "LRN" else 0
            bypass = algo == "LRN" and not st.used_fallback
            part_rows = rows - heavy
            alg = 8 * rows + (16 * passes + 8) * part_rows
            # RSM's per-partition sort reads an S tile twice, the second time from L2
            step = "sort + merge" if algo == "RSM" else "build/probe"
            model = (f"histogram read 8 B/row of R and S; {passes} passes x 16 + {step} 8 B/row of the "
                     f"rows that are partitioned ({part_rows}" + (f", {heavy} heavy S rows joined in the "
                                                                   f"histogram read" if heavy else "") + ")")
            if bypass:  # the kept S rows written compacted, R read once more for its heavy rows
                alg += 8 * (nS - heavy) + 8 * nR
                model += "; compacted S 8 B per kept row; heavy R count 8 B per R row"
        if mat:
            alg += 12 * int(m)
            model += "; 12 B per output row"
        achieved = alg / (pipe_ms / 1e3) / 1e9
        roofline = {"bound": "hbm", "kernel": f"all kernels of one {algo} join (pipeline)",
                    "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": None, "peak_source": peak_source, "algorithmic_bytes_per_join": alg,
                    "bytes_model": model, "timing": "CUDA events around the timed joins on their stream"}
    line = {
        "metric": metric, "value": value, "unit": "Mtuples/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": pipe_ms, "higher_is_better": True,
        "scaling": scaling, "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": workload_name, "global_batch": world * rows, "nR": nR, "nS": nS,
                   "radix_bits": st.radix_bits, "passes": st.passes,
                   "parallelism": ("one join on one GPU (on N > 1 GPUs the same join is spread over the ranks)"
                                   if scaling == "strong" else f"{world} independent joins (one per rank)"),
                   "l2": f"inputs {rows * 8 / 1e9:.1f} GB per step > 126 MB L2; no flush needed",
                   "generator": "on-GPU pk / fk / zipf (generator.cpp semantics)"},
        "gpu_launches": int(launches),
        "e2e": e2e,
        "roofline": roofline,
        "stats": {"used_fallback": st.used_fallback, "heavy_keys": st.heavy_keys,
                  "heavy_rows_S": st.heavy_rows_S, "imbalance": st.imbalance,
                  "max_part_S": st.max_part_S},
        "phases_ms": {k: v / K for k, v in phase.items()},
        "clocks": clocks.summary(),
        "matches": int(m),
    }
    if args.workload == "rho_c2" and world == 1 and not args.no_learned_block and args.log2_r is None:
        line["learned_vs_radix"] = learned_vs_radix(tbg, torch, dev, stream, args.steps, args.warmup)
    if host_rows is not None:
        line["cpu_baseline"] = cpu_baseline_line(host_rows, algo, mat)
    elif rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = {"value": None, "unavailable": "oracle/_ref/libtbref.so not built"}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def host_copy_rows(t, n):
    """The first n rows of a device relation as a host ROW array."""
    return t[:n].cpu().numpy().view(np.dtype([("key", "<u4"), ("payload", "<u4")]))


def cpu_baseline_line(host_rows, algo, mat):
    """cpu_baseline: the reference's own join on the rows the GPU joined (R
    whole, S whole or its stated prefix), at the physical core count and at
    the logical CPU count, median of 3 calls each."""
    R, S, nS_full = host_rows
    ref_algo = algo if algo in ("RHO", "RHT", "RSM", "PSM") else "RHO"
    best, runs, cpu = cpu_baseline_leg(R, S, ref_algo, mat)
    part = "all" if len(S) == nS_full else f"the first {len(S)} of {nS_full}"
    return {"value": best["Mtuples_s"], "unit": "Mtuples/s", "cores": best["threads"], "kind": "reference",
            "sample": f"reference {ref_algo}{'_mat' if mat else ''} (oracle/_ref, built from the reference's sources) "
                      f"on the workload's own rows copied from the GPU: R all {len(R)}, S {part} rows; median of 3 "
                      f"calls after 1 warm-up at {runs['physical']['threads']} threads (physical cores) and at "
                      f"{runs['logical']['threads']} threads (logical CPUs), its own Total Runtime; value = the "
                      f"faster",
            "host": cpu, "runs": runs}


# ------------------------------------------------------------------ sharded
def sharded_main(args, rank, world, local):
    """One |R| = 2^27, |S| = 2^30 uniform FK join spread over the ranks (strong
    scaling): rank r holds rows shard_rows(n, world, r) of R and of S.  Each
    step every rank splits its rows by shard (tbg_shard_split), an all-to-all
    (NCCL over NVLink) moves every piece to its shard's rank, each rank joins
    what it received (tbg_join_device) and the counts are all-reduced.  Every
    rank partitions only its share of R and S.  With one rank it is the
    single-GPU join."""
    algo, lr, ls, kind, param, _ = wl_spec(args.workload)
    lr = args.log2_r if args.log2_r is not None else lr
    ls = args.log2_s if args.log2_s is not None else ls
    nR, nS = 1 << lr, 1 << ls
    rlo, rhi = shard_rows(nR, world, rank)
    slo, shi = shard_rows(nS, world, rank)
    workload_name = (f"{algo} |R|=2^{lr} |S|=2^{ls} uniform FK 100% selectivity, count only, one join spread over "
                     f"the GPUs: each rank holds 1/N of R and S, splits its rows by key hash, all-to-all exchange, "
                     f"local joins, counts all-reduced")
    metric = "input Mtuples/s (|R|+|S|)/t, count-only equi-join, bit-exact"
    if args.impl == "reference":
        if rank != 0:
            return 0
        return reference_main(args, metric, {"workload": workload_name, "global_batch": nR + nS, "nR": nR,
                                             "nS": nS}, world, False, scaling="strong")
    import torch
    import torch.distributed as dist
    tbg = importlib.import_module("tee-bench_b200")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300), device_id=dev)
    # one stream (the current one) orders the splits, the exchange and the joins
    sh = torch.cuda.current_stream().cuda_stream
    full = torch.empty(max(nR, nS), dtype=torch.int64, device=dev)  # every rank draws the same relations
    tbg.gen_pk(full.data_ptr(), nR, 11111, sh)
    tR = full[rlo:rhi].clone()
    tbg.gen_fk(full.data_ptr(), nS, nR, 22222, sh)
    tS = full[slo:shi].clone()
    del full
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    cfg = tbg.config(algo)
    moved = {"rows": 0}

    def split(t, n):
        out = torch.empty_like(t)
        offs = tbg.shard_split(t.data_ptr(), t.numel(), n, out.data_ptr(), sh)
        moved["rows"] += t.numel() - (offs[rank + 1] - offs[rank])
        return out, offs

    def join(Rt, St):
        moved["joined"] = Rt.numel() + St.numel()
        return tbg.join_device(cfg, Rt.data_ptr(), Rt.numel(), St.data_ptr(), St.numel(), stream=sh)[1]

    def new_rows(n):
        return torch.empty(max(n, 1), dtype=torch.int64, device=dev)[:n]

    def step():
        return tbg.distributed_join_count(dist, tR, tS, split, join, new_rows)

    for _ in range(args.warmup):
        m = step()
    if m != nS:
        raise SystemExit(f"wrong match count {m} != {nS}")
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = tbg.kernel_launches()
    moved["rows"] = 0
    with ClockSampler(local) as clocks:
        ev0.record()
        for _ in range(args.steps):
            m = step()
        ev1.record()
        torch.cuda.synchronize()
    launches = tbg.kernel_launches() - l0
    K = args.steps
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist, dev)
    value = (nR + nS) * K / (ms / 1e3) / 1e6
    sent_rows = moved["rows"] / K
    e2e = None
    if args.e2e_steps > 0:  # every step: this rank's rows copied from pinned host memory, the count read back
        hR = torch.empty(tR.numel(), dtype=torch.int64, pin_memory=True)
        hS = torch.empty(tS.numel(), dtype=torch.int64, pin_memory=True)
        hR.copy_(tR)
        hS.copy_(tS)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.e2e_steps):
            tR.copy_(hR, non_blocking=True)
            tS.copy_(hS, non_blocking=True)
            m = step()  # the count is read back to the host
        e1.record()
        torch.cuda.synchronize()
        el = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist, dev)
        e2e = {"value": (nR + nS) * args.e2e_steps / el / 1e6, "unit": "Mtuples/s",
               "h2d_bytes_per_step": (tR.numel() + tS.numel()) * 8, "d2h_bytes_per_step": 8,
               "api": "distributed_join_count: tbg_shard_split + NCCL all-to-all + tbg_join_device per rank; "
                      "each rank's rows copied from pinned host memory each step", "count": int(m)}
    peak, peak_kind = read_peaks()
    local_rows = tR.numel() + tS.numel()
    joined = moved.get("joined", local_rows)
    # this rank's HBM bytes: split 8 (histogram) + 16 (scatter) per own row when
    # world > 1, the join 48 per received row (histogram 8, 2 passes x 16, build/probe 8)
    alg = (24 * local_rows if world > 1 else 0) + 48 * joined
    line = {
        "metric": metric, "value": value, "unit": "Mtuples/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": workload_name, "global_batch": nR + nS, "nR": nR, "nS": nS,
                   "rows_per_rank": local_rows, "nvlink_rows_sent_per_rank": sent_rows,
                   "parallelism": f"one join over {world} rank(s): key-hash split, all-to-all (NCCL), local RHO, "
                                  f"count all-reduce",
                   "l2": "inputs larger than the 126 MB L2; no flush needed"},
        "gpu_launches": int(launches),
        "e2e": e2e,
        "roofline": {"bound": "hbm", "kernel": "this rank's split and join kernels (pipeline)",
                     "achieved": alg / (ms / K / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (ms / K / 1e3) / 1e9 / peak, "traffic": None, "peak_source": peak_kind,
                     "algorithmic_bytes_per_rank": alg,
                     "nvlink_bytes_per_rank": sent_rows * 8,
                     "bytes_model": "split: histogram 8 + scatter 16 B per own row (world > 1); join: 48 B per "
                                    "received row"},
        "clocks": clocks.summary(),
        "matches": int(m),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline and reference_available():
        host_rows = (host_copy_rows(tR, nR), host_copy_rows(tS, min(tS.numel(), 1 << args.cpu_sample_log2)), nS)
        line["cpu_baseline"] = cpu_baseline_line(host_rows, "RHO", False)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ batch
def batch_algorithmic_bytes(dj, desc):
    """Bytes each join must move under the plan's choices: partitioned joins
    8 (histogram) + 16 (scatter) + 8 (build/probe) per row; direct joins read
    S once and R once per S slice."""
    choice = {c["log2_R"]: c for c in desc["classes"]}
    total = 0
    for (_, nR, _, nS) in dj:
        if not nR or not nS:
            continue
        c = choice[int(nR).bit_length() - 1]
        if c["bits"] > 0:
            total += 32 * (nR + nS)
        else:
            total += 8 * nS + 8 * nR * (-(-nS // c["capS"]))
    return total


def batch_reference_run(njoins, lo, hi, zf, max_rows, threads):
    """The reference's RHO (oracle/_ref) looped over the first joins of the
    seeded batch until max_rows input rows, as its driver runs one join per
    call.  Returns (Mtuples/s, seconds, joins, rows) or (None, why)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if O.ref() is None:
        return None, "oracle/_ref/libtbref.so not built"
    nR, nS, zipf = batch_sizes(njoins, lo, hi, zf)
    rng = np.random.default_rng(4)
    t = 0.0
    rows = 0
    n = 0
    for i in range(njoins):
        if rows and rows + nR[i] + nS[i] > max_rows:
            break
        R = np.zeros(nR[i], dtype=[("key", "<u4"), ("payload", "<u4")])
        R["key"] = rng.permutation(nR[i]).astype(np.uint32) + 1
        S = np.zeros(nS[i], dtype=R.dtype)
        if zipf[i]:
            w = 1.0 / np.arange(1, nR[i] + 1)
            cdf = np.cumsum(w)
            cdf /= cdf[-1]
            S["key"] = (np.searchsorted(cdf, rng.random(nS[i])) + 1).astype(np.uint32)
        else:
            S["key"] = rng.integers(1, nR[i] + 1, nS[i]).astype(np.uint32)
        c, _, rt_us = O.ref_join("RHO", R, S, nthreads=threads)
        if c != nS[i]:
            return None, f"reference RHO count {c} != {nS[i]} on join {i}"
        t += rt_us * 1e-6
        rows += int(nR[i] + nS[i])
        n += 1
    return (rows / t / 1e6, t, n, rows), None


def batch_main(args, rank, world, local):
    nj, lo, hi, zf = BATCH_WORKLOADS[args.workload]
    nj = args.joins or nj
    lo = args.log2_lo if args.log2_lo is not None else lo
    hi = args.log2_hi if args.log2_hi is not None else hi
    workload_name = (f"{nj} batched RHO joins, |R_i| log-uniform 2^{lo}..2^{hi}, |S_i| = k|R_i| k in 1..16, "
                     f"{int(zf * 100)}% Zipf z=1.0 else uniform FK, count only, one persistent launch (CUDA graph)")
    metric = "input Mtuples/s sum(|R_i|+|S_i|)/t over the batch, per-join bit-exact counts"
    if args.impl == "reference":
        if rank != 0:
            return 0
        threads = host_threads()
        steps = max(1, args.steps)
        res, why = None, None
        vals = []
        for _ in range(steps):
            res, why = batch_reference_run(nj, lo, hi, zf, 1 << 27, threads)
            if res is None:
                print(json.dumps({"impl": "reference", "unavailable": why}))
                return 0
            vals.append(res)
        v = statistics.median(r[0] for r in vals)
        _, t, n, rows = vals[-1]
        print(json.dumps({
            "impl": "reference", "metric": metric, "value": v, "unit": "Mtuples/s", "n_gpus": world,
            "steps": steps, "warmup": 0, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": workload_name, "global_batch": rows},
            "cpu_baseline": {"value": v, "unit": "Mtuples/s", "cores": threads, "kind": "reference",
                             "sample": f"reference RHO (oracle/_ref) looped over the first {n} joins of the "
                                       f"batch ({rows} rows), {threads} threads, its own Total Runtime"},
            "e2e": {"value": v, "unit": "Mtuples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return 0

    import torch
    import torch.distributed as dist
    tbg = importlib.import_module("tee-bench_b200")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:  # the rank's GPU is current before NCCL binds to it
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300), device_id=dev)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    with torch.cuda.stream(stream):
        buf, dj, zipf = make_batch_device(torch, tbg, nj, lo, hi, zf, seed=4 + rank, stream=sh)
    stream.synchronize()
    rows = sum(j[1] + j[3] for j in dj)
    want = [j[3] for j in dj]
    b = tbg.Batch(dj, tbg.config("RHO", radix_bits=-1 if args.no_autotune else 0), sh)
    desc = b.describe()
    counts = torch.empty(nj, dtype=torch.int64, device=dev)
    for _ in range(args.warmup):
        b.run(counts.data_ptr(), sh)
        b.sync()
    if counts.cpu().tolist() != want:
        raise SystemExit("wrong per-join counts")
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = tbg.kernel_launches()
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            b.run(counts.data_ptr(), sh)
        ev1.record(stream)
        torch.cuda.synchronize()
    b.sync()
    launches = tbg.kernel_launches() - l0
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms, dist, dev)
    K = args.steps
    value = job_mtuples(world, rows, K, ms / 1e3)
    peak, peak_kind = read_peaks()
    alg = batch_algorithmic_bytes(dj, desc)
    achieved = alg / (ms / K / 1e3) / 1e9

    # e2e through the public batch API: each step copies every join's inputs
    # from pinned host memory, replays the graph and reads the counts back
    e2e = None
    host = None
    if args.e2e_steps > 0:
        try:
            host = torch.empty(buf.numel(), dtype=torch.int64, pin_memory=True)
        except RuntimeError as ex:
            e2e = {"value": None, "unavailable": f"pinned host buffer of {buf.numel() * 8} bytes: {ex}"[:200]}
    if host is not None:
        host.copy_(buf)
        hcounts = torch.empty(nj, dtype=torch.int64, pin_memory=True)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.e2e_steps):
            with torch.cuda.stream(stream):
                buf.copy_(host, non_blocking=True)
            b.run(counts.data_ptr(), sh)
            with torch.cuda.stream(stream):
                hcounts.copy_(counts, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        el = e0.elapsed_time(e1) / 1e3
        el = max_over_ranks(el, dist, dev)
        if hcounts.tolist() != want:
            raise SystemExit("wrong per-join counts (e2e)")
        e2e = {"value": job_mtuples(world, rows, args.e2e_steps, el), "unit": "Mtuples/s",
               "h2d_bytes_per_step": int(buf.numel() * 8), "d2h_bytes_per_step": int(nj * 8),
               "api": "tbg_batch_run with every join's R_i, S_i copied from pinned host memory each step"}
        del host
    b.close()
    line = {
        "metric": metric, "value": value, "unit": "Mtuples/s", "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": workload_name, "global_batch": world * rows, "joins": nj,
                   "zipf_joins": int(zipf.sum()), "grid": desc["grid"], "tickets": desc["tickets"],
                   "autotune_ms": desc["tune_ms"],
                   "classes": [{k: c[k] for k in ("log2_R", "joins", "bits", "layout", "capS", "chunk")}
                               for c in desc["classes"]],
                   "l2": f"inputs {rows * 8 / 1e9:.1f} GB per step > 126 MB L2; no flush needed",
                   "generator": "on-GPU pk / fk / zipf per join (generator.cpp semantics)"},
        "gpu_launches": int(launches),
        "e2e": e2e,
        "roofline": {"bound": "hbm", "kernel": "k_batch (the batch's only kernel; one launch per step)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": alg,
                     "timing": "CUDA events around each graph replay on its stream"},
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = host_threads()
        res, why = batch_reference_run(nj, lo, hi, zf, 1 << 27, threads)
        if res:
            line["cpu_baseline"] = {"value": res[0], "unit": "Mtuples/s", "cores": threads, "kind": "reference",
                                    "sample": f"reference RHO (oracle/_ref) looped over the first {res[2]} joins "
                                              f"({res[3]} rows), its own timer"}
        else:
            line["cpu_baseline"] = {"value": None, "unavailable": why}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
