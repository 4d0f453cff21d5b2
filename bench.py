#!/usr/bin/env python
"""BPMax fill benchmark on B200: max-plus Gterms/s of the whole fill (and batched pairs/s).

    python bench.py [--gpus N --steps K --warmup W] [--workload single|small|balanced|batched|grad]
    python bench.py --impl reference ...   # the reference's own CPU fill on the host cores

One step = one complete fill of one sequence pair (default: strand 1 N1=1024, strand 2 N2=64,
uniform random ACGU from a seed, integer weights GC=3/AU=2/GU=1). One term = one max-plus
candidate (one fp32 add + one max); a fill evaluates C(M)C(N) + 2T(M)C(N) + 2C(M)T(N) + C(M) + C(N)
terms with C(n) = n(n^2-1)/6, T(n) = n(n+1)/2 (twice this is the reference's "bpmax OPS").
With N GPUs every rank fills its own pair (independent pairs, no collective): weak scaling.
Prints ONE JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from bpmax_b200 import workloads as W  # noqa: E402

REASON_COLS = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="single", choices=["single", "small", "balanced", "batched", "grad"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched pairs/s sub-measurement")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--pair", default=None, help="M,N: one custom uniform pair instead of the workload")
    ap.add_argument("--r0-only", default=None, metavar="M,N",
                    help="R0-only double max-plus microbenchmark of shape M x N (the reference's IPDPSW program), "
                         "one JSON line, then exit")
    return ap.parse_args()


def workload(name: str, rank: int, pair: str | None = None) -> W.Workload:
    seed = 2 + 1000 * rank
    if pair:
        m, n = (int(x) for x in pair.split(","))
        return W.single_pair(m, n, seed=seed)
    if name == "single":
        return W.single_pair(1024, 64, seed=seed)
    if name == "small":
        return W.single_pair(128, 32, seed=1 + 1000 * rank)
    if name == "balanced":
        return W.single_pair(256, 256, seed=3 + 1000 * rank)
    if name == "batched":
        return W.batched_uneven(512, seed=4 + 1000 * rank)
    return W.gradient_batch(64, 256, 64, seed=5 + 1000 * rank)


# ---------------------------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out" if os.path.isdir(os.path.join(ROOT, "gpurun_out")) else ".",
                                 f".clocks_{os.getpid()}.csv")

    def __enter__(self):
        q = "clocks.sm,clocks.max.sm,power.draw," + ",".join("clocks_event_reasons." + c for c in REASON_COLS)
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 3 + len(REASON_COLS):
                    continue
                try:
                    rows.append((float(parts[0]), float(parts[1]), float(parts[2]), parts[3:]))
                except ValueError:
                    continue
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        load = [r for r in rows if r[2] > 250.0] or rows
        reasons = sorted({REASON_COLS[i] for r in load for i, v in enumerate(r[3]) if v.lower().startswith("active")})
        return {"sm_mhz": statistics.median(r[0] for r in load), "sm_max_mhz": max(r[1] for r in rows),
                "power_w_max": max(r[2] for r in rows), "samples": len(load), "reasons": reasons}


# ---------------------------------------------------------------------------------- dist
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world, device: str = "cuda"):
    if world > 1:
        import torch
        import torch.distributed as dist

        dist.barrier()
        if device == "cuda":
            torch.cuda.synchronize()


def reduce_max(world, x: float, device: str = "cuda") -> float:
    """The max over ranks of x (one all-reduce; every rank calls it in the same order)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------------- CPU side
def cpu_sample_pair(wl_name: str):
    """Bounded sample of the workload for the reference's CPU fill: same strand-2 length and
    weights, strand 1 shortened so one fill takes ~10-20 s on 16 host cores."""
    if wl_name in ("single", "grad"):
        return W.single_pair(160, 64, seed=2), 32, "strand1 N1=160 prefix-size pair, strand2 N2=64, N_tile=32 (3x8)"
    if wl_name == "small":
        return W.single_pair(128, 32, seed=1), 16, "the full pair N1=128, N2=32, N_tile=16 (3x8)"
    if wl_name == "balanced":
        return W.single_pair(24, 256, seed=3), 64, "strand1 N1=24, strand2 N2=256, N_tile=64 (3x8)"
    return W.single_pair(100, 40, seed=4), 8, "one pair N1=100, N2=40, N_tile=8 (3x8)"


def run_reference_fill(pair_wl: W.Workload, n_tile: int):
    from oracle import oracle as O

    s1, s2 = pair_wl.pairs[0]
    threads = min(os.cpu_count() or 1, 128)
    t0 = time.perf_counter()
    out = O.ref_fill(s1, s2, pair_wl.weights, n_tile, 3, 8, threads=threads, sentinel=0.0)
    dt = time.perf_counter() - t0
    terms = W.terms(len(s1), len(s2))["total"]
    return terms, dt, threads, out


def cpu_baseline(wl_name: str):
    from oracle import oracle as O

    if not O.ref_available():
        return {"value": None, "unit": "Gterms/s", "cores": None, "kind": "reference",
                "sample": "oracle/_ref not built (needs the reference sources at build time)"}
    wl, T, desc = cpu_sample_pair(wl_name)
    terms, dt, threads, _ = run_reference_fill(wl, T)
    return {"value": terms / dt / 1e9, "unit": "Gterms/s", "cores": threads, "kind": "reference",
            "sample": f"{desc}; {terms:.3e} terms in {dt:.2f} s", "host_cpu": host_cpu()}


def host_cpu() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def mem_available_bytes() -> int:
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


# ---------------------------------------------------------------------------------- reference arm
def main_reference(args, world, rank):
    if rank != 0:
        return
    wl, T, desc = cpu_sample_pair(args.workload)
    from oracle import oracle as O

    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libbpmax_ref.so was not built"}))
        return
    for _ in range(args.warmup):
        run_reference_fill(wl, T)
    tot_terms, tot_t = 0, 0.0
    for _ in range(args.steps):
        terms, dt, threads, _ = run_reference_fill(wl, T)
        tot_terms += terms
        tot_t += dt
    v = tot_terms / tot_t / 1e9
    line = {"metric": "max-plus Gterms/s", "value": v, "unit": "Gterms/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": wl.name, "sample_of": args.workload, "N_tile": T, "MR": 3, "NR": 8},
            "cpu_baseline": {"value": v, "unit": "Gterms/s", "cores": threads, "kind": "reference",
                             "sample": desc, "host_cpu": host_cpu()},
            "e2e": {"value": v, "unit": "Gterms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------------- B200 arm
def main_b200(args, world, rank, local):
    from bpmax_b200 import Engine

    wl = workload(args.workload, rank, args.pair)
    eng = Engine(local)
    eng.set_weights(wl.weights)
    single = len(wl.pairs) == 1
    terms_step = wl.total_terms
    s1, s2 = wl.pairs[0]

    def step():
        if single:
            eng.score(s1, s2)
        elif args.workload == "grad":
            eng.grad_batch(wl.pairs)
        else:
            eng.score_batch(wl.pairs)
        return eng.last_timing()

    tuned = None
    if not single:  # batches: schedule chosen by the autotuner on these shapes (outside the timing)
        tuned, _ = eng.autotune(wl.pairs, trials=1)
    for _ in range(max(args.warmup, 0)):
        step()
    barrier(world)
    dev_ms, launches = 0.0, 0
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ms, n = step()
            dev_ms += ms
            launches += n
        barrier(world)
        wall = time.perf_counter() - t0
    clocks = clk.summary()
    dev_ms = reduce_max(world, dev_ms)
    value = terms_step * args.steps * world / (dev_ms * 1e-3) / 1e9

    # roofline: eager re-run with events around every launch
    prof = eng.profile_kernels()
    r0_ms, r0_n, r0_terms = prof["r0"]
    peak = eng.maxplus_peak()
    roofline = r0_roofline(wl, r0_ms, r0_n, r0_terms, peak, clocks)
    roofline["kernels"] = {k: {"ms": v[0], "launches": v[1], "terms": v[2]} for k, v in prof.items()}
    roofline["r0_share_of_step"] = r0_ms / sum(v[0] for v in prof.values())

    e2e = None
    if not args.no_e2e and single and len(s2) >= 8:
        e2e = measure_e2e(eng, wl, args, world)

    batched = None
    if not args.no_batched and single and args.workload == "single" and not args.pair and world == 1:
        batched = measure_batched(eng)
        eng.set_weights(wl.weights)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(args.workload)
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "error": str(e)}

    if rank == 0:
        M, N = len(s1), len(s2)
        line = {"metric": "max-plus Gterms/s", "value": value, "unit": "Gterms/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "impl": "b200",
                "config": {"workload": wl.name, "N1": M if single else None, "N2": N if single else None,
                           "pairs": len(wl.pairs), "terms_per_step": terms_step,
                           "weights": [float(x) for x in wl.weights],
                           "l2": "inputs larger than L2 (each step streams its F tables from HBM)",
                           "parallelism": f"independent pairs per rank x{world}", "autotuned": tuned},
                "pct_maxplus_peak": 100.0 * value * 1e9 / peak,
                "gpu_launches": launches, "wall_s": wall, "clocks": clocks, "roofline": roofline,
                "cpu_baseline": cpu, "e2e": e2e, "batched": batched}
        print(json.dumps(line))
    eng.close()


# DRAM bytes (read + write) per product item (one outer cell and one k1) of the R0 kernel with
# inner width 64, from one ncu capture of a 512x64 fill (profiles/r0_kernel_512x64.md): the
# kernel's traffic grows with the items it processes.
R0_DRAM_BYTES_PER_ITEM_NP64 = 16466


def r0_roofline(wl, r0_ms, r0_n, r0_terms, peak_terms_s, clocks):
    """Roofline of the dominant kernel (the R0+R3+R4 product): FP32-ALU bound. One max-plus term is
    one fp32 add + one max, counted as 2 FP32 operations as the reference counts its GFLOPS.
    achieved = algorithmic terms per launch / mean launch time (CUDA events on the launching stream).
    peak = the max-plus issue ceiling measured live on this GPU (register-resident add + 3-input max
    on every SM). Also reported: the nominal FP32-lane peak (148 SMs x 128 lanes x SM clock, 2 ops
    per term) and the HBM side of the same kernel (ncu DRAM bytes per launch vs measured copy peak)."""
    per_launch_s = r0_ms * 1e-3 / max(r0_n, 1)
    terms_per_launch = r0_terms / max(r0_n, 1)
    achieved = 2 * terms_per_launch / per_launch_s / 1e12  # TFLOP/s
    peak = 2 * peak_terms_s / 1e12
    out = {"bound": "fp32_alu", "kernel": "r0_kernel (R0+R3+R4 max-plus product)", "achieved": achieved, "peak": peak,
           "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
           "peak_source": "measured live: bpmax_gpu_maxplus_peak (packed fp32 add + 3-input max, every sum new, register resident, all SMs)",
           "ops_per_term": 2, "achieved_Gterms_s": achieved / 2 * 1e3, "launches": r0_n,
           "ms_per_launch": per_launch_s * 1e3, "terms_per_launch": terms_per_launch}
    mhz = clocks.get("sm_mhz") or 1965.0
    nominal = 148 * 128 * mhz * 1e6 / 1e12  # FP32 lane-ops/s in T
    out["nominal_fp32_peak"] = nominal
    out["frac_of_nominal_fp32"] = achieved / nominal
    if R0_DRAM_BYTES_PER_ITEM_NP64 and len(wl.pairs) == 1 and len(wl.pairs[0][1]) > 56 and len(wl.pairs[0][1]) <= 64:
        M = len(wl.pairs[0][0])
        items_per_launch = (M * (M * M - 1) / 6) / max(r0_n, 1)
        traffic = R0_DRAM_BYTES_PER_ITEM_NP64 * items_per_launch
        out["traffic"] = traffic
        hbm = measured_peaks().get("hbm_gbs")
        source = "MEASURED_PEAKS.json hbm_gbs (of measured)"
        if not hbm:
            hbm, source = 6650.0, "6.65 TB/s copy bandwidth measured earlier on this pool (of fallback)"
        gbs = traffic / per_launch_s / 1e9
        out["hbm"] = {"achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                      "peak_source": source,
                      "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per item, scaled to a launch"}
    return out


def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def measure_e2e(eng, wl, args, world):
    """The same fill through the reference-facing C call bpmax_gpu_fill: sequences from host
    memory in, the whole F table in the reference's layout back into pinned host memory."""
    s1, s2 = wl.pairs[0]
    M, N = len(s1), len(s2)
    T = 32 if N >= 64 else (16 if N >= 32 else 8)
    n = eng.reference_size(M, N, T)
    ns = (N + T - 1) // T
    d2h = M * (M + 1) // 2 * ns * ns * (T + 1) * T * 4
    if mem_available_bytes() < 2 * n * 4:
        return {"value": None, "unit": "Gterms/s", "skipped": f"host memory below 2x the {n * 4 / 1e9:.1f} GB F buffer"}
    import torch

    buf = torch.empty(n, dtype=torch.float32, pin_memory=True)
    out = buf.numpy()
    eng.fill(s1, s2, T, out=out)  # warm
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        _, score = eng.fill(s1, s2, T, out=out)
    barrier(world)
    wall = reduce_max(world, time.perf_counter() - t0)
    del out, buf
    return {"value": wl.total_terms * args.steps * world / wall / 1e9, "unit": "Gterms/s",
            "h2d_bytes_per_step": 4 * (M + N), "d2h_bytes_per_step": d2h, "N_tile": T,
            "api": "bpmax_gpu_fill (reference layout, pinned host buffer)", "s_per_step": wall / args.steps}


def measure_batched(eng):
    """512 uneven pairs: one batched graph (schedule from the autotuner) vs one fill per pair (both
    on this GPU)."""
    wl = W.batched_uneven(512, seed=4)
    eng.set_weights(wl.weights)
    tuned, tune_ms = eng.autotune(wl.pairs, trials=1)
    eng.score_batch(wl.pairs)
    ms_b = []
    for _ in range(3):
        eng.score_batch(wl.pairs)
        ms_b.append(eng.last_timing()[0])
    t0 = time.perf_counter()
    eng.score_each(wl.pairs)  # warm (captures one graph per shape)
    eng.score_each(wl.pairs)
    ms_e, launches_e = eng.last_timing()
    wall_e = time.perf_counter() - t0
    mb = statistics.median(ms_b)
    return {"workload": wl.name, "pairs": len(wl.pairs), "pairs_per_s_batched": len(wl.pairs) / (mb * 1e-3),
            "pairs_per_s_per_pair_launch": len(wl.pairs) / (ms_e * 1e-3), "ms_batched": mb, "ms_per_pair_launch": ms_e,
            "speedup": ms_e / mb, "terms": wl.total_terms, "Gterms_per_s_batched": wl.total_terms / (mb * 1e-3) / 1e9,
            "launches_per_pair_launch": launches_e, "wall_s_per_pair_pass": wall_e / 2,
            "autotuned": tuned, "autotune_best_ms": tune_ms}


R0_ONLY_PUBLISHED = "246.2 ... 343.8 GFLOPS at 16x1024 ... 16x3000 on a Xeon E-2278G, 8 cores (the reference's own R0-only code)"


def r0only_reference_time(M: int, N: int):
    """The reference's R0-only program (oracle/_ref/ospsqmax_time, random sequences as its driver
    draws them) on this host's cores: (seconds, threads), or None where it was not built."""
    from oracle import oracle as O

    if not os.path.exists(O._REF_R0_TIME):
        return None
    out = subprocess.run([O._REF_R0_TIME, str(M), str(N)], capture_output=True, text=True, check=True)
    t = float(next(l for l in out.stdout.splitlines() if l.startswith("Execution time")).split(":")[1].split()[0])
    return t, os.cpu_count()


def main_r0only(args, rank):
    """R0-only microbenchmark: terms = C(M) C(N) per fill; value = terms / summed device time."""
    from bpmax_b200 import Engine

    if rank != 0:
        return
    M, N = (int(x) for x in args.r0_only.split(","))
    rng = np.random.default_rng(11)
    s1 = rng.integers(0, 2**31 - 1, M).astype(np.int32)  # rand()-sized values, as the reference's driver
    s2 = rng.integers(0, 2**31 - 1, N).astype(np.int32)
    C = lambda n: n * (n * n - 1) // 6  # noqa: E731
    terms = C(M) * C(N)
    eng = Engine(0)
    peak = eng.maxplus_peak()
    for _ in range(max(args.warmup, 1)):
        eng.r0_only(s1, s2, want_table=False)
    ms = []
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            eng.r0_only(s1, s2, want_table=False)
            ms.append(eng.last_timing()[0])
    prof = eng.profile_kernels()
    t = sum(ms) / len(ms) * 1e-3
    v = terms / t / 1e9
    ms_ = M  # the reference's program on a bounded sample: same N, the largest M' <= M with C(M')C(N) <= 2e11
    while ms_ > 2 and C(ms_) * C(N) > 2e11:
        ms_ -= 1
    sample = (ms_, N)
    ref = None if args.no_cpu_baseline else r0only_reference_time(*sample)
    cpu = None
    if ref:
        cpu = {"value": C(sample[0]) * C(sample[1]) / ref[0] / 1e9, "unit": "Gterms/s", "cores": ref[1],
               "kind": "reference", "sample": f"ospsqmax_float {sample[0]}x{sample[1]}, {ref[0]:.3f} s",
               "host_cpu": host_cpu()}
    line = {"metric": "R0-only max-plus Gterms/s", "value": v, "unit": "Gterms/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (rand()-sized non-negative integers)",
            "config": {"workload": f"r0only_{M}x{N}", "M": M, "N": N, "terms_per_step": terms},
            "gflops": 2 * v, "pct_maxplus_peak": 100.0 * v * 1e9 / peak, "maxplus_peak_Gterms_s": peak / 1e9,
            "kernels": {k: {"ms": prof[k][0], "launches": prof[k][1]} for k in ("strand", "r0", "finalize")},
            "published_reference": R0_ONLY_PUBLISHED, "cpu_baseline": cpu, "clocks": clk.summary()}
    print(json.dumps(line))
    eng.close()


def main():
    args = parse_args()
    if args.r0_only:
        main_r0only(args, int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            main_reference(args, world, rank)
        else:
            main_b200(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
