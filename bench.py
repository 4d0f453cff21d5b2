#!/usr/bin/env python
"""BPMax fill benchmark on B200: max-plus Gterms/s of the whole fill (and batched pairs/s).

    python bench.py [--gpus N --steps K --warmup W] [--workload single|small|balanced|batched|grad]
    python bench.py --impl reference ...   # the reference's own CPU fill on the host cores

One step = one complete fill of one sequence pair (default: strand 1 N1=1024, strand 2 N2=64,
uniform random ACGU from a seed, integer weights GC=3/AU=2/GU=1). One term = one max-plus
candidate (one fp32 add + one max); a fill evaluates C(M)C(N) + 2T(M)C(N) + 2C(M)T(N) + C(M) + C(N)
terms with C(n) = n(n^2-1)/6, T(n) = n(n+1)/2 (twice this is the reference's "bpmax OPS").
With N GPUs every rank fills its own pair (independent pairs, no collective): weak scaling; a batched
workload is split over the ranks by estimated work instead (strong scaling), its scores gathered once.
The default line also carries the sub-measurements of the other configurations (batched pairs/s,
the balanced 256 x 256 pair, the reference's own published shapes 16 x 750, 32 x 1024 and 32 x 3000,
the forward + adjoint batch, the persistent fill against the graph of per-diagonal launches), bitwise
windows of the benched tables
against the reference's own fill ("parity"), and the reference's fill of a bounded sample timed on
the host cores ("cpu_baseline").
Prints ONE JSON line on rank 0.
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
    ap.add_argument("--no-autotune", action="store_true",
                    help="batches: keep the default schedule (no autotuner runs before the warm-up steps)")
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
        fd, self.path = tempfile.mkstemp(prefix="bpmax_clocks_", suffix=".csv")
        os.close(fd)

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
# Windows of the benched pairs that the reference fills on the host cores: F(i1, j1, ., .) with
# j1 < K depends only on seq1[0..K) and seq2, and with i1 >= M-K only on seq1[M-K..M), so the
# reference's fill of the prefix pair (seq1[:K], seq2) holds exactly the cells j1 < K of the full
# table and the fill of the suffix pair the cells i1 >= M-K. The prefix fill is also the bounded
# CPU sample that is timed (about 10 s of work on 16 host cores).
SAMPLES = {  # workload -> (prefix K, suffix K, N_tile of the reference fill)
    "single": (160, 96, 32),
    "small": (128, 0, 16),
    "balanced": (24, 24, 64),
    "grad": (160, 0, 32),
}


def cpu_sample(wl_name: str, wl: W.Workload):
    """(prefix pair workload, N_tile, description) of the bounded CPU sample of ``wl``."""
    if wl_name == "batched":  # the batch's first pair with N2 >= 9 (the reference needs N_sec >= 2, NR = 8)
        a, b = next(p for p in wl.pairs if len(p[1]) >= 9)
        n = len(b)
        T = 8 if n <= 16 else (16 if n <= 32 else 32)
        return W.Workload(f"batched_pair_{len(a)}x{n}", [(a, b)], wl.weights), T, \
            f"one pair of the batch, N1={len(a)}, N2={n}, N_tile={T} (3x8)"
    K, _, T = SAMPLES[wl_name]
    a, b = wl.pairs[0]
    K = min(K, len(a))
    what = "the full pair" if K == len(a) else f"the strand-1 prefix seq1[:{K}] of the benched pair"
    return W.Workload(f"{wl.name}_prefix{K}", [(a[:K], b)], wl.weights), T, \
        f"{what}, N1={K}, N2={len(b)}, N_tile={T} (3x8)"


def run_reference_fill(pair_wl: W.Workload, n_tile: int):
    """The reference's own fill (oracle/_ref, all host cores) of one pair, timed around its bpmax()
    call alone as V3/bpmax-wrapper.c:274-284 times it. Returns (terms, seconds, threads, table)."""
    from oracle import oracle as O

    s1, s2 = pair_wl.pairs[0]
    threads = min(os.cpu_count() or 1, 128)
    out, dt = O.ref_fill(s1, s2, pair_wl.weights, n_tile, 3, 8, threads=threads, sentinel=0.0, timed=True)
    terms = W.terms(len(s1), len(s2))["total"]
    return terms, dt, threads, out


def cpu_baseline(wl_name: str, wl: W.Workload):
    """Returns (cpu_baseline dict, (reference table of the prefix pair, K, N_tile) or None)."""
    from oracle import oracle as O

    if not O.ref_available():
        return {"value": None, "unit": "Gterms/s", "cores": None, "kind": "reference",
                "sample": "oracle/_ref not built (needs the reference sources at build time)"}, None
    swl, T, desc = cpu_sample(wl_name, wl)
    terms, dt, threads, out = run_reference_fill(swl, T)
    return ({"value": terms / dt / 1e9, "unit": "Gterms/s", "cores": threads, "kind": "reference",
             "sample": f"{desc}; {terms:.3e} terms in {dt:.2f} s (bpmax() alone)", "host_cpu": host_cpu()},
            (out, len(swl.pairs[0][0]), T))


def windows_vs_reference(eng, wl: W.Workload, K_pre: int, K_suf: int, T: int, ref_pre=None):
    """Bitwise comparison of windows of the engine's last fill (the full-size pair of ``wl``) with
    the reference's own fills of the prefix and suffix pairs: every cell the reference writes for
    the outer cells j1 < K_pre, and i1 >= M - K_suf. ref_pre: the prefix table when already filled."""
    from oracle import oracle as O

    if not O.ref_available():
        return {"checked": False, "why": "oracle/_ref not built"}
    s1, s2 = wl.pairs[0]
    M, N = len(s1), len(s2)
    out = {"against": "the reference's own fill (oracle/_ref) of the prefix / suffix pair, bitwise on every "
                      "cell it writes (reference layout, masks and halo rows included)", "N_tile": T}
    total_cells = total_bad = 0
    for name, K, lo in (("prefix", K_pre, 0), ("suffix", K_suf, M - K_suf)):
        if K <= 0:
            continue
        K = min(K, M)
        lo = 0 if name == "prefix" else M - K
        sub = s1[:K] if name == "prefix" else s1[M - K:]
        if name == "prefix" and ref_pre is not None and ref_pre[1] == K and ref_pre[2] == T:
            ref = ref_pre[0]
        else:
            ref = O.ref_fill(sub, s2, wl.weights, T, 3, 8, sentinel=0.0)
        win = eng.read_cells(0, lo, lo + K, lo, lo + K, N)
        iu, ju = np.triu_indices(K)
        mine = O.to_reference_layout(np.ascontiguousarray(win[iu, ju]), K, N, T)
        mask = O.reference_written_mask(K, N, T)
        bad = int(np.count_nonzero(mine.view(np.uint32)[mask] != ref.view(np.uint32)[mask]))
        cells = int(np.count_nonzero(mask))
        out[name] = {"outer_cells": f"{'j1' if name == 'prefix' else 'i1'} {'<' if name == 'prefix' else '>='} "
                                    f"{K if name == 'prefix' else M - K}", "K": K, "cells": cells, "mismatches": bad}
        total_cells += cells
        total_bad += bad
        del win, mine, mask, ref
    out["cells"] = total_cells
    out["mismatches"] = total_bad
    return out


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
    from oracle import oracle as O

    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libbpmax_ref.so was not built"}))
        return
    full = workload(args.workload, 0, args.pair)
    wl, T, desc = cpu_sample(args.workload, full)
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
            "config": {"workload": full.name, "sample_pair": wl.name, "N_tile": T, "MR": 3, "NR": 8},
            "cpu_baseline": {"value": v, "unit": "Gterms/s", "cores": threads, "kind": "reference",
                             "sample": f"{desc}; each step one fill of it, timed around bpmax() alone",
                             "host_cpu": host_cpu()},
            "e2e": {"value": v, "unit": "Gterms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------------- B200 arm
def main_b200(args, world, rank, local):
    from bpmax_b200 import Engine

    single = args.workload in ("single", "small", "balanced") or bool(args.pair)
    # one pair: every rank fills its own (weak scaling); a batch: the same batch on every rank, each
    # filling its LPT share by estimated work (strong scaling), scores gathered at the end
    wl = workload(args.workload, rank if single else 0, args.pair)
    eng = Engine(local)
    eng.set_weights(wl.weights)
    terms_step = wl.total_terms
    s1, s2 = wl.pairs[0]
    mine = list(range(len(wl.pairs)))
    if not single and world > 1:
        from bpmax_b200 import shard

        mine = shard.shares_of(wl.pairs, world)[rank]
    my_pairs = [wl.pairs[i] for i in mine]

    def step():
        if single:
            eng.score(s1, s2)
        elif args.workload == "grad":
            eng.grad_batch(my_pairs)
        else:
            eng.score_batch(my_pairs)
        return eng.last_timing()

    tuned = None
    if not single and not args.no_autotune:  # batches: schedule chosen by the autotuner on these shapes (untimed)
        tuned, _ = eng.autotune(my_pairs, trials=1)
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
    value = terms_step * args.steps * (world if single else 1) / (dev_ms * 1e-3) / 1e9
    gathered = None
    if not single and world > 1:  # every rank's scores into batch order (one object all-gather)
        from bpmax_b200 import shard

        scores, _ = shard.run_sharded(eng.score_batch, wl.pairs, rank, world)
        gathered = {"pairs": int(len(scores)), "ranks": world, "my_pairs": len(mine)}

    # roofline: eager re-run with events around every launch
    prof = eng.profile_kernels()
    r0_ms, r0_n, r0_terms = prof["r0"]
    peak = eng.maxplus_peak()
    roofline = r0_roofline(wl, r0_ms, r0_n, r0_terms, peak, clocks)
    roofline["kernels"] = {k: {"ms": v[0], "launches": v[1], "terms": v[2]} for k, v in prof.items()}
    roofline["r0_share_of_step"] = r0_ms / sum(v[0] for v in prof.values())

    # the reference's own fill of a bounded sample (the prefix pair), and bitwise windows of the
    # benched table against the reference (rank 0 of a one-GPU run; the engine still holds the table)
    cpu, parity, ref_pre = None, None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu, ref_pre = cpu_baseline(args.workload, wl)
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "error": str(e)}
        if single and args.workload in SAMPLES:
            K_pre, K_suf, T = SAMPLES[args.workload]
            try:
                parity = windows_vs_reference(eng, wl, K_pre, K_suf, T, ref_pre)
            except Exception as e:
                parity = {"checked": False, "error": str(e)}

    e2e = None
    if not args.no_e2e and single and len(s2) >= 8:
        e2e = measure_e2e(eng, wl, args, world, ref_pre)

    extra = {}
    if not args.no_batched and single and args.workload == "single" and not args.pair and world == 1:
        extra["batched"] = measure_batched(eng)
        extra["balanced"] = measure_balanced(eng, peak, with_reference=not args.no_cpu_baseline)
        extra["published_shapes"] = measure_published(eng, with_reference=not args.no_cpu_baseline)
        extra["grad"] = measure_grad(eng)
        extra["persistent"] = measure_persistent(local)
        eng.set_weights(wl.weights)

    if rank == 0:
        M, N = len(s1), len(s2)
        line = {"metric": "max-plus Gterms/s", "value": value, "unit": "Gterms/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
                "higher_is_better": True, "scaling": "weak" if single else "strong", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic", "impl": "b200",
                "config": {"workload": wl.name, "N1": M if single else None, "N2": N if single else None,
                           "pairs": len(wl.pairs), "terms_per_step": terms_step,
                           "weights": [float(x) for x in wl.weights],
                           "l2": "inputs larger than L2 (each step streams its F tables from HBM)",
                           "parallelism": (f"independent pairs per rank x{world}" if single else
                                           f"batch sharded over {world} ranks by estimated work (LPT)"),
                           "autotuned": tuned, "gathered": gathered},
                "pct_maxplus_peak": 100.0 * value * 1e9 / peak,
                "gpu_launches": launches, "wall_s": wall, "clocks": clocks, "roofline": roofline,
                "cpu_baseline": cpu, "parity": parity, "e2e": e2e, **extra}
        print(json.dumps(line))
    eng.close()


# DRAM bytes (read + write) per product item (one outer cell and one k1) of the R0 kernel with
# inner width 64: ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of a 512 x 64 fill
# (outer diagonal 256: 256 cells x 256 items, 1.079 GB) divided by its items. The kernel's traffic
# grows with the items it processes, so a launch's traffic is this figure times its items.
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
            hbm, source = 6650.0, "6.65 TB/s, an earlier copy-bandwidth measurement on a B200 (of fallback)"
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


def measure_e2e(eng, wl, args, world, ref_pre=None):
    """The same fill through the reference-facing C call bpmax_gpu_fill: sequences from host
    memory in, the whole F table in the reference's layout back into pinned host memory. With the
    reference's own fill of the prefix pair (ref_pre = (table, K, N_tile)), the last step's table is
    also compared with it, bitwise on every cell the reference writes for the outer cells j1 < K."""
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
    res = {"value": wl.total_terms * args.steps * world / wall / 1e9, "unit": "Gterms/s",
           "h2d_bytes_per_step": 4 * (M + N), "d2h_bytes_per_step": d2h, "N_tile": T,
           "api": "bpmax_gpu_fill (reference layout, pinned host buffer)", "s_per_step": wall / args.steps}
    if ref_pre is not None and ref_pre[2] == T:
        from oracle import oracle as O

        ref, K, _ = ref_pre
        cell_f = ns * ns * (T + 1) * T
        mine = np.ascontiguousarray(out.reshape(M, M, cell_f)[:K, :K])
        mask = O.reference_written_mask(K, N, T)
        bad = int(np.count_nonzero(mine.reshape(-1).view(np.uint32)[mask] != ref.view(np.uint32)[mask]))
        res["parity_reference_layout"] = {"outer_cells": f"j1 < {K}", "cells": int(np.count_nonzero(mask)),
                                          "mismatches": bad,
                                          "against": "the reference's own fill of the prefix pair (oracle/_ref)"}
        del mine, mask
    del out, buf
    return res


def measure_batched(eng):
    """512 uneven pairs: one batched graph (schedule from the autotuner) vs one fill per pair (both
    on this GPU)."""
    wl = W.batched_uneven(512, seed=4)
    eng.set_weights(wl.weights)
    tuned, tune_ms = eng.autotune(wl.pairs, trials=1)
    eng.score_batch(wl.pairs)
    ms_b = []
    t0 = time.perf_counter()
    for _ in range(3):
        eng.score_batch(wl.pairs)
        ms_b.append(eng.last_timing()[0])
    wall_b = (time.perf_counter() - t0) / 3
    eng.score_each(wl.pairs)  # warm (captures one graph per shape)
    t0 = time.perf_counter()
    eng.score_each(wl.pairs)
    wall_e = time.perf_counter() - t0
    ms_e, launches_e = eng.last_timing()
    mb = statistics.median(ms_b)
    return {"workload": wl.name, "pairs": len(wl.pairs), "pairs_per_s_batched": len(wl.pairs) / (mb * 1e-3),
            "pairs_per_s_per_pair_launch": len(wl.pairs) / (ms_e * 1e-3), "ms_batched": mb, "ms_per_pair_launch": ms_e,
            "speedup": ms_e / mb, "terms": wl.total_terms, "Gterms_per_s_batched": wl.total_terms / (mb * 1e-3) / 1e9,
            "launches_per_pair_launch": launches_e, "wall_s_per_pair_pass": wall_e, "wall_s_batched": wall_b,
            "speedup_wall": wall_e / wall_b,
            "speedup_note": "speedup: summed device time of the per-pair fills (cached graphs) over the batched "
                            "fill's device time; speedup_wall: host wall clock of both passes, host work included",
            "autotuned": tuned, "autotune_best_ms": tune_ms}


def measure_persistent(device: int):
    """The persistent fill (one launch per width class walking the outer diagonals with device-side
    dependency counters; the classes of a batch one after another) against the graph of per-diagonal
    launches, on this GPU: median fill ms of three runs of each, single pairs and the 512-pair batch.
    A separate engine, so that no autotuned schedule of the other measurements overrides the mode."""
    from bpmax_b200 import Engine
    e = Engine(device)
    out = {}
    try:
        def med(f):
            f()
            runs = []
            for _ in range(3):
                f()
                runs.append(e.last_timing()[0])
            return statistics.median(runs)
        e.set_weights(W.INTEGER_WEIGHTS)
        for M, N in ((1024, 64), (200, 64), (200, 16)):
            a, b = W.pair(M, N, 2)
            r = {}
            for mode, key in ((0, "graph_ms"), (1, "persistent_ms")):
                e.set_tuning("persistent", mode)
                r[key] = med(lambda: e.score(a, b))
            r["speedup"] = r["graph_ms"] / r["persistent_ms"]
            out[f"{M}x{N}"] = r
        wl = W.batched_uneven(512, seed=4)
        e.set_weights(wl.weights)
        r = {}
        for mode, key in ((0, "graph_ms"), (2, "persistent_ms")):
            e.set_tuning("persistent", mode)
            r[key] = med(lambda: e.score_batch(wl.pairs))
        r["speedup"] = r["graph_ms"] / r["persistent_ms"]
        out[wl.name] = r
    finally:
        e.close()
    return out


def measure_balanced(eng, peak, with_reference=True):
    """Configuration 3: one 256 x 256 pair, uniform and GC-rich (P(G) = P(C) = 0.35): fill rate, the
    product kernel's roofline, and bitwise windows against the reference's own fill."""
    out = {}
    for tag, gc in (("uniform", False), ("gc_rich", True)):
        wl = W.single_pair(256, 256, seed=3, gc_rich=gc)
        s1, s2 = wl.pairs[0]
        eng.set_weights(wl.weights)
        eng.score(s1, s2)  # warm-up (captures the graph)
        ms = []
        for _ in range(2):
            eng.score(s1, s2)
            ms.append(eng.last_timing()[0])
        t = statistics.median(ms)
        d = {"workload": wl.name, "ms_per_fill": t, "value": wl.total_terms / (t * 1e-3) / 1e9, "unit": "Gterms/s"}
        if not gc:
            prof = eng.profile_kernels()
            r0_ms, r0_n, r0_terms = prof["r0"]
            d["roofline"] = r0_roofline(wl, r0_ms, r0_n, r0_terms, peak, {})
            d["roofline"]["kernels"] = {k: {"ms": v[0], "launches": v[1], "terms": v[2]} for k, v in prof.items()}
        if with_reference:
            K_pre, K_suf, T = SAMPLES["balanced"]
            try:
                d["parity"] = windows_vs_reference(eng, wl, K_pre, K_suf, T)
            except Exception as e:
                d["parity"] = {"checked": False, "error": str(e)}
        out[tag] = d
    return out


# The reference's own published whole-fill shapes (short strand 1, long strand 2) and its published
# times for them on 8 cores of a Xeon E-2278G (TPDS/experiments/bpmax_final.xlsx, sheet E2278G): a
# different machine, reported beside the B200 time, not measured here. Each entry: (M, N, parity
# prefix K of strand 1, reference N_tile, published ms).
PUBLISHED_SHAPES = ((16, 750, 16, 64, 730.0), (32, 1024, 8, 64, 9710.0), (32, 3000, 0, 64, 188200.0))


def measure_published(eng, with_reference=True):
    """The reference's published shapes: B200 fill ms (median of two after a warm-up) and, where K > 0,
    the reference's own fill of the strand-1 prefix pair compared bitwise with the same cells of the
    GPU table (K = M: the whole table)."""
    out = {"reference_published": "TPDS V3 whole fill, Xeon E-2278G, 8 cores (bpmax_final.xlsx)"}
    for M, N, K, T, pub in PUBLISHED_SHAPES:
        try:
            wl = W.single_pair(M, N, seed=6)
            s1, s2 = wl.pairs[0]
            eng.set_weights(wl.weights)
            eng.score(s1, s2)  # warm-up (captures the graph)
            ms = []
            for _ in range(2):
                eng.score(s1, s2)
                ms.append(eng.last_timing()[0])
            t = statistics.median(ms)
            d = {"ms_per_fill": t, "value": wl.total_terms / (t * 1e-3) / 1e9, "unit": "Gterms/s",
                 "reference_published_ms": pub, "ratio_to_published": pub / t}
        except Exception as e:  # reported, not fatal
            out[f"{M}x{N}"] = {"error": str(e)}
            continue
        if with_reference and K > 0:
            try:
                d["parity"] = windows_vs_reference(eng, wl, K, 0, T)
            except Exception as e:
                d["parity"] = {"checked": False, "error": str(e)}
        out[f"{M}x{N}"] = d
    return out


def measure_grad(eng):
    """Configuration 5: 64 pairs of 256 x 64, 12 weights from U[0.5, 4]: the forward fill plus the
    adjoint pass (exact d score / d weights); pairs/s with the forward / backward split."""
    wl = W.gradient_batch(64, 256, 64, seed=5)
    eng.set_weights(wl.weights)
    eng.grad_batch(wl.pairs)  # warm-up (captures the graph)
    fwd, tot = [], []
    for _ in range(2):
        eng.score_batch(wl.pairs)
        fwd.append(eng.last_timing()[0])
        eng.grad_batch(wl.pairs)
        tot.append(eng.last_timing()[0])
    f, t = statistics.median(fwd), statistics.median(tot)
    return {"workload": wl.name, "pairs": len(wl.pairs), "pairs_per_s": len(wl.pairs) / (t * 1e-3),
            "ms_forward": f, "ms_backward": t - f, "ms_total": t,
            "Gterms_per_s_forward": wl.total_terms / (f * 1e-3) / 1e9}


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
