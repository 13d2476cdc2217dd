#!/usr/bin/env python
"""Benchmark of the 1M-gate plain placement iteration on B200.

One step = one plain composite iteration of the HAPR placement hot path on
the 1,000,000-gate / 1,200,000-net synthetic netlist (die 1200 x 1200):
net-spring attraction (k = 1) + Barnes-Hut repulsion (theta 0.5, k 0.5,
min_dist 0.1) + DCT-II Poisson density force (1024 x 1024 grid, GEMM form) +
damped Euler step + congestion counting (512 x 512) and FP64 HPWL. Every
step starts from the same device-resident state (the seeded uniform
placement, checkpointed with fx_design_save_state and restored inside the
step), so each timed step does the same work; the configured 500-iteration run is reported beside it
("trajectory").

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fluxion|reference]

Prints one JSON line (rank 0). With N > 1 (torchrun, one process per GPU)
every rank runs an independent replica of the workload ("replicas only": the
path does not shard), timing is the max over ranks and `value` is the sum of
iterations over all ranks divided by that time.

--impl reference times the reference's CPU implementation of the same
iteration on all of this host's cores (the oracle port of the Rust path, the
reference's own BarnesHutTree.cpp and its scipy DCT): every timed step is one
full iteration; only rank 0 runs it, and it never loads the CUDA library.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "neon-physics-fluxion_b200"))
sys.path.insert(0, str(ROOT))

METRIC = "1M-gate force iterations/s"
UNIT = "iterations/s"
# fx_force_iterate reads back HPWL + total overflow (16 B), max overflow (4),
# density energy (8) and the walk's error word (4) after the last iteration
ITER_STATS_D2H = 32


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fluxion", choices=["fluxion", "reference"])
    ap.add_argument("--gates", type=int, default=1_000_000)
    ap.add_argument("--nets", type=int, default=1_200_000)
    ap.add_argument("--die", type=float, default=1200.0)
    ap.add_argument("--bins", type=int, default=1024)
    ap.add_argument("--cong", type=int, default=512)
    ap.add_argument("--precision", default="i8",
                    choices=["fp32", "3xtf32", "tf32", "bf16", "simt", "i8"],
                    help="DCT GEMMs: fp32 (= simt, CUDA cores), 3xtf32, tf32, bf16 (tensor cores)")
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--bh-walk", default="fast", choices=["fast", "exact"],
                    help="Barnes-Hut walk: hardware rsqrt (default) or the bit-reproducible one")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--trajectory", type=int, default=500,
                    help="iterations of the full run reported beside the steps (0: skip)")
    ap.add_argument("--workload", default="plain",
                    choices=["plain", "small", "serve", "leaves", "precision", "attention"],
                    help="plain: the 1M-gate iteration; serve: the request stream; "
                         "leaves: the batched leaf placement; precision: the DCT sweep; "
                         "attention: every level of the 1M-gate hierarchy")
    ap.add_argument("--clusters", type=int, default=16_384, help="leaves: clusters")
    ap.add_argument("--leaf-iters", type=int, default=300, help="leaves: force iterations")
    ap.add_argument("--leaf-precision", default="ieee", choices=["ieee", "fast"],
                    help="leaves: pair-term arithmetic (FX_LEAF_IEEE or FX_LEAF_FAST)")
    ap.add_argument("--leaf-schedule", type=int, default=0,
                    help="leaves: FX_LEAF_* schedule (0 = autotune)")
    ap.add_argument("--no-per-cluster", action="store_true",
                    help="leaves: skip the one-launch-per-cluster comparison run")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: arrivals per second")
    ap.add_argument("--duration", type=float, default=10.0, help="serve: arrival window (s)")
    ap.add_argument("--slots", type=int, default=8, help="serve: concurrent jobs")
    ap.add_argument("--pool", type=int, default=16, help="serve: distinct netlists")
    return ap.parse_args(argv)


PREC = {"fp32": 3, "simt": 3, "3xtf32": 0, "tf32": 1, "bf16": 2, "i8": 4}
PREC_DTYPE = {"fp32": "f32 (DCT GEMMs FP32 on CUDA cores)",
              "3xtf32": "f32 (DCT GEMMs 3xTF32, FP32 accumulate)",
              "tf32": "f32 (DCT GEMMs TF32, FP32 accumulate)",
              "bf16": "f32 (DCT GEMMs BF16, FP32 accumulate)", "simt": "f32",
              "i8": "f32 (DCT GEMMs on the tensor cores from exact 8-bit slices, int32 "
                    "accumulate)"}


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 100 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(device)], stdout=self.tmp,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.tmp.flush()
        rows = [l.split(",") for l in Path(self.tmp.name).read_text().splitlines() if l.strip()]
        os.unlink(self.tmp.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [c.strip() for c in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of each
# stage's kernels at the default 1M-gate workload, from single ncu captures
# (`--set full -s 1 -c 1` of the bench command with --steps 2 --warmup 3;
# summaries under profiles/). A stage missing here reports traffic null.
NCU_DRAM_BYTES = {
    # with --precision 3xtf32: 6 x tc_gemm_kernel<0> (21.000 MB + 0.011 MB
    # each) + dens_charge_kernel (8.393 MB); dens_scatter runs in the
    # previous step's fused kernel
    "density": 6 * 21_010_944 + 8_393_472,
}
# The same per walk kernel (the --bh-walk choice), with its warp
# instructions per launch (smsp__inst_executed.sum), threads per warp
# instruction (smsp__thread_inst_executed_per_inst_executed.ratio) and what
# bounds it; the walk's roofline is the issue rate, 4 warp instructions per
# SM per cycle.
NCU_WALK = {
    "exact": {"dram": 61_725_696, "inst": 1_390_529_927, "tpi": 20.07,
              "limiter": "instruction issue: 87% issue-active, 0.5% of DRAM peak, "
                         "82% warps active"},
    # bh_batch_walk_kernel<64, false>: 59.529 MB read + 1.481 MB written
    "fast": {"dram": 61_009_920, "inst": 587_039_746, "tpi": 31.77,
             "limiter": "instruction issue: 83% issue-active (ALU pipe 66%, FMA 33%), "
                        "1.1% of DRAM peak, 52% warps active"},
}


# ---------------------------------------------------------------------------
# Replicas (N > 1, "replicas only"): every rank runs the whole workload on its
# own GPU; the job's time is the slowest rank's and its throughput the work of
# all ranks over that time.
def max_over_ranks(v: float, dist=None, device: str = "cpu") -> float:
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units: float, seconds: float, dist=None, device: str = "cpu") -> float:
    """sum of units over ranks / max of seconds over ranks"""
    if dist is None:
        return units / seconds
    import torch
    u = torch.tensor([units], dtype=torch.float64, device=device)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(u.item()) / max_over_ranks(seconds, dist, device)


def algorithmic(n, m, p, a, G, gc):
    """Compulsory HBM bytes (each array read once, each output written once)
    and flops per iteration, by stage."""
    b = {
        # adj_ptr, adj_idx, own x/y, v, BH force, area, E fields, new x/y, v,
        # density accumulator update
        "attract_integrate": 4 * (n + 1) + 4 * a + 8 * n + 8 * n + 8 * n + 4 * n
        + 8 * G * G + 8 * n + 8 * n + 8 * G * G,
        # keys+idx written, positions read
        "bh_keys": 8 * n + 8 * n,
        # 4 passes: read keys+idx, write keys+idx (histogram pass re-reads keys)
        "bh_sort": 4 * (8 * n + 8 * n + 4 * n),
        # gather sorted positions, prefix sums, nodes (child, range, com, meta)
        "bh_tree": 4 * n + 8 * n + 8 * n + 16 * n + 4 * n + (n - 1) * (8 + 8 + 16 + 8 + 8),
        # sorted positions, perm, nodes read once, force written
        "bh_walk": 8 * n + 4 * n + (n - 1) * (8 + 8 + 16 + 8) + 8 * n,
        # charge grid, 4 GEMM operands in+out, field
        "density": 8 * G * G + 4 * G * G + 4 * (3 * 4 * G * G) + 4 * G * G + 8 * G * G,
        # net_ptr, pins, positions, difference array RMW, counts
        "congestion": 4 * (m + 1) + 4 * p + 8 * n + 2 * 4 * (gc + 1) ** 2 + 4 * gc * gc,
    }
    f = {"density": 4 * 2 * G ** 3}  # 8 G^3: the four dense G x G DCT GEMMs of one solve
    return b, f


# ---------------------------------------------------------------------------
def cpu_iteration_sample(syn, x, y, bins, cong, threads, bh_stride, cong_stride):
    """Seconds per plain iteration of the CPU path, from a bounded sample.

    attraction (oracle restatement of placer.rs:243-255, full), Barnes-Hut
    (the reference's BarnesHutTree.cpp: full build + every bh_stride-th
    point's walk, scaled), DCT density (the reference's scipy dctn/idctn,
    full), damped step (full), congestion (congestion.rs:11-62 on every
    cong_stride-th net, scaled) and HPWL (full)."""
    from oracle import oracle as orc
    c = syn.circuit
    ap, ai = syn.adj
    area = (c.gate_widths * c.gate_heights).astype(np.float64)
    t = {}
    t0 = time.perf_counter()
    fa = orc.attraction_f32(ap, ai, x, y, 1.0)
    t["attraction"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    orc.bh_reference(x, y, 0.5, 0.5, 0.1, threads, stride=len(x))
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    bh = orc.bh_reference(x, y, 0.5, 0.5, 0.1, threads, stride=bh_stride)
    t_samp = time.perf_counter() - t0
    t["barnes_hut"] = t_build + max(t_samp - t_build, 0.0) * bh_stride
    t0 = time.perf_counter()
    dens = orc.density_forces(x, y, area, c.chip_width, c.chip_height, bins, 0.7, 1e-4)
    t["density"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    fx = (fa[0] + bh[0].astype(np.float32)) + dens["fx"].astype(np.float32)
    fy = (fa[1] + bh[1].astype(np.float32)) + dens["fy"].astype(np.float32)
    xx, yy = x.copy(), y.copy()
    vx, vy = np.zeros_like(xx), np.zeros_like(yy)
    orc.integrate(xx, yy, vx, vy, fx, fy, 0.1, 0.9, (0.0, 0.0, c.chip_width, c.chip_height))
    t["integrate"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    orc.congestion_sample(c.net_ptr, c.net_gate, xx, yy, c.chip_width, c.chip_height,
                          cong, cong, cong_stride)
    t["congestion"] = (time.perf_counter() - t0) * cong_stride
    t0 = time.perf_counter()
    orc.hpwl_f32(c.net_ptr, c.net_gate, xx, yy)
    t["hpwl"] = time.perf_counter() - t0
    return sum(t.values()), t


class SynthCache:
    def __init__(self, args):
        import fluxion_b200 as fx
        self.syn = fx.synth_plain(args.seed, args.gates, args.nets, args.die)
        self.circuit = self.syn.circuit
        self.placement = self.syn.placement
        self.adj = None


def plain_config(args, pins, adj_entries, world):
    """The `config` of the plain-1M line; both arms print it."""
    b_alg, _ = algorithmic(args.gates, args.nets, pins, adj_entries, args.bins, args.cong)
    B_iter = sum(b_alg.values())
    return {"workload": f"plain-1M: {args.gates} gates, {args.nets} nets "
                        f"({pins} pins, {adj_entries} adjacency entries), die {args.die:g}, "
                        f"BH theta 0.5, DCT {args.bins}^2 ({args.precision}), congestion "
                        f"{args.cong}^2",
            "seed": args.seed, "parallelism": "replicas" if world > 1 else "single",
            "l2": "working set per iteration ~%d MB > 126 MB L2" % (B_iter // 2**20)}


def cpu_iteration_full(orc, s, adj, x, y, bins, cong, threads, sample=1):
    """One plain iteration of the CPU path from (x, y) at rest; returns the
    seconds of each stage. Every stage runs in full when sample == 1:
    attraction (restatement of placer.rs:243-255 over the adjacency, 1
    thread), Barnes-Hut (the reference's BarnesHutTree.cpp: sequential build,
    walk of every point on `threads` threads), the DCT density force (the
    reference's scipy dctn/idctn solve, FP64), the damped step, congestion
    (the literal loops of congestion.rs:11-62 over every net on `threads`
    threads) and the f32 HPWL. sample > 1 (warm-up only) walks every
    sample-th point and counts every sample-th net."""
    ap, ai = adj
    area = (s.gate_widths * s.gate_heights).astype(np.float64)
    t = {}
    t0 = time.perf_counter()
    fa = orc.attraction_f32(ap, ai, x, y, 1.0)
    t["attraction"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    bh = orc.bh_reference(x, y, 0.5, 0.5, 0.1, threads, stride=sample)
    t["barnes_hut"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    dens = orc.density_forces(x, y, area, s.chip_width, s.chip_height, bins, 0.7, 1e-4)
    t["density"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    fx = (fa[0] + bh[0].astype(np.float32)) + dens["fx"].astype(np.float32)
    fy = (fa[1] + bh[1].astype(np.float32)) + dens["fy"].astype(np.float32)
    xx, yy = x.copy(), y.copy()
    vx, vy = np.zeros_like(xx), np.zeros_like(yy)
    orc.integrate(xx, yy, vx, vy, fx, fy, 0.1, 0.9, (0.0, 0.0, s.chip_width, s.chip_height))
    t["integrate"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    if sample == 1:
        orc.congestion_parallel(s.net_ptr, s.net_gate, xx, yy, s.chip_width, s.chip_height,
                                cong, cong, threads)
    else:
        orc.congestion_sample(s.net_ptr, s.net_gate, xx, yy, s.chip_width, s.chip_height,
                              cong, cong, sample)
    t["congestion"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    orc.hpwl_f32(s.net_ptr, s.net_gate, xx, yy)
    t["hpwl"] = time.perf_counter() - t0
    return t


def run_reference(args, rank, world):
    """The reference arm: the CPU implementation of the same iteration on all
    host threads. The netlist comes from the generator built into the
    oracle's own library (the same seeded bytes as the GPU arm); the CUDA
    library is never loaded. Every timed step is one full, unsampled
    iteration from the seeded start positions; the warm-up steps run the
    same stages on a 1/16 sample (every 16th walked point and counted net),
    which warms the code, pools and caches without the full cost."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    from oracle import oracle as orc
    orc.build()
    s = orc.synth_plain(args.seed, args.gates, args.nets, args.die)
    adj = orc.build_adjacency(s.num_gates, s.net_ptr, s.net_gate)
    x, y = s.gate_x.copy(), s.gate_y.copy()
    for _ in range(args.warmup):
        cpu_iteration_full(orc, s, adj, x, y, args.bins, args.cong, threads, sample=16)
    per, parts = [], {}
    t_all = time.perf_counter()
    for _ in range(args.steps):
        t = cpu_iteration_full(orc, s, adj, x, y, args.bins, args.cong, threads)
        per.append(sum(t.values()))
        for k, v in t.items():
            parts[k] = parts.get(k, 0.0) + v / args.steps
    wall = time.perf_counter() - t_all
    sec = wall / args.steps
    value = 1.0 / sec
    sample = (f"{args.steps} full plain iterations on {args.gates} gates from the seeded start "
              f"positions, every stage unsampled: attraction (1 thread), the reference "
              f"BarnesHutTree.cpp (sequential build, walk on {threads} threads), the scipy DCT "
              f"solve, the damped step, the literal congestion loops over all nets on "
              f"{threads} threads, HPWL")
    out = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 (density solve FP64, scipy)", "data": "synthetic",
           "config": plain_config(args, s.num_pins, len(adj[1]), world),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                            "kind": "port", "sample": sample},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0},
           "stage_seconds": {k: round(v, 4) for k, v in parts.items()},
           "step_seconds_min_max": [round(min(per), 3), round(max(per), 3)]}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
def run_fluxion(args, rank, world, local_rank):
    import fluxion_b200 as fx

    dist = None
    if world > 1:
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
        dist = tdist

    def barrier():
        if dist is not None:
            dist.barrier()

    dev = f"cuda:{local_rank}"

    sc = SynthCache(args)
    c, p = sc.circuit, sc.placement
    ctx = fx.Context(local_rank)
    d = fx.Design(ctx, c)
    cfg = fx.iter_cfg(density_bins=args.bins, dct_precision=PREC[args.precision],
                      cong_cols=args.cong, cong_rows=args.cong,
                      bh_walk=fx.FX_BH_EXACT if args.bh_walk == "exact" else fx.FX_BH_FAST)
    # The start state of every step: the seeded uniform placement (the state
    # the reference arm and the CPU baseline time too), velocities zero,
    # checkpointed on the device.
    d.set_positions(p.gate_x, p.gate_y)
    x0, y0 = p.gate_x.copy(), p.gate_y.copy()
    d.save_state()

    def step():
        d.restore_state()
        return d.force_iterate(cfg, 1)

    # In the timed region only the stages the roofline lines report carry
    # events (the walk and the density solve; two events each per step).
    # Each step is one public single-iteration call on the resident state,
    # which (after two eager calls per ping-pong parity in the warm-up)
    # replays the library's cached CUDA graph of the whole call; the graph
    # records those stage events itself, read after every call.
    ctx.set_profiling(True, stages=("bh_walk", "density"))
    # at least four warm-up calls: the graph of each parity is captured by
    # the second call of that parity, so every timed call is a replay
    warmup_run = max(args.warmup, 4)
    for _ in range(warmup_run):
        step()
    ctx.synchronize()
    launches0 = ctx.kernel_launches()
    ctx.reset_stage_times()
    clocks = ClockSampler(local_rank)
    time.sleep(0.3)
    barrier()
    ctx.synchronize()
    ctx.mark(0)
    for _ in range(args.steps):
        st = step()
    ctx.mark(1)
    ctx.synchronize()
    ms = ctx.elapsed_ms(0, 1)
    barrier()
    clk = clocks.stop()
    ctx.set_profiling(False)
    launches = ctx.kernel_launches() - launches0
    stages = ctx.stage_times()
    # The breakdown of the other stages comes from a separate pass with
    # events on every stage (about 0.03 ms per step), outside the timed region.
    ctx.reset_stage_times()
    ctx.set_profiling(True)
    for _ in range(min(args.steps, 50)):
        step()
    ctx.synchronize()
    ctx.set_profiling(False)
    all_stages = ctx.stage_times()
    stages = {k: (stages[k] if k in ("bh_walk", "density") else all_stages[k]) for k in all_stages}
    ms_max = max_over_ranks(ms, dist, dev)
    value = world * args.steps / (ms_max / 1e3)

    # End to end through the public call with host buffers: every step
    # copies the start positions in from pinned host memory, runs the
    # iteration and reads the new positions and statistics back. The host
    # refill of the buffers between steps is outside the timed intervals.
    e2e = None
    if not args.no_e2e:
        try:
            import torch
            ax = torch.empty(c.num_gates, dtype=torch.float32).pin_memory().numpy()
            ay = torch.empty(c.num_gates, dtype=torch.float32).pin_memory().numpy()
            pinned = True
        except Exception:
            ax = np.empty(c.num_gates, np.float32)
            ay = np.empty(c.num_gates, np.float32)
            pinned = False
        e2e_s = 0.0
        for i in range(args.warmup + args.steps):
            ax[...] = x0
            ay[...] = y0
            ctx.synchronize()
            barrier()
            t0 = time.perf_counter()
            d.force_iterate(cfg, 1, ax, ay)
            if i >= args.warmup:
                e2e_s += time.perf_counter() - t0
        e2e_s = max_over_ranks(e2e_s, dist, dev)
        e2e = {"value": world * args.steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": 8 * c.num_gates,
               "d2h_bytes_per_step": 8 * c.num_gates + ITER_STATS_D2H,
               "call": "fx_force_iterate(iters=1) with host x/y"
                       f"{' (pinned)' if pinned else ''} per step"}

    # The whole configured run: `trajectory` iterations from the seeded
    # uniform placement in one call (the reference's math contracts the
    # netlist, so later iterations are cheaper than the timed steps).
    traj = None
    if args.trajectory > 0:
        d.set_positions(p.gate_x, p.gate_y)
        ctx.synchronize()
        ctx.mark(2)
        tst = d.force_iterate(cfg, args.trajectory)
        ctx.mark(3)
        ctx.synchronize()
        tms = ctx.elapsed_ms(2, 3)
        traj = {"iterations": args.trajectory, "value": args.trajectory / (tms / 1e3),
                "unit": UNIT, "final_hpwl": tst.hpwl,
                "final_total_overflow": tst.total_overflow}

    n, m, pn, a = d.n, d.m, d.p, d.a
    G, gc = args.bins, args.cong
    b_alg, f_alg = algorithmic(n, m, pn, a, G, gc)
    per_iter = {k: stages[k][0] / max(stages[k][1], 1) for k in stages if stages[k][1]}
    # the dominant kernel of the step's critical path: the density stage runs
    # on the side stream, overlapped (its own roofline is reported apart)
    dom = max((k for k in per_iter if k != "density"), key=per_iter.get)
    hbm, bf16, src = peaks()
    if dom == "density" and PREC[args.precision] != 3:
        ach = f_alg["density"] / (per_iter[dom] * 1e-3) / 1e12
        peak = bf16 if args.precision == "bf16" else bf16 / 2
        roof = {"bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                "frac": ach / peak, "traffic": NCU_DRAM_BYTES.get(dom), "kernel": dom,
                "peak_source": f"{src} bf16 dense" + ("" if args.precision == "bf16"
                                                      else " / 2 (tf32)")}
    else:
        ach = b_alg[dom] / (per_iter[dom] * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                "frac": ach / hbm, "traffic": NCU_DRAM_BYTES.get(dom), "kernel": dom,
                "algorithmic_bytes": b_alg[dom], "peak_source": f"{src} HBM copy"}
    walk_ncu = NCU_WALK.get(args.bh_walk) if dom == "bh_walk" else None
    if walk_ncu:
        roof["traffic"] = walk_ncu["dram"]
        roof["limiter"] = walk_ncu["limiter"]
    if walk_ncu and args.gates == 1_000_000:
        inst, tpi = walk_ncu["inst"], walk_ncu["tpi"]
        mhz = (clk.get("sm_mhz") or 1965.0) if isinstance(clk, dict) else 1965.0
        peak_i = 4 * 148 * mhz * 1e6
        ach_i = inst / (per_iter[dom] * 1e-3)
        roof["issue"] = {"achieved": ach_i, "peak": peak_i, "unit": "warp inst/s",
                         "frac": ach_i / peak_i, "inst_per_launch": inst,
                         "simt_efficiency": tpi / 32.0,
                         "peak_source": "4 warp instructions per SM per cycle x 148 SMs x "
                                        "median SM clock during the timed region"}
    if args.gates != 1_000_000 or args.bins != 1024 or (dom == "density" and
                                                        args.precision != "3xtf32"):
        roof["traffic"] = None  # the captures are of the default workload
    dens_roof = None
    if "density" in per_iter:
        fl = f_alg["density"] * 6 / 4  # six GEMMs per step (no potential)
        d_tf = fl / (per_iter["density"] * 1e-3) / 1e12
        code = PREC[args.precision]
        halves = code != 0 and args.bins % 256 == 0  # the even/odd half products
        executed = d_tf / 2 if halves else d_tf
        if code == 3:
            pk, ps = 148 * 128 * 2 * 1.965e9 / 1e12, "nominal FP32 CUDA cores 148 x 128 x 2 x 1.965 GHz"
            bound, unit = "fp32-pipe", "TFLOP/s"
        elif code == 4:
            # 21 slice-pair int8 products per GEMM; int8 dense = twice the bf16 rate
            executed *= 21
            pk, ps = 2 * bf16, f"{src} bf16 dense x 2 (int8)"
            bound, unit = "tensor (int8)", "TOPS"
        else:
            pk = bf16 if args.precision == "bf16" else bf16 / 2
            ps = f"{src} bf16 dense" + ("" if args.precision == "bf16" else " / 2 (tf32)")
            bound, unit = "tensor", "TFLOP/s"
        dens_roof = {"bound": bound, "algorithmic_tflops": d_tf, "executed": executed,
                     "unit_executed": unit, "peak": pk, "frac": executed / pk,
                     "peak_source": ps,
                     "flops": "algorithmic: the dense GEMM form, 6 x 2 G^3 per step",
                     "note": ("split in two half-size products by the DCT's even/odd symmetry; "
                              if halves else "") + "side stream, overlapped with Barnes-Hut: its "
                                                   "span includes time it yields"}
    B_iter = sum(b_alg.values())
    it_ms = ms_max / args.steps

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as orc
        orc.build()
        sc.adj = d.adjacency()
        sec, parts = cpu_iteration_sample(sc, x0, y0, G, gc, 1, 16, 256)
        cpu = {"value": 1.0 / sec, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": "one plain iteration at the timed steps' start positions on 1 core: "
                         "attraction/integrate/HPWL (oracle restatement) and scipy DCT in "
                         "full; reference BarnesHutTree.cpp walk of every 16th point and "
                         "congestion of every 256th net, scaled",
               "stage_seconds": {k: round(v, 4) for k, v in parts.items()}}

    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": it_ms,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": PREC_DTYPE[args.precision], "data": "synthetic",
           "config": plain_config(args, pn, a, world),
           "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
           "clocks": clk,
           "iteration_roofline": {"bytes": B_iter, "achieved_gbs": B_iter / (it_ms * 1e-3) / 1e9,
                                  "frac_of_hbm": B_iter / (it_ms * 1e-3) / 1e9 / hbm},
           "stage_ms_per_iter": {k: round(v, 4) for k, v in per_iter.items()},
           "warmup_steps_run": warmup_run,
           "density_roofline": dens_roof,
           "step_hpwl": st.hpwl, "trajectory": traj,
           "bh_walk": ("FX_BH_FAST (hardware rsqrt)" if args.bh_walk == "fast"
                       else "FX_BH_EXACT (bit-reproducible rsqrt)")}
    if rank == 0:
        print(json.dumps(out), flush=True)
    d.close()
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
SERVE_METRIC = "served placement/ECO jobs/s (p50/p99 latency)"


class ServeWorkload:
    """The serving request stream: Poisson arrivals at `rate` for `duration`
    seconds; 70 % PLACE jobs on netlists of log-uniform 5k-500k gates (die side
    1.2 sqrt(N), drawn from a pool of `pool` seeded netlists), 30 % ECO jobs
    that move 1 % of a resident design's gates by N(0, 2 density bins) and run
    50 plain iterations. The first `pool` PLACE jobs keep their designs
    resident as ECO targets."""

    def __init__(self, args, fx):
        rng = np.random.default_rng(args.seed + 1)
        lo, hi = np.log(5_000), np.log(500_000)
        sizes = sorted(int(np.exp(rng.uniform(lo, hi))) for _ in range(args.pool))
        self.circuits = [fx.synth_plain(args.seed + 7 * i, n, int(1.2 * n), 1.2 * float(np.sqrt(n))).circuit
                         for i, n in enumerate(sizes)]
        self.part = fx.part_cfg(mode=fx.FX_PART_FP64, power_iterations=30, tol=0.0)
        t, self.jobs = 0.0, []
        resident = []  # (job index, circuit index)
        while True:
            t += rng.exponential(1.0 / args.rate)
            if t > args.duration:
                break
            if rng.random() < 0.7 or not resident:
                ci = int(rng.integers(len(self.circuits)))
                keep = len(resident) < args.pool
                if keep:
                    resident.append((len(self.jobs), ci))
                self.jobs.append(dict(t=t, kind="place", ci=ci, keep=keep))
            else:
                ji, ci = resident[int(rng.integers(len(resident)))]
                c = self.circuits[ci]
                k = max(1, c.num_gates // 100)
                g = rng.choice(c.num_gates, k, replace=False).astype(np.int32)
                G = min(1024, max(128, int(round(np.sqrt(c.num_gates) / 128.0)) * 128))
                sig = 2.0 * c.chip_width / G
                self.jobs.append(dict(t=t, kind="eco", target=ji, ci=ci, gates=g,
                                      dx=rng.normal(0, sig, k).astype(np.float32),
                                      dy=rng.normal(0, sig, k).astype(np.float32)))

    def desc(self, fx, j, ids):
        if j["kind"] == "place":
            return fx.Server.place_desc(self.circuits[j["ci"]], keep_resident=j["keep"],
                                        part=self.part)
        return fx.Server.eco_desc(ids[j["target"]], j["gates"], j["dx"], j["dy"], iterations=50)

    def bytes_in(self, j):
        c = self.circuits[j["ci"]]
        if j["kind"] == "place":
            return 4 * (c.num_nets + 1) + 4 * c.num_pins + 8 * c.num_gates
        return 12 * len(j["gates"])


def _pct(v, q):
    return float(np.percentile(np.asarray(v), q)) if len(v) else None


def run_serve(args, rank, world, local_rank):
    """Open-loop serving run (arrivals at their Poisson times, results polled
    as they finish), then the same jobs one at a time on one slot (the serial
    GPU baseline); each job's HPWL must agree between the two."""
    import threading
    import fluxion_b200 as fx
    if world > 1:
        args.seed += 1000 * rank
    wl = ServeWorkload(args, fx)
    n_jobs = len(wl.jobs)

    def served(slots, open_loop, scale=1.0):
        sv = fx.Server(device=local_rank, slots=slots)
        ids, res = {}, {}
        try:
            # warm-up: one PLACE per pool netlist size class is not needed;
            # load the kernels once with a small job outside the timing
            sv.submit(fx.Server.place_desc(wl.circuits[0], part=wl.part))
            sv.poll(-1)
            launches0 = sv.stats()["launches"]
            t0 = time.perf_counter()
            if open_loop:
                err = []

                def submitter():
                    try:
                        for i, j in enumerate(wl.jobs):
                            delay = t0 + j["t"] * scale - time.perf_counter()
                            if delay > 0:
                                time.sleep(delay)
                            ids[i] = sv.submit(wl.desc(fx, j, ids))
                    except Exception as e:  # reported after the run
                        err.append(e)

                th = threading.Thread(target=submitter)
                th.start()
                while len(res) < n_jobs and not (err and not th.is_alive() and
                                                 len(res) >= len(ids)):
                    r = sv.poll(100)
                    if r is not None:
                        res[r["job_id"]] = r
                th.join()
                if err:
                    raise err[0]
            else:
                for i, j in enumerate(wl.jobs):
                    ids[i] = sv.submit(wl.desc(fx, j, ids))
                    r = sv.poll(-1)
                    res[r["job_id"]] = r
            wall = time.perf_counter() - t0
            launches = sv.stats()["launches"] - launches0
        finally:
            sv.close()
        out = [res[ids[i]] for i in range(n_jobs)]
        return out, wall, launches

    clocks = ClockSampler(local_rank)
    mix, wall_mix, launches = served(args.slots, True)
    clk = clocks.stop()
    ser, wall_ser, _ = served(1, False)
    # the same arrivals stretched to ~70 % of the capacity the first run
    # reached (when it was overloaded), so the latencies are service, not queue
    offered = n_jobs / args.duration
    cap = n_jobs / wall_mix
    load70 = None
    if offered > 0.7 * cap:
        scale = offered / (0.7 * cap)
        m70, wall70, _ = served(args.slots, True, scale)
        lat70 = [1e3 * (r["end_s"] - r["submit_s"]) for r in m70]
        load70 = {"offered_rate": n_jobs / (args.duration * scale), "jobs_s": n_jobs / wall70,
                  "p50": _pct(lat70, 50), "p99": _pct(lat70, 99),
                  "eco_p50": _pct([l for l, j in zip(lat70, wl.jobs) if j["kind"] == "eco"], 50),
                  "place_p50": _pct([l for l, j in zip(lat70, wl.jobs)
                                     if j["kind"] == "place"], 50),
                  "hpwl_max_rel_diff_vs_serial": max(
                      abs(a["hpwl"] - b["hpwl"]) / max(abs(b["hpwl"]), 1e-30)
                      for a, b in zip(m70, ser))}
        mix = mix + m70  # both served runs are checked below
    bad = [r for r in mix + ser if r["status"] != 0]
    if bad:
        raise RuntimeError(f"{len(bad)} serving jobs failed: {bad[0]['error']}")
    mix = mix[:n_jobs]
    lat = [1e3 * (r["end_s"] - r["submit_s"]) for r in mix]
    svc = [1e3 * (r["end_s"] - r["start_s"]) for r in ser]
    rel = max(abs(a["hpwl"] - b["hpwl"]) / max(abs(b["hpwl"]), 1e-30) for a, b in zip(mix, ser))
    jobs_s = n_jobs / wall_mix
    serial_s = n_jobs / wall_ser
    if world > 1:
        import torch.distributed as tdist
        jobs_s = replica_throughput(n_jobs, wall_mix, tdist, f"cuda:{local_rank}")
    kinds = [j["kind"] for j in wl.jobs]
    bin_ = sum(wl.bytes_in(j) for j in wl.jobs) / n_jobs
    out = {"metric": SERVE_METRIC, "value": jobs_s, "unit": "jobs/s", "n_gpus": world,
           "steps": n_jobs, "warmup": 1, "ms_per_step": 1e3 * wall_mix / n_jobs,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32 (FP64 HPWL/reductions)", "data": "synthetic",
           "config": {"workload": f"serve: Poisson {args.rate:g} req/s for {args.duration:g} s, "
                      f"70% PLACE (partition FP64-30 + leaves + refine) on {args.pool} netlists "
                      f"of 5k-500k gates, 30% ECO (1% moves, 50 plain iterations)",
                      "slots": args.slots, "jobs": n_jobs, "place": kinds.count("place"),
                      "eco": kinds.count("eco"), "seed": args.seed,
                      "pool_gates": [c.num_gates for c in wl.circuits]},
           "latency_ms": {"p50": _pct(lat, 50), "p90": _pct(lat, 90), "p99": _pct(lat, 99),
                          "max": max(lat)},
           "offered_rate": n_jobs / args.duration,
           "latency_at_70pct_load_ms": load70,
           "serial": {"value": serial_s, "unit": "jobs/s",
                      "service_ms": {"p50": _pct(svc, 50), "p99": _pct(svc, 99)},
                      "how": "same jobs, one at a time on one slot (closed loop)"},
           "service_ms_by_kind": {
               k: {"n": sum(1 for j in wl.jobs if j["kind"] == k),
                   "serial_p50": _pct([1e3 * (r["end_s"] - r["start_s"]) for r, j in
                                       zip(ser, wl.jobs) if j["kind"] == k], 50),
                   "serial_mean": float(np.mean([1e3 * (r["end_s"] - r["start_s"])
                                                 for r, j in zip(ser, wl.jobs)
                                                 if j["kind"] == k] or [0.0])),
                   "served_p50": _pct([1e3 * (r["end_s"] - r["start_s"]) for r, j in
                                       zip(mix, wl.jobs) if j["kind"] == k], 50)}
               for k in ("place", "eco")},
           "speedup_vs_serial": jobs_s / serial_s,
           "hpwl_max_rel_diff_vs_serial": rel,
           "e2e": {"value": jobs_s, "unit": "jobs/s", "h2d_bytes_per_step": bin_,
                   "d2h_bytes_per_step": 248,
                   "call": "fx_serve_submit/fx_serve_poll with host netlists and moves"},
           "gpu_launches": launches, "clocks": clk}
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_serve_reference(args, rank, world):
    """The reference's CPU flow for the same jobs on a bounded sample: PLACE =
    build_adjacency + build_hierarchy + place_gates_in_leaf per leaf + refine
    (the oracle's restatements of main.rs:74-111); ECO = one plain iteration
    on the CPU path (attraction, Barnes-Hut via BarnesHutTree.cpp, scipy DCT,
    congestion) scaled to 50. Jobs are taken in order until ~20 s."""
    if rank != 0:
        return
    import fluxion_b200 as fx
    from oracle import oracle as orc
    orc.build()
    wl = ServeWorkload(args, fx)
    threads = os.cpu_count() or 1
    done, spent, adj = 0, 0.0, {}
    for j in wl.jobs:
        if spent > 20.0 and done > 0:
            break
        c = wl.circuits[j["ci"]]
        t0 = time.perf_counter()
        if j["ci"] not in adj:
            adj[j["ci"]] = orc.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
        ap, ai = adj[j["ci"]]
        if j["kind"] == "place":
            tr = orc.build_hierarchy(c.num_gates, ap, ai, c.chip_width, c.chip_height)
            x = np.zeros(c.num_gates, np.float32)
            y = np.zeros(c.num_gates, np.float32)
            lp, lg = tr["leaf_ptr"], tr["leaf_gate"]
            for l in range(len(lp) - 1):
                orc.place_leaf(lg[lp[l]:lp[l + 1]], ap, ai, tr["region"][l], 50,
                               out_x=x, out_y=y)
            # one refine iteration (two congestion passes), scaled to the 30
            # the GPU runs typically take: the reference counts every cell of
            # every net's bounding box, seconds per pass at 100k gates
            t1 = time.perf_counter()
            orc.refine(c.net_ptr, c.net_gate, x, y, c.chip_width, c.chip_height, max_iters=1)
            spent += (time.perf_counter() - t1) * (30.0 / 2.0 - 1.0)
        else:
            x = np.random.default_rng(0).uniform(0, c.chip_width, c.num_gates).astype(np.float32)
            y = np.random.default_rng(1).uniform(0, c.chip_height, c.num_gates).astype(np.float32)

            class S:
                pass
            sc = S()
            sc.circuit, sc.adj = c, (ap, ai)
            G = min(1024, max(128, int(round(np.sqrt(c.num_gates) / 128.0)) * 128))
            sec, _ = cpu_iteration_sample(sc, x, y, G, 256, threads, 16, 64)
            spent += 49 * sec  # 50 iterations, one measured
        spent += time.perf_counter() - t0
        done += 1
    value = done / spent
    out = {"metric": SERVE_METRIC, "value": value, "unit": "jobs/s", "impl": "reference",
           "n_gpus": world, "steps": done, "warmup": 0, "ms_per_step": 1e3 * spent / done,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic",
           "config": {"workload": "serve (same job stream as --impl fluxion)", "seed": args.seed},
           "cpu_baseline": {"value": value, "unit": "jobs/s", "cores": threads, "kind": "port",
                            "sample": f"the first {done} jobs of the stream, run one after "
                                      "another on the CPU (PLACE: hierarchy and leaves in "
                                      "full, refine as 1 iteration scaled to 30; ECO: 1 of "
                                      "50 plain iterations timed, scaled)"},
           "e2e": {"value": value, "unit": "jobs/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
LEAF_METRIC = "batched leaf placement: cluster-iterations/s"


def run_leaves(args, rank, world, local_rank):
    """Batched leaf placement (16,384 clusters of log-uniform 16-128 gates,
    1.5 nets/gate of degree 2-8, unit boxes, 300 iterations): one step = one
    fx_hapr_place_leaves call over all clusters. `value` from the kernel's
    device time (CUDA events on its stream), `e2e` from the whole call (host
    leaf lists in, positions out); the per-cluster-launch schedule and the
    CPU restatement of place_gates_in_leaf (placer.rs:210-287) beside it."""
    import fluxion_b200 as fx
    syn = fx.synth_leaves(args.seed + rank, args.clusters, 16, 128, 1.5)
    c = syn.circuit
    lp, region = syn.leaf_ptr, syn.region
    lg = np.arange(c.num_gates, dtype=np.int32)
    sizes = np.diff(lp).astype(np.int64)
    pairs = int((sizes * (sizes - 1) // 2).sum())
    # the call uploads the caller's lists and positions plus what it derives:
    # the in-leaf adjacency (row offsets, int16 neighbour slots) and the order
    ap_all, ai_all = fx.build_adjacency(c)
    leaf_of = np.empty(c.num_gates, np.int64)
    leaf_of[lg] = np.repeat(np.arange(len(sizes)), sizes)
    in_leaf = int((leaf_of[np.repeat(np.arange(c.num_gates), np.diff(ap_all))]
                   == leaf_of[ai_all]).sum())
    h2d_bytes = (4 * (len(lp) + c.num_gates) + 16 * args.clusters + 8 * c.num_gates
                 + 4 * (c.num_gates + 1) + 2 * in_leaf + 4 * args.clusters)
    ctx = fx.Context(local_rank)
    d = fx.Design(ctx, c)
    fast = args.leaf_precision == "fast"
    cfg = fx.leaf_cfg(force_iterations=args.leaf_iters, schedule=args.leaf_schedule,
                      precision=fx.FX_LEAF_FAST if fast else fx.FX_LEAF_IEEE)
    x, y, sched = d.place_leaves(lp, lg, region, cfg)  # tunes the schedule unless given
    cfg.schedule = sched
    for _ in range(max(0, args.warmup - 1)):
        d.place_leaves(lp, lg, region, cfg)
    ctx.synchronize()
    ctx.reset_stage_times()
    ctx.set_profiling(True)
    launches0 = ctx.kernel_launches()
    clocks = ClockSampler(local_rank)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        x2, y2, _ = d.place_leaves(lp, lg, region, cfg)
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    ctx.set_profiling(False)
    launches = ctx.kernel_launches() - launches0
    kms = ctx.stage_times()["leaf"][0] / args.steps
    assert np.array_equal(x, x2) and np.array_equal(y, y2)
    # per-cluster launches (one launch per leaf), once
    pc_ms, same = None, None
    if not args.no_per_cluster:
        pc = fx.leaf_cfg(force_iterations=args.leaf_iters, schedule=fx.FX_LEAF_PER_CLUSTER,
                         precision=cfg.precision)
        ctx.reset_stage_times()
        ctx.set_profiling(True)
        xp, yp, _ = d.place_leaves(lp, lg, region, pc)
        ctx.set_profiling(False)
        pc_ms = ctx.stage_times()["leaf"][0]
        same = bool(np.array_equal(xp, x) and np.array_equal(yp, y))
    d.close()
    ctx.close()
    units = args.clusters * args.leaf_iters
    ops = 17.0 * pairs * args.leaf_iters  # placer.rs:259-270, per unordered pair
    achieved = ops / (kms * 1e-3) / 1e12
    lane_peak = 148 * 128 * 1.965e9 / 1e12
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as orc
        orc.build()
        ap, ai = fx.build_adjacency(c)
        k = min(args.clusters, 256)
        t1 = time.perf_counter()
        ox = np.zeros(c.num_gates, np.float32)
        oy = np.zeros(c.num_gates, np.float32)
        for l in range(k):
            orc.place_leaf(lg[lp[l]:lp[l + 1]], ap, ai, region[4 * l:4 * l + 4],
                           args.leaf_iters, out_x=ox, out_y=oy)
        sec = (time.perf_counter() - t1) * args.clusters / k
        cpu = {"value": units / sec, "unit": "cluster-iterations/s", "cores": 1, "kind": "port",
               "sample": f"place_gates_in_leaf restated, first {k} of {args.clusters} clusters "
                         "on 1 core, scaled"}
    out = {"metric": LEAF_METRIC, "value": world * units / (kms * 1e-3),
           "unit": "cluster-iterations/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": kms, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": f"leaves: {args.clusters} clusters of 16-128 gates "
                      f"({c.num_gates} gates, {pairs} pairs), {args.leaf_iters} iterations",
                      "schedule": int(sched), "seed": args.seed,
                      "precision": ("FX_LEAF_FAST (hardware rsqrt pair term)" if fast else
                                    "FX_LEAF_IEEE (bit-exact with place_gates_in_leaf)")},
           "roofline": {"bound": "fp32-pipe", "achieved": achieved, "peak": lane_peak,
                        "unit": "Tops/s", "frac": achieved / lane_peak, "traffic": None,
                        "kernel": ("leaf_pairs_kernel" if sched in (
                            fx.FX_LEAF_PAIR64, fx.FX_LEAF_PAIR128, fx.FX_LEAF_PAIR256)
                            else "leaf_batch_kernel"),
                        "peak_source": "nominal 148 SMs x 128 FP32 lanes x 1.965 GHz, 17 ops "
                                       "per unordered pair"},
           "per_cluster_launches_ms": pc_ms,
           "speedup_vs_per_cluster": None if pc_ms is None else pc_ms / kms,
           "same_result_as_per_cluster": same, "cpu_baseline": cpu,
           "e2e": {"value": world * units * args.steps / wall, "unit": "cluster-iterations/s",
                   "h2d_bytes_per_step": h2d_bytes,
                   "d2h_bytes_per_step": 8 * c.num_gates,
                   "call": "fx_hapr_place_leaves with host leaf lists and regions (the "
                           "in-leaf adjacency it derives on the host is uploaded too)"},
           "gpu_launches": launches, "clocks": clk}
    if rank == 0:
        print(json.dumps(out), flush=True)


PREC_METRIC = "density solve precision sweep (field/force rel. L2 vs FP64, tensor TFLOP/s)"
# plain iterations after which the HPWL delta is reported, in one run: the
# reference's plain iteration contracts the netlist within ~100 iterations and
# amplifies small differences on the way, so early counts show the solve's
# precision and later ones the divergence of the trajectories
HPWL_ITERS = (3, 10, 50)


def run_precision(args, rank, world, local_rank):
    """The density step's precision sweep on a 4M-gate netlist from the same
    generator (die 2400 x 2400): for G = 2048 and 4096 and each DCT precision
    (BF16, TF32, 3xTF32, SIMT FP32; FP32 accumulation throughout), the
    field / force / potential relative L2 error against the FP64 FFT oracle
    (scipy dctn/idctn of force_electrostatic.py), the density stage's device
    time and GEMM throughput, and the HPWL of a plain run against the SIMT
    FP32 run after each count of HPWL_ITERS. HPWL and energy are FP64
    reductions on the device."""
    if rank != 0:
        return
    import fluxion_b200 as fx
    from oracle import oracle as orc
    t_start = time.perf_counter()
    n = 4_000_000
    s = fx.synth_plain(args.seed, n, int(1.2 * n), 2400.0)
    c, p = s.circuit, s.placement
    ctx = fx.Context(local_rank)
    d = fx.Design(ctx, c)
    d.set_positions(p.gate_x, p.gate_y)
    area = (c.gate_widths * c.gate_heights).astype(np.float64)
    codes = {"bf16": fx.FX_DCT_BF16, "tf32": fx.FX_DCT_TF32, "3xtf32": fx.FX_DCT_FP32,
             "i8_slices": fx.FX_DCT_I8, "fp32_simt": fx.FX_DCT_SIMT}
    _, bf16_peak, src = peaks()

    def rel(a, b):
        return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))

    rows = []
    print(f"precision sweep: set-up {time.perf_counter() - t_start:.1f} s", file=sys.stderr,
          flush=True)
    for G in (2048, 4096):
        ref = orc.density_forces(p.gate_x, p.gate_y, area, c.chip_width, c.chip_height, G,
                                 0.7, 1.0)
        hp = {}
        for name, code in codes.items():
            t_phase = time.perf_counter()
            d.set_positions(p.gate_x, p.gate_y)  # the oracle's positions
            out = d.density(G, 0.7, 1.0, code, grids=True)
            ctx.reset_stage_times()
            ctx.set_profiling(True)
            reps = 3
            for _ in range(reps):
                d.density(G, 0.7, 1.0, code)
            ctx.set_profiling(False)
            ms = ctx.stage_times()["density"][0] / reps
            # executed: the even/odd half GEMMs (G a multiple of 256, not
            # 3xTF32) do G^3 each instead of 2 G^3; 3xTF32 runs three MMAs
            # (FX_DCT_I8: 21 8-bit slice-pair products per GEMM, int8 ops)
            halves = G % 256 == 0 and code != fx.FX_DCT_FP32
            flops = 6 * (1.0 if halves else 2.0) * G ** 3 * (
                3 if code == fx.FX_DCT_FP32 else 21 if code == fx.FX_DCT_I8 else 1)
            fld = float(np.sqrt((np.linalg.norm(out["ex"] - ref["ex"]) ** 2 +
                                 np.linalg.norm(out["ey"] - ref["ey"]) ** 2) /
                                (np.linalg.norm(ref["ex"]) ** 2 + np.linalg.norm(ref["ey"]) ** 2)))
            frc = float(np.sqrt((np.linalg.norm(out["fx"] - ref["fx"]) ** 2 +
                                 np.linalg.norm(out["fy"] - ref["fy"]) ** 2) /
                                (np.linalg.norm(ref["fx"]) ** 2 + np.linalg.norm(ref["fy"]) ** 2)))
            cfg = fx.iter_cfg(density_bins=G, dct_precision=code, density_weight=1e-4,
                              cong_cols=512, cong_rows=512)
            x0, y0 = p.gate_x.copy(), p.gate_y.copy()
            hpwl_at, done = {}, 0
            for it in HPWL_ITERS:  # one run, continued on the device
                st = (d.force_iterate(cfg, it, x0, y0) if done == 0
                      else d.force_iterate(cfg, it - done))
                done = it
                hpwl_at[it] = st.hpwl
            hp[name] = hpwl_at
            print(f"precision sweep: G={G} {name}: {time.perf_counter() - t_phase:.1f} s",
                  file=sys.stderr, flush=True)
            # int8 dense: twice the bf16 rate (nominal ratio); tf32: half
            peak = (bf16_peak if code == fx.FX_DCT_BF16 else
                    2 * bf16_peak if code == fx.FX_DCT_I8 else bf16_peak / 2)
            rows.append({"G": G, "precision": name, "field_rel_l2": fld, "force_rel_l2": frc,
                         "phi_rel_l2": rel(out["phi"], ref["phi"]),
                         "energy_rel": abs(out["energy"] - ref["energy"]) / abs(ref["energy"]),
                         "density_ms": ms,
                         "tensor_tflops_executed": (flops / (ms * 1e-3) / 1e12
                                                    if code != fx.FX_DCT_SIMT else None),
                         "tensor_frac_of_measured": (flops / (ms * 1e-3) / 1e12 / peak
                                                     if code != fx.FX_DCT_SIMT else None),
                         "hpwl_after_iters": {str(k): v for k, v in hpwl_at.items()}})
        for r in rows:
            if r["G"] == G:
                r["hpwl_delta_vs_fp32"] = {
                    str(it): (hp[r["precision"]][it] - hp["fp32_simt"][it]) / hp["fp32_simt"][it]
                    for it in HPWL_ITERS}
    d.close()
    ctx.close()
    best = max((r for r in rows if r["G"] == 4096 and r["tensor_tflops_executed"]),
               key=lambda r: r["tensor_tflops_executed"])
    out = {"metric": PREC_METRIC, "value": best["tensor_tflops_executed"], "unit": "TFLOP/s",
           "n_gpus": 1, "steps": 3, "warmup": 1, "ms_per_step": best["density_ms"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "bf16/tf32/3xtf32/fp32 (FP32 accumulate), int8 slices (int32 accumulate)",
           "data": "synthetic",
           "config": {"workload": f"precision: {n} gates, die 2400, G in (2048, 4096), "
                                  "target density 0.7, weight 1", "seed": args.seed,
                      "peak_source": f"{src} bf16 dense (tf32: half, int8: twice)"},
           "value_is": f"{best['precision']} at G=4096, executed tensor FLOP/s of the 6 GEMMs",
           "sweep": rows}
    print(json.dumps(out), flush=True)


SMALL_METRIC = "plain-small run (10k gates, 200 iterations): iterations/s"


def run_small(args, rank, world, local_rank):
    """BASELINE config 1 in full: 10,000 gates, 12,000 nets, die 120 x 120,
    200 iterations of attraction (k = 1) + Barnes-Hut (theta 0.5) + damped
    step with 64 x 64 congestion, on the GPU and in the oracle (one core);
    the two runs must end on identical positions."""
    if rank != 0:
        return
    import fluxion_b200 as fx
    from oracle import oracle as orc
    orc.build()
    sy = fx.synth_plain(args.seed, 10_000, 12_000, 120.0)
    c, p = sy.circuit, sy.placement
    iters = 200
    cfg = fx.iter_cfg(density_bins=0, cong_cols=64, cong_rows=64, bh_walk=fx.FX_BH_EXACT)
    ctx = fx.Context(local_rank)
    d = fx.Design(ctx, c)
    x, y = p.gate_x.copy(), p.gate_y.copy()
    d.force_iterate(cfg, iters, x, y)  # warm-up (allocations, graph path)
    runs = []
    for _ in range(max(3, args.warmup)):
        x, y = p.gate_x.copy(), p.gate_y.copy()
        ctx.synchronize()
        t0 = time.perf_counter()
        st = d.force_iterate(cfg, iters, x, y)
        runs.append(time.perf_counter() - t0)
    d.close()
    ctx.close()
    gpu_s = float(np.median(runs))
    rp, ri = orc.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
    ox, oy = p.gate_x.copy(), p.gate_y.copy()
    vx, vy = np.zeros_like(ox), np.zeros_like(oy)
    t0 = time.perf_counter()
    for _ in range(iters):
        fa_x, fa_y = orc.attraction_f32(rp, ri, ox, oy, 1.0)
        b = orc.bh_forces(ox, oy, 0.5, 0.5, float(np.float32(0.1)))
        orc.integrate(ox, oy, vx, vy, fa_x + b["fx32"], fa_y + b["fy32"], 0.1, 0.9,
                      (0.0, 0.0, c.chip_width, c.chip_height))
        orc.congestion(c.net_ptr, c.net_gate, ox, oy, c.chip_width, c.chip_height, 64, 64)
    cpu_s = time.perf_counter() - t0
    same = bool(np.array_equal(ox, x) and np.array_equal(oy, y))
    out = {"metric": SMALL_METRIC, "value": iters / gpu_s, "unit": "iterations/s", "n_gpus": 1,
           "steps": len(runs), "warmup": 1, "ms_per_step": 1e3 * gpu_s / iters,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic",
           "config": {"workload": "plain-small: 10000 gates, 12000 nets, die 120, BH theta 0.5, "
                                  "congestion 64^2, 200 iterations (one call)", "seed": args.seed},
           "positions_identical_to_oracle": same, "final_hpwl": st.hpwl,
           "cpu_baseline": {"value": iters / cpu_s, "unit": "iterations/s", "cores": 1,
                            "kind": "port", "sample": "the same 200 iterations in full "
                                                      "(oracle restatement, 1 core)"},
           "e2e": {"value": iters / gpu_s, "unit": "iterations/s",
                   "h2d_bytes_per_step": 8 * c.num_gates / iters,
                   "d2h_bytes_per_step": (8 * c.num_gates + 32) / iters,
                   "call": "fx_force_iterate(iters=200) with host x/y"}}
    print(json.dumps(out), flush=True)


ATTN_METRIC = "attention passes/s (compute_all_attention over the hierarchy, top-10)"
ATTN_TOP_K = 10


def attention_setup(args, rank):
    """The plain netlist, its device hierarchy (default partition config) and
    the levels with at least two clusters, as host CSR lists."""
    import fluxion_b200 as fx
    syn = fx.synth_plain(args.seed + rank, args.gates, args.nets, args.die)
    return syn, fx


def attention_levels(fx, d):
    tree = d.partition(fx.part_cfg())
    lv = fx.hierarchy_levels(tree["leaf_ptr"], tree["leaf_gate"], tree["leaf_depth"])
    return tree, [(t, cp, cg) for t, (cp, cg) in enumerate(lv) if len(cp) - 1 >= 2]


def attention_cpu_sample(c, levels, k_max=16):
    """compute_level_attention restated in C++ with hash sets, on k sampled
    clusters per level, scaled to the whole level by the cost of each phase:
    net sets (one scan of every net per cluster) x n/k, intersections x
    n(n-1)/(k(k-1)), top-k sorts x n/k. Returns (seconds per pass, sample)."""
    from oracle import oracle as orc
    orc.build()
    total, samp = 0.0, 0
    for _, cp, cg in levels:
        n = len(cp) - 1
        k = min(n, k_max)
        rows = np.linspace(0, n - 1, k).round().astype(np.int32)
        rows = np.unique(rows)
        k = len(rows)
        _, _, t = orc.attention_sample(c.net_ptr, c.net_gate, cp, cg, rows, ATTN_TOP_K)
        total += t[0] * n / k + t[1] * (n * (n - 1)) / max(k * (k - 1), 1) + t[2] * n / k
        samp += k
    return total, samp


def run_attention(args, rank, world, local_rank):
    """(f.4) attention scores, compute_all_attention (attention.rs:33-48),
    over every level of the plain netlist's hierarchy: one step = one
    fx_attention_tree call with the host leaf lists in and every level's
    top-10 lists out. `value` from the device time of the levels (stage
    events), `e2e` from the call's wall time; the dense n x n score matrices
    are not requested (fx_attention returns them per level on request)."""
    syn, fx = attention_setup(args, rank)
    c = syn.circuit
    ctx = fx.Context(local_rank)
    d = fx.Design(ctx, c)
    tree, levels = attention_levels(fx, d)
    first = d.attention(tree, ATTN_TOP_K)
    for _ in range(max(0, args.warmup - 1)):
        d.attention(tree, ATTN_TOP_K)
    ctx.synchronize()
    ctx.reset_stage_times()
    ctx.set_profiling(True)
    launches0 = ctx.kernel_launches()
    clocks = ClockSampler(local_rank)
    t0 = time.perf_counter()
    same = True
    for _ in range(args.steps):
        got = d.attention(tree, ATTN_TOP_K)
        same = same and all(np.array_equal(a["top_k"], b["top_k"]) for a, b in zip(got, first))
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    ctx.set_profiling(False)
    launches = ctx.kernel_launches() - launches0
    dev_ms = ctx.stage_times()["attention"][0] / args.steps
    n_cl = [len(cp) - 1 for _, cp, _ in levels]
    d.close()
    ctx.close()
    # algorithmic bytes of one pass: per level, the pin lists read once
    # (net_ptr, net_gate), each pin's cluster (one 4-byte gather), the level's
    # cluster lists and the top-k lists written
    p = int(c.net_ptr[-1])
    alg = sum(4 * (c.num_nets + 1) + 8 * p + 4 * (len(cp) + len(cg)) + 4 * (len(cp) - 1)
              * ATTN_TOP_K for _, cp, cg in levels)
    hbm, _, peak_src = peaks()
    achieved = alg / (dev_ms * 1e-3) / 1e9
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        sec, k = attention_cpu_sample(c, levels)
        cpu = {"value": 1.0 / sec, "unit": "passes/s", "cores": 1, "kind": "port",
               "sample": f"{k} sampled clusters over {len(levels)} levels through the C++ "
                         "hash-set restatement of compute_level_attention, each phase scaled "
                         "to the whole level"}
    L = len(tree["leaf_ptr"]) - 1
    h2d = 4 * (2 * L + 1 + len(tree["leaf_gate"])) + 4 * L * len(levels)
    d2h = sum(4 * n * ATTN_TOP_K for n in n_cl)
    out = {"metric": ATTN_METRIC, "value": world * 1e3 / dev_ms, "unit": "passes/s",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
           "data": "synthetic",
           "config": {"workload": f"attention: {args.gates} gates, {args.nets} nets, "
                                  f"{len(levels)} levels of 2..{max(n_cl)} clusters, top "
                                  f"{ATTN_TOP_K}", "seed": args.seed,
                      "l2": "inputs (pins, pair keys) larger than L2 at the deep levels"},
           "levels": n_cl, "same_result_every_step": bool(same), "cpu_baseline": cpu,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                        "frac": achieved / hbm, "traffic": None,
                        "kernel": "all kernels of a pass (stage events)",
                        "algorithmic_bytes_per_pass": alg, "peak_source": peak_src,
                        "limiter": "shared-memory atomics and dependent loads of the "
                                   "per-row counting (attn_rows_kernel), not bandwidth"},
           "e2e": {"value": world * args.steps / wall, "unit": "passes/s",
                   "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                   "call": "fx_attention_tree with the host leaf lists (one call per pass)"},
           "gpu_launches": launches, "clocks": clk}
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_attention_reference(args, rank, world):
    """The reference's single-threaded compute_all_attention restated in C++
    (hash sets), timed on a bounded sample of clusters per level and scaled."""
    if rank != 0:
        return
    import fluxion_b200 as fx
    from oracle import oracle as orc
    syn = fx.synth_plain(args.seed, args.gates, args.nets, args.die)
    c = syn.circuit
    ap, ai = orc.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
    t = orc.build_hierarchy(c.num_gates, ap, ai, c.chip_width, c.chip_height)
    lv = fx.hierarchy_levels(t["leaf_ptr"], t["leaf_gate"], t["leaf_depth"])
    levels = [(d, cp, cg) for d, (cp, cg) in enumerate(lv) if len(cp) - 1 >= 2]
    per = []
    for i in range(args.warmup + args.steps):
        sec, k = attention_cpu_sample(c, levels, k_max=8)
        if i >= args.warmup:
            per.append(sec)
    sec = float(np.mean(per))
    out = {"metric": ATTN_METRIC, "value": 1.0 / sec, "unit": "passes/s", "impl": "reference",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
           "data": "synthetic",
           "config": {"workload": f"attention: {args.gates} gates, {args.nets} nets, "
                                  f"{len(levels)} levels, top {ATTN_TOP_K}", "seed": args.seed},
           "cpu_baseline": {"value": 1.0 / sec, "unit": "passes/s", "cores": 1, "kind": "port",
                            "sample": f"{k} sampled clusters per pass (the oracle's hierarchy), "
                                      "each phase scaled to the whole level"},
           "e2e": {"value": 1.0 / sec, "unit": "passes/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_leaves_reference(args, rank, world):
    """place_gates_in_leaf (placer.rs:210-287, the oracle's restatement) over
    the same clusters on all host threads, on a bounded sample of clusters."""
    if rank != 0:
        return
    from concurrent.futures import ThreadPoolExecutor
    import fluxion_b200 as fx
    from oracle import oracle as orc
    orc.build()
    syn = fx.synth_leaves(args.seed, args.clusters, 16, 128, 1.5)
    c, lp, region = syn.circuit, syn.leaf_ptr, syn.region
    lg = np.arange(c.num_gates, dtype=np.int32)
    ap, ai = fx.build_adjacency(c)
    threads = os.cpu_count() or 1
    ox = np.zeros(c.num_gates, np.float32)
    oy = np.zeros(c.num_gates, np.float32)

    def one(l):  # ctypes releases the GIL during the call
        orc.place_leaf(lg[lp[l]:lp[l + 1]], ap, ai, region[4 * l:4 * l + 4], args.leaf_iters,
                       out_x=ox, out_y=oy)

    k = min(args.clusters, 64 * threads)
    per = []
    with ThreadPoolExecutor(threads) as ex:
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            list(ex.map(one, range(k)))
            if i >= args.warmup:
                per.append((time.perf_counter() - t0) * args.clusters / k)
    sec = float(np.mean(per))
    value = args.clusters * args.leaf_iters / sec
    out = {"metric": LEAF_METRIC, "value": value, "unit": "cluster-iterations/s",
           "impl": "reference", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": 1e3 * sec, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": f"leaves: {args.clusters} clusters, {args.leaf_iters} "
                                  "iterations", "seed": args.seed},
           "cpu_baseline": {"value": value, "unit": "cluster-iterations/s", "cores": threads,
                            "kind": "port", "sample": f"first {k} clusters per step on "
                                                      f"{threads} threads, scaled"},
           "e2e": {"value": value, "unit": "cluster-iterations/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.workload == "small":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "metric": SMALL_METRIC,
                              "unavailable": "timed in full as cpu_baseline of the fluxion arm"}))
            return
        run_small(args, rank, world, local_rank)
        return
    if args.workload == "precision":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "metric": PREC_METRIC,
                              "unavailable": "the FP64 oracle is part of the fluxion arm's "
                                             "line (error baseline, not a timed arm)"}))
            return
        run_precision(args, rank, world, local_rank)
        return
    if args.workload == "leaves":
        args.steps = max(1, min(args.steps, 20))  # a step is a whole 300-iteration batch
        if args.impl == "reference":
            run_leaves_reference(args, rank, world)
            return
        run_leaves(args, rank, world, local_rank)
        return
    if args.workload == "attention":
        args.steps = max(1, min(args.steps, 50))
        if args.impl == "reference":
            args.steps, args.warmup = min(args.steps, 3), min(args.warmup, 1)
            run_attention_reference(args, rank, world)
            return
        run_attention(args, rank, world, local_rank)
        return
    if args.workload == "serve":
        if args.impl == "reference":
            run_serve_reference(args, rank, world)
        else:
            if world > 1:
                import torch
                import torch.distributed as tdist
                torch.cuda.set_device(local_rank)
                tdist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
            run_serve(args, rank, world, local_rank)
            if world > 1:
                tdist.barrier()
                tdist.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_fluxion(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
