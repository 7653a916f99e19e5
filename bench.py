"""Benchmark of the multichannel VEGAS hot path (2->4, 15 channels, 100 bins,
1e6 accepted points per iteration) on B200, and of the reference's own CPU
implementation of the same workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl chili|reference]
                    [--workload multichannel|batched]

One step = one MultiChannel::operator() iteration: 1e6 accepted points
(generation, PreProcess, combined weight over all 15 channels, integrand,
StatsData, per-channel grid histograms and alpha training) followed by the
alpha and grid adaptation.  The PreProcess is the physical region with the
usual cuts (incoming momentum fractions <= 1, pT > 30 GeV, |eta| < 99,
Delta R > 0.4), where every channel covers the same phase space.  After the
plain path, the learned proposal (spline flow + channel-weight network) is
trained on the GPU and measured on the same integrand; the line reports both
paths and selects the one with the lower variance x time per point.  Rank 0
prints one JSON line.

--workload batched: 512 uneven integrands (camel functions and 2->n
multichannel integrands) advanced together, one persistent graph-replayed
launch per iteration; one step = one adapting iteration of every task.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

TIMED_KERNELS = ["k_mc_forward", "k_pp_nodes", "k_pp_items", "k_pp_chains", "k_pp_channel", "k_pp_combine",
                 "k_mc_weight", "k_mc_accum"]
FLOW_KERNELS = ["k_flow_layer", "k_flow_layer_bwd", "k_flow_wgrad", "k_alpha_train", "k_alpha_eval", "k_flow_phys",
                "k_flow_batch", "k_pp_nodes", "k_pp_items", "k_pp_chains", "k_pp_channel"]
METRIC = "time to 0.1% error & unweighted events/s: flow vs plain VEGAS, 1 B200, FP64"
UNIT = "unweighted events/s"
SEED = 7

# The two multichannel workloads: the 2->4 iteration (the headline) and the
# large 2->6 case. channels(): the channel set; fkind: the integrand.
WORKLOADS = {
    "multichannel": {"n_out": 4, "bins": 100, "ncalls": 1_000_000, "fkind": "PROPAGATOR", "flow_layers": 6,
                     "flow_hidden": 128, "flow_depth": 2,
                     "metric": METRIC, "dims": 10, "channels": 15,
                     "describe": "multichannel 2->4 propagator integrand, sqrt(S)=1 TeV, 10 dims",
                     "unweighted_target": None},
    "large": {"n_out": 6, "bins": 200, "ncalls": 10_000_000, "fkind": "PROPAGATOR_TOP2", "flow_layers": 10,
              "flow_hidden": 256, "flow_depth": 3,
              "metric": "time to 0.1% error & unweighting efficiency, 2->6 (45 channels, 200 bins, 1e7 "
                        "points/iteration): flow vs plain VEGAS, 1 B200, FP64",
              "dims": 16, "channels": 45,
              "describe": "multichannel 2->6, product of the two largest pair propagators x t-channel factors, "
                          "sqrt(S)=1 TeV, 16 dims",
              "unweighted_target": 1_000_000},
}
WL = WORKLOADS["multichannel"]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="chili", choices=["chili", "reference"])
    ap.add_argument("--ncalls", type=int, default=None, help="points per iteration (default: the workload's)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-flow", action="store_true")
    ap.add_argument("--flow-steps", type=int, default=200)
    ap.add_argument("--flow-batch", type=int, default=65536)
    ap.add_argument("--flow-long-steps", type=int, default=600,
                    help="also train a second flow this many steps and report it beside the 200-step one "
                         "(0: skip)")
    ap.add_argument("--workload", default="multichannel", choices=["multichannel", "large", "batched", "vegas"],
                    help="multichannel: the 2->4 iteration with the learned proposal beside it; large: the "
                         "2->6 case (45 channels, 200 bins, 1e7 points per iteration, 10-layer flow, 1e6 "
                         "unweighted events); batched: 512 uneven integrands in one persistent graph-replayed "
                         "launch per iteration; vegas: plain VEGAS on the 4-d camel (50 bins, 1e5 points per "
                         "iteration) and its materialised points")
    ap.add_argument("--batch-scale", type=float, default=1.0,
                    help="batched: point counts times this factor (small cases for profiling)")
    ap.add_argument("--no-sequential", action="store_true",
                    help="batched: skip the one-call-per-task comparison")
    ap.add_argument("--gen-points", type=int, default=100_000_000,
                    help="vegas: points per launch of the materialised generation")
    ap.add_argument("--no-t01", action="store_true", help="vegas: skip the time-to-0.1%% run")
    ap.add_argument("--no-others", action="store_true",
                    help="multichannel: skip the compact runs of the other workloads")
    ap.add_argument("--no-unweighting", action="store_true",
                    help="multichannel: skip the unweighting-quantile and event-output measurements")
    ap.add_argument("--log-iterations", action="store_true",
                    help="multichannel: one line per iteration on stderr (points tried, weighted, accepted), "
                         "to normalise per-launch profiler counters")
    return ap.parse_args()


def workload_config(ncalls):
    return {"workload": WL["describe"],
            "channels": WL["channels"], "bins_per_dim": WL["bins"], "points_per_iteration": ncalls,
            "seed": SEED, "alpha_adapted": True, "alpha_guard": True,
            "preprocess": "physical region and cuts: x1, x2 <= 1, pT > 30 GeV, |eta| < 99, dR > 0.4",
            "l2": "per-step working set > L2 (momenta of the tried points: "
                  f"~{ncalls * 1.7 * 4 * (WL['n_out'] + 2) * 8 / 1e6:.0f} MB)"}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        import tempfile
        self.path = os.path.join(tempfile.gettempdir(), f"chili_bench_clocks_{os.getpid()}_{index}.csv")

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                mhz.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


# ------------------------------------------------------------------ chili arm
def unweighted_events(st, info):
    """Expected unweighted events of an iteration: N <w> / w_max = sum / w_max."""
    return st.sum / info.weight_max if info.weight_max > 0 else 0.0


def run_chili(args, rank, world, local_rank):
    import torch

    from chili_b200 import abi, channels, gpu, workloads

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    cs = workloads.channel_set(WL["n_out"])
    ctx = gpu.Context(local_rank)
    # a stream of our own, current for torch too: the library's kernels, the
    # collectives and the timing events share it (torch's default stream is
    # the legacy NULL stream, which does not order the library's own stream)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_channels(cs)
    ctx.uniform_grids(cs.nch, ctx.ndims, WL["bins"])
    ctx.set_integrand(getattr(abi, "CHILI_FUNC_" + WL["fkind"]), channels.propagator_params())
    ctx.set_preprocess_cuts(cs.sqrts)
    params = workloads.mc_params(args.ncalls, iterations=args.warmup + args.steps)
    seed = SEED + 1000 * rank  # disjoint streams per rank (weak scaling)
    counter = 0

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # N > 1: the reference's MPI mode (MultiChannel.hh:184-212): every rank
    # integrates its own counter stream, the training data and StatsData are
    # summed by one NCCL all-reduce per iteration, every rank adapts alike
    synced = world > 1
    if synced:
        from chili_b200 import parallel
        rank_obj = parallel.GpuRank(ctx, seed, counter, shared_stream=True)

    def one_step():
        if synced:
            mst, info = parallel.synced_iteration(rank_obj, params, device=dev)
            return mst, info, (mst[3] / mst[2] if mst[2] > 0 else 0.0) / world
        st, info = ctx.multichannel_iterate(params, seed=seed, counter=rank_obj_counter[0], guard=True)
        rank_obj_counter[0] += info.points_tried
        return st.as_tuple(), info, unweighted_events(st, info)

    rank_obj_counter = [counter]
    n_iter = [0]

    def logged(out):
        if args.log_iterations:
            info = out[1]
            print(f"iteration {n_iter[0]}: tried {info.points_tried} weighted {info.points_weighted} "
                  f"accepted {info.points_accepted} drawn {info.points_drawn} chunks {info.chunks}",
                  file=sys.stderr, flush=True)
        n_iter[0] += 1
        return out

    for _ in range(args.warmup):
        logged(one_step())
    torch.cuda.synchronize(dev)
    barrier()
    torch.cuda.synchronize(dev)

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.set_option("kernel_timing", 1)  # CUDA events around each kernel of the timed region
    l0 = ctx.launches
    weighted = 0
    drawn = 0
    pooled = np.zeros(6)
    history = []
    unw = 0.0
    tried = 0
    with ClockSampler(local_rank) as clk:
        ev0.record(stream)
        t_wall0 = time.perf_counter()
        for _ in range(args.steps):
            st_t, info, u_step = logged(one_step())
            tried += info.points_tried
            weighted += info.points_weighted
            drawn += info.points_drawn
            unw += u_step
            pooled += np.array(st_t) * np.array([1, 0, 0, 1, 1, 1])
            mean, err = gpu.stats_mean_error(pooled)
            history.append((time.perf_counter() - t_wall0, err / abs(mean) if mean else float("inf")))
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    launches = ctx.launches - l0
    ms = ev0.elapsed_time(ev1)
    barrier()
    # max over ranks of the device time; totals summed
    t = torch.tensor([ms, unw, float(tried), float(args.ncalls * args.steps)], dtype=torch.float64, device=dev)
    if world > 1:
        tmax = t[:1].clone()
        torch.distributed.all_reduce(tmax, op=torch.distributed.ReduceOp.MAX)
        tsum = t[1:].clone()
        torch.distributed.all_reduce(tsum)
        ms_max, unw_tot, tried_tot, acc_tot = tmax.item(), *tsum.tolist()
    else:
        ms_max, unw_tot, tried_tot, acc_tot = ms, unw, float(tried), float(args.ncalls * args.steps)
    mean, err = gpu.stats_mean_error(pooled)
    t01 = next((h[0] for h in history if h[1] <= 1e-3), None)

    kernel_ms = {k: ctx.kernel_time(k) for k in TIMED_KERNELS}
    kernel_ms = {k: v for k, v in kernel_ms.items() if v[1] > 0}
    roof = roofline(kernel_ms, weighted, args.ncalls * args.steps, ms, dev, drawn=drawn)
    # where the step's device time goes: the timed kernel classes, the small
    # per-round kernels, the end-of-iteration adaptation, and the rest (the
    # device idle while the host reads a round's counts back and launches)
    main_ms = sum(v[0] for v in kernel_ms.values())
    other_ms = ctx.kernel_time("round_other")[0]
    end_ms = ctx.kernel_time("iteration_end")[0]
    time_split = {"kernels_ms_per_step": main_ms / args.steps, "round_other_ms_per_step": other_ms / args.steps,
                  "iteration_end_ms_per_step": end_ms / args.steps,
                  "rest_ms_per_step": (ms - main_ms - other_ms - end_ms) / args.steps}

    plain = {"value": unw_tot / (ms_max / 1e3), "ms_per_step": ms_max / args.steps,
             "points_per_step": tried_tot / args.steps, "integral": mean, "rel_error": err / abs(mean),
             "rel_var_per_point": (err / abs(mean)) ** 2 * tried_tot, "time_to_0p1pct_s": t01,
             "unweighting_efficiency": unw_tot / tried_tot if tried_tot else None}
    flow = flow_long = None
    if not args.no_flow and world == 1:
        flow = measure_flow(ctx, args, dev, stream, plain)
        if args.flow_long_steps > 0:
            flow_long = measure_flow(ctx, args, dev, stream, plain, train_steps=args.flow_long_steps)

    ctx.set_option("kernel_timing", 0)  # no per-kernel events around the event-output calls
    unw_q = unw_out = None
    if not args.no_unweighting:
        unw_q = quantile_unweighting(ctx, seed=4242 + rank)
        if WL["unweighted_target"]:
            unw_out = measure_unweighted_target(ctx, info.weight_max, dev, rank, WL["unweighted_target"])
        else:
            unw_out = measure_unweighted_output(ctx, info.weight_max, dev, rank)

    e2e = None
    if not args.no_e2e:
        if WL["unweighted_target"]:
            if unw_out is None:
                raise SystemExit("bench.py: the large workload's e2e is its event output (drop --no-unweighting)")
            # 1e7-point iterations: the uniforms would not fit pinned host memory
            # twice; the end-to-end path is the event output to the host
            e2e = {"value": unw_out["events_per_s"], "unit": UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": unw_out["d2h_bytes_per_call"], "steps": unw_out["calls"],
                   "path": unw_out["path"]}
        else:
            e2e = measure_e2e(ctx, params, args, dev, rank)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args)
    others = None
    if world == 1 and WL is WORKLOADS["multichannel"] and not args.no_others:
        others = compact_other_workloads(args, dev, rank)

    if rank == 0:
        selected = "plain"
        if flow and flow.get("variance_x_time_ratio") is not None and flow["variance_x_time_ratio"] < 1.0:
            selected = "flow"
        value = flow["value"] if selected == "flow" else unw_tot / (ms_max / 1e3)
        line = {
            "metric": WL["metric"], "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (on-device Philox4x32-10 uniforms)",
            "config": workload_config(args.ncalls),
            "parallelism": f"dp{world}: ranks synchronised by one NCCL all-reduce of the training data per "
                           f"iteration" if world > 1 else "single GPU",
            "points_per_s": acc_tot / (ms_max / 1e3),
            "tried_points_per_s": tried_tot / (ms_max / 1e3),
            "weighted_points_per_step": weighted / args.steps,
            "unweighting_efficiency": unw_tot / acc_tot,
            "integral": mean, "rel_error": err / abs(mean),
            "time_to_0p1pct_s": t01,
            "clocks": clk.summary(),
            "gpu_launches": launches,
            "roofline": roof,
            "time_split": time_split,
            "paths": {"selected": selected, "plain": plain, "flow": flow, "flow_long_training": flow_long},
            "unweighted_output": unw_out,
            "unweighting_quantile": unw_q,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "other_workloads": others,
        }
        print(json.dumps(line), flush=True)
    ctx.close()


# ------------------------------------------- the other workloads, compactly
def compact_other_workloads(args, dev, rank):
    """Short, time-bounded runs of the other benchmark configurations beside
    the headline, so that one default run records them all: the plain VEGAS
    camel (4-d, 50 bins, 1e5 points per iteration) with its materialised
    points, the 512-integrand batch and the 2->6 / 45-channel / 200-bin
    workload (1e7 points per iteration, plain path).  Device time by CUDA
    events on a stream of their own."""
    import torch

    from chili_b200 import abi, channels, gpu, workloads
    out = {}
    stream = torch.cuda.Stream(dev)
    prev = torch.cuda.current_stream(dev)
    torch.cuda.set_stream(stream)
    try:
        # plain VEGAS
        cfg = dict(workloads.VEGAS_CAMEL)
        ctx = gpu.Context(dev.index)
        ctx.set_stream(stream.cuda_stream)
        ctx.uniform_grids(1, cfg["dims"], cfg["bins"])
        ctx.set_integrand(abi.CHILI_FUNC_CAMEL, workloads.camel_params(cfg["dims"]))
        sd = torch.zeros(6, dtype=torch.float64, device=dev)
        import ctypes as C

        def vstep(k):
            ctx.call("chili_gpu_vegas_iterate", cfg["ncalls"], cfg["seed"], k * cfg["ncalls"], None,
                     float(cfg["alpha"]), 1, C.c_void_p(sd.data_ptr()), None)
        for k in range(5):
            vstep(k)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(50):
            vstep(5 + k)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / 50
        mat = vegas_materialised(ctx, dev, stream, cfg, n=50_000_000, reps=5)
        out["vegas"] = {"workload": "plain VEGAS, 4-d camel, 50 bins, alpha 1.5, 1e5 points per iteration",
                        "ms_per_iteration": ms, "points_per_s": cfg["ncalls"] / (ms / 1e3),
                        "materialised_points_per_s": mat["points_per_s"],
                        "materialised_hbm_frac": mat["roofline"]["frac"],
                        "full_line": "python bench.py --workload vegas"}
        ctx.close()
        # the 512 batched integrands
        tasks = workloads.batched_tasks(seed=BATCH_SEED + rank)
        ctx = gpu.Context(dev.index)
        ctx.set_stream(stream.cuda_stream)
        ctx.batch_set(tasks)
        ctx.batch_iterate(1, seed=BATCH_SEED)
        ctx.batch_iterate(1, seed=BATCH_SEED)
        l0 = ctx.launches
        bms, calls = 0.0, 0.0
        for _ in range(3):
            st, info = ctx.batch_iterate(1, seed=BATCH_SEED)
            bms += info.ms_per_iteration
            calls += float(st[0][:, 0].sum())
        out["batched"] = {"workload": "512 integrands (256 camels D 2-12, 256 multichannel 2->n), one adapting "
                                      "iteration each per step (fixed budget)",
                          "ms_per_iteration": bms / 3,
                          "points_per_s": calls / (bms / 1e3), "launches_per_iteration": (ctx.launches - l0) / 3,
                          "full_line": "python bench.py --workload batched"}
        ctx.close()
        # 2->6, 45 channels, 200 bins, 1e7 points per iteration
        wl = WORKLOADS["large"]
        cs = workloads.channel_set(6)
        ctx = gpu.Context(dev.index)
        ctx.set_stream(stream.cuda_stream)
        ctx.set_channels(cs)
        ctx.uniform_grids(cs.nch, ctx.ndims, wl["bins"])
        ctx.set_integrand(abi.CHILI_FUNC_PROPAGATOR_TOP2, channels.propagator_params())
        ctx.set_preprocess_cuts(cs.sqrts)
        params = workloads.mc_params(wl["ncalls"], iterations=6)
        c = 0
        for _ in range(3):
            st, info = ctx.multichannel_iterate(params, seed=SEED, counter=c, guard=True)
            c += info.points_tried
        e0.record(stream)
        unw, tried = 0.0, 0
        for _ in range(3):
            st, info = ctx.multichannel_iterate(params, seed=SEED, counter=c, guard=True)
            c += info.points_tried
            unw += unweighted_events(st, info)
            tried += info.points_tried
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / 3
        out["large"] = {"workload": wl["describe"] + ", 45 channels, 200 bins, 1e7 accepted points per iteration, "
                                                     "plain path", "ms_per_iteration": ms,
                        "unweighted_events_per_s": unw / (3 * ms / 1e3),
                        "tried_points_per_s": tried / (3 * ms / 1e3),
                        "full_line": "python bench.py --workload large"}
        ctx.close()
    finally:
        torch.cuda.set_stream(prev)
    return out


# Per-kernel figures of the committed ncu capture (the multichannel 2->4
# summary under profiles/): FP64 operations (2*DFMA + DADD + DMUL, executed)
# and DRAM bytes (read + write) per point of the kernel's basis: drawn
# counters for the forward kernel (it runs over every drawn point of a
# chunk), weighted points for the rest.
KERNEL_COUNTERS = {
    "k_mc_forward": {"fp64_ops_per_point": 1868.7, "dram_bytes_per_point": 424.4, "basis": "drawn",
                     "source": "profiles/multichannel_2to4_kernels.md"},
    "k_pp_nodes": {"fp64_ops_per_point": 24.0, "dram_bytes_per_point": 838.1, "basis": "weighted",
                     "source": "profiles/multichannel_2to4_kernels.md"},
    "k_pp_items": {"fp64_ops_per_point": 9343.5, "dram_bytes_per_point": 1316.3, "basis": "weighted",
                     "source": "profiles/multichannel_2to4_kernels.md"},
    "k_pp_chains": {"fp64_ops_per_point": 3684.0, "dram_bytes_per_point": 597.0, "basis": "weighted",
                     "source": "profiles/multichannel_2to4_kernels.md"},
    "k_pp_channel": {"fp64_ops_per_point": 684.0, "dram_bytes_per_point": 1077.4, "basis": "weighted",
                     "source": "profiles/multichannel_2to4_kernels.md"},
    "k_pp_combine": {"fp64_ops_per_point": 724.0, "dram_bytes_per_point": 416.2, "basis": "weighted",
                     "source": "profiles/multichannel_2to4_kernels.md"},
    "k_mc_accum": {"fp64_ops_per_point": 300.0, "dram_bytes_per_point": 32.3, "basis": "weighted",
                     "source": "profiles/multichannel_2to4_kernels.md"}
}


def fp64_peak_tflops(dev):
    """FP64 peak measured here: cuBLAS DGEMM 8192^3, best of 5."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize(dev)
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def roofline(kernel_ms, weighted, accepted, step_ms, dev, drawn=None):
    """The FP64 roofline of the multichannel step (the binding resource:
    every point evaluates every channel's inverse map, mostly
    transcendental-function expansions).  For the dominant kernel of the
    timed region (by CUDA-event time): achieved = its FP64 operations per
    weighted point (2 DFMA + DADD + DMUL, the committed ncu counters; a
    property of the per-point work, not of the batch size) x the weighted
    points of one launch / the launch's average CUDA-event duration, against
    the cuBLAS DGEMM peak measured in this run.  traffic = its measured DRAM
    bytes per launch (the phased pass keeps intermediates in HBM: the ratio
    to its zero algorithmic bytes is the waste).  `step` gives the same view
    for all kernels of the step, and the HBM view of the materialised event
    record (204 B per accepted point)."""
    dom = max(kernel_ms, key=lambda k: kernel_ms[k][0])
    ms, launches = kernel_ms[dom]
    peak = fp64_peak_tflops(dev)
    hbm = measured_peaks().get("hbm_gbs")
    c = KERNEL_COUNTERS.get(dom)
    drawn = drawn or weighted

    def points(k):  # the points a kernel class processes: drawn (forward) or weighted
        return drawn if KERNEL_COUNTERS.get(k, {}).get("basis") == "drawn" else weighted
    per_launch = points(dom) / max(launches, 1)
    out = {"kernel": dom, "bound": "fp64", "launches": launches, "ms_per_launch": ms / max(launches, 1),
           "points_per_launch": per_launch, "points_basis": KERNEL_COUNTERS.get(dom, {}).get("basis", "weighted"),
           "share_of_kernel_time": ms / sum(v[0] for v in kernel_ms.values()),
           "peak": peak, "unit": "TFLOP/s", "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
           "kernel_ms": {k: round(v[0], 4) for k, v in kernel_ms.items()}}
    if c:
        ach = c["fp64_ops_per_point"] * per_launch / (ms / max(launches, 1) / 1e3) / 1e12
        out.update(achieved=ach, frac=ach / peak, fp64_ops_per_point=c["fp64_ops_per_point"],
                   traffic=c["dram_bytes_per_point"] * per_launch, algorithmic_bytes=0,
                   counters_source=c["source"])
    else:
        out.update(achieved=None, frac=None, traffic=None)
    # the whole step: each kernel class's count times the points it processed
    ops_tot = sum(KERNEL_COUNTERS[k]["fp64_ops_per_point"] * points(k) for k in kernel_ms if k in KERNEL_COUNTERS)
    dram_tot = sum(KERNEL_COUNTERS[k]["dram_bytes_per_point"] * points(k) for k in kernel_ms if k in KERNEL_COUNTERS)
    ops, dram = ops_tot / weighted, dram_tot / weighted
    sec = step_ms / 1e3
    out["step"] = {
        "fp64": {"ops_per_weighted_point": ops, "achieved": ops_tot / sec / 1e12, "unit": "TFLOP/s",
                 "frac": ops_tot / sec / 1e12 / peak},
        "hbm_event_record": {"bytes_per_accepted_point": 204, "achieved": 204 * accepted / sec / 1e9, "unit": "GB/s",
                             "peak": hbm, "frac": 204 * accepted / sec / 1e9 / hbm if hbm else None},
        "dram_bytes_per_weighted_point": dram,
        "seconds": sec, "weighted_points": weighted, "drawn_points": drawn, "accepted_points": accepted,
    }
    return out


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def measure_flow(ctx, args, dev, stream, plain, train_steps=None):
    """The learned proposal on the same context (grids and channel weights as
    the plain path left them): online training on the GPU, one beta
    adaptation pass, then `steps` timed passes of as many points as a plain
    step generates. Device time by CUDA events on the context's stream."""
    import torch
    from chili_b200 import abi, gpu
    n = int(round(plain["points_per_step"]))
    train_steps = args.flow_steps if train_steps is None else train_steps
    fp = abi.FlowParams.defaults(batch=args.flow_batch, layers=WL["flow_layers"], lr=1e-3,
                                 hidden=WL["flow_hidden"], depth=WL["flow_depth"])
    # one-time costs (first launch of each kernel, first allocations) outside
    # the timed training: three steps and one sampling pass on a throwaway
    # network, then a fresh one
    ctx.flow_init(fp)
    ctx.flow_train(3, seed=SEED + 76, counter=0)
    ctx.flow_iterate(n, seed=SEED + 75, counter=0)
    torch.cuda.synchronize(dev)
    ctx.flow_init(fp)
    k0 = {k: ctx.kernel_time(k) for k in FLOW_KERNELS}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    em = torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e0.record(stream)
    loss = ctx.flow_train(train_steps, seed=SEED + 77, counter=0)
    em.record(stream)
    w1 = time.perf_counter()
    ctx.flow_iterate(n, seed=SEED + 78, counter=0, adapt_beta=True)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    w2 = time.perf_counter()
    train_s = e0.elapsed_time(e1) / 1e3
    split = {"steps_device_s": e0.elapsed_time(em) / 1e3, "beta_pass_device_s": em.elapsed_time(e1) / 1e3,
             "steps_wall_s": w1 - w0, "beta_pass_wall_s": w2 - w1}
    k1 = {k: ctx.kernel_time(k) for k in FLOW_KERNELS}
    ctx.flow_iterate(n, seed=SEED + 79, counter=0)  # warm-up
    torch.cuda.synchronize(dev)
    pooled = np.zeros(6)
    unw, history = 0.0, []
    e0.record(stream)
    t_wall0 = time.perf_counter()
    for s in range(args.steps):
        st, info = ctx.flow_iterate(n, seed=SEED + 100 + s, counter=0)
        unw += st.sum / info.weight_max if info.weight_max > 0 else 0.0
        pooled += np.array(st.as_tuple()) * np.array([1, 0, 0, 1, 1, 1])
        m_, e_ = gpu.stats_mean_error(pooled)
        history.append((time.perf_counter() - t_wall0, e_ / abs(m_) if m_ else float("inf")))
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    k2 = {k: ctx.kernel_time(k) for k in FLOW_KERNELS}
    mean, err = gpu.stats_mean_error(pooled)
    rv = (err / abs(mean)) ** 2 * pooled[0]
    t_step = ms / 1e3 / args.steps
    t_plain = plain["ms_per_step"] / 1e3
    ratio = (rv * t_step / n) / (plain["rel_var_per_point"] * t_plain / plain["points_per_step"])
    t01 = next((h[0] for h in history if h[1] <= 1e-3), None)
    pull = (mean - plain["integral"]) / np.hypot(err, plain["rel_error"] * abs(plain["integral"]))
    # tensor-core roofline of the coupling layers: the conditioners' useful
    # products (FLOPs from the layer shapes) over the layer kernels' CUDA-event
    # time, against the sustained cuBLAS bf16 figure (the kernels run inside
    # long passes); training runs the forward products, the two data-gradient
    # products of the same shapes and the weight-gradient products (3x)
    f_pt = flow_flops_per_point(ctx.ndims, WL["flow_layers"], WL["flow_hidden"], WL["flow_depth"])
    peak_bf16 = measured_peaks().get("bf16_tflops_sustained") or measured_peaks().get("bf16_tflops")
    lay_ms = k2["k_flow_layer"][0] - k1["k_flow_layer"][0]
    tr_ms = sum(k1[k][0] - k0[k][0] for k in ("k_flow_layer", "k_flow_layer_bwd", "k_flow_wgrad"))
    tensor = {"flops_per_point_per_pass": f_pt, "peak": peak_bf16, "unit": "TFLOP/s",
              "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained (cuBLAS bf16, seconds-long loop)"}
    if lay_ms > 0:
        a = f_pt * n * args.steps / (lay_ms / 1e3) / 1e12
        tensor["pass"] = {"achieved": a, "frac": a / peak_bf16 if peak_bf16 else None, "kernel_ms": lay_ms}
    if tr_ms > 0:
        a = 3 * f_pt * args.flow_batch * train_steps / (tr_ms / 1e3) / 1e12
        tensor["training"] = {"achieved": a, "frac": a / peak_bf16 if peak_bf16 else None, "kernel_ms": tr_ms}
    return {
        "value": unw / (ms / 1e3), "unit": UNIT, "ms_per_step": t_step * 1e3, "points_per_step": n,
        "integral": mean, "rel_error": err / abs(mean), "rel_var_per_point": rv,
        "rel_var_reduction_vs_plain": plain["rel_var_per_point"] / rv,
        "unweighting_efficiency": unw / pooled[0],
        "unweighting_gain_vs_plain": (unw / pooled[0]) / plain["unweighting_efficiency"],
        "time_to_0p1pct_s": t01,
        "time_to_0p1pct_with_training_s": (t01 + train_s) if t01 is not None else None,
        "variance_x_time_ratio": ratio, "pull_vs_plain": pull,
        "training": {"steps": train_steps, "batch": args.flow_batch, "layers": WL["flow_layers"],
                     "hidden": f"{WL['flow_depth']} x {WL['flow_hidden']} (unit {WL['flow_hidden'] - 1} the "
                               f"constant 1; " + ("weights resident in shared memory" if WL["flow_hidden"] == 128
                                                   and WL["flow_depth"] == 2 else "weights streamed per tile") + ")",
                     "seconds": train_s, "split": split,
                     "loss_first": float(np.mean(loss[:10])), "loss_last": float(np.mean(loss[-10:])),
                     "kernel_ms": {k: round(k1[k][0] - k0[k][0], 3) for k in FLOW_KERNELS if k1[k][0] > k0[k][0]}},
        "kernel_ms": {k: round(k2[k][0] - k1[k][0], 3) for k in FLOW_KERNELS if k2[k][0] > k1[k][0]},
        "gpu_launches_note": "flow kernels: tcgen05 coupling layers, FP64 phase space, phased weight pass",
        "tensor_roofline": tensor,
    }


def flow_flops_per_point(dims, layers, hidden, depth):
    """Useful tensor-core FLOPs of one flow pass per point: per coupling layer
    2 H da (first product; the channel embedding is a one-hot lookup),
    2 (depth - 1) H^2 (hidden products) and 2 (49 db) H (spline parameters)."""
    from chili_b200 import flowspec
    tot = 0
    for m in flowspec.masks(dims, layers):
        da, db = int(m.sum()), int((~m).sum())
        tot += 2 * hidden * da + 2 * (depth - 1) * hidden * hidden + 2 * flowspec.PER_DIM * db * hidden
    return tot


def measure_unweighted_output(ctx, w_max, dev, rank, n=4_000_000, reps=8):
    """The unweighting stage end to end: n points drawn, weighted, hit-or-miss
    against the last iteration's largest weight, and the kept events
    (momenta, weight, channel) written to pinned host memory."""
    import torch
    ne = ctx.n_ext
    cap = n // 4
    out = (torch.empty((cap, ne, 4), dtype=torch.float64, pin_memory=True).numpy(),
           torch.empty(cap, dtype=torch.float64, pin_memory=True).numpy(),
           torch.empty(cap, dtype=torch.int32, pin_memory=True).numpy())
    seed = 97 + rank
    ctx.generate_unweighted(n, w_max, seed=seed, counter=0, max_events=cap, out=out)  # warm-up
    torch.cuda.synchronize(dev)
    kept = 0
    t0 = time.perf_counter()
    for r in range(reps):
        _, _, _, info = ctx.generate_unweighted(n, w_max, seed=seed, counter=(r + 1) * n, max_events=cap, out=out)
        kept += info.kept
    dt = time.perf_counter() - t0
    written = min(kept // reps, cap)
    return {"events_per_s": kept / dt, "points_per_s": n * reps / dt, "efficiency": kept / (n * reps),
            "w_max": w_max, "overweight_last_call": int(info.overweight), "points_per_call": n,
            "d2h_bytes_per_call": int(written * (ne * 32 + 12)),
            "path": "chili_gpu_generate_unweighted with pinned host outputs, wall clock"}


def quantile_unweighting(ctx, seed, n=2_000_000, q=0.999):
    """Unweighting efficiency <v> / w_q with w_q the q-quantile of the
    nonzero values |v| of n drawn points instead of their maximum, in the
    reference's Percentile convention (Statistics.hh:22-59: the
    (floor(k q) + 1)-th smallest of k values); <v> is over all n points
    (zeros of rejected points included, as in StatsData).  The values come
    from chili_gpu_generate_unweighted with a vanishing w_max, which keeps
    every nonzero value and returns it unchanged."""
    wgt = np.empty(n)
    _, v, _, _ = ctx.generate_unweighted(n, 1e-300, seed=seed, counter=0, max_events=n, out=(None, wgt, None))
    mean = float(np.sum(v)) / n
    nz = np.sort(np.abs(v))
    if len(nz) == 0:
        return {"quantile": q, "points": n, "nonzero": 0}
    w_q = float(nz[int(len(nz) * q)])
    return {"quantile": q, "w_max_quantile": w_q, "w_max_sample": float(nz[-1]),
            "efficiency": mean / w_q, "efficiency_with_max": mean / float(nz[-1]),
            "overweight_fraction": float(np.mean(nz > w_q)), "points": n, "nonzero": int(len(nz)),
            "path": "chili_gpu_generate_unweighted values on the adapted channels, host sort"}


def measure_unweighted_target(ctx, w_max, dev, rank, target, chunk=20_000_000, limit_s=60.0):
    """`target` unweighted events written to pinned host memory, chunk after
    chunk of drawn points (w_max = the last iteration's largest weight),
    stopping at the target or after limit_s seconds."""
    import torch
    ne = ctx.n_ext
    cap = target
    out = (torch.empty((cap, ne, 4), dtype=torch.float64, pin_memory=True).numpy(),
           torch.empty(cap, dtype=torch.float64, pin_memory=True).numpy(),
           torch.empty(cap, dtype=torch.int32, pin_memory=True).numpy())
    seed = 97 + rank
    ctx.generate_unweighted(1_000_000, w_max, seed=seed, counter=0, max_events=cap, out=out)  # warm-up
    torch.cuda.synchronize(dev)
    kept, pts, calls, over = 0, 0, 0, 0
    t0 = time.perf_counter()
    while kept < target and time.perf_counter() - t0 < limit_s:
        view = tuple(b[kept:] for b in out)
        _, _, _, info = ctx.generate_unweighted(chunk, w_max, seed=seed, counter=(calls + 1) * chunk,
                                                max_events=cap - kept, out=view)
        kept += min(info.kept, cap - kept)
        pts += chunk
        calls += 1
        over += info.overweight
    dt = time.perf_counter() - t0
    return {"events_per_s": kept / dt, "events": kept, "target": target, "reached": kept >= target,
            "seconds": dt, "points": pts, "points_per_s": pts / dt, "efficiency": kept / pts, "w_max": w_max,
            "overweight": over, "calls": calls, "points_per_call": chunk,
            "d2h_bytes_per_call": int(kept / max(calls, 1) * (ne * 32 + 12)),
            "path": "chili_gpu_generate_unweighted with pinned host outputs, wall clock"}


def measure_e2e(ctx, params, args, dev, rank):
    """Same metric through the C ABI with HOST buffers: each step's uniforms
    come from pinned host memory (the library uploads the rows it consumes,
    overlapped with the mapping), the StatsData and iteration record come
    back to the host."""
    import torch
    from chili_b200 import gpu, workloads
    D = ctx.ndims
    n_u = int(args.ncalls * 3.0) + 4096
    rng = np.random.default_rng(1234 + rank)
    bufs = []
    for _ in range(2):
        t = torch.empty((n_u, D + 1), dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = workloads.uniforms53(rng, (n_u, D + 1))
        bufs.append(t.numpy())
    steps = max(2, min(args.steps, 5))
    ctx.multichannel_iterate(params, u=bufs[0], guard=True)  # warm-up
    torch.cuda.synchronize(dev)
    unw = 0.0
    rows = 0
    t0 = time.perf_counter()
    for s in range(steps):
        st, info = ctx.multichannel_iterate(params, u=bufs[s % 2], guard=True)
        unw += unweighted_events(st, info)
        rows += info.points_tried
    dt = time.perf_counter() - t0
    # the PCIe floor: the same bytes as one pinned host-to-device copy
    nb = int(rows / steps)
    src = torch.from_numpy(bufs[0][:nb])
    dst = torch.empty(src.shape, dtype=torch.float64, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dst.copy_(src, non_blocking=True)
    e0.record()
    for _ in range(3):
        dst.copy_(src, non_blocking=True)
    e1.record()
    e1.synchronize()
    copy_ms = e0.elapsed_time(e1) / 3
    del dst
    return {"value": unw / dt, "unit": UNIT, "h2d_bytes_per_step": int(nb * (D + 1) * 8),
            "d2h_bytes_per_step": int(2 * 48 + 32), "steps": steps, "ms_per_step": dt / steps * 1e3,
            "h2d_copy_ms": copy_ms, "h2d_gbs": nb * (D + 1) * 8 / copy_ms / 1e6,
            "path": "chili_gpu_multichannel_iterate with host uniforms (pinned) and host StatsData"}


# ------------------------------------------------------------- reference arm
def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_ncalls():
    """Points per reference iteration: the workload's own 1e6 for the 2->4
    workload (like for like with the GPU step); the 2->6 workload's 1e7
    points would take minutes per iteration on the host, so a bounded sample
    of 2000 points per core."""
    return WL["ncalls"] if WL["n_out"] <= 4 else 2000 * cpu_cores()


def _ref_mpi(ncalls):
    from oracle.mpi_ranks import RefMPI
    return RefMPI(cpu_cores(), n_out=WL["n_out"], bins=WL["bins"], ncalls=ncalls, fkind=WL["fkind"], seed=SEED,
                  cuts=True)


def cpu_baseline(args, kind="reference"):
    """The reference (oracle/_ref) timed on the host in its MPI mode
    (MultiChannel.hh:184-212) over one process per core: one iteration of
    the workload's points after one warm-up iteration."""
    from oracle import ref
    if not ref.available():
        return {"value": None, "unavailable": "oracle/_ref not built"}
    ncalls = reference_ncalls()
    with _ref_mpi(ncalls) as M:
        M.iterate()  # warm-up: the iteration on uniform grids
        st, w_max, tried, sec = M.iterate()
    cores = M.nranks
    return {"value": (st[3] / w_max if w_max > 0 else 0.0) / sec, "unit": UNIT, "cores": cores, "kind": kind,
            "points_per_s": M.ncalls_rank * cores / sec, "seconds": sec,
            "sample": f"one MultiChannel iteration of {M.ncalls_rank * cores} accepted points in the reference's "
                      f"MPI mode ({cores} host processes of {M.ncalls_rank} points, training data summed, every "
                      f"rank adapting alike), after one warm-up iteration; time = the slowest rank"}


def run_reference(args, rank, world):
    """The reference's own CPU implementation of the step: one
    MultiChannel::operator() iteration of the workload's points with the
    alpha and grid adaptation, in the reference's MPI mode over one process
    per host core (ncalls / size points per rank, training data and StatsData
    summed, Train on every rank; MultiChannel.hh:184-212).  Each step's time
    is the slowest rank's iteration plus its Train (the uniforms are drawn
    before the clock starts); the unweighted events of a step are its summed
    values over the largest weight of all its points, as on the GPU."""
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libchili_ref.so not built"}))
        return
    ncalls = reference_ncalls()
    unw, secs = 0.0, 0.0
    pooled = np.zeros(6)
    history = []
    from chili_b200.gpu import stats_mean_error
    with _ref_mpi(ncalls) as M:
        for _ in range(args.warmup):
            M.iterate()
        for _ in range(args.steps):
            st, w_max, tried, sec = M.iterate()
            unw += st[3] / w_max if w_max > 0 else 0.0
            secs += sec
            pooled += np.array(st) * np.array([1, 0, 0, 1, 1, 1])
            m_, e_ = stats_mean_error(pooled)
            history.append((secs, e_ / abs(m_) if m_ else float("inf")))
    cores = M.nranks
    value = unw / secs
    mean, err = stats_mean_error(pooled)
    line = {
        "impl": "reference", "metric": WL["metric"], "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (host uniforms)", "config": workload_config(M.ncalls_rank * cores),
        "parallelism": f"the reference's MPI mode over {cores} host processes",
        "points_per_s": M.ncalls_rank * cores * args.steps / secs, "integral": mean, "rel_error": err / abs(mean),
        "time_to_0p1pct_s": next((h[0] for h in history if h[1] <= 1e-3), None),
        "unweighting_efficiency": unw / (M.ncalls_rank * cores * args.steps),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"each step: one MultiChannel iteration of {M.ncalls_rank * cores} accepted "
                                   f"points in the reference's MPI mode ({cores} processes of {M.ncalls_rank}), "
                                   f"time = the slowest rank's iteration and Train"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------- plain VEGAS workload
VEGAS_METRIC = "VEGAS points/s and time to 0.1% error, 4-d camel (50 bins, alpha 1.5, 1e5 points/iteration), FP64"
VEGAS_UNIT = "points/s"
# FP64 operations (2*DFMA + DADD + DMUL, executed) per point of the point
# loop the iteration kernels share (k_vegas_iter, and k_vegas_step, which
# adds the last block's fold and adaptation: O(dims * bins) once per
# iteration), and DRAM bytes per launch, from the committed ncu capture of
# the 1e5-point iteration (profiles/vegas_camel_kernels.md)
VEGAS_COUNTERS = {"fp64_ops_per_point": 180.1, "dram_bytes_per_launch": 32.5e3,
                  "source": "profiles/vegas_camel_kernels.md"}


def vegas_config(cfg):
    return {"workload": f"plain VEGAS, {cfg['dims']}-d camel (sigma 0.1, centres 1/3 and 2/3, unit integral)",
            "bins_per_dim": cfg["bins"], "grid_alpha": cfg["alpha"], "points_per_iteration": cfg["ncalls"],
            "seed": cfg["seed"], "refine": "none",
            "l2": "flushed between timed iterations (256 MB write outside the timed events); the uniforms are "
                  "generated on the device"}


def run_vegas(args, rank, world, local_rank):
    """Config 1 of the benchmark definition: plain VEGAS (Vegas::operator(),
    Vegas.cc:18-52) on the 4-d camel.  One step = one iteration of 1e5
    points with the grid adaptation, fused in one kernel (on-device
    uniforms, map, camel, StatsData and histogram in shared memory) plus the
    fold and the adaptation.  Beside it: the materialised points
    (chili_gpu_vegas_generate: x and f*J written to HBM, 40 B per point),
    the HBM-bound form of the same map, and the time to 0.1% pooled error."""
    import ctypes as C

    import torch

    from chili_b200 import abi, gpu, workloads
    cfg = dict(workloads.VEGAS_CAMEL)
    n = args.ncalls if args.ncalls else cfg["ncalls"]
    cfg["ncalls"] = n
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.Stream(dev)  # current for torch too (the flush and the events share it)
    torch.cuda.set_stream(stream)
    ctx = gpu.Context(local_rank)
    ctx.set_stream(stream.cuda_stream)
    params = workloads.camel_params(cfg["dims"])
    ctx.uniform_grids(1, cfg["dims"], cfg["bins"])
    ctx.set_integrand(abi.CHILI_FUNC_CAMEL, params)
    seed = cfg["seed"] + 1000 * rank
    stats_dev = torch.zeros((args.warmup + args.steps, 6), dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step(k, counter):
        ctx.call("chili_gpu_vegas_iterate", n, seed, counter, None, float(cfg["alpha"]), 1,
                 C.c_void_p(stats_dev[k].data_ptr()), None)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    counter = 0
    for k in range(args.warmup):
        step(k, counter)
        counter += n
    torch.cuda.synchronize(dev)
    barrier()
    torch.cuda.synchronize(dev)
    ctx.set_option("kernel_timing", 1)
    l0 = ctx.launches
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local_rank) as clk:
        for k in range(args.steps):
            flush.fill_(k & 0xff)  # L2 flushed between the timed iterations, outside their events
            evs[k][0].record(stream)
            step(args.warmup + k, counter)
            evs[k][1].record(stream)
            counter += n
        torch.cuda.synchronize(dev)
    launches = ctx.launches - l0
    kname = "k_vegas_step"
    kms, kl = ctx.kernel_time(kname)
    if kl == 0:  # the iteration ran as separate point, fold and adaptation kernels
        kname = "k_vegas_iter"
        kms, kl = ctx.kernel_time(kname)
    ctx.set_option("kernel_timing", 0)
    ms = sum(a.elapsed_time(b) for a, b in evs)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms_max = t.item()
    st = stats_dev[args.warmup:].cpu().numpy()
    pooled = (st * np.array([1, 0, 0, 1, 1, 1])).sum(axis=0)
    mean, err = gpu.stats_mean_error(pooled)
    c = VEGAS_COUNTERS
    peak = fp64_peak_tflops(dev)
    roof = {"kernel": kname, "bound": "fp64", "launches": kl, "ms_per_launch": kms / max(kl, 1),
            "share_of_step": kms / ms, "peak": peak, "unit": "TFLOP/s",
            "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
            "achieved": c["fp64_ops_per_point"] * n * kl / (kms / 1e3) / 1e12 if kl else None,
            "fp64_ops_per_point": c["fp64_ops_per_point"], "counters_source": c["source"],
            "traffic": c["dram_bytes_per_launch"], "algorithmic_bytes": 0,
            "note": "fused mode: uniforms drawn in the kernel, grid and histogram in L1/shared memory; "
                    "a 1e5-point launch is latency-bound (see materialised for the HBM-bound form)"}
    roof["frac"] = roof["achieved"] / peak if roof["achieved"] else None

    mat = vegas_materialised(ctx, dev, stream, cfg, n=args.gen_points)
    t01 = None if args.no_t01 else vegas_time_to_target(ctx, cfg, params, seed + 17, dev)
    e2e = None if args.no_e2e else vegas_e2e(ctx, cfg, args, dev, rank)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline_vegas(cfg)
    if rank == 0:
        line = {
            "metric": VEGAS_METRIC, "value": n * args.steps * world / (ms_max / 1e3), "unit": VEGAS_UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (on-device Philox4x32-10 uniforms)", "config": vegas_config(cfg),
            "parallelism": f"dp{world}: independent replicas" if world > 1 else "single GPU",
            "integral": mean, "rel_error": err / abs(mean), "time_to_0p1pct": t01,
            "clocks": clk.summary(), "gpu_launches": launches, "roofline": roof, "materialised": mat,
            "e2e": e2e, "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    ctx.close()


def vegas_materialised(ctx, dev, stream, cfg, n=100_000_000, reps=10):
    """chili_gpu_vegas_generate on the adapted grid: n points, x (8 dims B)
    and f*J (8 B) written per point; outputs (4 GB) far larger than L2."""
    import torch
    D = cfg["dims"]
    x = torch.empty((n, D), dtype=torch.float64, device=dev)
    w = torch.empty(n, dtype=torch.float64, device=dev)
    for r in range(3):
        ctx.vegas_generate(n, seed=cfg["seed"], counter=r * n, out=(x, w))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for r in range(reps):
        ctx.vegas_generate(n, seed=cfg["seed"], counter=(3 + r) * n, out=(x, w))
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / reps
    hbm = measured_peaks().get("hbm_gbs")
    b = 8 * (D + 1)
    achieved = b * n / (ms / 1e3) / 1e9
    mean = float(w.mean().item())
    del x, w
    return {"points_per_s": n / (ms / 1e3), "points_per_launch": n, "ms_per_launch": ms,
            "mean_weight": mean,
            "roofline": {"kernel": "k_vegas_generate", "bound": "hbm", "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm if hbm else None,
                         "algorithmic_bytes_per_point": b,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured copy bandwidth)",
                         "traffic": vegas_gen_traffic(n),
                         "traffic_source": "profiles/vegas_camel_kernels.md (40 B/point less the L2-resident "
                                           "tail, from captures at 4e6 and 2.5e7 points)"}}


# DRAM bytes of a k_vegas_generate launch of n points, from the committed
# ncu captures at 4e6 and 2.5e7 points (profiles/vegas_camel_kernels.md):
# 40 B per point written, less the ~60 MB of the output still in L2 when
# the kernel ends (99.9 MB and 939.5 MB measured)
def vegas_gen_traffic(n):
    return 40.0 * n - 60.1e6


def vegas_time_to_target(ctx, cfg, params, seed, dev, target=1e-3, max_iter=4000):
    """Wall time of Vegas iterations from a uniform grid until the pooled
    relative error is at most `target` (each iteration's StatsData read back
    to decide, as Vegas::Optimize does, Vegas.cc:56-61)."""
    import torch

    from chili_b200 import gpu
    ctx.uniform_grids(1, cfg["dims"], cfg["bins"])
    torch.cuda.synchronize(dev)
    pooled = np.zeros(6)
    t0 = time.perf_counter()
    it = 0
    rel = float("inf")
    while it < max_iter:
        st = ctx.vegas_iterate(cfg["ncalls"], seed=seed, counter=it * cfg["ncalls"], alpha=cfg["alpha"])
        pooled += np.array(st.as_tuple()) * np.array([1, 0, 0, 1, 1, 1])
        it += 1
        m, e = gpu.stats_mean_error(pooled)
        rel = e / abs(m)
        if rel <= target:
            break
    dt = time.perf_counter() - t0
    return {"seconds": dt if rel <= target else None, "iterations": it, "points": it * cfg["ncalls"],
            "rel_error": rel, "integral": float(gpu.stats_mean_error(pooled)[0]),
            "path": "chili_gpu_vegas_iterate per iteration with host StatsData, wall clock"}


def vegas_e2e(ctx, cfg, args, dev, rank):
    """The iteration through the C ABI with HOST buffers: the step's uniforms
    from pinned host memory (copied inside the call) and StatsData back."""
    import torch

    from chili_b200 import workloads
    n, D = cfg["ncalls"], cfg["dims"]
    rng = np.random.default_rng(4321 + rank)
    bufs = []
    for _ in range(2):
        t = torch.empty((n, D), dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = workloads.uniforms53(rng, (n, D))
        bufs.append(t.numpy())
    ctx.vegas_iterate(n, u=bufs[0], alpha=cfg["alpha"])
    torch.cuda.synchronize(dev)
    steps = max(5, args.steps)
    t0 = time.perf_counter()
    for s in range(steps):
        ctx.vegas_iterate(n, u=bufs[s % 2], alpha=cfg["alpha"])
    dt = time.perf_counter() - t0
    return {"value": n * steps / dt, "unit": VEGAS_UNIT, "h2d_bytes_per_step": n * D * 8,
            "d2h_bytes_per_step": 48, "steps": steps, "ms_per_step": dt / steps * 1e3,
            "path": "chili_gpu_vegas_iterate with host uniforms (pinned) and host StatsData, wall clock"}


def _vegas_ref_run(cfg, warmup, steps, target=None, max_iter=4000):
    from chili_b200.gpu import stats_mean_error
    from oracle.mpi_ranks import RefVegasMPI
    with RefVegasMPI(cpu_cores(), dims=cfg["dims"], bins=cfg["bins"], alpha=cfg["alpha"], ncalls=cfg["ncalls"],
                     seed=cfg["seed"]) as M:
        for _ in range(warmup):
            M.iterate()
        secs, pooled = 0.0, np.zeros(6)
        for _ in range(steps):
            st, sec = M.iterate()
            secs += sec
            pooled += np.array(st) * np.array([1, 0, 0, 1, 1, 1])
        t01 = None
        if target:
            M.edges = np.tile(np.arange(cfg["bins"] + 1, dtype=np.float64) / cfg["bins"], (cfg["dims"], 1))
            acc, tot, it = np.zeros(6), 0.0, 0
            while it < max_iter:
                st, sec = M.iterate()
                tot += sec
                it += 1
                acc += np.array(st) * np.array([1, 0, 0, 1, 1, 1])
                m, e = stats_mean_error(acc)
                if e / abs(m) <= target:
                    t01 = {"seconds": tot, "iterations": it, "points": it * M.ncalls_rank * M.nranks,
                           "rel_error": e / abs(m), "integral": m}
                    break
    return secs, pooled, M


def cpu_baseline_vegas(cfg, steps=20):
    from oracle import ref
    if not ref.available():
        return {"value": None, "unavailable": "oracle/_ref not built"}
    secs, pooled, M = _vegas_ref_run(cfg, 1, steps)
    pts = M.ncalls_rank * M.nranks * steps
    return {"value": pts / secs, "unit": VEGAS_UNIT, "cores": M.nranks, "kind": "reference",
            "sample": f"{steps} Vegas iterations of {M.ncalls_rank * M.nranks} points in the reference's MPI mode "
                      f"({M.nranks} processes of {M.ncalls_rank}), after one warm-up; time = the slowest rank "
                      f"plus the adaptation"}


def run_reference_vegas(args, rank, world):
    if rank != 0:
        return
    from oracle import ref
    from chili_b200 import workloads
    from chili_b200.gpu import stats_mean_error
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libchili_ref.so not built"}))
        return
    cfg = dict(workloads.VEGAS_CAMEL)
    if args.ncalls:
        cfg["ncalls"] = args.ncalls
    from oracle.mpi_ranks import RefVegasMPI
    with RefVegasMPI(cpu_cores(), dims=cfg["dims"], bins=cfg["bins"], alpha=cfg["alpha"], ncalls=cfg["ncalls"],
                     seed=cfg["seed"]) as M:
        for _ in range(args.warmup):
            M.iterate()
        secs, pooled = 0.0, np.zeros(6)
        for _ in range(args.steps):
            st, sec = M.iterate()
            secs += sec
            pooled += np.array(st) * np.array([1, 0, 0, 1, 1, 1])
        # time to 0.1% pooled error from a uniform grid
        M.edges = np.tile(np.arange(cfg["bins"] + 1, dtype=np.float64) / cfg["bins"], (cfg["dims"], 1))
        acc, tot, it, t01 = np.zeros(6), 0.0, 0, None
        while it < 4000:
            st, sec = M.iterate()
            tot += sec
            it += 1
            acc += np.array(st) * np.array([1, 0, 0, 1, 1, 1])
            m_, e_ = stats_mean_error(acc)
            if e_ / abs(m_) <= 1e-3:
                t01 = {"seconds": tot, "iterations": it, "rel_error": e_ / abs(m_), "integral": m_}
                break
    pts = M.ncalls_rank * M.nranks
    mean, err = stats_mean_error(pooled)
    value = pts * args.steps / secs
    cfg["ncalls"] = pts
    line = {
        "impl": "reference", "metric": VEGAS_METRIC, "value": value, "unit": VEGAS_UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (host uniforms)", "config": vegas_config(cfg),
        "parallelism": f"the reference's MPI mode over {M.nranks} host processes",
        "integral": mean, "rel_error": err / abs(mean), "time_to_0p1pct": t01,
        "cpu_baseline": {"value": value, "unit": VEGAS_UNIT, "cores": M.nranks, "kind": "reference",
                         "sample": f"each step: one Vegas iteration of {pts} points in the reference's MPI mode "
                                   f"({M.nranks} processes of {M.ncalls_rank}), time = the slowest rank plus the "
                                   f"adaptation"},
        "e2e": {"value": value, "unit": VEGAS_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------ batched workload
BATCH_METRIC = "integrand points/s over 512 uneven integrands, one adapting iteration each per step, FP64"
BATCH_UNIT = "points/s"
BATCH_SEED = 2024


def batched_config(tasks, world):
    kinds = [t["kind"] for t in tasks]
    return {"workload": "512 batched integrands: 256 camel functions (dims 2-12, sigma in [0.05, 0.2], centres in "
                        "[0.2, 0.8], 50 bins, grid alpha 1.5) + 256 multichannel 2->n propagator integrands "
                        "(n = 2..5, sqrt(S) in [200, 2000] GeV, 50 bins, channel weights adapted); points per "
                        "integrand log-uniform in [1e4, 1e6]; every drawn point is one call (fixed budget: the "
                        "reference's retry loop, option batch_retry, never finishes this batch: one task's channel "
                        "weights turn NaN after three iterations under it, as the C oracle shows)",
            "tasks": len(tasks), "camel_tasks": kinds.count("camel"),
            "multichannel_tasks": kinds.count("multichannel"),
            "points_per_iteration": int(sum(t["ncalls"] for t in tasks)), "seed": BATCH_SEED,
            "l2": "L2 flushed (256 MiB write) before every timed iteration",
            "parallelism": f"{world} ranks, each its own 512 integrands (no collective)" if world > 1
            else "single GPU"}


def sequential_batched_ms(tasks, local_rank):
    """The same tasks one call each through the single-integrand entry points
    (chili_gpu_vegas_iterate, chili_gpu_multichannel_iterate), second
    iteration of each timed by wall clock around the synchronous call."""
    from chili_b200 import abi, channels, gpu, workloads
    c = gpu.Context(local_rank)
    total = 0.0
    for k, t in enumerate(tasks):
        if t["kind"] == "camel":
            c.uniform_grids(1, t["dims"], t["bins"])
            c.set_integrand(abi.CHILI_FUNC_CAMEL, t["params"])
            run = lambda ctr: c.vegas_iterate(t["ncalls"], seed=BATCH_SEED + k, counter=ctr,
                                              alpha=t["grid_alpha"], adapt=True)
        else:
            cs = t["channels"]
            c.set_channels(cs)
            c.uniform_grids(cs.nch, cs.ndims, t["bins"])
            c.set_integrand(t["fkind"], t["params"])
            c.set_preprocess(t["pre"])
            p = workloads.mc_params(t["ncalls"], grid_alpha=t["grid_alpha"], beta=t["beta"],
                                    min_alpha=t["min_alpha"])
            run = lambda ctr: c.multichannel_iterate(p, seed=BATCH_SEED + k, counter=ctr)
        run(0)
        c.synchronize()
        t0 = time.perf_counter()
        run(1 << 32)
        c.synchronize()
        total += time.perf_counter() - t0
    c.close()
    return total * 1e3


def run_batched(args, rank, world, local_rank):
    import torch

    from chili_b200 import gpu, workloads

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    tasks = workloads.batched_tasks(seed=BATCH_SEED + rank, scale=args.batch_scale)
    npts = sum(t["ncalls"] for t in tasks)
    stream = torch.cuda.Stream(dev)
    ctx = gpu.Context(local_rank)
    ctx.set_stream(stream.cuda_stream)
    ctx.batch_set(tasks)
    t0 = time.perf_counter()
    _, info = ctx.batch_iterate(1, seed=BATCH_SEED)  # picks block size and points per thread, captures the graph
    setup_s = time.perf_counter() - t0
    for _ in range(max(args.warmup, 3) - 1):
        ctx.batch_iterate(1, seed=BATCH_SEED)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    ctx.set_option("kernel_timing", 0)
    torch.cuda.synchronize(dev)
    barrier()
    l0 = ctx.launches
    dev_ms, wall = 0.0, 0.0
    retry_rounds = 0
    pooled = np.zeros((len(tasks), 6))
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            stream.synchronize()
            w0 = time.perf_counter()
            st, info = ctx.batch_iterate(1, seed=BATCH_SEED)  # host StatsData read back inside the call
            wall += time.perf_counter() - w0
            dev_ms += info.ms_per_iteration
            retry_rounds += info.retry_rounds
            pooled += st[0]
    torch.cuda.synchronize(dev)
    launches = ctx.launches - l0
    barrier()
    t = torch.tensor([dev_ms, wall], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms_max, wall_max = t.tolist()
    seq_ms = None
    if not args.no_sequential and rank == 0:
        seq_ms = sequential_batched_ms(tasks, local_rank)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline_batched()
    if rank == 0:
        # points = StatsData calls (with the fixed budget, every drawn point;
        # the reference arm counts its calls, rejections included)
        calls = float(pooled[:, 0].sum())
        value = calls * world / (ms_max / 1e3)
        per_iter = ms_max / args.steps
        kinds = np.array([t["kind"] == "camel" for t in tasks])
        line = {
            "metric": BATCH_METRIC, "value": value, "unit": BATCH_UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_iter,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (on-device Philox4x32-10 uniforms, key seed + task)",
            "config": batched_config(tasks, world),
            "autotune": {"block": info.block, "points_per_thread": info.points_per_thread,
                         "units_per_iteration": info.units, "first_call_s": setup_s},
            "calls_per_iteration": calls / args.steps, "accepted_per_iteration": npts,
            "retry_rounds_timed": retry_rounds,
            "sequential": None if seq_ms is None else {
                "ms_per_iteration": seq_ms, "points_per_s": calls / args.steps / (seq_ms / 1e3),
                "batched_speedup": seq_ms / per_iter,
                "path": "one chili_gpu_vegas_iterate / chili_gpu_multichannel_iterate call per task "
                        "(multichannel with the reference's retry loop)"},
            "nonzero_fraction": {"camel": float(pooled[kinds, 5].sum() / pooled[kinds, 0].sum()),
                                 "multichannel": float(pooled[~kinds, 5].sum() / pooled[~kinds, 0].sum())},
            "clocks": clk.summary(),
            "gpu_launches": launches,
            "roofline": batched_roofline(per_iter, calls / args.steps, dev),
            "e2e": {"value": calls * world / wall_max, "unit": BATCH_UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(st.nbytes),
                    "path": "chili_gpu_batch_iterate (graph replay + host StatsData of every task) by wall clock; "
                            "the uniforms are counter-based and drawn in the kernel, as the reference draws its "
                            "own"},
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    ctx.close()


# One iteration's kernels per drawn point, all tasks together (the small case
# keeps the tasks' mix: every point count scaled by 1/16), from the committed
# ncu capture (the batched-integrands summary under profiles/): FP64
# operations (2*DFMA + DADD + DMUL, executed) and DRAM bytes (read + write).
BATCH_COUNTERS = {"fp64_ops_per_point": 3623.3, "dram_bytes_per_point": 651.0,
                  "source": "profiles/batched_integrands.md"}


def batched_roofline(ms_per_iter, npts, dev):
    """The iteration's kernels together (k_batch_eval for the camel tasks;
    k_bt_forward, the phased k_pp_* weight pass and k_bt_accum for the
    multichannel ones) against the FP64 peak measured in this run, over the
    iteration's npts calls; the algorithmic HBM traffic is nil
    (counter-based uniforms, grids and histograms in L2; the phased buffers
    of one task tile)."""
    peak = fp64_peak_tflops(dev)
    c = BATCH_COUNTERS
    achieved = c["fp64_ops_per_point"] * npts / (ms_per_iter / 1e3) / 1e12
    return {"kernel": "k_batch_eval + k_bt_forward + k_pp_* + k_bt_accum (one iteration)", "bound": "fp64",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
            "traffic": c["dram_bytes_per_point"] * npts, "counters_source": c["source"],
            "note": "ms_per_iter is the whole iteration (evaluation, folds, adaptation)"}


def _ref_batch_init():
    global _WB
    # the reference's Vegas prints its result to stdout: keep the workers quiet
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    sys.path.insert(0, ROOT)
    from chili_b200 import abi, workloads
    from oracle import ref
    _WB = {"tasks": workloads.batched_tasks(seed=BATCH_SEED), "ref": ref, "abi": abi, "wl": workloads,
           "rng": np.random.default_rng(os.getpid())}


BATCH_SAMPLE_CALLS = 20000


def _ref_batch_step(k):
    """One iteration of task k through the reference's own Vegas or
    MultiChannel object and its own random numbers (points capped at
    BATCH_SAMPLE_CALLS); returns (points drawn, seconds)."""
    t = _WB["tasks"][k]
    ref, wl = _WB["ref"], _WB["wl"]
    n = min(t["ncalls"], BATCH_SAMPLE_CALLS)
    seed = int(_WB["rng"].integers(1, 2 ** 31))
    if t["kind"] == "camel":
        t0 = time.perf_counter()
        ref.vegas_run(t["dims"], t["bins"], t["grid_alpha"], t["params"], seed, n, 1)
        return n, time.perf_counter() - t0
    p = wl.mc_params(n, iterations=1, grid_alpha=t["grid_alpha"], beta=t["beta"], min_alpha=t["min_alpha"])
    R = ref.MultiChannel(t["channels"], t["bins"], p, t["fkind"], t["params"], pre=t["pre"])
    t0 = time.perf_counter()
    st = R.run_native(seed, 1)  # StatsData n counts every drawn point (rejections add a 0)
    return int(st.n), time.perf_counter() - t0


def _batch_pool(cores):
    import multiprocessing as mp
    return mp.get_context("spawn").Pool(cores, initializer=_ref_batch_init)


def cpu_baseline_batched(steps=1):
    """The reference's own code on the host cores: one iteration of every
    16th task (32 tasks, points capped at 20000 each), tasks spread over all
    cores; points/s = points drawn / wall time."""
    from oracle import ref
    if not ref.available():
        return {"value": None, "unavailable": "oracle/_ref not built"}
    cores = cpu_cores()
    sample = list(range(0, 512, 16))
    with _batch_pool(cores) as pool:
        pool.map(_ref_batch_step, sample[:cores])  # warm-up
        t0 = time.perf_counter()
        pts = 0
        for _ in range(steps):
            pts += sum(r[0] for r in pool.map(_ref_batch_step, sample))
        dt = time.perf_counter() - t0
    return {"value": pts / dt, "unit": BATCH_UNIT, "cores": cores, "kind": "reference",
            "sample": f"one iteration of every 16th task (32 tasks, at most {BATCH_SAMPLE_CALLS} points each; "
                      f"multichannel tasks with the reference's retry loop) per step, tasks spread over {cores} "
                      f"cores"}


def run_reference_batched(args, rank, world):
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libchili_ref.so not built"}))
        return
    from chili_b200 import workloads
    tasks = workloads.batched_tasks(seed=BATCH_SEED)
    cores = cpu_cores()
    sample = list(range(0, 512, 16))
    pts = 0
    with _batch_pool(cores) as pool:
        for _ in range(args.warmup):
            pool.map(_ref_batch_step, sample)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            pts += sum(r[0] for r in pool.map(_ref_batch_step, sample))
        dt = time.perf_counter() - t0
    value = pts / dt
    line = {
        "impl": "reference", "metric": BATCH_METRIC, "value": value, "unit": BATCH_UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (host uniforms)", "config": batched_config(tasks, 1),
        "cpu_baseline": {"value": value, "unit": BATCH_UNIT, "cores": cores, "kind": "reference",
                         "sample": f"each step: one iteration of every 16th task (32 tasks, at most "
                                   f"{BATCH_SAMPLE_CALLS} points each), tasks spread over {cores} cores"},
        "e2e": {"value": value, "unit": BATCH_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    global WL
    args = parse()
    if args.workload in WORKLOADS:
        WL = WORKLOADS[args.workload]
    if args.ncalls is None and args.workload in WORKLOADS:
        args.ncalls = WL["ncalls"]
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        if args.workload == "batched":
            run_reference_batched(args, rank, world)
        elif args.workload == "vegas":
            run_reference_vegas(args, rank, world)
        else:
            run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local_rank))
    try:
        if args.workload == "batched":
            run_batched(args, rank, world, local_rank)
        elif args.workload == "vegas":
            run_vegas(args, rank, world, local_rank)
        else:
            run_chili(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
