#!/usr/bin/env python
"""Spectral placement throughput: placements per second on the B200 path.

One step is one greedy placement: every catalog orientation's page over the
current layout (legal-translation FFT correlation of occupancy + proximity,
fused threshold / score / top-k, exact recount and rescoring), the page merge,
and the stamp of the chosen copy (rasterise, dilate, update counts, occupancy,
exact EDT and the environment spectrum for the next step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

Under torchrun (N > 1) each rank packs an independent seeded job (replicas:
the path has no data exchange between jobs); value = all ranks' placements /
max over ranks of the device time.  --impl reference times the reference's
own CPU implementation of the same per-orientation page (compiled from its
sources, single-threaded on Linux) on the host cores.
"""

from __future__ import annotations

import argparse
import ctypes
import importlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
METRIC = "placements/s at 256^3 grid x512 orients: learned-proposal vs exhaustive GPU"
UNIT = "placements/s"
# dram__bytes_read.sum + dram__bytes_write.sum of one pass_a256_kernel launch,
# mean of the four launches captured in profiles/step_kernels_rounded256_o16.md
# (211,964,672 / 211,798,016 / 211,456,000 / 211,373,312 bytes).
PASS_A256_DRAM_BYTES = 211648000
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cpp-max-packer_b200", "weights",
                               "proposal_rounded256.npz")


def pkg(name):
    return importlib.import_module("cpp-max-packer_b200." + name)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def step_model(fft_shape, env_shape, orientations, ms_per_step, hbm_gbs):
    """Whole-step figures for one exhaustive placement step, beside the
    pass-A kernel roofline.

    Bytes: the floor of a fully fused design with FFT length L per axis,
    P = L^3 and Ph = (L/2 + 1) L^2 complex-FP32 half spectra (8 B each).  Per
    orientation it reads the kernel spectrum once (8 Ph) and makes one round
    trip of an inverse-transform intermediate (16 Ph).  Per step it reads the
    two environment spectra once (16 Ph), runs two forward environment
    transforms (48 Ph), the EDT (24 B per window cell) and the stamp and
    occupancy update (2 B per cell):
        bytes_step = 24 Ph O + 64 Ph + 26 E^3.
    FLOPs: 2.5 P log2 P per real transform; a step inverts a binary and a
    proximity correlation per orientation and transforms both environment
    fields forward: (2 O + 2) transforms.  The paged pipeline prunes to
    legal translations, so it does less than this full-range count.
    """
    import math

    L = [int(v) for v in fft_shape]
    P = L[0] * L[1] * L[2]
    Ph = (L[0] // 2 + 1) * L[1] * L[2]
    E3 = int(env_shape[0]) * int(env_shape[1]) * int(env_shape[2])
    O = int(orientations)
    bytes_step = 24 * Ph * O + 64 * Ph + 26 * E3
    flops_step = 2.5 * P * math.log2(P) * (2 * O + 2) if P > 1 else 0.0
    seconds = ms_per_step / 1000.0
    achieved = bytes_step / seconds / 1e9 if seconds > 0 else 0.0
    return {"model_bytes_per_step": int(bytes_step), "achieved": round(achieved, 1), "peak": hbm_gbs,
            "unit": "GB/s", "frac": round(achieved / hbm_gbs, 4) if hbm_gbs > 0 else None,
            "floor_ms_per_step": round(bytes_step / (hbm_gbs * 1e9) * 1000.0, 3) if hbm_gbs > 0 else None,
            "ms_per_step": round(ms_per_step, 4), "fft_flops_per_step": flops_step,
            "fft_tflops": round(flops_step / seconds / 1e12, 3) if seconds > 0 else 0.0}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def timed_steps(stream, fn, dist):
    """Runs fn() between a barrier + synchronize on both sides with CUDA
    events on the library's stream; returns (ms, result)."""
    import torch

    if dist:
        import torch.distributed as tdist

        tdist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    out = fn()
    end.record(stream)
    torch.cuda.synchronize()
    if dist:
        import torch.distributed as tdist

        tdist.barrier()
    return start.elapsed_time(end), out


def max_over_ranks(ms, placed, world):
    """(max ms over ranks, placements summed over ranks).  The exchanged pair
    sits on the device the process group's backend serves: CUDA under NCCL,
    the host under gloo."""
    if world == 1:
        return ms, float(placed)
    import torch
    import torch.distributed as tdist

    device = "cuda" if tdist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([ms, float(placed)], device=device)
    gathered = [torch.zeros_like(t) for _ in range(world)]
    tdist.all_gather(gathered, t)
    return max(float(g[0]) for g in gathered), sum(float(g[1]) for g in gathered)


def reset_layout(session):
    while session.placements:
        session.remove_last()


def run_ours(args, rank, world, local_rank):
    import torch

    compute, session_mod, workloads, lib_mod = pkg("compute"), pkg("session"), pkg("workloads"), pkg("_lib")
    proposal = pkg("proposal")
    torch.cuda.set_device(local_rank)
    ctx = compute.Context(local_rank)
    lib = lib_mod.lib()
    wl = workloads.WORKLOADS[args.workload](seed=2 + rank) if args.workload != "box64_cuboid_cube24" else \
        workloads.WORKLOADS[args.workload]()
    if args.orientations:
        wl.catalog = wl.catalog[: args.orientations]
    O = len(wl.catalog)
    t0 = time.time()
    session = session_mod.Session(wl.obj, wl.container, wl.origin, wl.pitch, wl.catalog, wl.pair_clearance,
                                  wl.wall_clearance, context=ctx)
    open_s = time.time() - t0
    stream = torch.cuda.ExternalStream(lib.spk_context_stream(ctx.handle))
    dist = world > 1
    weights = args.weights if args.weights else DEFAULT_WEIGHTS
    learned = args.mode == "learned" and os.path.exists(weights)
    k = min(args.k, O)

    with ClockSampler(local_rank) as clocks:
        # Exhaustive arm: every orientation paged at every step.
        session.greedy(args.warmup)
        session.stats(reset=True)
        launches0 = ctx.launches
        exhaustive_offset = int(launches0)
        ex_ms, ex_placed = timed_steps(stream, lambda: session.greedy(args.steps), dist)
        ex_launches = ctx.launches - launches0
        page_stats = session.stats(reset=True)
        ex_ms, ex_total = max_over_ranks(ex_ms, len(ex_placed), world)
        ex_value = ex_total / (ex_ms / 1000.0) if ex_ms > 0 else 0.0
        ex_sequence = [(p.orientation_index, p.translation) for p in session.placements]

        ln_value, ln_ms, ln_placed, fallbacks, ln_launches, ln_sequence = None, None, [], 0, 0, []
        learned_offset = None
        if learned:
            net = proposal.Proposal(seed=0, context=ctx)
            net.load(weights)
            reset_layout(session)
            proposal.greedy_proposed(session, net, k, args.warmup)
            launches0 = ctx.launches
            learned_offset = int(launches0)
            ln_ms, (ln_placed, fallbacks) = timed_steps(
                stream, lambda: proposal.greedy_proposed(session, net, k, args.steps), dist)
            ln_launches = ctx.launches - launches0
            ln_ms, ln_total = max_over_ranks(ln_ms, len(ln_placed), world)
            ln_value = ln_total / (ln_ms / 1000.0) if ln_ms > 0 else 0.0
            ln_sequence = [(p.orientation_index, p.translation) for p in session.placements]

    if args.no_extras:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": round(ln_value if learned else ex_value, 4), "unit": UNIT,
                              "profiling_run": True, "exhaustive_value": round(ex_value, 4),
                              "ms_per_step": round((ln_ms if learned else ex_ms) / max(args.steps, 1), 4),
                              "gpu_launches": int(ln_launches if learned else ex_launches),
                              # library launches before the learned timed steps (an ncu -s skip count)
                              "launches_before_learned_steps": learned_offset,
                              "launches_before_exhaustive_steps": exhaustive_offset,
                              "page_stats": page_stats}))
        session.close()
        ctx.close()
        return

    # Roofline of pass A (the dominant spectral pass), timed with events on the
    # context stream around each launch during two further exhaustive steps.
    lib.spk_context_set_profiling(ctx.handle, 1)
    session.greedy(2)
    launches_arr = np.zeros(4, np.uint64)
    total_ms = np.zeros(4, np.float64)
    lib.spk_context_pass_times(ctx.handle, launches_arr.ctypes.data, total_ms.ctypes.data, 4)
    pass_bytes = np.zeros(4, np.float64)
    lib.spk_context_pass_bytes(ctx.handle, pass_bytes.ctypes.data, 4)
    lib.spk_context_set_profiling(ctx.handle, 0)
    hbm, peak_kind = peaks()
    launches_a = max(int(launches_arr[0]), 1)
    bytes_a = pass_bytes[0] / launches_a  # algorithmic bytes per pass-A launch (one orientation)
    avg_a_ms = total_ms[0] / launches_a
    achieved = bytes_a / (avg_a_ms / 1000.0) / 1e9 if avg_a_ms > 0 else 0.0
    pass_share = {name: round(float(total_ms[i] / max(total_ms.sum(), 1e-9)), 3)
                  for i, name in enumerate(["spectral_z", "inverse_y", "inverse_x_epilogue", "merge_exact"])}

    # End to end through the public API with host buffers: the proposal
    # (predictions out), page queries in, pages out, the chosen copy placed.
    e2e_steps = max(1, min(args.steps, 8))
    pipeline = pkg("pipeline")
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    e2e_placed, h2d, d2h = 0, 0, 0
    for _ in range(e2e_steps):
        if learned:
            orients, _ = proposal.propose(session, net, k)
            orients = [int(o) for o in orients]
            d2h += 4 * O + 8 * k
        else:
            orients = list(range(O))
        pages = session.pages(orients)
        h2d += ctypes.sizeof(pipeline.PageQueryC) * len(orients)
        d2h += (ctypes.sizeof(pipeline.CandidateC) * 32 + 4 + ctypes.sizeof(pipeline.PageReportC)) * len(orients)
        heads = [next(c for c in p if c.direct_zero_overlap) for p in pages if any(c.direct_zero_overlap for c in p)]
        if not heads and learned:
            pages = session.pages(range(O))
            h2d += ctypes.sizeof(pipeline.PageQueryC) * O
            d2h += (ctypes.sizeof(pipeline.CandidateC) * 32 + 4 + ctypes.sizeof(pipeline.PageReportC)) * O
            heads = [next(c for c in p if c.direct_zero_overlap) for p in pages if any(c.direct_zero_overlap for c in p)]
        if not heads:
            break
        best = min(heads, key=lambda c: (c.score, c.orientation_index, c.translation[2], c.translation[1],
                                         c.translation[0]))
        session.place(best.orientation_index, best.translation)
        h2d += 8 + 24
        e2e_placed += 1
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t1
    e2e = {"value": round(e2e_placed / e2e_s, 4) if e2e_s > 0 else 0.0, "unit": UNIT,
           "h2d_bytes_per_step": int(h2d / max(e2e_placed, 1)), "d2h_bytes_per_step": int(d2h / max(e2e_placed, 1)),
           "steps": e2e_placed, "path": "propose + pages + place" if learned else "pages + place"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(wl, O)

    if rank == 0:
        value = ln_value if learned else ex_value
        ms = ln_ms if learned else ex_ms
        same = 0
        for a, b in zip(ex_sequence, ln_sequence):
            if a != b:
                break
            same += 1
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / max(args.steps, 1), 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32 spectra, fp64 exact scores, u8 fields, bf16 proposal network",
            "data": "synthetic (seeded rounded-box STL container, spherical-harmonic blob item, seeded SO(3) catalog)",
            "config": {"workload": wl.name, "grid": list(session.environment_shape), "fft": list(session.fft_shape),
                       "orientations": O, "object_triangles": int(len(wl.obj.triangles)),
                       "container_triangles": int(len(wl.container.triangles)) if hasattr(wl.container, "triangles")
                       else 0,
                       "mode": f"learned proposal (top {k} of {O}, exhaustive fallback)" if learned else "exhaustive",
                       "l2": "working set above L2 (all orientations' kernel spectra stay in HBM)",
                       "session_open_s": round(open_s, 2), "parallelism": f"replicas x{world}",
                       "page_stats_exhaustive": page_stats},
            "exhaustive": {"value": round(ex_value, 4), "ms_per_step": round(ex_ms / max(args.steps, 1), 4),
                           "gpu_launches": int(ex_launches),
                           "step_model": step_model(session.fft_shape, session.environment_shape, O,
                                                    ex_ms / max(args.steps, 1), hbm)},
            "gpu_launches": int(ln_launches if learned else ex_launches),
            "roofline": {"bound": "hbm", "kernel": "pass_a256_kernel (spectral z pass)",
                         "achieved": round(achieved, 1), "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": round(achieved / hbm, 4),
                         # DRAM read + write bytes of one pass_a256 launch (one orientation), cold-cache ncu
                         # capture of the same kernel on this workload's 256^3 window; see profiles/.
                         "traffic": PASS_A256_DRAM_BYTES if tuple(session.fft_shape) == (256, 256, 256) else None,
                         "algorithmic_bytes_per_launch": int(bytes_a), "avg_launch_ms": round(avg_a_ms, 5),
                         "pass_share": pass_share},
            "e2e": e2e,
            "clocks": clocks.summary(),
        }
        if learned:
            line["proposal"] = {"k": k, "weights": os.path.relpath(weights, os.path.dirname(os.path.abspath(__file__))),
                                "learned_over_exhaustive": round(value / ex_value, 3) if ex_value else None,
                                "fallback_steps": int(fallbacks),
                                "same_placements_as_exhaustive": f"{same} of first {len(ex_sequence)}"}
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if learned:
        net.close()
    session.close()
    ctx.close()


def reference_sample(wl, z_planes: int = 16, orientation: int = 0, barrier=None):
    """The reference's own correlate_binary_cpu + correlate_proximity_cpu
    (compiled from its sources; FP64 FFT with a Bluestein stand-in for
    pocketfft) for one orientation's kernel against the lowest `z_planes`
    planes of the workload's environment window (the empty layout's container
    blocker and proximity).  Preparation runs before `barrier`; only the two
    correlations are timed.  Returns (seconds, sampled padded cells, full
    padded cells, kernel shape, window shape)."""
    from oracle.bindings import Ref, ref_voxelize_container

    geometry = pkg("geometry")
    ref = Ref()
    obj = ref.asset(wl.object_stl)
    kfirst, kshape, kernel = obj.voxelize_object(wl.origin, wl.pitch, wl.catalog[orientation])
    if wl.container_stl:
        container = ref.asset(wl.container_stl, container=True)
        v, t, b = container.mesh()
        bounds = list(b)
    else:
        container = tuple(wl.container)
        bounds = [0, 0, 0, *wl.container]
    first, shape = geometry.environment_window(bounds, wl.origin, wl.pitch)
    sub_shape = (shape[0], shape[1], min(z_planes, shape[2]))
    mask = ref_voxelize_container(ref, container, wl.origin, wl.pitch, first, sub_shape, wl.wall_clearance)
    prox = ref.build_proximity(sub_shape, mask)
    if barrier is not None:
        barrier.wait()
    t0 = time.perf_counter()
    b = ref.correlate(False, sub_shape, kshape, first, kfirst, mask, kernel)
    p = ref.correlate(True, sub_shape, kshape, first, kfirst, prox, kernel)
    seconds = time.perf_counter() - t0
    if isinstance(b, str) or isinstance(p, str):
        raise RuntimeError(f"reference correlation failed: {b if isinstance(b, str) else p}")
    padded_sample = float(np.prod([e + k - 1 for e, k in zip(sub_shape, kshape)]))
    padded_full = float(np.prod([e + k - 1 for e, k in zip(shape, kshape)]))
    return seconds, padded_sample, padded_full, tuple(int(v) for v in kshape), tuple(int(v) for v in sub_shape)


def _sample_worker(workload, z_planes, orientation, barrier, queue):
    try:
        wl = pkg("workloads").WORKLOADS[workload]()
        queue.put((orientation, reference_sample(wl, z_planes, orientation, barrier)))
    except Exception as exc:  # reported to the parent, which fails the measurement
        try:
            barrier.abort()
        except Exception:
            pass
        queue.put((orientation, f"{type(exc).__name__}: {exc}"))


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_throughput(wl, z_planes: int = 16, workers: int = 0):
    """Reference CPU placements/s for the workload: `workers` processes (one
    per host core by default; spawned, so they are safe beside a CUDA
    context) each correlate a different orientation's sampled page at the
    same time.  The reference parallelises its FFT only on Windows, so on
    this host concurrency comes from independent orientations, which is how a
    multi-core caller would use it.  Each sample is scaled by P log P to the
    full page; the step takes ceil(O / workers) rounds of the slowest worker.
    Returns (placements/s, workers, description)."""
    import multiprocessing as mp

    O = len(wl.catalog)
    workers = max(1, min(workers or host_cores(), O, 128))
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(workers)
    queue = ctx.Queue()
    stride = max(1, O // workers)
    procs = [ctx.Process(target=_sample_worker, args=(wl.name, z_planes, (i * stride) % O, barrier, queue))
             for i in range(workers)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=1800) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    errors = [r for _, r in results if isinstance(r, str)]
    if errors:
        raise RuntimeError(errors[0])
    scaled = [scaled_step_seconds(r[0], r[1], r[2], 1) for _, r in results]
    rounds = -(-O // workers)
    step = max(scaled) * rounds
    sec = [r[0] for _, r in results]
    r0 = results[0][1]
    desc = (f"reference correlate_binary_cpu + correlate_proximity_cpu (FP64, Bluestein stand-in for pocketfft) "
            f"in {workers} concurrent processes, each one orientation's ~{r0[3]} kernel against the lowest "
            f"{r0[4][2]} z-planes of the window ({min(sec):.1f}-{max(sec):.1f} s, {r0[1]:.3g} padded cells); "
            f"each scaled by P log P to the full {r0[2]:.3g}-cell page, slowest worker x {rounds} rounds "
            f"for {O} orientations per placement")
    return 1.0 / step, workers, desc


def scaled_step_seconds(seconds, padded_sample, padded_full, orientations):
    return seconds * (padded_full * np.log2(padded_full)) / (padded_sample * np.log2(padded_sample)) * orientations


def cpu_baseline(wl, orientations):
    """Reported baseline only: the reference's own CPU correlation work for a
    bounded sample of the same workload on all host cores, scaled to a
    placement step."""
    cores = host_cores()
    try:
        from oracle.bindings import REF_SO

        if not os.path.exists(REF_SO) or not wl.object_stl:
            return None
        value, cores, desc = reference_throughput(wl)
        return {"value": round(value, 8), "unit": UNIT, "cores": cores, "kind": "reference", "sample": desc}
    except Exception as exc:  # the baseline is reported, never required
        return {"value": None, "unit": UNIT, "cores": cores, "kind": "reference", "sample": f"unavailable: {exc}"}


def run_reference(args, rank, world):
    """The reference's own CPU implementation of the path (compiled from its
    sources into oracle/_ref), on every host core: each step is one bounded
    concurrent sample (see reference_throughput), scaled to placements/s of
    the same workload."""
    if rank != 0:
        return
    workloads = pkg("workloads")
    wl = workloads.WORKLOADS[args.workload]()
    if args.orientations:
        wl.catalog = wl.catalog[: args.orientations]
    O = len(wl.catalog)
    try:
        from oracle.bindings import REF_SO

        if not os.path.exists(REF_SO):
            print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libspk_ref.so missing"}))
            return
        for _ in range(args.warmup):
            reference_sample(wl, z_planes=2)
        values = []
        desc, cores = "", 1
        for _ in range(args.steps):
            v, cores, desc = reference_throughput(wl)
            values.append(v)
        value = float(np.mean(values))
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": round(value, 8), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000.0 / value, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": wl.name, "orientations": O, "mode": "exhaustive"},
            "cpu_baseline": {"value": round(value, 8), "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": desc},
            "e2e": {"value": round(value, 8), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }), flush=True)
    except Exception as exc:
        print(json.dumps({"impl": "reference", "unavailable": f"{type(exc).__name__}: {exc}"}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rounded256_blob_hopf512")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--orientations", type=int, default=0, help="use the first N catalog entries (profiling runs)")
    ap.add_argument("--no-extras", action="store_true", help="skip the roofline and e2e passes (profiling runs)")
    ap.add_argument("--mode", default="learned", choices=["learned", "exhaustive"],
                    help="headline path (the exhaustive path is always timed beside it)")
    ap.add_argument("--k", type=int, default=32, help="orientations the proposal pages per step")
    ap.add_argument("--weights", default="", help="proposal network parameters (.npz)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as tdist

            tdist.destroy_process_group()


if __name__ == "__main__":
    main()
