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
# The page pipeline's passes as the library's per-pass timing reports them.
PASSES = [
    ("pass_a256_batch_kernel", "spectral z: environment spectrum read once per batch of orientations, kernel z "
                               "finish, conjugate product, inverse z"),
    ("pass_b1_256_batch_kernel", "inverse y over the legal z planes, a batch of orientations per launch"),
    ("pass_b2_256_batch_kernel", "inverse x with the fused threshold / score / top-k epilogue, a batch of "
                                 "orientations per launch"),
    ("merge_kernel + exact_kernel", "key merge and exact recount"),
    ("pass_stage256_kernel", "pipelined stage: pass A of one batch of 16 orientations with B1 and B2 of the two "
                             "batches before it, their blocks interleaved in one launch"),
]
# DRAM read + write bytes per launch of each kernel on the 256^3 workload,
# from the ncu capture summarised in profiles/page_passes_rounded256_o16.md
# (dram__bytes.sum.per_second x duration; each launch there does the same
# work as in the 512-orientation workload).
NCU_DRAM_BYTES = {
    "pass_a256_batch_kernel": 2232506604,
    "pass_b1_256_batch_kernel": 3796781901,
    "pass_b2_256_batch_kernel": 1862432076,
}
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


class profiler_region:
    """cudaProfilerStart/Stop around one timed arm, so that a profiler started
    with --profile-from-start off records only that arm's launches."""

    def __init__(self, active: bool):
        self.active = active

    def __enter__(self):
        if self.active:
            import torch

            torch.cuda.profiler.start()
        return self

    def __exit__(self, *exc):
        if self.active:
            import torch

            torch.cuda.synchronize()
            torch.cuda.profiler.stop()


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
        # Exhaustive arm: every orientation paged at every step (a profiling
        # run of the learned arm alone may skip it).
        skip_exhaustive = args.no_extras and args.profile_region == "learned"
        session.greedy(0 if skip_exhaustive else args.warmup)
        session.stats(reset=True)
        launches0 = ctx.launches
        exhaustive_offset = int(launches0)
        with profiler_region(args.profile_region == "exhaustive"):
            ex_ms, ex_placed = timed_steps(stream, lambda: session.greedy(0 if skip_exhaustive else args.steps),
                                           dist)
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
            with profiler_region(args.profile_region == "learned"):
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

    # Roofline of the page passes, timed with events on the context stream
    # around each launch: during six further steps of the headline path (the
    # learned steps when the proposal is on), and during two further
    # exhaustive steps.  The bench line's roofline is the pass with the
    # largest share of the headline path's time.
    hbm, peak_kind = peaks()
    full256 = tuple(session.fft_shape) == (256, 256, 256)

    def profile_passes(run_steps):
        lib.spk_context_set_profiling(ctx.handle, 1)
        run_steps()
        launches_arr = np.zeros(len(PASSES), np.uint64)
        total_ms = np.zeros(len(PASSES), np.float64)
        lib.spk_context_pass_times(ctx.handle, launches_arr.ctypes.data, total_ms.ctypes.data, len(PASSES))
        pass_bytes = np.zeros(len(PASSES), np.float64)
        lib.spk_context_pass_bytes(ctx.handle, pass_bytes.ctypes.data, len(PASSES))
        lib.spk_context_set_profiling(ctx.handle, 0)
        out = []
        for i, (kernel, what) in enumerate(PASSES):
            n = max(int(launches_arr[i]), 1)
            avg_ms = total_ms[i] / n
            per_launch = pass_bytes[i] / n
            achieved_i = per_launch / (avg_ms / 1000.0) / 1e9 if avg_ms > 0 and per_launch > 0 else None
            out.append({"kernel": kernel, "work": what, "launches": int(launches_arr[i]),
                        "share": round(float(total_ms[i] / max(total_ms.sum(), 1e-9)), 3),
                        "avg_launch_ms": round(avg_ms, 5), "algorithmic_bytes_per_launch": int(per_launch),
                        "achieved_gbs": round(achieved_i, 1) if achieved_i else None,
                        "frac": round(achieved_i / hbm, 4) if achieved_i else None,
                        "traffic": NCU_DRAM_BYTES.get(kernel) if full256 else None})
        return out

    passes_exhaustive = profile_passes(lambda: session.greedy(2))
    passes = profile_passes(lambda: proposal.greedy_proposed(session, net, k, 6)) if learned else passes_exhaustive
    # The candidates for the roofline: every pass but the merge and recount.
    dominant = max((p for i, p in enumerate(passes) if i != 3 and p["launches"]), key=lambda p: p["share"])

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
        cpu = cpu_baseline(args.workload, O)
    broad = broad_phase_line(ctx, with_cpu=rank == 0 and world == 1 and not args.no_cpu_baseline)
    stl = stl_export_line(ctx, with_cpu=rank == 0 and world == 1 and not args.no_cpu_baseline)

    if rank == 0:
        config = reference_config(args.workload, world)
        config["orientations"] = O
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
            "config": config,
            "mode": f"learned proposal (top {k} of {O}, exhaustive fallback)" if learned else "exhaustive",
            "fft": list(session.fft_shape), "session_open_s": round(open_s, 2), "page_stats_exhaustive": page_stats,
            "exhaustive": {"value": round(ex_value, 4), "ms_per_step": round(ex_ms / max(args.steps, 1), 4),
                           "gpu_launches": int(ex_launches),
                           "step_model": step_model(session.fft_shape, session.environment_shape, O,
                                                    ex_ms / max(args.steps, 1), hbm)},
            "gpu_launches": int(ln_launches if learned else ex_launches),
            "roofline": {"bound": "hbm", "kernel": f"{dominant['kernel']} ({dominant['work']})",
                         "achieved": dominant["achieved_gbs"], "peak": hbm,
                         "peak_kind": f"{peak_kind} (burst copy bandwidth; each launch is timed alone)",
                         "unit": "GB/s", "frac": dominant["frac"], "traffic": dominant["traffic"],
                         "algorithmic_bytes_per_launch": dominant["algorithmic_bytes_per_launch"],
                         "avg_launch_ms": dominant["avg_launch_ms"], "share": dominant["share"],
                         "passes": passes, "passes_measured_on": "learned steps" if learned else "exhaustive steps",
                         "passes_exhaustive": passes_exhaustive},
            "e2e": e2e,
            "clocks": clocks.summary(),
            "validator_broad_phase": broad,
            "stl_export": stl,
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


def broad_phase_line(ctx, with_cpu: bool, copies: int = 3580):
    """The validator broad phase (spk_broad_phase) on a full fill's number of
    copies of the bench item: pairs per second through the C ABI with host
    buffers (bounds in, unresolved pairs out), and, as its CPU baseline, the
    oracle's plain-C pair loop on one host core over the same bounds, whose
    pair list must be the same."""
    bp = pkg("broad_phase_bench")
    lo, hi, fin = bp.layout(copies)
    pairs = copies * (copies - 1) // 2
    seconds, got = bp.time_device(lo, hi, fin, 0.0, 10, ctx)
    line = {"metric": "copy pairs tested per second", "copies": copies, "pairs": pairs,
            "unresolved_pairs": int(len(got)), "value": round(pairs / seconds, 1), "ms_per_call": round(seconds * 1e3, 3),
            "path": "spk_posed_bounds on the host, spk_broad_phase with host buffers"}
    if with_cpu:
        from oracle.bindings import C

        t0 = time.perf_counter()
        want, count = C().broad_phase(lo, hi, fin, None, 0.0)
        cpu_s = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": round(pairs / cpu_s, 1), "unit": "pairs/s", "cores": 1, "kind": "port",
                                "sample": f"all {pairs} pairs of the same layout (oracle_broad_phase)",
                                "same_pairs": bool(np.array_equal(got, want))}
    return line


def stl_export_line(ctx, with_cpu: bool, copies: int = 512, cpu_copies: int = 16):
    """STL export of a placement sequence (spk_export_stl): triangles per
    second through the C ABI with host buffers (poses in, the file's bytes
    out), for `copies` posed copies of the bench item; as its CPU baseline,
    the reference build's own record loop (RigidTransform, libm hypot) on one
    host core over the first `cpu_copies` poses, whose bytes must match."""
    bp, geometry = pkg("broad_phase_bench"), pkg("geometry")
    obj, stl_bytes, t, q = bp.poses(copies)
    triangles = copies * len(obj.triangles)
    out = np.zeros(84 + 50 * triangles, np.uint8)  # the caller's file buffer, touched once
    size = geometry.export_stl(obj, t, q, context=ctx, out=out)  # device buffers and first-call costs
    repeats = 3
    t0 = time.perf_counter()
    for _ in range(repeats):
        size = geometry.export_stl(obj, t, q, context=ctx, out=out)
    seconds = (time.perf_counter() - t0) / repeats
    line = {"metric": "STL triangles exported per second", "copies": copies, "triangles": triangles,
            "bytes": int(size), "value": round(triangles / seconds, 1), "ms_per_call": round(seconds * 1e3, 3),
            "path": "spk_export_stl into a host buffer (poses in, the file's bytes out)"}
    if with_cpu:
        from oracle.bindings import Ref

        asset = Ref().asset(stl_bytes)
        t1 = time.perf_counter()
        want = asset.export_stl(t[:cpu_copies], q[:cpu_copies])
        cpu_s = time.perf_counter() - t1
        sample = cpu_copies * len(obj.triangles)
        head = geometry.export_stl(obj, t[:cpu_copies], q[:cpu_copies], context=ctx)
        line["cpu_baseline"] = {"value": round(sample / cpu_s, 1), "unit": "triangles/s", "cores": 1,
                                "kind": "reference",
                                "sample": f"the first {cpu_copies} copies ({sample} triangles), record loop of "
                                          "result_export.cpp:1034-1123 in the reference build",
                                "same_bytes": head == want}
    return line


def _page_worker(workload, worker, orientations, warmup_orientations, barrier, queue):
    """One host process of the reference arm: the reference's own session on
    the workload's empty layout (container blocker, proximity and kernels
    built by the reference's code), untimed warm-up pages, then whole pages
    of `orientations` after `barrier`.  Reports (worker, seconds per page,
    start, end) with perf_counter times, or an error string."""
    try:
        from oracle.bindings import Ref

        spec = pkg("workloads").SPECS[workload]()
        ref = Ref()
        obj = ref.asset(spec.object_stl)
        container = tuple(spec.container_box) if spec.container_box is not None else \
            ref.asset(spec.container_stl, container=True)
        catalog = ref.catalog(1) if spec.catalog_kind == "cube" else ref.catalog(4, spec.raw_quaternions())
        session = ref.session(obj, container, spec.pair_clearance, spec.wall_clearance, spec.origin, spec.pitch,
                              catalog)
        for o in warmup_orientations:  # the first builds the environment fields
            session.page(o % len(catalog))
        barrier.wait()
        start = time.perf_counter()
        times = []
        for o in orientations:
            t0 = time.perf_counter()
            session.page(o % len(catalog))
            times.append(time.perf_counter() - t0)
        queue.put((worker, times, start, time.perf_counter()))
    except Exception as exc:  # reported to the parent, which fails the measurement
        try:
            barrier.abort()
        except Exception:
            pass
        queue.put((worker, f"{type(exc).__name__}: {exc}", 0.0, 0.0))


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_pages(workload: str, pages: int, workers: int = 0, first_orientation: int = 0, warmup: int = 1):
    """Whole pages of the reference's own spectral pipeline
    (build_spectral_pipeline, spectral_pipeline.cpp:914-1876: the kernel's
    raster, the binary and proximity FFT correlations, the page scan and the
    exact recount), compiled from its sources into oracle/_ref, for `pages`
    distinct orientations spread over `workers` concurrent processes (one per
    host core by default; spawned, so they are safe beside a CUDA context),
    after `warmup` untimed pages (at least one per worker).  The reference
    parallelises its FFT only on Windows (fft_execution.cpp:201), so on this
    host concurrency comes from independent orientations, which is how a
    multi-core caller would use it.  Returns (wall seconds from the common
    start to the last page's end, per-page seconds, workers)."""
    import multiprocessing as mp

    workers = max(1, min(workers or host_cores(), pages))
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(workers)
    queue = ctx.Queue()
    share = [list(range(first_orientation + w, first_orientation + pages, workers)) for w in range(workers)]
    per_worker = max(1, -(-warmup // workers))
    warm = [[first_orientation + pages + w * per_worker + i for i in range(per_worker)] for w in range(workers)]
    procs = [ctx.Process(target=_page_worker, args=(workload, w, share[w], warm[w], barrier, queue))
             for w in range(workers)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=3600) for _ in procs]
    for p in procs:
        p.join(timeout=120)
    errors = [r[1] for r in results if isinstance(r[1], str)]
    if errors:
        raise RuntimeError(errors[0])
    start = min(r[2] for r in results)
    end = max(r[3] for r in results)
    per_page = [t for r in results for t in r[1]]
    return end - start, per_page, workers


def reference_config(workload: str, world: int) -> dict:
    """The arms' shared config, computed without this library: the window
    from the workload's container bounds and lattice (the reference's
    GridWindow rule, spectral_pipeline.cpp:107-140: a one-cell halo)."""
    import math

    spec = pkg("workloads").SPECS[workload]()
    assets = pkg("assets")
    if spec.container_box is not None:
        lo, hi = np.zeros(3), np.array(spec.container_box, np.float64)
        container_triangles = 0
    else:
        mesh = assets.accept_stl(spec.container_stl, role="container")
        lo, hi = mesh.bounds
        container_triangles = int(len(mesh.triangles))
    grid = [int(math.ceil((hi[a] - spec.origin[a]) / spec.pitch)) -
            int(math.floor((lo[a] - spec.origin[a]) / spec.pitch)) + 2 for a in range(3)]
    orientations = spec.catalog_count if spec.catalog_kind == "hopf" else 24
    return {"workload": workload, "grid": grid, "orientations": orientations,
            "object_triangles": int(len(assets.accept_stl(spec.object_stl).triangles)),
            "container_triangles": container_triangles,
            "l2": "working set above L2 (all orientations' kernel spectra stay in HBM)",
            "parallelism": f"replicas x{world}"}


def page_sample_description(pages, wall, per_page, cores, orientations, warmup):
    return (f"{pages} whole pages of the reference's build_spectral_pipeline (kernel raster, FP64 binary and "
            f"proximity FFT correlations with the oracle build's FFT in place of pocketfft, page scan, exact "
            f"recount), distinct orientations on the empty layout after {warmup} warm-up pages, {cores} concurrent "
            f"processes, {wall:.1f} s wall ({min(per_page):.1f}-{max(per_page):.1f} s per page); a step is one page, "
            f"and placements/s = pages / {orientations} (pages per placement) / wall")


def cpu_baseline(workload: str, orientations: int):
    """Reported baseline only: one whole reference page per host core, run
    concurrently (a bounded sample of the same workload), scaled linearly by
    the orientation count to placements/s."""
    cores = host_cores()
    try:
        from oracle.bindings import REF_SO

        if not os.path.exists(REF_SO):
            return None
        wall, per_page, cores = reference_pages(workload, cores)
        value = (len(per_page) / orientations) / wall
        return {"value": round(value, 8), "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": page_sample_description(len(per_page), wall, per_page, cores, orientations, cores)}
    except Exception as exc:  # the baseline is reported, never required
        return {"value": None, "unit": UNIT, "cores": cores, "kind": "reference", "sample": f"unavailable: {exc}"}


def run_reference(args, rank, world):
    """The reference's own CPU implementation of the path (compiled from its
    sources into oracle/_ref), on every host core, loading nothing of this
    library: each timed step is one whole page of a distinct orientation
    (all steps run concurrently, one process per core), and placements/s is
    the pages completed / the orientations a placement pages / the wall time
    of the timed steps."""
    if rank != 0:
        return
    try:
        from oracle.bindings import REF_SO

        if not os.path.exists(REF_SO):
            print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libspk_ref.so missing"}))
            return
        config = reference_config(args.workload, world)
        O = args.orientations or config["orientations"]
        config["orientations"] = O
        wall, per_page, cores = reference_pages(args.workload, args.steps, workers=min(host_cores(), args.steps),
                                                warmup=args.warmup)
        value = (len(per_page) / O) / wall
        desc = page_sample_description(len(per_page), wall, per_page, cores, O, args.warmup)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": round(value, 8), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000.0 * wall / max(args.steps, 1), 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded rounded-box STL container, spherical-harmonic blob item, seeded SO(3) catalog)",
            "config": config, "mode": "exhaustive (the reference pages every orientation)",
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
    ap.add_argument("--profile-region", default="", choices=["", "learned", "exhaustive"],
                    help="bracket that arm's timed steps with cudaProfilerStart/Stop (ncu --profile-from-start off)")
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
