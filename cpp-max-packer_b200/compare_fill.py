"""Full greedy fill with the learned proposal against the exhaustive fill.

    python cpp-max-packer_b200/compare_fill.py [--workload rounded256_blob_hopf512] [--k 32]
        [--configs 32,64,32:4]

--configs runs one exhaustive fill and then a learned fill per entry: "k"
pages the k proposed orientations, "k:m" also widens by k at a time while
fewer than m paged orientations admit a copy
(spk_session_greedy_proposed_adaptive), "m:k_min:k_max:margin" pages every
orientation predicted within the margin of the k_min-th best, and
"s:k:n:k2" pages k proposed orientations for the first n copies and k2
after them (k2 = 0: the exhaustive step).

Both fills start from the empty container and run until no orientation
admits a copy.
- The exhaustive fill pages every orientation at every step.
- The learned fill pages the k proposed orientations. It falls back to the
  exhaustive step whenever none of them admits a copy, so it also ends only
  when no orientation admits one.

Every placement of either fill is an exact candidate: it has a zero exact
overlap recount, and its score is the exact FP64 score. Printed per fill:
- copies placed and the device time;
- for the learned fill, its fallback steps;
- the packed-count ratio, learned copies over exhaustive copies.
"""

from __future__ import annotations

import argparse
import importlib
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pkg(name):
    return importlib.import_module("cpp-max-packer_b200." + name)


def fill(session, step, chunk=64, max_copies=100000, log=print):
    """Runs `step(n)` (returns the copies placed, and the fallback count)
    until a call places fewer than asked; returns (copies, fallbacks, seconds)."""
    copies, fallbacks = 0, 0
    t0 = time.perf_counter()
    while copies < max_copies:
        placed, fb = step(chunk)
        copies += placed
        fallbacks += fb
        if placed < chunk:
            break
        if copies % (chunk * 8) == 0:
            log(f"  {copies} copies, {time.perf_counter() - t0:.1f} s")
    return copies, fallbacks, time.perf_counter() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="rounded256_blob_hopf512")
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--k", type=int, default=32)
    ap.add_argument("--weights", default=os.path.join(HERE, "weights", "proposal_rounded256.npz"))
    ap.add_argument("--max-copies", type=int, default=100000)
    ap.add_argument("--report", default="")
    ap.add_argument("--configs", default="", help="comma-separated learned configurations: k, k:min_feasible, "
                                                  "or m:k_min:k_max:margin")
    args = ap.parse_args()
    compute, session_mod, workloads, proposal = pkg("compute"), pkg("session"), pkg("workloads"), pkg("proposal")
    ctx = compute.Context(0)
    wl = workloads.WORKLOADS[args.workload](seed=args.seed)

    def open_session():
        return session_mod.Session(wl.obj, wl.container, wl.origin, wl.pitch, wl.catalog, wl.pair_clearance,
                                   wl.wall_clearance, context=ctx)

    s = open_session()
    print("exhaustive fill", flush=True)
    ex = fill(s, lambda n: (len(s.greedy(n)), 0), max_copies=args.max_copies)
    ex_scores = [p.score for p in s.placements]
    s.close()
    net = proposal.Proposal(seed=0, context=ctx)
    net.load(args.weights)
    configs = [c for c in args.configs.split(",") if c] or [str(args.k)]
    report = {
        "workload": wl.name, "orientations": len(wl.catalog),
        "exhaustive": {"copies": ex[0], "seconds": round(ex[2], 2), "placements_per_s": round(ex[0] / ex[2], 3)},
        "learned": [],
    }
    for config in configs:
        margin, switch_at, k_late = None, None, None
        if config.startswith("s:"):
            _, k, switch_at, k_late = config.split(":")
            k, m, switch_at, k_late = int(k), 0, int(switch_at), int(k_late)
        elif config.startswith("m:"):
            _, k_min, k_max, margin = config.split(":")
            k, m, k_max, margin = int(k_min), 0, int(k_max), float(margin)
        else:
            k, _, m = config.partition(":")
            k, m = int(k), int(m or 0)
        s = open_session()
        print(f"learned fill k={k} min_feasible={m} margin={margin}", flush=True)
        widened = [0]

        def learned(n):
            if switch_at is not None:
                total, fallbacks = 0, 0
                while total < n:
                    done = len(s.placements)
                    want = min(n - total, switch_at - done) if done < switch_at else n - total
                    if done < switch_at:
                        placed, fb = proposal.greedy_proposed(s, net, k, want)
                    elif k_late == 0:
                        placed, fb = s.greedy(want), 0
                    else:
                        placed, fb = proposal.greedy_proposed(s, net, k_late, want)
                    total += len(placed)
                    fallbacks += fb
                    if len(placed) < want:
                        break
                return total, fallbacks
            if margin is not None:
                placed, fb, paged = proposal.greedy_proposed_margin(s, net, k, k_max, margin, n)
                widened[0] += paged
            elif m:
                placed, fb, w = proposal.greedy_proposed_adaptive(s, net, k, m, n)
                widened[0] += w
            else:
                placed, fb = proposal.greedy_proposed(s, net, k, n)
            return len(placed), fb

        ln = fill(s, learned, max_copies=args.max_copies)
        ln_scores = [p.score for p in s.placements]
        s.close()
        entry = {"k": k, "min_feasible": m, "copies": ln[0], "fallback_steps": ln[1], "widenings": widened[0],
                 "margin": margin, "k_max": k_max if margin is not None else None,
                 "switch_at": switch_at, "k_late": k_late,
                 "mean_paged": round(widened[0] / max(ln[0], 1), 2) if margin is not None else None,
                 "seconds": round(ln[2], 2), "placements_per_s": round(ln[0] / ln[2], 3),
                 "packed_count_ratio": round(ln[0] / ex[0], 4) if ex[0] else None,
                 "speed_over_exhaustive": round((ln[0] / ln[2]) / (ex[0] / ex[2]), 3) if ex[2] and ln[2] else None,
                 "same_prefix": next((i for i, (a, b) in enumerate(zip(ex_scores, ln_scores)) if a != b),
                                     min(len(ex_scores), len(ln_scores))),
                 "mean_score": sum(ln_scores) / max(len(ln_scores), 1)}
        report["learned"].append(entry)
        print(json.dumps(entry), flush=True)
    report["exhaustive"]["mean_score"] = sum(ex_scores) / max(len(ex_scores), 1)
    print(json.dumps(report), flush=True)
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)
    net.close()
    ctx.close()


if __name__ == "__main__":
    main()
