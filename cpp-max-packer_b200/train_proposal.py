"""Trains the orientation proposal network on labels from the exhaustive method.

    python cpp-max-packer_b200/train_proposal.py --out cpp-max-packer_b200/weights/proposal_rounded256.npz

Labels come from the exhaustive GPU path.
- **Items.** Each training item is a seeded spherical-harmonic blob in the
  rounded-box container of the 256^3 workload, with that seed's 512-orientation
  SO(3) catalog.
- **Labelled layouts.** The greedy fill runs from the empty container. Layouts
  are labelled at every step early on, then at every `--stride`-th step.
- **Labels.** At each labelled layout, every orientation's certified page gives
  that orientation's best exact score among copies that pass the exact recount.
  The label is the orientation's gap to the layout's best score, clipped to
  `--cap` and scaled to [0, 1]. Orientations with no admissible copy get 1.
- **Policy layouts.** A second set of layouts follows the proposal policy
  itself (a DAgger round). A given network fills the container with the
  proposed greedy, and a layout is labelled every `--policy-stride` steps through
  the whole fill. The states the learned fill reaches late, in a nearly full
  container, are then covered too.
- **Training.** Runs on the device with the library's own forward and backward
  kernels (Adam, mean squared error).
- **Evaluation.** Held-out seeds measure the regret of paging only the top-k
  proposals. Regret is the best proposed score minus the best score overall.
  The untrained network and a random k-subset are measured the same way.
"""

from __future__ import annotations

import argparse
import importlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pkg(name):
    return importlib.import_module("cpp-max-packer_b200." + name)


def best_scores(session, orientations):
    """Each orientation's best admissible exact score (inf when none)."""
    pages = session.pages(orientations)
    out = np.full(len(orientations), np.inf)
    for i, page in enumerate(pages):
        for c in page:
            if c.direct_zero_overlap:
                out[i] = c.score
                break
    return out


LABEL = "linear"


def labels_from(best, cap):
    """Each orientation's gap to the layout's best score as a target in [0, 1].
    'log': (log10(gap + 1e-5) + 5) / 5, so gaps of 1e-5 .. 1 spread evenly and
    the near-best orientations, which decide the top k, stay apart; 'linear':
    gap clipped to `cap`, over `cap`.  No admissible copy: 1."""
    top = best.min()
    if not np.isfinite(top):
        return None
    gap = np.where(np.isfinite(best), best - top, np.inf)
    if LABEL == "log":
        y = np.clip((np.log10(np.where(np.isfinite(gap), gap, 1.0) + 1e-5) + 5.0) / 5.0, 0.0, 1.0)
    else:
        y = np.minimum(np.where(np.isfinite(gap), gap, cap), cap) / cap
    return np.where(np.isfinite(gap), y, 1.0).astype(np.float32)


def open_session(seed, orientations, context):
    workloads, session_mod = pkg("workloads"), pkg("session")
    wl = workloads.rounded256_blob_hopf512(seed=seed, orientations=orientations)
    s = session_mod.Session(wl.obj, wl.container, wl.origin, wl.pitch, wl.catalog, wl.pair_clearance,
                            wl.wall_clearance, context=context)
    return s, wl


def labelled_steps(dense, stride, total):
    return [t for t in range(total) if t < dense or (t - dense) % stride == 0]


def generate(seeds, total_steps, dense, stride, orientations, cap, context, log=print):
    """Dataset over the training seeds (crops, items, samples)."""
    proposal = pkg("proposal")
    crops, items, sc, si, sl, best_log = [], [], [], [], [], []
    for seed in seeds:
        t0 = time.time()
        s, wl = open_session(seed, orientations, context)
        O = len(wl.catalog)
        _, it = proposal.session_features(s)
        item_base = sum(len(x) for x in items)
        items.append(it)
        marks = set(labelled_steps(dense, stride, total_steps))
        for step in range(total_steps):
            if step in marks:
                best = best_scores(s, range(O))
                lab = labels_from(best, cap)
                if lab is None:
                    break
                crop_index = len(crops)
                crops.append(proposal.session_crop(s))
                sc.append(np.full(O, crop_index, np.uint32))
                si.append(item_base + np.arange(O, dtype=np.uint32))
                sl.append(lab)
                best_log.append(float(best.min()))
            if not s.greedy(1):
                break
        s.close()
        log(f"seed {seed}: {len(crops)} layouts so far, {time.time() - t0:.1f} s")
    return proposal.ProposalDataset(np.stack(crops), np.concatenate(items), np.concatenate(sc), np.concatenate(si),
                                    np.concatenate(sl))


def generate_policy(seeds, net, k, stride, orientations, cap, context, item_base_count=0, log=print):
    """Layouts along the proposed-greedy fill of `net`, labelled every `stride` steps until the fill ends."""
    proposal = pkg("proposal")
    crops, items, sc, si, sl = [], [], [], [], []
    for seed in seeds:
        t0 = time.time()
        s, wl = open_session(seed, orientations, context)
        O = len(wl.catalog)
        _, it = proposal.session_features(s)
        item_base = item_base_count + sum(len(x) for x in items)
        items.append(it)
        copies = 0
        while True:
            best = best_scores(s, range(O))
            lab = labels_from(best, cap)
            if lab is None:
                break
            crops.append(proposal.session_crop(s))
            sc.append(np.full(O, len(crops) - 1, np.uint32))
            si.append(item_base + np.arange(O, dtype=np.uint32))
            sl.append(lab)
            placed, _ = proposal.greedy_proposed(s, net, k, stride)
            copies += len(placed)
            if len(placed) < stride:
                break
        s.close()
        log(f"policy seed {seed}: {copies} copies, {len(crops)} layouts so far, {time.time() - t0:.1f} s")
    return crops, items, sc, si, sl


def merge_datasets(a, crops, items, sc, si, sl):
    """Appends policy layouts (indices relative to their own lists) to dataset a."""
    proposal = pkg("proposal")
    if not crops:
        return a
    sc = [x + len(a.crops) for x in sc]
    return proposal.ProposalDataset(np.concatenate([a.crops, np.stack(crops)]), np.concatenate([a.items] + items),
                                    np.concatenate([a.sample_crop] + sc), np.concatenate([a.sample_item] + si),
                                    np.concatenate([a.sample_label] + sl))


def fill_copies(seed, net, k, orientations, context, chunk=64):
    """Copies placed by a full proposed-greedy fill (and its fallback steps)."""
    proposal = pkg("proposal")
    s, _ = open_session(seed, orientations, context)
    copies, fallbacks = 0, 0
    while True:
        placed, fb = proposal.greedy_proposed(s, net, k, chunk)
        copies += len(placed)
        fallbacks += fb
        if len(placed) < chunk:
            break
    s.close()
    return copies, fallbacks


def evaluate(nets, seeds, steps, orientations, k, context, rng_seed=0, log=print):
    """Mean regret and top-k hit rate of each net (and a random subset) on
    held-out seeds, following the exhaustive greedy's layouts."""
    proposal = pkg("proposal")
    rng = np.random.default_rng(rng_seed)
    stats = {name: {"regret": [], "hit": []} for name in list(nets) + ["random"]}
    for seed in seeds:
        s, wl = open_session(seed, orientations, context)
        O = len(wl.catalog)
        for _ in range(steps):
            best = best_scores(s, range(O))
            if not np.isfinite(best.min()):
                break
            winner = int(np.argmin(best))
            for name, net in nets.items():
                chosen, _ = proposal.propose(s, net, k)
                chosen = chosen.astype(np.int64)
                stats[name]["regret"].append(float(best[chosen].min() - best.min()))
                stats[name]["hit"].append(float(winner in set(chosen.tolist())))
            pick = rng.choice(O, size=k, replace=False)
            stats["random"]["regret"].append(float(best[pick].min() - best.min()))
            stats["random"]["hit"].append(float(winner in set(pick.tolist())))
            if not s.greedy(1):
                break
        s.close()
    out = {}
    for name, st in stats.items():
        r = np.array(st["regret"])
        out[name] = {"mean_regret": float(np.mean(np.where(np.isfinite(r), r, 1.0))),
                     "infeasible_steps": int(np.sum(~np.isfinite(r))), "hit_rate": float(np.mean(st["hit"])),
                     "steps": len(r)}
        log(f"{name}: {out[name]}")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train-seeds", type=int, nargs="+", default=list(range(100, 112)))
    ap.add_argument("--eval-seeds", type=int, nargs="+", default=[2, 7])
    ap.add_argument("--steps", type=int, default=100, help="greedy steps per training seed")
    ap.add_argument("--dense", type=int, default=20, help="label every step below this one")
    ap.add_argument("--stride", type=int, default=10, help="then label every stride-th step")
    ap.add_argument("--orientations", type=int, default=512)
    ap.add_argument("--cap", type=float, default=0.25)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--k", type=int, default=32)
    ap.add_argument("--eval-steps", type=int, default=15)
    ap.add_argument("--init-seed", type=int, default=7)
    ap.add_argument("--policy-seeds", type=int, nargs="*", default=list(range(200, 208)))
    ap.add_argument("--policy-stride", type=int, default=25)
    ap.add_argument("--policy-weights", default="", help="network whose fills give the policy layouts")
    ap.add_argument("--fill-seed", type=int, default=-1, help="held-out item for a full learned fill after training")
    ap.add_argument("--fill-k", type=int, nargs="+", default=[32], help="proposal sizes of those fills")
    ap.add_argument("--label", choices=["log", "linear"], default="linear")
    ap.add_argument("--out", default=os.path.join(HERE, "weights", "proposal_rounded256.npz"))
    ap.add_argument("--report", default="")
    args = ap.parse_args()

    global LABEL
    LABEL = args.label
    compute, proposal = pkg("compute"), pkg("proposal")
    ctx = compute.Context(0)
    t0 = time.time()
    data = generate(args.train_seeds, args.steps, args.dense, args.stride, args.orientations, args.cap, ctx)
    if args.policy_weights and args.policy_seeds:
        policy = proposal.Proposal(seed=0, context=ctx)
        policy.load(args.policy_weights)
        extra = generate_policy(args.policy_seeds, policy, args.k, args.policy_stride, args.orientations, args.cap,
                                ctx, item_base_count=len(data.items))
        data = merge_datasets(data, *extra)
        policy.close()
    t_gen = time.time() - t0
    print(f"dataset: {len(data.crops)} layouts, {len(data.sample_label)} samples, {t_gen:.1f} s", flush=True)
    net = proposal.Proposal(seed=args.init_seed, context=ctx)
    untrained = proposal.Proposal(seed=args.init_seed, context=ctx)
    t1 = time.time()
    losses = []
    for phase, lr in enumerate((args.lr, args.lr / 4)):
        losses.append(net.train(data, args.batch, args.train_steps // 2, lr, seed=1000 + phase))
    losses = np.concatenate(losses)
    t_train = time.time() - t1
    print(f"training: {args.train_steps} steps of {args.batch} in {t_train:.1f} s; loss {losses[:50].mean():.4f} -> "
          f"{losses[-50:].mean():.4f}", flush=True)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    np.savez_compressed(args.out, parameters=net.get_parameters(),
                        meta=json.dumps({"train_seeds": args.train_seeds, "policy_seeds": args.policy_seeds
                                         if args.policy_weights else [], "policy_stride": args.policy_stride,
                                         "steps": args.steps, "dense": args.dense,
                                         "stride": args.stride, "orientations": args.orientations, "cap": args.cap,
                                         "label": args.label,
                                         "batch": args.batch, "train_steps": args.train_steps, "lr": args.lr,
                                         "init_seed": args.init_seed, "layouts": len(data.crops),
                                         "samples": len(data.sample_label)}))
    ev = evaluate({"trained": net, "untrained": untrained}, args.eval_seeds, args.eval_steps, args.orientations,
                  args.k, ctx)
    report = {"layouts": len(data.crops), "samples": int(len(data.sample_label)), "generate_s": t_gen,
              "train_s": t_train, "loss_first": float(losses[:50].mean()), "loss_last": float(losses[-50:].mean()),
              "eval": ev, "k": args.k}
    if args.fill_seed >= 0:
        report["fill"] = []
        for k in args.fill_k:
            t_fill = time.time()
            copies, fallbacks = fill_copies(args.fill_seed, net, k, args.orientations, ctx)
            report["fill"].append({"seed": args.fill_seed, "k": k, "copies": copies, "fallback_steps": fallbacks,
                                   "seconds": round(time.time() - t_fill, 1)})
            print(report["fill"][-1], flush=True)
    print(json.dumps(report), flush=True)
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)
    net.close()
    untrained.close()
    ctx.close()


if __name__ == "__main__":
    main()
