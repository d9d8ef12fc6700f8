"""Train the learned orientation proposal on the plain method's results.

    python -m psacking_b200.train_proposal [--train-seeds N] [--epochs E] [--out PATH]

Config 4 of the benchmark set: the config-2 distribution (128^3 tray, 100
seeded items of superellipsoids and box unions, 24 orientations).  Training
runs use seeds 10000.. (disjoint from the evaluation seeds 0..9).  Every item
of a training run gives 24 (tray state, orientation, score) tuples: its
orientations' exact results from the plain search (psb_pack_staged_detail).
The network is trained with the engine's own forward and backward kernels
(Adam, masked softmax cross-entropy against the plain search's rank-based
soft target), then evaluated on held-out runs: top-k recall of a best
orientation, and density and items/s of the gated packing loop against the
plain one.  Writes the parameters and the evaluation to --out (npz).
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import proposal as PR
from . import workloads
from .rotations import orientation_maps

TRAIN_SEED0 = 10000
TEST_SEEDS = tuple(range(10))


def density(tray: np.ndarray) -> float:
    """Occupied voxels over the occupied bounding box (packer.py:582-601)."""
    idx = np.argwhere(tray > 0)
    if len(idx) == 0:
        return 0.0
    ext = idx.max(axis=0) - idx.min(axis=0) + 1
    return float(len(idx) / np.prod(ext))


def evaluate(prop, seeds=TEST_SEEDS, topk=4, margin=0.5, tray_dims=workloads.TRAY2):
    """Plain vs gated packing on held-out seeds: density, items placed, time."""
    import torch
    maps = orientation_maps(24)
    tray = PR.Tray(tray_dims)
    out = {"plain": {"density": [], "placed": [], "ms": []}, "learned": {"density": [], "placed": [], "ms": []},
           "fallbacks": 0, "items": 0}
    try:
        for seed in seeds:
            seq = PR.sorted_by_volume(workloads.config2_items(seed))
            for name in ("plain", "learned"):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                res, final, stats = tray.pack(seq, maps, prop=prop if name == "learned" else None, topk=topk,
                                              margin=margin)
                torch.cuda.synchronize()
                out[name]["ms"].append(1e3 * (time.perf_counter() - t0))
                out[name]["density"].append(density(final))
                out[name]["placed"].append(sum(r.found for r in res))
                if name == "learned":
                    out["items"] += int(stats[0])
                    out["fallbacks"] += int(stats[1])
    finally:
        tray.close()
    summ = {}
    for name in ("plain", "learned"):
        d = out[name]
        summ[name] = {"density_mean": float(np.mean(d["density"])), "placed_mean": float(np.mean(d["placed"])),
                      "items_per_s": float(100 * len(seeds) / (sum(d["ms"]) / 1e3))}
    summ["density_gap_pp"] = 100 * (summ["plain"]["density_mean"] - summ["learned"]["density_mean"])
    summ["speedup"] = summ["learned"]["items_per_s"] / summ["plain"]["items_per_s"]
    summ["fallback_rate"] = out["fallbacks"] / max(1, out["items"])
    summ["per_seed"] = out
    return summ


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train-seeds", type=int, default=300)
    ap.add_argument("--test-seeds", type=int, default=len(TEST_SEEDS))
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--gates", default="4:0,4:0.3,6:0,6:0.3,8:0,8:0.3",
                    help="top-k:margin pairs evaluated on the held-out seeds")
    ap.add_argument("--out", default=str(PR.WEIGHTS))
    ap.add_argument("--eval-only", default=None, help="evaluate the gates of an existing weights file")
    args = ap.parse_args(argv)
    if args.eval_only:
        prop = PR.load(Path(args.eval_only))
        for g in args.gates.split(","):
            topk, margin = int(g.split(":")[0]), float(g.split(":")[1])
            ev = evaluate(prop, seeds=tuple(range(args.test_seeds)), topk=topk, margin=margin)
            print(json.dumps({"topk": topk, "margin": margin, **{k: v for k, v in ev.items() if k != "per_seed"}}),
                  flush=True)
        return

    t0 = time.time()
    train_recs = PR.generate(range(TRAIN_SEED0, TRAIN_SEED0 + args.train_seeds))
    test_recs = PR.generate(range(args.test_seeds))
    t_gen = time.time() - t0
    print(f"data: {len(train_recs)} training items ({24 * len(train_recs)} orientation results), "
          f"{len(test_recs)} held-out items, {t_gen:.1f} s", flush=True)
    t1 = time.time()
    prop = PR.train(train_recs, epochs=args.epochs, batch=args.batch, lr=args.lr)
    t_train = time.time() - t1
    untrained = PR.Proposal(PR.init_params(0))
    recall = {}
    for k in (1, 4, 6, 8):
        recall[k] = {"train": PR.topk_recall(prop, train_recs[:2000], k=k),
                     "held_out": PR.topk_recall(prop, test_recs, k=k),
                     "untrained": PR.topk_recall(untrained, test_recs, k=k)}
        print(f"top-{k} recall: train {recall[k]['train']:.3f}, held-out {recall[k]['held_out']:.3f} "
              f"(untrained network {recall[k]['untrained']:.3f})", flush=True)
    print(f"training {t_train:.1f} s", flush=True)
    gates = [(int(a), float(b)) for a, b in (g.split(":") for g in args.gates.split(","))]
    evals = []
    for topk, margin in gates:
        ev = evaluate(prop, seeds=tuple(range(args.test_seeds)), topk=topk, margin=margin)
        evu = evaluate(untrained, seeds=tuple(range(args.test_seeds)), topk=topk, margin=margin)
        row = {"topk": topk, "margin": margin, "plain_items_per_s": ev["plain"]["items_per_s"],
               "learned_items_per_s": ev["learned"]["items_per_s"], "speedup": ev["speedup"],
               "density_plain": ev["plain"]["density_mean"], "density_learned": ev["learned"]["density_mean"],
               "density_gap_pp": ev["density_gap_pp"], "fallback_rate": ev["fallback_rate"],
               "untrained_density_gap_pp": evu["density_gap_pp"], "untrained_fallback_rate": evu["fallback_rate"]}
        evals.append(row)
        print(json.dumps(row), flush=True)
    ok = [r for r in evals if r["density_gap_pp"] <= 1.0]
    best = max(ok, key=lambda r: r["speedup"]) if ok else min(evals, key=lambda r: r["density_gap_pp"])
    print("chosen gate:", json.dumps(best), flush=True)
    untrained.close()
    meta = {"train_seeds": args.train_seeds, "train_items": len(train_recs), "epochs": args.epochs,
            "topk": best["topk"], "margin": best["margin"], "recall": json.dumps(recall),
            "evals": json.dumps(evals)}
    PR.save(prop, Path(args.out), **meta)
    print("saved", args.out)


if __name__ == "__main__":
    main()
