"""Training and evaluation of the learned initial guess.

Pairs (features, converged (u, v)) come from plain Newton (midpoint guess) on
seeded scenes: the small height-field surface and the 64-surface mixed-degree
scene, at seeds other than the evaluation seeds.  The network is trained on
the GPU by the engine's own kernels (nrt_mlp_train: BF16 tensor-core forward
and backward, Adam) and evaluated on unseen seeds against plain Newton:
Newton evaluations per ray and per converged solve, fallback rate, hit/miss
agreement and throughput.

    python -m nrt.learned [--pairs 4000000] [--epochs 20] [--out models/init_mlp.nrt]
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import lib_module as L
from . import scenes

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEFAULT_MODEL = os.path.join(PKG, "models", "init_mlp.nrt")


def training_scenes(pairs: int):
    """Seeded training scenes: height-field seeds 1.. (256x256) and mixed-degree
    seeds 101.. (640x360, 2 jittered samples), alternating."""
    k = 0
    while True:
        yield scenes.heightfield_scene(1 + k, 256, 256, 1)
        yield scenes.mixed_degree_scene(101 + k, 640, 360, 2)
        k += 1


def collect(pairs: int = 4_000_000, verbose: bool = True, miss_ratio: float = 0.0, which=None):
    """Pairs from solves that converged (target: their (u, v)) and, up to
    miss_ratio times as many, from solves that did not (target (-1, -1))."""
    import torch

    feats, targs, have = [], [], 0
    opts = L.default_opts(schedule=L.SCHED_WAVEFRONT, hull_cull=2)
    gen = torch.Generator(device="cuda").manual_seed(7)
    for sc in (which or training_scenes(pairs)):
        scene = L.Scene(sc.surfaces)
        rays = L.camera_rays(sc.camera)
        f, t, _ = scene.collect_training_data(rays, opts, capacity=16 * rays[0].numel())
        scene.close()
        conv = t[:, 0] >= 0
        fc, tc, fm, tm = f[conv], t[conv], f[~conv], t[~conv]
        keep = min(fm.shape[0], int(miss_ratio * fc.shape[0]))
        pick = torch.randperm(fm.shape[0], generator=gen, device="cuda")[:keep]
        f = torch.cat([fc, fm[pick]])
        t = torch.cat([tc, tm[pick]])
        take = min(f.shape[0], pairs - have)
        feats.append(f[:take].clone())
        targs.append(t[:take].clone())
        have += take
        if verbose:
            print(f"  {sc.name}: {f.shape[0]} pairs (total {have})", flush=True)
        if have >= pairs:
            break
    return torch.cat(feats), torch.cat(targs)


def train(features, targets, epochs: int = 20, batch: int = 4096, lr: float = 1e-3, seed: int = 0):
    mlp = L.Mlp(seed=seed)
    t0 = time.perf_counter()
    losses = mlp.train(features, targets, epochs=epochs, batch=batch, lr=lr, seed=seed)
    return mlp, losses, time.perf_counter() - t0


def evaluate(mlp, sc=None, learned_iters: int = 3, hull_cull: int = 2, reps: int = 5):
    """Plain vs learned guess on one scene (wavefront, FP64 final step off)."""
    import torch

    sc = sc or scenes.mixed_degree_scene(1)
    scene = L.Scene(sc.surfaces)
    scene.set_mlp(mlp)
    rays = L.camera_rays(sc.camera)
    n = rays[0].numel()
    W = L.SCHED_WAVEFRONT
    res = {}
    for tag, opts in [("plain", L.default_opts(hull_cull=hull_cull, schedule=W)),
                      ("learned", L.default_opts(hull_cull=hull_cull, schedule=W, init_mode=L.INIT_LEARNED,
                                                 learned_iters=learned_iters))]:
        scene.enable_counters(True)
        out = {k: v.cpu().numpy() for k, v in scene.intersect(rays, opts).items()}
        c = scene.counters()
        scene.enable_counters(False)
        for _ in range(2):
            scene.intersect(rays, opts, extra=False)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(reps):
            scene.intersect(rays, opts, extra=False)
        e.record()
        torch.cuda.synchronize()
        ms = s.elapsed_time(e) / reps
        hit = out["patch"] >= 0
        res[tag] = {"ms": round(ms, 3), "mrays_s": round(n / ms / 1e3, 2), "hit_rate": round(float(hit.mean()), 5),
                    "evals_per_ray": round(c["newton_evals"] / n, 3),
                    "solves_per_ray": round(c["newton_solves"] / n, 3),
                    "evals_per_hit_solve": round(float(out["iters"][hit].mean()), 3),
                    "learned_solves_per_ray": round(c["learned_solves"] / n, 3),
                    "fallback_rate": round(c["learned_fallbacks"] / max(1, c["learned_solves"]), 4),
                    "patch": out["patch"], "t": out["t"]}
    a, b = res["plain"], res["learned"]
    both = (a["patch"] >= 0) & (b["patch"] >= 0)
    agree = float(((a["patch"] >= 0) == (b["patch"] >= 0)).mean())
    rel = np.abs(a["t"][both] - b["t"][both]) / np.abs(a["t"][both])
    same = float((a["patch"][both] == b["patch"][both]).mean())
    for r in (a, b):
        r.pop("patch"), r.pop("t")
    res["learned_vs_plain"] = {"hit_agreement": round(agree, 6), "t_rel_gt_1e-4": float((rel > 1e-4).mean()),
                               "same_patch": same}
    scene.close()
    return res


def load_or_train(path: str = DEFAULT_MODEL, pairs: int = 1_000_000, epochs: int = 20):
    """The committed model if present, else a freshly trained one (not saved)."""
    if os.path.exists(path):
        return L.Mlp.load(path), {"source": os.path.relpath(path, PKG)}
    feats, targs = collect(pairs, verbose=False)
    mlp, losses, secs = train(feats, targs, epochs=epochs)
    return mlp, {"source": f"trained now on {feats.shape[0]} pairs", "train_s": round(secs, 2),
                 "final_loss": float(losses[-1])}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=4_000_000)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=DEFAULT_MODEL)
    ap.add_argument("--learned-iters", type=int, default=3)
    args = ap.parse_args()
    t0 = time.perf_counter()
    feats, targs = collect(args.pairs)
    print(f"collected {feats.shape[0]} pairs in {time.perf_counter() - t0:.1f} s", flush=True)
    mlp, losses, secs = train(feats, targs, args.epochs, args.batch, args.lr)
    print(f"trained {args.epochs} epochs in {secs:.2f} s; loss per epoch {np.round(losses, 5).tolist()}", flush=True)
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    mlp.save(args.out)
    res = evaluate(mlp, learned_iters=args.learned_iters)
    meta = {"model": os.path.basename(args.out), "pairs": int(feats.shape[0]), "epochs": args.epochs,
            "batch": args.batch, "lr": args.lr, "train_s": round(secs, 2), "loss": [float(x) for x in losses],
            "eval_unseen_mixed64_seed1": res}
    # the model's metadata beside it: how it was trained and what it gained on an unseen scene
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(meta, f, indent=1)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
