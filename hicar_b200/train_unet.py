"""Train the learned preconditioner's U-Net on synthetic terrains and save its
parameters (FP32 .npy), e.g.

    python -m hicar_b200.train_unet --nx 128 --ny 128 --nz 32 --terrains 16 \\
        --samples 8 --steps 2000 --out hicar_b200/weights/unet_128x128x32.npy

    python -m hicar_b200.train_unet --source composite --terrains 4096 \\
        --out hicar_b200/weights/unet_mg_128x128x32.npy

The composite source trains the second stage of HICARW_PRECOND_MG_LEARNED
(z = M(r) + theta U(r'), r' = r - A M(r)) online: each seeded terrain's plain-solver iterates
give (residual, error) pairs after the V-cycle (learned.composite_pairs), the
pairs enter a replay buffer, and a few Adam steps follow each terrain, so that
thousands of terrains stream through without being stored.

Terrains are the seeded generator's cases (hicar_b200.cases, seeds
--seed0 .. --seed0 + terrains - 1); the samples of a terrain are random
residuals and/or the residuals of the plain solver's iterates on the terrain's
own right-hand side (--source), and the loss is the residual loss
mean((A z - rhat)^2) of hicar_b200.learned.train.  The network is
convolutional, so parameters trained on one grid size serve any other
(load_params / UNet.set_params)."""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")
DEFAULT_WEIGHTS = os.path.join(WEIGHTS_DIR, "unet_128x128x32.npy")
COMPOSITE_WEIGHTS = os.path.join(WEIGHTS_DIR, "unet_mg_128x128x32.npy")


def load_params(path: str = DEFAULT_WEIGHTS):
    """FP32 parameter vector saved by this module."""
    if not os.path.exists(path):
        raise FileNotFoundError(f"no trained U-Net parameters at {path} (run python -m hicar_b200.train_unet)")
    return np.load(path).astype(np.float32)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=128)
    ap.add_argument("--ny", type=int, default=128)
    ap.add_argument("--nz", type=int, default=32)
    ap.add_argument("--terrains", type=int, default=16)
    ap.add_argument("--samples", type=int, default=8, help="random residuals per terrain")
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed0", type=int, default=1000)
    ap.add_argument("--hills", type=int, default=20)
    ap.add_argument("--source", default="random", choices=["random", "solver", "mixed", "composite"],
                    help="residuals: random fields, the plain solver's iterates, half of each, or the "
                         "composite preconditioner's residuals after the V-cycle (online)")
    ap.add_argument("--steps-per-terrain", type=int, default=2, help="composite: Adam steps after each terrain")
    ap.add_argument("--buffer", type=int, default=64, help="composite: replay buffer of samples")
    ap.add_argument("--max-minutes", type=float, default=0.0,
                    help="composite: stop streaming terrains after this much wall time (0: all terrains)")
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    if args.out is None:
        args.out = COMPOSITE_WEIGHTS if args.source == "composite" else DEFAULT_WEIGHTS

    import torch

    from . import cases, learned as L
    net = L.UNet(args.nx, args.ny, args.nz, seed=args.seed0)
    if args.source == "composite":
        t0 = time.time()
        stream = (cases.build_case(args.nx, args.ny, args.nz, seed=args.seed0 + t, adv_den=True,
                                   n_hills=args.hills) for t in range(args.terrains))
        hist, used = L.train_online(net, stream, steps_per_terrain=args.steps_per_terrain, batch=args.batch,
                                    lr=args.lr, lr_decay_every=max(1, args.terrains // 4), buffer=args.buffer,
                                    seed=args.seed0, log_every=max(1, args.terrains // 16),
                                    time_limit_s=60.0 * args.max_minutes)
        torch.cuda.synchronize()
        p = net.params().cpu().numpy()
        os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
        np.save(args.out, p)
        info = {"grid": [args.nx, args.ny, args.nz], "terrains": used, "terrains_requested": args.terrains,
                "source": "composite",
                "pairs_per_terrain": len(L.SOLVER_ITERS), "solver_iterations_logged": list(L.SOLVER_ITERS),
                "steps": len(hist), "steps_per_terrain": args.steps_per_terrain, "batch": args.batch,
                "buffer": args.buffer, "lr": args.lr, "seed0": args.seed0, "hills": args.hills,
                "cycle": {k: (list(v) if isinstance(v, tuple) else v) for k, v in L.MG_CYCLE.items()},
                "loss_first": float(np.mean(hist[:10])), "loss_last": float(np.mean(hist[-50:])),
                "train_s": time.time() - t0, "params": int(p.size)}
        with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
            json.dump(info, f, indent=1)
        print(json.dumps(info))
        return
    t0 = time.time()
    pairs = []
    for t in range(args.terrains):
        case = cases.build_case(args.nx, args.ny, args.nz, seed=args.seed0 + t, adv_den=True, n_hills=args.hills)
        if args.source in ("random", "mixed"):
            pairs += L.training_pairs(case, net, args.samples if args.source == "random" else args.samples // 2,
                                      seed=args.seed0 + t)
        if args.source in ("solver", "mixed"):
            pairs += L.training_pairs(case, net, args.samples if args.source == "solver" else args.samples // 2,
                                      seed=args.seed0 + t, source="solver")
    torch.cuda.synchronize()
    t_data = time.time() - t0
    t0 = time.time()
    hist = []
    lr = args.lr
    for phase in range(4):  # step-decayed learning rate
        hist += L.train(net, pairs, steps=args.steps // 4, lr=lr, batch=args.batch, seed=args.seed0 + phase)
        lr *= 0.5
    torch.cuda.synchronize()
    t_train = time.time() - t0
    p = net.params().cpu().numpy()
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    np.save(args.out, p)
    info = {"grid": [args.nx, args.ny, args.nz], "terrains": args.terrains, "samples": args.samples,
            "source": args.source,
            "steps": args.steps, "batch": args.batch, "lr": args.lr, "seed0": args.seed0,
            "loss_first": float(np.mean(hist[:10])), "loss_last": float(np.mean(hist[-50:])),
            "data_s": t_data, "train_s": t_train, "params": int(p.size)}
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(info, f, indent=1)
    print(json.dumps(info))


if __name__ == "__main__":
    main()
