"""Train the learned preconditioner on pairs harvested from the plain solver.

For each seeded problem the plain mixed-precision solver (precond_hprsdft) runs from a random
start; at a few points of its convergence history every band's CG gradient is cut into patch
pairs (input: the gradient scaled to unit RMS; target: the screened-kinetic correction
sigma (T + sigma)^-1 of it, solved on the device by CG on the finite-difference kinetic
operator).  The pairs of all problems are pooled on the device and the network is trained
there by the library's own forward/backward kernels and Adam.

    python -m rsdft_develop_b200.lpc_train --config c1 --seeds 101 102 103 --pairs 20000 \\
        --out rsdft_develop_b200/weights/lpc_h0.30.npy

The weights depend on the grid spacing through T (the kinetic operator scales as 1/h^2);
configurations with the same h share them.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import api, synth

WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")


def default_weights_path(h: float) -> str:
    return os.path.join(WEIGHTS_DIR, f"lpc_h{h:.2f}.npy")


def harvest(cfg_name: str, seed: int, npairs: int, patch: int, sigma: float, iters: int,
            schedule=(0, 2, 5, 10), init_seed: int = 1):
    """(x, t) pairs from the plain solver's states on problem (cfg_name, seed), host arrays."""
    prob = synth.make_problem(synth.get_config(cfg_name, seed=seed))
    per = [npairs // len(schedule)] * len(schedule)
    per[-1] += npairs - sum(per)
    xs, ts = [], []
    with api.BandUpdate(prob, precision=api.PREC_MIXED, pc_mode=api.PC_HPRSDFT) as g:
        g.random_wf(init_seed + seed)
        g.gram_schmidt()
        g.lpc_dataset(npairs, patch)
        done = 0
        for i, sw in enumerate(schedule):
            if sw > done:
                g.calc_sweep(sw - done)
                done = sw
            g.lpc_harvest(per[i], sigma=sigma, iters=iters, seed=seed * 1000 + i)
        n = g.lpc_status()[3]
        x, t = g.lpc_dataset_get(0, n, patch)
    xs.append(x)
    ts.append(t)
    return np.concatenate(xs), np.concatenate(ts)


def train(cfg_name: str = "c1", seeds=(101, 102, 103), npairs: int = 20000, patch: int = 16,
          sigma: float = 2.5, iters: int = 30, epochs: int = 30, batch: int = 64, lr: float = 2e-3,
          init: int = 1, margin: int = 4):
    """Harvest npairs pairs over the seeded problems and train; returns (weights, losses, info)."""
    t0 = time.time()
    per = [npairs // len(seeds)] * len(seeds)
    per[-1] += npairs - sum(per)
    xs, ts = [], []
    for s, n in zip(seeds, per):
        x, t = harvest(cfg_name, s, n, patch, sigma, iters)
        xs.append(x)
        ts.append(t)
    x = np.concatenate(xs)
    t = np.concatenate(ts)
    t_harvest = time.time() - t0
    prob = synth.make_problem(synth.get_config(cfg_name, seed=seeds[0]))
    with api.BandUpdate(prob, precision=api.PREC_MIXED, pc_mode=api.PC_HPRSDFT) as g:
        g.lpc_init(init)
        g.lpc_dataset(x.shape[0], patch)
        g.lpc_dataset_add(x, t)
        t1 = time.time()
        losses = g.lpc_train(epochs=epochs, batch=batch, lr=lr, margin=margin)
        t_train = time.time() - t1
        w = g.lpc_get_weights()
    info = {"config": cfg_name, "h": prob.h, "seeds": list(seeds), "pairs": int(x.shape[0]), "patch": patch,
            "sigma": sigma, "target_cg_iters": iters, "epochs": epochs, "batch": batch, "lr": lr,
            "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
            "harvest_s": round(t_harvest, 2), "train_s": round(t_train, 2)}
    return w, losses, info


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--config", default="c1")
    ap.add_argument("--seeds", type=int, nargs="+", default=[101, 102, 103])
    ap.add_argument("--pairs", type=int, default=20000)
    ap.add_argument("--patch", type=int, default=16)
    ap.add_argument("--sigma", type=float, default=2.5)
    ap.add_argument("--iters", type=int, default=30)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    w, losses, info = train(args.config, tuple(args.seeds), args.pairs, args.patch, args.sigma, args.iters,
                            args.epochs, args.batch, args.lr)
    out = args.out or default_weights_path(info["h"])
    os.makedirs(os.path.dirname(out), exist_ok=True)
    np.save(out, w)
    with open(os.path.splitext(out)[0] + ".json", "w") as f:
        json.dump(dict(info, losses=[float(v) for v in losses]), f, indent=1)
    print(json.dumps(info))


if __name__ == "__main__":
    main()
