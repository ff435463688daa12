"""Train the learned smooth-face flag from the plain method's own runs.

Samples come from FP64 WENO runs of the engine itself (the plain form): a
circularly polarised Alfven wave (smooth) at 64^3, 128^3 and 256^3 and a
magnetised blast (shocks, contacts, smooth ambient) at 64^3 and 128^3,
several snapshots each, all three sweeps.  Each
sample holds the 35 features the reconstruction kernel computes and the
relative change the linear optimal weights would make to the cell's face
values.  The network is trained on the GPU (cumc_mlp_train) to predict
"change < delta".

    python -m cumc3d_b200.train_flag --out cumc3d_b200/data/flag_mlp.npy
"""
import argparse
import json
import os
import time

import numpy as np

from . import capi, engine, models

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "data", "flag_mlp.npy")
DELTA = 1e-6


def harvest(spec, prim, eps, snapshots, stride):
    s = engine.Solver(spec)
    s.set_state(prim, eps)
    s.initial_update()
    rows, done = [], 0
    for st in snapshots:
        if st > done:
            s.evolve(1e30, st - done)
            done = st
        for d in range(3):
            rows.append(s.learn_harvest(d, stride))
    s.close()
    return np.concatenate(rows)


def training_set(n=64, stride=3):
    """Snapshots at n^3 and at 2n, 4n (strides scaled to keep each grid's
    share similar): the features of smooth data shift with resolution (the
    relative variation across a stencil falls as 1/n)."""
    smooth, rough = [], []
    for m, st in ((n, stride), (2 * n, 8 * stride), (4 * n, 64 * stride)):
        sa, pa, ea = models.alfven_3d(m, recon="weno")
        smooth.append(harvest(sa, pa, ea, [0, 20], st))
        if m <= 2 * n:
            sb, pb, eb = models.blast_3d(m, radius=0.2, p_in=1.0)
            sb["positivity_fallback"] = 1
            sb["fix_periodic_normal_faces"] = 1
            rough.append(harvest(sb, pb, eb, [10, 30, 60], st))
    return np.concatenate(smooth), np.concatenate(rough)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--stride", type=int, default=3)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--delta", type=float, default=DELTA)
    ap.add_argument("--seed", type=int, default=20261203)
    args = ap.parse_args(argv)
    t0 = time.time()
    smooth, rough = training_set(args.n, args.stride)
    data = np.concatenate([smooth, rough])
    rng = np.random.default_rng(args.seed)
    rng.shuffle(data)
    n_tr = int(0.9 * len(data))
    P, losses = engine.mlp_train(data[:n_tr], engine.mlp_init(args.seed), steps=args.steps, batch=args.batch,
                                 lr=args.lr, delta=args.delta, seed=args.seed)
    held = data[n_tr:]
    z = engine.mlp_infer(P, held[:, :capi.LEARN_NF])
    y = held[:, capi.LEARN_NF] < args.delta
    flagged = z > 0
    summary = {
        "samples": int(len(data)), "smooth_samples": int(len(smooth)), "rough_samples": int(len(rough)),
        "delta": args.delta, "steps": args.steps, "batch": args.batch, "lr": args.lr,
        "loss_first": float(losses[:50].mean()), "loss_last": float(losses[-50:].mean()),
        "heldout_accuracy": float((flagged == y).mean()),
        "heldout_false_flag_rate": float((flagged & ~y).sum() / max(1, (~y).sum())),
        "heldout_recall": float((flagged & y).sum() / max(1, y.sum())),
        "seconds": time.time() - t0,
    }
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    np.save(args.out, P.astype(np.float32))
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(summary, f, indent=1)
    print(json.dumps(summary))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
