"""Train the learned preconditioner on the GPU and save its weights.

    python -m rigidfibers_kth_b200.train_preconditioner --out rigidfibers_kth_b200/mlp_weights.npy

Pairs (fiber, one of its 8 nearest neighbours) from seeded layouts (M =
250..2000, seeds from 5000): Gaussian clouds and uniform boxes, each
evolved by 0..--max-steps time steps first (the sedimented states a run
goes through); minibatch Adam with the library's own forward/backward
kernels.
"""
import argparse
import json
import time

import numpy as np

from .learned import train_preconditioner


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--samples", type=int, default=200_000)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--kinds", default="cloud,box", help="layout kinds: cloud (Gaussian), box (uniform)")
    ap.add_argument("--max-steps", type=int, default=25, help="evolve each layout by 0..max_steps steps")
    args = ap.parse_args()
    t0 = time.time()
    w, losses, var = train_preconditioner(args.samples, args.epochs, args.batch, args.lr,
                                          kinds=tuple(args.kinds.split(",")), max_steps=args.max_steps)
    np.save(args.out, w)
    print(json.dumps({"samples": args.samples, "epochs": args.epochs, "kinds": args.kinds, "max_steps": args.max_steps,
                      "final_mse": losses[-1], "target_var": var,
                      "seconds": time.time() - t0}))


if __name__ == "__main__":
    main()
