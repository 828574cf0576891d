"""Train the learned preconditioner on the GPU and write the parameters the package ships
(caffe_old_b200/data/precond_params.npy).

Training pairs come from the first steps on several seeds (Re ~ U[100, 300]) of the IB channel
case (--case channel) or of the sphere-in-a-box case (--case sphere, the 8x4x4 box of the
25.2M-cell configuration):
* the (b, x*) of every pressure-correction solve;
* residual/correction pairs (b - A x_k, x* - x_k) from plain re-solves truncated after 8, 32
  and 128 iterations;
* multi-scale synthetic pairs (A e, e).

The steps themselves run with the plain FP64 p' solve (--form fp64) or, where a plain step is
too slow (a 25M-cell lattice), with the learned + mixed form in pyramid mode (--form levels);
either way every solve reaches the same 1e-8 FP64 residual, and the truncated re-solves are the
plain solver's.  All pairs live in HBM on one handle, and the network is trained there by the
library's tensor-core forward and backward passes (Adam, energy-norm loss).

  python -m caffe_old_b200.train_precond [--case channel|sphere] [--dims 256 128 128] [--seeds 1 2 3 4]
                                         [--steps-per-seed 4] [--form fp64|levels] [--random 128]
                                         [--train-steps 1500] [--out path]
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import cases as C
from . import precond as P
from .solver import make_solver


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="channel", choices=("channel", "sphere"))
    ap.add_argument("--form", default="fp64", choices=("fp64", "levels"))
    ap.add_argument("--dims", type=int, nargs=3, default=(256, 128, 128))
    ap.add_argument("--seeds", type=int, nargs="+", default=(11, 12, 13, 14))
    ap.add_argument("--steps-per-seed", type=int, default=4)
    ap.add_argument("--snapshots", type=int, default=3)
    ap.add_argument("--random", type=int, default=128)
    ap.add_argument("--train-steps", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=2e-4)
    ap.add_argument("--net-from", type=int, default=1, help="first pyramid level that runs the network")
    ap.add_argument("--out", default=P.DEFAULT_WEIGHTS)
    args = ap.parse_args(argv)
    dims = tuple(args.dims)
    t0 = time.time()
    per_solve = 1 + args.snapshots
    handles = []
    store = None
    for q, seed in enumerate(args.seeds):
        if args.case == "channel":
            nodes, spec, _ = C.config4_channel_sphere(dims, seed=seed)
        else:
            re = float(np.random.default_rng(seed).uniform(100.0, 300.0))
            nodes, spec, _ = C.config5_sphere(dims, re=re)
        s = make_solver(nodes, spec.replace(p_form="fp64" if args.form == "fp64" else "learned_mixed"))
        if args.form == "levels":
            P.set_mode(s, "levels")
        cap = args.steps_per_seed * spec.n_inner * spec.n_pcorr * per_solve
        if store is None:
            # the first seed's handle holds every pair and trains; the others hand theirs over
            store = s
            total = cap * len(args.seeds) + args.random
            P.record_pairs(s, total, args.snapshots)
        else:
            P.record_pairs(s, cap, args.snapshots)
        for _ in range(args.steps_per_seed):
            s.solve()
        if s is not store:
            P.copy_pairs(store, s)
            s.close()
        else:
            P.record_pairs(s, 0)
        handles.append(seed)
    P.add_random_pairs(store, args.random, seed=7)
    n = P.pair_count(store)
    t1 = time.time()
    P.set_options(store, "auto", args.net_from)
    net_to = len(P.pyramid_dims(dims)) - 1
    before = {m: float(P.evaluate(store, m).mean()) for m in ("jacobi", "levels")}
    params, hist = P.train(store, P.identity_params(0), steps=args.train_steps, batch=args.batch, lr=args.lr, seed=1)
    after = float(P.evaluate(store, "network").mean())
    t2 = time.time()
    store.close()
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    np.save(args.out, params.astype(np.float32))
    info = {"case": args.case, "form": args.form, "net_from": args.net_from, "net_to": net_to, "pairs": n, "seeds": list(args.seeds), "dims": list(dims),
            "train_steps": args.train_steps, "batch": args.batch, "lr": args.lr, "pair_generation_s": round(t1 - t0, 1),
            "training_s": round(t2 - t1, 1), "loss_jacobi": before["jacobi"], "loss_levels": before["levels"],
            "loss_network": after, "loss_first_steps": [float(v) for v in hist[:5]],
            "loss_last_steps": [float(v) for v in hist[-5:]], "out": args.out}
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(info, f, indent=1)
    print(json.dumps(info), flush=True)
    return info


if __name__ == "__main__":
    main()
