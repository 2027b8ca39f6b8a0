"""Train the learned coarse-level smoother on the GPU and write its weight file.

    python -m rochpcg_b200.train_smoother [--out PATH] [--count 4096] [--epochs 40]

Training set: ``count`` (residual, error) pairs from the plain FP32 V-cycle,
half on 64^3 and half on 128^3 grids, with b ~ N(0,1) from seeds 1..count
(seeds 1..count/2 on 64^3, the rest on 128^3); the pairs live on MG level 2
(16^3 and 32^3 grids).  Forward, backward and Adam run in the library's
tcgen05 kernels.  The script then evaluates on held-out seeds and records the
flexible-CG iteration counts of the plain mixed V-cycle and of the learned one
on a solve of the evaluation grid (b ~ N(0,1), seed 9999), all stored with the
weights.  The network is evaluated as an odd function of the residual
((N(r) - N(-r)) / 2) and trained on the error's energy norm by default.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def evaluate_loss(S, sets, kind: int = 1) -> float:
    """Mean relative error of N(r) against e over the pairs: energy norm
    (N(r)-e).A(N(r)-e) / e.Ae for kind 1, squared 2-norm for kind 0."""
    from rochpcg_b200 import learned as LS

    tot, n = 0.0, 0
    for P in sets:
        inv = LS.sample_norms(P.e, P.dims, P.count, kind)
        loss, _ = S.loss_grad(P.r, P.e, inv, P.dims, P.count, 1.0 / P.count, kind)
        tot += loss * P.count
        n += P.count
    return tot / n


def cg_iterations(S, n: int, seed: int, first_level: int = 2) -> dict:
    import rochpcg_b200 as R
    from rochpcg_b200.rhs import normal_rhs

    P = R.Problem(n, n, n)
    P.set_rhs(normal_rhs(P.rows[0], seed))
    P.cg(1000, 1e-9, mode=R.MODE_MIXED)  # warm-up (graph capture)
    mixed = P.cg(1000, 1e-9, mode=R.MODE_MIXED)
    P.set_smoother(S, first_level)
    P.cg(1000, 1e-9, mode=R.MODE_LEARNED)
    learned = P.cg(1000, 1e-9, mode=R.MODE_LEARNED)
    out = dict(grid=n, seed=seed, mixed_iters=mixed["niters"], mixed_s=mixed["seconds"],
               learned_iters=learned["niters"], learned_s=learned["seconds"], fallback_iter=P.last_fallback(),
               learned_true_residual=P.true_residual())
    P.set_smoother(None)
    P.close()
    return out


def main(argv=None):
    from rochpcg_b200 import learned as LS

    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--out", default=LS.DEFAULT_WEIGHTS)
    ap.add_argument("--count", type=int, default=4096)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--lr0", type=float, default=2e-3)
    ap.add_argument("--lr1", type=float, default=1e-4)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--symmetry", type=int, default=1, help="0 plain, 1 odd (two branches), 2 tied odd weights")
    ap.add_argument("--kind", type=int, default=1, help="loss: 0 squared 2-norm, 1 energy norm")
    ap.add_argument("--eval-grid", type=int, default=256)
    args = ap.parse_args(argv)

    t0 = time.time()
    half = args.count // 2
    small = LS.make_pairs(64, 2, 1, half, batch=min(64, half))
    large = LS.make_pairs(128, 2, 1 + half, args.count - half, batch=min(8, args.count - half))
    t_pairs = time.time() - t0
    held = [LS.make_pairs(64, 2, 100001, 32), LS.make_pairs(128, 2, 200001, 32)]

    w0 = LS.jacobi_weights(1.0, 0.02, args.seed, twin=8 if args.symmetry == LS.TIED else 1)
    S0 = LS.Smoother(w0, symmetry=args.symmetry)
    loss_init = evaluate_loss(S0, held, args.kind)
    cg_init = cg_iterations(S0, args.eval_grid, 9999)
    S = LS.Smoother(w0, symmetry=args.symmetry)
    t1 = time.time()
    hist = S.train([small, large], args.epochs, args.lr0, args.lr1, args.seed, kind=args.kind)
    t_train = time.time() - t1
    loss_trained = evaluate_loss(S, held, args.kind)
    cg_eval = cg_iterations(S, args.eval_grid, 9999)
    meta = dict(
        network="3x3x3 conv, 1->16->16->1, ReLU, BF16 weights/activations, FP32 accumulate",
        pairs=dict(count=args.count, grids=[64, 128], level=2, seeds=[1, args.count],
                   rhs="N(0,1) SplitMix64+Box-Muller by natural row id", error="A_level^-1 r, FP64 MG-PCG to 1e-8"),
        training=dict(epochs=args.epochs, lr0=args.lr0, lr1=args.lr1, seed=args.seed, batch_points=262144,
                      loss=["squared 2-norm", "energy norm"][args.kind],
                      init="damped Jacobi (omega 1) + uniform noise 0.02", epoch_loss=[float(v) for v in hist]),
        heldout=dict(seeds=[100001, 100032, 200001, 200032], loss_jacobi_init=loss_init, loss_trained=loss_trained),
        cg_init=cg_init, cg=cg_eval, seconds=dict(pairs=t_pairs, train=t_train))
    S.save(args.out, **meta)
    print(json.dumps(meta, indent=1))


if __name__ == "__main__":
    main()
