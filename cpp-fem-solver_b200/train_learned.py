"""Train the learned-IC(0) network on generated diffusion systems (GPU).

    python cpp-fem-solver_b200/train_learned.py --systems 2000 --grid 256 --corr 0.1

Training systems are -div(k grad u) problems with log k a squared-exponential
Gaussian random field, one per seed 0..systems-1 (variance uniform in [1, 4]
per seed).  The network is local (three message-passing hops), so it trains
on 256^2 grids with correlation length 0.1 -- 25.6 cells per correlation
length, the same local statistics as the 512^2 / 0.05 benchmark systems.
Each step runs this library's own forward and backward kernels on one system
and applies Adam.  At the end, PCG iterations to 1e-8 with the trained
network and with plain IC(0) are compared on held-out seeds (2000+) at the
benchmark size, and the weights are written to weights/learned_ic0.bin,
where B2S_PC_LEARNED_IC0 finds them.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load():
    if "b2s" in sys.modules:
        return sys.modules["b2s"]
    spec = importlib.util.spec_from_file_location("b2s", os.path.join(HERE, "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["b2s"] = mod
    spec.loader.exec_module(mod)
    return mod


def _gen(args):
    grid, corr, seed = args
    b2s = load()
    return seed, b2s.gen_grf_diffusion(grid, seed, corr=corr)


def evaluate(b2s, ctx, learner, seeds, grid, corr, tol=1e-8):
    out = []
    for s in seeds:
        n, rp, ci, v = b2s.gen_grf_diffusion(grid, s, corr=corr)
        A = b2s.CSR(ctx, n, n, rp, ci, v)
        b = b2s.uniform(s, n)
        rows = {}
        for name, M in (("ic0", b2s.Precond(ctx, A, b2s.PC_IC0)), ("learned", learner.precond(A))):
            x, st = b2s.solve(ctx, A, b, b2s.PCG, M, tol=tol, maxit=20000)
            rows[name] = dict(iterations=st["iterations"], relres_true=st["relres_true"], ms=st["solve_ms"])
        out.append(dict(seed=s, **rows))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--systems", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=1)
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--corr", type=float, default=0.1)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--probes", type=int, default=4)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--eval", type=int, default=8, help="held-out systems at 512^2 / 0.05")
    ap.add_argument("--out", default=os.path.join(HERE, "weights", "learned_ic0.bin"))
    ap.add_argument("--log", default=None)
    args = ap.parse_args()

    # generate on host cores first (spawned workers, before any GPU work)
    t0 = time.time()
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        data = dict(pool.map(_gen, [(args.grid, args.corr, s) for s in range(args.systems)], chunksize=8))
    t_gen = time.time() - t0

    b2s = load()
    ctx = b2s.Context(0)
    learner = b2s.Learner(ctx, seed=args.seed)
    log = []
    t1 = time.time()
    step = 0
    for ep in range(args.epochs):
        order = np.random.default_rng(ep).permutation(args.systems)
        run = []
        for k in order:
            n, rp, ci, v = data[int(k)]
            A = b2s.CSR(ctx, n, n, rp, ci, v)
            lr = args.lr * (0.5 * (1 + np.cos(np.pi * step / (args.epochs * args.systems))))
            loss = learner.step(A, nprobes=args.probes, seed=1000003 * ep + int(k), lr=lr)
            run.append(loss)
            step += 1
            if step % 100 == 0:
                log.append(dict(step=step, loss=float(np.mean(run[-100:]))))
                print(json.dumps(log[-1]), flush=True)
    t_train = time.time() - t1
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    learner.save(args.out)
    ev = evaluate(b2s, ctx, learner, list(range(2000, 2000 + args.eval)), 512, 0.05)
    it_ic0 = float(np.mean([e["ic0"]["iterations"] for e in ev]))
    it_lrn = float(np.mean([e["learned"]["iterations"] for e in ev]))
    summary = dict(systems=args.systems, epochs=args.epochs, grid=args.grid, corr=args.corr, steps=step,
                   gen_s=t_gen, train_s=t_train, first_loss=log[0]["loss"] if log else None,
                   last_loss=log[-1]["loss"] if log else None, heldout=ev, iterations_ic0=it_ic0,
                   iterations_learned=it_lrn, weights=args.out)
    print(json.dumps(summary))
    if args.log:
        with open(args.log, "w") as f:
            json.dump(dict(summary=summary, log=log), f, indent=1)


if __name__ == "__main__":
    main()
