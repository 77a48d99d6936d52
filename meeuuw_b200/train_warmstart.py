"""Train the warm-start U-Net on snapshots of the device time stepper and report what it buys.

    python -m meeuuw_b200.train_warmstart --n 128 --runs 20 --steps 110 --epochs 20 \
        --out meeuuw_b200/weights/unet_fk128.npz      (20 runs x 100 recorded steps = 2000 snapshots)

Every number printed comes from the device: the snapshots are generated by ``GPUModel`` (mixed
precision, 1e-8 relative Stokes residual), the network trains with the library's tensor-core
kernels, and the evaluation reruns held-out models with the zero, previous-step and gated learned
initial guesses.
"""
import argparse
import json
import math
import time
from dataclasses import replace

import numpy as np
import torch

from . import configs
from .unet import UNet, cold_start_gain, compare_guesses, generate_dataset, train


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--runs", type=int, default=20)
    ap.add_argument("--steps", type=int, default=110)
    ap.add_argument("--skip", type=int, default=10)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--eval-steps", type=int, default=20)
    ap.add_argument("--eval-n", type=int, nargs="*", default=[128])
    ap.add_argument("--out", default="meeuuw_b200/weights/unet_fk128.npz")
    ap.add_argument("--report", default=None)
    ap.add_argument("--load", default=None, help="evaluate these weights instead of training")
    ap.add_argument("--cold-cases", type=int, default=8)
    a = ap.parse_args(argv)
    log = lambda s: print(s, flush=True)
    if a.load:
        net = UNet.load(a.load)
        report = dict(weights=a.load, eval={})
    else:
        t0 = time.time()
        Xs, Ys, meta = generate_dataset(a.n, a.runs, a.steps, a.skip, a.seed, log=log)
        torch.cuda.synchronize()
        t1 = time.time()
        log(f"dataset: {Xs.shape[0]} snapshots in {t1 - t0:.1f} s")
        net = UNet(base=32, levels=4, seed=a.seed)
        losses = train(net, Xs, Ys, a.epochs, a.batch, a.lr, a.seed, log=log)
        torch.cuda.synchronize()
        t2 = time.time()
        log(f"training: {a.epochs} epochs in {t2 - t1:.1f} s")
        net.save(a.out, n_net=a.n, runs=a.runs, steps=a.steps, epochs=a.epochs, final_mse=losses[-1])
        del Xs, Ys
        report = dict(dataset_s=t1 - t0, train_s=t2 - t1, snapshots=len(meta), losses=losses, eval={})
    # cold starts on held-out models (seeds and temperatures the training never saw)
    rng = np.random.default_rng(777)
    cases = []
    for i in range(a.cold_cases):
        Ra = math.exp(rng.uniform(math.log(1e4), math.log(1e6)))
        c = math.exp(rng.uniform(0.0, math.log(1e5)))
        cases.append((replace(configs.fk_convection(a.n), name=f"heldout{i}", Ra=Ra, fk_gamma=math.log(c),
                              seed=900000 + i), 500000 + i))
    for sb in (0, 20):
        g = cold_start_gain(net, cases, steps_before=sb, n_net=a.n, log=log)
        report[f"cold_start_after_{sb}_steps"] = g
        z = sum(x[1] for x in g)
        l = sum(x[2] for x in g)
        log(f"cold starts after {sb} steps: zero guess {z} outer iterations, learned guess {l}")
    for n in a.eval_n:
        cfg = replace(configs.fk_convection(n), seed=12345)
        ev = compare_guesses(net, cfg, a.eval_steps, n_net=a.n)
        report["eval"][n] = {k: {kk: vv for kk, vv in v.items() if kk != "steps"} for k, v in ev.items()}
        report["eval"][n]["per_step"] = {k: [s["outer"] for s in v["steps"]] for k, v in ev.items()}
        log(f"eval {n}: " + json.dumps(report["eval"][n]))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)
    return report


if __name__ == "__main__":
    main()
