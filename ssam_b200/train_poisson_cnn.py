"""Trains the Poisson warm-start network (ssam_cnn_*) on the GPU.

Training set: 4096 pairs (f, u) at n^3 = 128^3 -- f = gaussian_rhs_torch(8,
n, seed) for 512 seeds (8 right-hand sides each), u = A^-1 f, the exact
discrete solution of the 7-point problem (poisson_dst.solve, a type-I sine
transform solve, checked here with the FP64 residual kernel).  The pairs are
regenerated on the device for every batch instead of being stored (64 GB at
FP32).  Seeds of the training set start at 100000, so the benchmark and test
right-hand sides (small seeds) are never seen in training.

Each step is one forward + backward through the library's tcgen05 kernels
(ssam_cnn_gradient) and one Adam step (ssam_cnn_adam_step); the learning rate
follows a linear warm-up and a cosine decay.  Writes the weights (the
ssam_cnn_save format) and a JSON-lines log of the loss, the held-out
warm-start residual and the step time.

    python -m ssam_b200.train_poisson_cnn --epochs 4 \
        --out ssam_b200/data/poisson_cnn_n128.bin
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

TRAIN_SEED0 = 100000
EVAL_SEED = 99


def main(argv=None):
    import torch

    import ssam_b200 as ssam
    from ssam_b200 import poisson_dst
    from ssam_b200.workloads import gaussian_rhs_torch

    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--pairs", type=int, default=4096)
    ap.add_argument("--epochs", type=float, default=4.0)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--init", default=None, help="weights to start from")
    ap.add_argument("--out", default="ssam_b200/data/poisson_cnn_n128.bin")
    ap.add_argument("--log", default=None)
    ap.add_argument("--eval-every", type=int, default=64)
    a = ap.parse_args(argv)

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    nbatches = a.pairs // a.batch
    steps = int(round(a.epochs * nbatches))
    net = ssam.WarmStartCNN(a.n, a.batch, seed=a.seed)
    if a.init:
        net.load(a.init)
    log_path = a.log or os.path.splitext(a.out)[0] + ".log"
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    logf = open(log_path, "w")

    def log(rec):
        logf.write(json.dumps(rec) + "\n")
        logf.flush()
        print(json.dumps(rec), flush=True)

    f_eval = gaussian_rhs_torch(a.batch, a.n, EVAL_SEED, dev)
    u_eval = poisson_dst.solve(f_eval)
    worst = max(ssam.poisson_residual(f_eval, u_eval))
    if worst > 1e-10:
        raise RuntimeError(f"sine-transform targets have residual {worst:.3g}")

    def evaluate():
        w = net.forward(f_eval)
        rel_res = ssam.poisson_residual(f_eval, w)
        err = ((w - u_eval).flatten(1).norm(dim=1) / u_eval.flatten(1).norm(dim=1)).tolist()
        return max(rel_res), max(err)

    log({"event": "start", "n": a.n, "batch": a.batch, "pairs": a.pairs, "steps": steps,
         "lr": a.lr, "params": net.num_params, "target_residual": worst})
    g = torch.Generator().manual_seed(a.seed)
    order = []
    t_start = time.time()
    t_steps = 0.0
    for step in range(steps):
        if not order:
            order = torch.randperm(nbatches, generator=g).tolist()
        seed = TRAIN_SEED0 + order.pop()
        f = gaussian_rhs_torch(a.batch, a.n, seed, dev)
        u = poisson_dst.solve(f)
        if step < a.warmup:
            lr = a.lr * (step + 1) / a.warmup
        else:
            p = (step - a.warmup) / max(1, steps - a.warmup)
            lr = a.lr * (0.05 + 0.95 * 0.5 * (1 + math.cos(math.pi * p)))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        loss = net.gradient(f, u)
        net.adam_step(lr)
        torch.cuda.synchronize()
        t_steps += time.perf_counter() - t0
        if not math.isfinite(loss):
            raise RuntimeError(f"loss is {loss} at step {step}")
        if step % a.eval_every == 0 or step == steps - 1:
            res, err = evaluate()
            log({"step": step, "loss": loss, "lr": lr, "eval_warm_start_residual": res,
                 "eval_rel_error": err, "ms_per_step": 1e3 * t_steps / (step + 1),
                 "elapsed_s": time.time() - t_start})
    net.save(a.out)
    res, err = evaluate()
    log({"event": "done", "steps": steps, "eval_warm_start_residual": res,
         "eval_rel_error": err, "ms_per_step": 1e3 * t_steps / max(1, steps),
         "elapsed_s": time.time() - t_start, "weights": os.path.basename(a.out)})
    logf.close()


if __name__ == "__main__":
    main()
