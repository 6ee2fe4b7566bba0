"""Trains the Poisson warm-start network (ssam_cnn_*) on the GPU.

Training set: 4096 pairs (f, u) at n^3 = 128^3 -- f = gaussian_rhs_torch(8,
n, seed) for 512 seeds (8 right-hand sides each; with --mix m, a fraction m
of the batches are poisson_dst.random_spectrum_rhs instead, so the network
also meets the rough and smooth inputs that residuals inside defect
correction are) and u the plain solver's answer (ssam_poisson_solve: FP32
Jacobi sweeps inside the FP64 defect correction, to --target-tol relative
residual, 64 right-hand sides per solve).  The solutions are kept on the
device in FP32 (8 MiB each); the right-hand sides are regenerated from their
seeds for every batch.  A sample of the solutions is compared with the exact
discrete solution (poisson_dst.solve, a type-I sine transform).  With
--targets exact the sine-transform solutions are used directly.  Seeds of the
training set start at 100000, so the benchmark and test right-hand sides
(small seeds) are never seen in training.

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
    ap.add_argument("--targets", choices=["solver", "exact"], default="solver")
    ap.add_argument("--target-tol", type=float, default=1e-4)
    ap.add_argument("--mix", type=float, default=0.5,
                    help="fraction of batches with random-spectrum right-hand sides")
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

    n_spec = int(round(a.mix * nbatches))

    def rhs(i):
        """Right-hand sides of training batch i."""
        if i >= nbatches - n_spec:
            return poisson_dst.random_spectrum_rhs(a.batch, a.n, TRAIN_SEED0 + 50000 + i, dev)
        return gaussian_rhs_torch(a.batch, a.n, TRAIN_SEED0 + i, dev)

    f_eval = gaussian_rhs_torch(a.batch, a.n, EVAL_SEED, dev)
    u_eval = poisson_dst.solve(f_eval)
    f_spec = poisson_dst.random_spectrum_rhs(a.batch, a.n, EVAL_SEED, dev)
    u_spec = poisson_dst.solve(f_spec)
    worst = max(ssam.poisson_residual(f_eval, u_eval) + ssam.poisson_residual(f_spec, u_spec))
    if worst > 1e-10:
        raise RuntimeError(f"sine-transform solution has residual {worst:.3g}")

    def rel_err(w, u):
        return ((w - u).flatten(1).norm(dim=1) / u.flatten(1).norm(dim=1)).max().item()

    def evaluate():
        w = net.forward(f_eval)
        return {"eval_warm_start_residual": max(ssam.poisson_residual(f_eval, w)),
                "eval_rel_error": rel_err(w, u_eval),
                "eval_spectrum_rel_error": rel_err(net.forward(f_spec), u_spec)}

    log({"event": "start", "n": a.n, "batch": a.batch, "pairs": a.pairs, "steps": steps,
         "lr": a.lr, "params": net.num_params, "targets": a.targets, "mix": a.mix})

    # the plain solver's answers for every training pair, 64 rhs per solve
    solved = None
    if a.targets == "solver":
        t0 = time.time()
        solved = torch.empty((nbatches * a.batch, a.n, a.n, a.n), dtype=torch.float32,
                             device=dev)
        per = max(1, 64 // a.batch)
        sweeps = 0
        dev_rel = None
        for c0 in range(0, nbatches, per):
            ids = list(range(c0, min(nbatches, c0 + per)))
            f = torch.cat([rhs(i) for i in ids])
            u = torch.zeros_like(f)
            st = ssam.poisson_solve(f, u, tol=a.target_tol, sweep_dtype="f32",
                                    sweeps_per_correction=2000, max_sweeps=400000)
            if not st["converged"]:
                raise RuntimeError(f"plain solver did not converge: {st}")
            sweeps += st["sweeps"]
            solved[c0 * a.batch:(c0 + len(ids)) * a.batch] = u.float()
            if c0 == 0:
                exact = poisson_dst.solve(f[:a.batch])
                dev_rel = rel_err(u[:a.batch], exact)
            del f, u
        log({"event": "targets", "solver_sweeps": sweeps, "seconds": time.time() - t0,
             "tol": a.target_tol, "max_rel_error_vs_exact_first_batch": dev_rel})
    g = torch.Generator().manual_seed(a.seed)
    order = []
    t_start = time.time()
    t_steps = 0.0
    for step in range(steps):
        if not order:
            order = torch.randperm(nbatches, generator=g).tolist()
        idx = order.pop()
        f = rhs(idx)
        if solved is not None:
            u = solved[idx * a.batch:(idx + 1) * a.batch].double()
        else:
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
            log({"step": step, "loss": loss, "lr": lr, **evaluate(),
                 "ms_per_step": 1e3 * t_steps / (step + 1), "elapsed_s": time.time() - t_start})
    net.save(a.out)
    log({"event": "done", "steps": steps, **evaluate(),
         "ms_per_step": 1e3 * t_steps / max(1, steps), "elapsed_s": time.time() - t_start,
         "weights": os.path.basename(a.out)})
    logf.close()


if __name__ == "__main__":
    main()
