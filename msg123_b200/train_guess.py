"""Train the learned Newton initial guess on steps the GPU solver generates.

Recipe (train_stream, the default): heterogeneous fields of 128x128x96 cells (the block
generator with sigma_lnK drawn in [0.5, 1.5]; the 25.2M-cell workload's depth, layer
thickness and water table), each advanced over a whole event -- the
rain and the drainage after it -- by the solver settings of the value path with the plain
extrapolation guess (mixed precision, AMG kept for 4 steps, two-pow kr, adaptive dt);
every accepted step (features before the step, the head increment after it) is one
sample, 20,000 in all.  The samples stream through a bounded store on the device
(reservoir sampling keeps it a uniform sample of every step so far), and AdamW steps on
the project's own forward/backward kernels follow each collected step, then a last pass
over the store.  Writes msg123_b200/weights/guess_cnn.npy (float32, msg_gpu_cnn_nparam
values).  `train` is the earlier fixed-set recipe (all samples kept, trained afterwards).

    python -m msg123_b200.train_guess [--fields 400] [--steps 50] [--cap 1000]
"""
import argparse
import json
import os
import time

import numpy as np

from .config import make_config
from .learned import Cnn, generate
from .solver import GpuSolver

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "weights", "guess_cnn.npy")


def train(fields=12, steps=16, iters=2400, seed=0, shape=(128, 128, 48), out=WEIGHTS, log=None):
    rng = np.random.default_rng(seed)
    probs = [make_config("hetero", shape=shape, seed=5000 + k, sigma=float(rng.uniform(0.5, 1.5)))
             for k in range(fields)]
    cnn = Cnn(seed=seed)
    t0 = time.time()
    n = generate(cnn, probs, steps_per_problem=steps, amg_lag=1, precision=1)
    t_gen = time.time() - t0
    l0 = float(np.mean([cnn.loss_grad(k, want_grad=False)[0] for k in range(n)]))
    t0 = time.time()
    lr = [2e-3, 1e-3, 5e-4]
    for k, rate in enumerate(lr):
        cnn.train(iters=iters // len(lr), lr=rate, weight_decay=1e-5, seed=seed + k)
    t_train = time.time() - t0
    l1 = float(np.mean([cnn.loss_grad(k, want_grad=False)[0] for k in range(n)]))
    w = cnn.get_weights()
    os.makedirs(os.path.dirname(out), exist_ok=True)
    np.save(out, w)
    info = dict(samples=n, shape=list(shape), fields=fields, steps=steps, iters=iters, loss_before=l0,
                loss_after=l1, gen_s=t_gen, train_s=t_train)
    if log:
        print(json.dumps(info))
    return info


SOLVER = dict(guess_mode=1, precision=1, amg_lag=4, vg_form=1, jv_mode=1)


def train_stream(fields=400, steps=50, cap=1000, iters_per_step=2, final_iters=3000, seed=0, shape=(128, 128, 96),
                 lr=(2e-3, 5e-4), out=WEIGHTS, log=None, init=None):
    """Streaming recipe: fields x steps generated samples, `iters_per_step` AdamW steps after
    each (learning rate decaying geometrically from lr[0] to lr[1]), then `final_iters` over
    the store.  Returns a summary dict (and saves the weights when `out` is set)."""
    rng = np.random.default_rng(seed)
    cnn = Cnn(seed=seed)
    if init is not None:
        cnn.set_weights(init)
    cnn.set_capacity(cap, seed)
    total = max(fields * steps, 1)
    done, skipped, t_solve, t_train = 0, 0, 0.0, 0.0
    rate = lambda f: lr[0] * (lr[1] / lr[0]) ** min(f, 1.0)
    for k in range(fields):
        p = make_config("hetero", shape=shape, seed=5000 + k, sigma=float(rng.uniform(0.5, 1.5)))
        with GpuSolver(p, **SOLVER) as g:
            g.init_state()
            g.advance(nsteps=1)                    # the first step has no previous increment
            for _ in range(steps):
                t0 = time.time()
                rc, st = g.advance(nsteps=1)
                t_solve += time.time() - t0
                if rc != 0 or st["accepted"] != 1:
                    skipped += 1
                    break
                cnn.collect(g)
                done += 1
                t0 = time.time()
                cnn.train(iters=iters_per_step, lr=rate(done / total), weight_decay=1e-5, seed=seed * 7919 + done)
                t_train += time.time() - t0
        if log and (k + 1) % 25 == 0:
            print(json.dumps(dict(fields=k + 1, samples=done, store=cnn.nsamples(), solve_s=round(t_solve, 1),
                                  train_s=round(t_train, 1))), flush=True)
        if out and (k + 1) % 100 == 0:             # a checkpoint, so a cut-off run still leaves weights
            os.makedirs(os.path.dirname(out) or ".", exist_ok=True)
            np.save(out, cnn.get_weights())
    t0 = time.time()
    last = cnn.train(iters=final_iters, lr=lr[1], weight_decay=1e-5, seed=seed + 17)
    t_train += time.time() - t0
    n = cnn.nsamples()
    loss = float(np.mean([cnn.loss_grad(i, want_grad=False)[0] for i in range(0, n, max(n // 200, 1))]))
    w = cnn.get_weights()
    if out:
        os.makedirs(os.path.dirname(out), exist_ok=True)
        np.save(out, w)
    info = dict(samples=done, store=n, fields=fields, steps=steps, shape=list(shape), final_loss=loss,
                last_window_loss=last, solve_s=t_solve, train_s=t_train, stopped_fields=skipped)
    if log:
        print(json.dumps(info), flush=True)
    cnn.close()
    return info, w


def load(cnn, path=WEIGHTS):
    cnn.set_weights(np.load(path))
    return cnn


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--fields", type=int, default=400)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--cap", type=int, default=1000)
    ap.add_argument("--iters-per-step", type=int, default=2)
    ap.add_argument("--final-iters", type=int, default=3000)
    ap.add_argument("--out", default=WEIGHTS)
    a = ap.parse_args()
    train_stream(a.fields, a.steps, a.cap, a.iters_per_step, a.final_iters, out=a.out, log=True)
