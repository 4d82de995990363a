"""Train the learned Newton initial guess on steps the GPU solver generates.

Recipe: heterogeneous fields of 128x128x48 cells (the block generator with sigma_lnK
drawn in [0.5, 1.5]), each advanced with the mixed-precision AMG solver from the plain
extrapolation guess; every accepted step (features before the step, the head increment
after it) is one sample.  AdamW on the project's own tensor-core forward/backward
kernels.  Writes msg123_b200/weights/guess_cnn.npy (float32, msg_gpu_cnn_nparam values).

    python -m msg123_b200.train_guess [--fields 12] [--steps 16] [--iters 2400]
"""
import argparse
import json
import os
import time

import numpy as np

from .config import make_config
from .learned import Cnn, generate

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


def load(cnn, path=WEIGHTS):
    cnn.set_weights(np.load(path))
    return cnn


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--fields", type=int, default=12)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--iters", type=int, default=2400)
    ap.add_argument("--out", default=WEIGHTS)
    a = ap.parse_args()
    train(a.fields, a.steps, a.iters, out=a.out, log=True)
