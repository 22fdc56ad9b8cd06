"""Training and evaluation of the learned preconditioner (the U-Net of
asd2g_unet_*).

Data: GFM pressure systems produced by this library's own solver on 256x256
grids -- two to four droplets per domain, density ratio log-uniform in
[1, 1000] (eight log-spaced ratios, one session each), random smooth
divergence fields as right-hand sides (plus the surface-tension jumps the
assembly adds) -- each solved to a relative residual of 1e-10 by the
MG-preconditioned FCG.  A pair is what the network sees inside the two-level
preconditioner of ASD2G_SOLVER_UNET: the features of r1 = r - A V(r), the
residual one FP32 V-cycle leaves, and the unit-RMS error it must supply; r is
the right-hand side for half of the pairs and the residual of a later MG-FCG
iterate (1 to 12 iterations) for the other half.  The pairs stay on the device; training is Adam on shuffled
mini-batches with cosine decay, by default on the energy loss (the relative
A-norm error that the best multiple of the output leaves, the quantity the
solver's omega step minimises).

    python -m asd2_b200.train_unet --samples 20000 --epochs 3

PyTorch only provides the device tensors; every kernel is the library's.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

DEFAULT_WEIGHTS = os.path.join(HERE, "unet_weights.npz")
RATIOS = tuple(float(r) for r in np.geomspace(1.0, 1000.0, 8))
MAX_PAIR_ITERS = 12


def generate(samples: int, n: int = 256, seed: int = 0, log=print):
    """(feats [S][n][n][4], targets [S][n][n]) as CUDA tensors."""
    import torch
    from asd2_b200 import api
    from asd2_b200 import workloads as W
    rng = np.random.Generator(np.random.PCG64(seed))
    feats = torch.empty(samples, n, n, 4, device="cuda")
    targets = torch.empty(samples, n, n, device="cuda")
    sessions = {}
    t0 = time.time()
    for k in range(samples):
        ratio = RATIOS[int(rng.integers(len(RATIOS)))]
        c = W.multi_droplet(n, seed=int(rng.integers(1 << 31)), count=int(rng.integers(2, 5)), rho_ratio=ratio)
        if ratio not in sessions:
            sessions[ratio] = api.Session(api.Params.from_case(c))
        s = sessions[ratio]
        s.upload("ls", c.ls)
        s.apply_bc("ls", "P")
        s.heaviside()
        s.kappa()
        s.upload("div", W.smooth_field(n, n, rng, modes=int(rng.integers(2, 12)),
                                       amplitude=float(10 ** rng.uniform(-1, 1.5))))
        s.assemble_gfm(1e-3, recompute_kappa=False)
        r = s.solve_pressure(api.MGPCG, tol=1e-10, maxit=2000, dt=1e-3)
        if r["status"] != 0:
            raise RuntimeError(f"training system {k} did not converge: {r}")
        # the first residual, or one of a later Krylov iterate (what the network meets inside the solve)
        s.training_pair(feats[k], targets[k], iters=int(rng.integers(0, MAX_PAIR_ITERS + 1)) if k % 2 else 0)
        if log and (k + 1) % 2000 == 0:
            s.sync()
            log(f"generated {k + 1}/{samples} systems in {time.time() - t0:.1f} s")
    for s in sessions.values():
        s.close()
    torch.cuda.synchronize()
    return feats, targets


def train(feats, targets, epochs: int = 3, batch: int = 16, lr: float = 1e-3, seed: int = 0, log=print,
          loss: str = "energy"):
    """Adam over shuffled mini-batches with cosine learning-rate decay;
    returns the network and the per-epoch mean losses.  loss "energy": the
    relative A-norm error the best multiple of u leaves against the error
    target (what the solver's omega step minimises); "residual": 1 -
    cos^2(A u, r1), the relative residual instead (targets unused); "mse":
    relative squared error against the targets."""
    import torch
    from asd2_b200 import api
    S, n = feats.shape[0], feats.shape[1]
    net = api.UNet(batch, n, n)
    net.init(seed)
    g = torch.Generator().manual_seed(seed)
    steps_total = epochs * (S // batch)
    step, history = 0, []
    t0 = time.time()
    for ep in range(epochs):
        perm = torch.randperm(S, generator=g).cuda()
        losses = []
        for b0 in range(0, S - batch + 1, batch):
            idx = perm[b0:b0 + batch]
            fb = feats[idx].contiguous()
            cur = lr * 0.5 * (1.0 + np.cos(np.pi * step / max(steps_total, 1)))
            if loss == "energy":
                losses.append(net.train_step_energy(fb, targets[idx].contiguous(), batch, n, n, cur))
            elif loss == "residual":
                losses.append(net.train_step_residual(fb, batch, n, n, cur))
            else:
                losses.append(net.train_step(fb, targets[idx].contiguous(), batch, n, n, cur))
            step += 1
        history.append(float(np.mean(losses)))
        if log:
            log(f"epoch {ep + 1}/{epochs}: mean {loss} loss {history[-1]:.4f} ({time.time() - t0:.1f} s)")
    if net.error_flag():
        raise RuntimeError("a tensor-core wait timed out during training")
    return net, history


def save(net, path, meta):
    np.savez(path, params=net.params(), meta=json.dumps(meta))


def load_params(path=DEFAULT_WEIGHTS):
    z = np.load(path)
    return z["params"], json.loads(str(z["meta"]))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=20000)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--loss", choices=("energy", "residual", "mse"), default="energy")
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    args = ap.parse_args()
    t0 = time.time()
    feats, targets = generate(args.samples, seed=args.seed)
    t_gen = time.time() - t0
    net, hist = train(feats, targets, args.epochs, args.batch, args.lr, args.seed, loss=args.loss)
    meta = dict(samples=args.samples, epochs=args.epochs, batch=args.batch, lr=args.lr, seed=args.seed, loss=args.loss,
                grid=256, ratios=list(RATIOS), loss_history=hist, seconds_generate=t_gen,
                seconds_total=time.time() - t0)
    save(net, args.out, meta)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
