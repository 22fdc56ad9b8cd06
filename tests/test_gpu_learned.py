"""The learned preconditioner inside the pressure solve (ASD2G_SOLVER_UNET):
flexible CG in FP64 with the V-cycle plus the U-Net correction, judged on the
FP64 residual like the MG-FCG.

  * with the committed trained weights, a 256^2 two-droplet system converges
    to 1e-8 without the Jacobi-PCG fallback, its true FP64 residual meets
    the tolerance, and the pressure agrees with a 1e-12 MG-FCG solve to 1e-6;
  * an untrained network still converges (the V-cycle carries it and the
    A-norm optimal step weighs the correction), and a cap that stops the
    learned phase early hands the system to Jacobi-PCG (last_fallback = 1);
  * a training pair satisfies its defining identity A e1 = r1: the 5-point
    operator of the pair's coefficient channels applied to the target is
    parallel to the residual channel (both are FP32 roundings);
  * the same pair taken at a later Krylov iterate satisfies it too.
"""
import os

import numpy as np
import pytest
import torch

from asd2_b200 import api
from asd2_b200 import train_unet as T
from asd2_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _system(n=256, count=2, ratio=300.0, seed=11):
    c = W.multi_droplet(n, seed=seed, count=count, rho_ratio=ratio)
    s = api.Session(api.Params.from_case(c))
    s.upload("ls", c.ls)
    s.apply_bc("ls", "P")
    s.heaviside()
    s.kappa()
    s.upload("div", W.smooth_field(n, n, np.random.default_rng(seed)))
    s.assemble_gfm(1e-3, recompute_kappa=False)
    return s


def _stencil(f, v):
    d, ce, cn = f[..., 1], f[..., 2], f[..., 3]
    y = d * v
    y[:, :-1, :] -= ce[:, :-1, :] * v[:, 1:, :]
    y[:, 1:, :] -= ce[:, :-1, :] * v[:, :-1, :]
    y[:, :, :-1] -= cn[:, :, :-1] * v[:, :, 1:]
    y[:, :, 1:] -= cn[:, :, :-1] * v[:, :, :-1]
    return y


@pytest.mark.skipif(not os.path.exists(T.DEFAULT_WEIGHTS), reason="no trained weights in the package")
def test_trained_learned_solve_converges():
    n = 256
    s = _system(n)
    ref = s.solve_pressure(api.MGPCG, tol=1e-12, maxit=10000, dt=1e-3)
    assert ref["status"] == 0
    p_ref = s.download("ps")[3:-3, 3:-3].copy()
    params, _ = T.load_params()
    net = api.UNet(1, n, n)
    net.set_params(params)
    s.set_preconditioner_net(net)
    r = s.solve_pressure(api.UNET, tol=1e-8, maxit=10000, dt=1e-3)
    assert r["status"] == 0, r
    assert s.last_fallback() == 0
    assert s.true_residual() <= 1e-8
    mg = s.solve_pressure(api.MGPCG, tol=1e-8, maxit=10000, dt=1e-3)
    assert r["iters"] <= mg["iters"] + 2, (r, mg)
    s.solve_pressure(api.UNET, tol=1e-8, maxit=10000, dt=1e-3)
    p = s.download("ps")[3:-3, 3:-3]
    assert np.abs(p - p_ref).max() <= 1e-6 * np.abs(p_ref).max()
    assert net.error_flag() == 0
    s.close()


def test_untrained_network_and_fallback():
    n = 128
    s = _system(n, count=2, ratio=100.0, seed=3)
    net = api.UNet(1, n, n)
    net.init(seed=1)
    s.set_preconditioner_net(net)
    r = s.solve_pressure(api.UNET, tol=1e-8, maxit=10000, dt=1e-3)
    assert r["status"] == 0 and s.last_fallback() == 0, r
    assert s.true_residual() <= 1e-8
    # a cap of 3 iterations ends the learned phase unconverged: the Jacobi-PCG
    # fallback runs (with the same cap) and reports not converged
    r = s.solve_pressure(api.UNET, tol=1e-8, maxit=3, dt=1e-3)
    assert s.last_fallback() == 1
    assert r["status"] == api.NOT_CONVERGED, r
    s.close()


@pytest.mark.parametrize("iters", [0, 5])
def test_training_pair_identity(iters):
    n = 128
    s = _system(n, count=3, ratio=1000.0, seed=7)
    r = s.solve_pressure(api.MGPCG, tol=1e-12, maxit=10000, dt=1e-3)
    assert r["status"] == 0
    f = torch.empty(1, n, n, 4, device="cuda")
    t = torch.empty(1, n, n, device="cuda")
    s.training_pair(f, t, iters=iters)
    s.sync()
    assert torch.isfinite(f).all() and torch.isfinite(t).all()
    assert abs(float(f[..., 0].pow(2).mean().sqrt()) - 1.0) < 1e-4
    assert abs(float(t.pow(2).mean().sqrt()) - 1.0) < 1e-4
    a, r1 = _stencil(f.double(), t.double()), f[..., 0].double()
    a[0, 0, 0] = 0.0  # the pinned cell's row is not part of the system
    cos = float((a * r1).sum() / (a.norm() * r1.norm()))
    assert cos > 0.999, cos
    s.close()
