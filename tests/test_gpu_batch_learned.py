"""The learned preconditioner inside the batched solver
(asd2g_batch_set_preconditioner_net + asd2g_batch_solve_with(..., UNET)):
uneven instances, one launch per phase, one network pass per size group.

  * each instance gives what a single session's learned solve gives on the
    same system: iteration counts within two, pressure within 1e-7 of its
    maximum (both at 1e-10), true FP64 residual within the tolerance, no
    fallback; a zero right-hand side converges at once beside the others;
  * the smallest instance also agrees with the oracle's FP64 PCG (1e-12);
  * an untrained network still converges; a cap that stops the learned phase
    hands the batch to the batched MG-FCG (fallback reported);
  * instances whose sides are not multiples of 8 are refused.
"""
import os

import numpy as np
import pytest

from asd2_b200 import api
from asd2_b200 import train_unet as T
from asd2_b200 import workloads as W
from oracle.pyoracle import Oracle
from tests.helpers import fluid_from_case, grid_from_case, interior, params_for

pytestmark = pytest.mark.gpu
O = Oracle()

SHAPES = [(64, 64), (96, 96), (64, 64), (128, 64), (160, 160)]
RATIOS = [1000.0, 10.0, 300.0, 1.0, 50.0]


def _inputs(k, nx, ny):
    c = W.droplet(nx, seed=200 + k, ny=ny, rho_ratio=RATIOS[k % len(RATIOS)])
    g, f = grid_from_case(c), fluid_from_case(c)
    with api.Session(params_for(g, f)) as s:
        s.upload("ls", c.ls)
        s.apply_bc("ls", "P")
        s.heaviside()
        s.kappa()
        X = (np.arange(g.nx + 6) - 2.5) * g.dx
        Y = (np.arange(g.ny + 6) - 2.5) * g.dy
        div = np.outer(np.sin(3 * X + k), np.cos(2 * Y)) * 10.0
        if k == 2:
            div[:] = 0.0
        s.upload("div", div)
        data = {f_: s.download(f_) for f_ in ("ls", "H", "kappa", "div")}
    if k == 2:
        data["kappa"][:] = 0.0  # no curvature jump either: b = 0
    return g, f, data


def _net(trained=True):
    net = api.UNet(1, 160, 160)
    if trained:
        params, _ = T.load_params()
        net.set_params(params)
    else:
        net.init(seed=5)
    return net


def _batch(items, dts):
    b = api.Batch([params_for(g, f) for g, f, _ in items])
    for k, (_, _, d) in enumerate(items):
        for fld in ("ls", "H", "kappa", "div"):
            b.upload(k, fld, d[fld])
    b.assemble(dts)
    return b


@pytest.mark.skipif(not os.path.exists(T.DEFAULT_WEIGHTS), reason="no trained weights in the package")
def test_batched_learned_matches_sessions_and_oracle():
    items = [_inputs(k, nx, ny) for k, (nx, ny) in enumerate(SHAPES)]
    dts = np.array([1e-3 * (1 + 0.1 * k) for k in range(len(items))])
    net = _net()
    with _batch(items, dts) as b:
        b.set_preconditioner_net(net)
        r = b.solve(tol=1e-10, maxit=2000, solver=api.UNET)
        assert r["status"] == 0 and not r["fallback"], r
        got = [b.download(k, "ps") for k in range(len(items))]
    for k, (g, f, d) in enumerate(items):
        ps = got[k]
        if k == 2:
            assert r["iters"][k] == 0 and np.abs(interior(ps)).max() == 0.0
            continue
        with api.Session(params_for(g, f)) as s:
            for fld in ("ls", "H", "kappa", "div"):
                s.upload(fld, d[fld])
            s.assemble_gfm(dts[k], recompute_kappa=False)
            s.set_preconditioner_net(net)
            rs = s.solve_pressure(api.UNET, tol=1e-10, maxit=2000, dt=dts[k])
            assert rs["status"] == 0 and not s.last_fallback(), rs
            ps_ref = s.download("ps")
            assert abs(int(r["iters"][k]) - rs["iters"]) <= 2, (k, r["iters"][k], rs["iters"])
            scale = np.abs(interior(ps_ref)).max()
            assert np.abs(interior(ps) - interior(ps_ref)).max() <= 1e-7 * scale, k
            s.upload("ps", ps)
            assert s.true_residual() <= 1e-9, k
            s.set_preconditioner_net(None)
        if k == 0:  # the smallest instance against the oracle's FP64 PCG
            sysd = O.gfm_assemble(g, f, dts[k], d["ls"], d["kappa"].copy(), d["H"], d["div"], recompute_kappa=False)
            x, _, _, _ = O.pcg(g, sysd, tol=1e-12, maxit=500000)
            ps_ora = O.scatter(g, x)
            e = np.abs(interior(ps) - interior(ps_ora)).max() / np.abs(interior(ps_ora)).max()
            assert e <= 1e-7, e
    net.close()


def test_batched_learned_untrained_and_fallback():
    items = [_inputs(k, nx, ny) for k, (nx, ny) in enumerate(SHAPES[:2])]
    dts = np.array([1e-3, 2e-3])
    net = _net(trained=False)
    with _batch(items, dts) as b:
        b.set_preconditioner_net(net)
        r = b.solve(tol=1e-8, maxit=2000, solver=api.UNET)
        assert r["status"] == 0 and not r["fallback"], r
        assert (r["resid"] <= 1e-8).all()
        # a cap of 3 iterations stops the learned phase: the batched MG-FCG
        # takes over (with the same cap, so it reports non-convergence)
        r = b.solve(tol=1e-10, maxit=3, solver=api.UNET)
        assert r["fallback"] and r["status"] == api.NOT_CONVERGED, r
        # and the plain batched solve is unaffected by the attached network
        r = b.solve(tol=1e-8, maxit=2000)
        assert r["status"] == 0
    net.close()


def test_batched_learned_needs_multiples_of_8():
    items = [_inputs(0, 64, 64), _inputs(1, 60, 64)]
    net = _net(trained=False)
    with _batch(items, np.array([1e-3, 1e-3])) as b:
        with pytest.raises(api.Asd2gError):
            b.set_preconditioner_net(net)
    net.close()
