"""Batched GFM pressure solves (asd2g_batch_*): uneven instances assembled
and solved together, one launch per phase.  Each instance must give what a
single session gives on the same inputs: the batched pressure agrees with the
session's MG-FCG pressure (both solved to 1e-10) to 1e-7 of its maximum, the
true FP64 residual of the batched pressure (recomputed by a session on the
same system) meets the tolerance, P = PS / dt, and instances stop on their
own (a zero right-hand side converges at once beside the others)."""
import numpy as np
import pytest

from asd2_b200 import api
from asd2_b200 import workloads as W
from tests.helpers import fluid_from_case, grid_from_case, interior, params_for

pytestmark = pytest.mark.gpu

SHAPES = [(48, 48), (64, 40), (96, 96), (130, 70), (200, 200), (256, 128)]


def _inputs(k, nx, ny):
    c = W.droplet(nx, seed=100 + k, ny=ny, rho_ratio=[1000, 10, 300, 1, 1000, 50][k % 6])
    g, f = grid_from_case(c), fluid_from_case(c)
    with api.Session(params_for(g, f)) as s:
        s.upload("ls", c.ls)
        s.apply_bc("ls", "P")
        s.heaviside()
        s.kappa()
        X = (np.arange(g.nx + 6) - 2.5) * g.dx
        Y = (np.arange(g.ny + 6) - 2.5) * g.dy
        div = np.outer(np.sin(3 * X + k), np.cos(2 * Y)) * 10.0
        if k == 3:
            div[:] = 0.0
        s.upload("div", div)
        data = {f_: s.download(f_) for f_ in ("ls", "H", "kappa", "div")}
    if k == 3:
        data["kappa"][:] = 0.0  # no curvature jump either: b = 0
    return g, f, data


def test_batch_matches_sessions():
    items = [_inputs(k, nx, ny) for k, (nx, ny) in enumerate(SHAPES)]
    params = [params_for(g, f) for g, f, _ in items]
    dts = np.array([1e-3 * (1 + 0.1 * k) for k in range(len(items))])
    with api.Batch(params) as b:
        for k, (_, _, d) in enumerate(items):
            for fld in ("ls", "H", "kappa", "div"):
                b.upload(k, fld, d[fld])
        b.assemble(dts)
        r = b.solve(tol=1e-10, maxit=2000)
        assert r["status"] == 0, r
        got = [(b.download(k, "ps"), b.download(k, "p")) for k in range(len(items))]
    for k, (g, f, d) in enumerate(items):
        with api.Session(params_for(g, f)) as s:
            for fld in ("ls", "H", "kappa", "div"):
                s.upload(fld, d[fld])
            s.assemble_gfm(dts[k], recompute_kappa=False)
            rs = s.solve_pressure(api.MGPCG, tol=1e-10, maxit=2000, dt=dts[k])
            ps_ref = s.download("ps")
            ps, p = got[k]
            if k == 3:
                assert r["iters"][k] == 0 and np.abs(interior(ps)).max() == 0.0
                continue
            assert abs(int(r["iters"][k]) - rs["iters"]) <= 2, (k, r["iters"][k], rs["iters"])
            scale = np.abs(interior(ps_ref)).max()
            assert np.abs(interior(ps) - interior(ps_ref)).max() <= 1e-7 * scale, k
            np.testing.assert_allclose(interior(p), interior(ps) / dts[k], rtol=1e-15)
            s.upload("ps", ps)
            assert s.true_residual() <= 1e-9, k


def test_tile_shapes_agree_and_tuning_picks_fastest(monkeypatch):
    """Every multigrid tile shape solves the batch to the same pressure (the
    smoothing of a cell does not depend on the tiling; only the order of the
    dot-product sums does), and the tuned batch keeps the shape whose trial
    was fastest."""
    cases = [_inputs(k, nx, ny) for k, (nx, ny) in enumerate(SHAPES)]
    dts = [1e-3 * (1 + k) for k in range(len(cases))]
    ps = []
    for shape in ("0", "1", "2", None):
        if shape is None:
            monkeypatch.delenv("ASD2G_MG_TILE", raising=False)
        else:
            monkeypatch.setenv("ASD2G_MG_TILE", shape)
        with api.Batch([params_for(g, f) for g, f, _ in cases]) as b:
            for i, (_, _, data) in enumerate(cases):
                for f_, a in data.items():
                    b.upload(i, f_, a)
            b.assemble(dts)
            r = b.solve(tol=1e-10, maxit=10000)
            assert r["status"] == 0, r
            (rows, cols), ms = b.tile_shape()
            if shape is not None:
                assert (rows, cols) == [(16, 32), (32, 32), (16, 64)][int(shape)]
                assert ms == [0.0, 0.0, 0.0]
            else:
                assert all(m > 0 for m in ms)
                assert (rows, cols) == [(16, 32), (32, 32), (16, 64)][int(np.argmin(ms))]
            ps.append([interior(b.download(i, "ps")) for i in range(len(cases))])
    for other in ps[1:]:
        for a, ref in zip(other, ps[0]):
            assert np.abs(a - ref).max() <= 1e-7 * max(np.abs(ref).max(), 1e-300)
