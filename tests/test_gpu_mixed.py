"""Mixed precision (ASD2G_PRECISION_MIXED): level-set advection and
reinitialisation in FP32, the rest of the step in FP64, pressure by the
FP32-preconditioned FP64 flexible CG.  The FP64 session of the same case is
the reference; the bars are the measured FP32 errors with a margin of about
ten:
  * one reinitialisation of an exact distance function (droplet at rest):
    phi within 2e-6 of its maximum (the subcell root is taken in its
    non-cancelling form in FP32);
  * one revolution of the 128^2 perturbed circle: |phi| error <= 5e-4,
    interface-cell mask identical, area of phi >= 0 identical;
  * ten full droplet steps at 128^2: phi within 2e-5, pressure within 5e-4
    (max) and 5e-5 (L2) of its FP64 values, smoothed volume within 5e-8
    (relative).  The volume bar is not ten times the measured error: FP32 phi
    carries 6e-8 relative rounding, and the measured differences after ten
    steps (-9.8e-9 with the per-cell reinitialisation passes, -1.7e-8 with
    the packed ones) wander by that much from step to step.
The FP64 volume integrals are checked against the restatement's H and HS.
"""
import numpy as np
import pytest

from asd2_b200 import api
from asd2_b200 import workloads as W
from oracle.pyoracle import Oracle
from tests.helpers import fluid_from_case, grid_from_case, interior, params_for

pytestmark = pytest.mark.gpu
O = Oracle()


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _run_steps(c, prec, steps, solver):
    g, f = grid_from_case(c), fluid_from_case(c)
    with api.Session(params_for(g, f, precision=prec)) as s:
        s.upload("ls", c.ls)
        s.upload("u", c.u)
        s.upload("v", c.v)
        s.apply_bc("ls", "P")
        dt = s.update_dt()
        for _ in range(steps):
            r = s.droplet_step(dt, reinit_mode=api.REINIT_MINRK2, solver=solver, tol=1e-10, maxit=200000)
            assert r["status"] == 0, r
            dt = r["dt_next"]
        out = {k: interior(s.download(k)) for k in ("ls", "u", "v", "p")}
        out["vol"] = s.last_volume()
    return out


def test_mixed_reinit_of_distance_function():
    c = W.droplet(128, seed=7)
    ref = _run_steps(c, api.PRECISION_FP64, 1, api.MGPCG)
    mix = _run_steps(c, api.PRECISION_MIXED, 1, api.MGPCG)
    assert _rel(mix["ls"], ref["ls"]) <= 2e-6


def test_mixed_level_set_revolution():
    lc = W.perturbed_circle(128, seed=3)
    g = grid_from_case(lc)
    outs = {}
    for prec in (api.PRECISION_FP64, api.PRECISION_MIXED):
        p = api.Params(lc.nx, lc.ny, lc.dx, lc.dy, bc_u=lc.bc_u, bc_v=lc.bc_v, bc_p=lc.bc_p, precision=prec)
        with api.Session(p) as s:
            s.upload("ls", lc.ls)
            s.upload("u", lc.u)
            s.upload("v", lc.v)
            for _ in range(200):
                s.ls_step(lc.dt, api.REINIT_MINRK2)
            outs[prec] = (s.download("ls"), s.volume())
    (l64, v64), (l32, v32) = outs[api.PRECISION_FP64], outs[api.PRECISION_MIXED]
    assert np.abs(interior(l32) - interior(l64)).max() <= 5e-4
    assert np.array_equal(O.interface_mask(g, l32), O.interface_mask(g, l64))
    assert v32[0] == v64[0]
    assert abs(v32[1] - v64[1]) <= 1e-4 * v64[1]


@pytest.mark.parametrize("nx,ny,mode", [(150, 97, api.REINIT_MINRK2), (37, 211, api.REINIT_MINRK2_SUSSMAN),
                                         (300, 64, api.REINIT_ORIGINAL), (150, 97, api.REINIT_MINRK2_SUSSMAN)])
def test_mixed_level_set_ragged_grids(nx, ny, mode):
    """The FP32 advection stage works on 64-column strips and row pairs:
    grids whose sizes are not multiples of either (and narrow ones) must
    track the FP64 step as closely as the square case does, in every
    reinitialisation mode the FP32 path implements.

    Measured after 30 steps (max |phi32 - phi64|): MinRK2 2e-5 to 7e-5, all
    of it at interface cells with |phi0| ~ 1e-5 where the subcell distance is
    tiny and -c / nd amplifies FP32 rounding; Original and MinRK2 + Sussman
    ~1.4e-6; 99% of the cells within 2e-6 in every mode.  Bars: about ten
    times those."""
    h = 1.0 / max(nx, ny)
    X = (np.arange(nx + 6) - 3 + 0.5)[:, None] * h
    Y = (np.arange(ny + 6) - 3 + 0.5)[None, :] * h
    xc, yc = 0.5 * nx * h, 0.45 * ny * h
    r0 = 0.3 * min(nx, ny) * h
    th = np.arctan2(Y - yc, X - xc)
    ls = np.ascontiguousarray(r0 * (1.0 + 0.05 * np.cos(3 * th)) - np.sqrt((X - xc) ** 2 + (Y - yc) ** 2))
    # rotation about the centre: u on west faces (a function of y only), v on south faces
    u = np.ascontiguousarray(-2.0 * np.pi * (Y + 0.0 * X - yc))
    v = np.ascontiguousarray(2.0 * np.pi * (X + 0.0 * Y - xc))
    dt = 0.25 * h / (2.0 * np.pi * max(nx, ny) * h)
    outs = {}
    for prec in (api.PRECISION_FP64, api.PRECISION_MIXED):
        p = api.Params(nx, ny, h, h, bc_u=("neumann",) * 4, bc_v=("neumann",) * 4, bc_p=("neumann",) * 4,
                       precision=prec)
        with api.Session(p) as s:
            s.upload("ls", ls)
            s.upload("u", u)
            s.upload("v", v)
            s.apply_bc("ls", "P")
            for _ in range(30):
                s.ls_step(dt, mode)
            outs[prec] = (s.download("ls"), s.volume())
    (l64, v64), (l32, v32) = outs[api.PRECISION_FP64], outs[api.PRECISION_MIXED]
    assert np.isfinite(l32).all()
    d = np.abs(interior(l32) - interior(l64))
    assert d.max() <= (5e-4 if mode == api.REINIT_MINRK2 else 2e-5)
    assert np.quantile(d, 0.99) <= 2e-5
    assert abs(v32[1] - v64[1]) <= 1e-4 * v64[1]


def test_mixed_droplet_steps():
    c = W.droplet(128, seed=7)
    ref = _run_steps(c, api.PRECISION_FP64, 10, api.PCG)
    mix = _run_steps(c, api.PRECISION_MIXED, 10, api.MGPCG)
    assert _rel(mix["ls"], ref["ls"]) <= 2e-5
    assert _rel(mix["p"], ref["p"]) <= 5e-4
    l2 = np.sqrt(((mix["p"] - ref["p"]) ** 2).mean()) / np.sqrt((ref["p"] ** 2).mean())
    assert l2 <= 5e-5
    assert abs(mix["vol"][1] - ref["vol"][1]) <= 5e-8 * ref["vol"][1]


def test_volume_integrals_match_restatement():
    c = W.droplet(96, seed=2)
    g, f = grid_from_case(c), fluid_from_case(c)
    ls = c.ls.copy()
    O.bc(g, "p", ls)
    H, HS = O.heaviside(g, ls), O.smooth_heaviside(g, ls)
    with api.Session(params_for(g, f)) as s:
        s.upload("ls", ls)
        sharp, smooth = s.volume()
    assert abs(sharp - interior(H).sum() * g.dx * g.dy) <= 1e-12 * sharp
    assert abs(smooth - interior(HS).sum() * g.dx * g.dy) <= 1e-12 * smooth
