"""Batched full droplet step (asd2g_batch_step): every phase of the step is
one launch over the whole batch of uneven droplets.  Each instance must give
what a single session's asd2g_droplet_step (MG-FCG solve) gives on the same
inputs:

  * after the first step the level set, curvature and Heaviside fields are
    bit-identical (the advection velocity is the initial one, and the batched
    stencil kernels run the single-grid tile functions);
  * velocity and pressure agree to 1e-7 of their maxima and the next dt to
    1e-7 relative (both pressure solves stop at 1e-10; their dot products sum
    in different block orders);
  * after a second step the level set still agrees to 1e-9 of its maximum;
  * the FP64 volume check matches the session's to 1e-12.
"""
import numpy as np
import pytest

from asd2_b200 import api
from asd2_b200 import workloads as W
from tests.helpers import fluid_from_case, grid_from_case, interior, params_for

pytestmark = pytest.mark.gpu

SIDES = [(48, 48), (64, 96), (96, 64), (128, 128), (70, 130), (160, 96)]


def _case(k, nx, ny):
    c = W.droplet(nx, seed=200 + k, ny=ny, rho_ratio=[1000, 10, 300, 1, 100, 30][k], mu_ratio=[100, 1, 10, 3, 30, 1][k])
    return c, grid_from_case(c), fluid_from_case(c)


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("reinit", [api.REINIT_MINRK2, api.REINIT_ORIGINAL, api.REINIT_SUSSMAN,
                                    api.REINIT_MINRK2_SUSSMAN])
def test_batch_step_matches_sessions(reinit):
    cases = [_case(k, nx, ny) for k, (nx, ny) in enumerate(SIDES)]
    sessions, init, dts = [], [], []
    for c, g, f in cases:
        # the batch runs the per-phase MG-FCG kernels; the sessions run the
        # same ones (not the one-launch solve) so only summation order differs
        s = api.Session(params_for(g, f, solver_flags=api.FLAG_NO_PERSIST_MG))
        s.upload("ls", c.ls)
        s.upload("u", c.u)
        s.upload("v", c.v)
        s.apply_bc("ls", "P")
        init.append({k: s.download(k) for k in ("ls", "u", "v")})
        dts.append(s.update_dt())
        sessions.append(s)
    b = api.Batch([params_for(g, f) for _, g, f in cases])
    for i, st in enumerate(init):
        for k, a in st.items():
            b.upload(i, k, a)
    ref1 = []
    for s, dt in zip(sessions, dts):
        r = s.droplet_step(dt, reinit_mode=reinit, solver=api.MGPCG, tol=1e-10, maxit=10000)
        assert r["status"] == 0
        ref1.append(dict(r=r, vol=s.last_volume(), **{k: s.download(k) for k in ("ls", "kappa", "H", "u", "v", "ps")}))
    out = b.step(dts, reinit_mode=reinit, tol=1e-10, maxit=10000)
    assert out["status"] == 0, out
    sharp, smooth = b.volume()
    for i, ref in enumerate(ref1):
        for k in ("ls", "kappa", "H"):
            assert np.array_equal(b.download(i, k), ref[k]), (i, k)
        for k in ("u", "v", "ps"):
            assert _rel(interior(b.download(i, k)), interior(ref[k])) <= 1e-7, (i, k)
        assert abs(out["dt_next"][i] - ref["r"]["dt_next"]) <= 1e-7 * ref["r"]["dt_next"], i
        assert abs(sharp[i] - ref["vol"][0]) <= 1e-12 * ref["vol"][0]
        assert abs(smooth[i] - ref["vol"][1]) <= 1e-12 * ref["vol"][1]
    # a second step from each side's own state
    dts2 = []
    for s, ref in zip(sessions, ref1):
        r = s.droplet_step(ref["r"]["dt_next"], reinit_mode=reinit, solver=api.MGPCG, tol=1e-10, maxit=10000)
        assert r["status"] == 0
        dts2.append(ref["r"]["dt_next"])
    out2 = b.step(out["dt_next"], reinit_mode=reinit, tol=1e-10, maxit=10000)
    assert out2["status"] == 0
    for i, s in enumerate(sessions):
        assert _rel(interior(b.download(i, "ls")), interior(s.download("ls"))) <= 1e-9, i
        assert _rel(interior(b.download(i, "ps")), interior(s.download("ps"))) <= 1e-7, i
        s.close()
    b.close()


def test_batch_step_mixed_orders_and_reinit_counts():
    """Instances with time orders 0, 1, 2, 2 and reinitialisation pseudo-time
    limits of 2.25 (the default), 1 and 4 cells (5, about 2 and about 8
    pseudo-steps) in one batch: each still gives its session's step (level
    set bit-identical, velocity and pressure to 1e-7)."""
    import dataclasses
    spec = [(0, 0.0), (1, 1.0), (2, 4.0), (2, 0.0)]  # (time order, ls_max_atime in cells; 0: default)
    cases, params, init, dts, sessions = [], [], [], [], []
    for k, (order, mt) in enumerate(spec):
        c, g, f = _case(k, *SIDES[k])
        f = dataclasses.replace(f, time_order=order)
        p = params_for(g, f, ls_max_atime=mt * min(g.dx, g.dy))
        s = api.Session(params_for(g, f, ls_max_atime=mt * min(g.dx, g.dy), solver_flags=api.FLAG_NO_PERSIST_MG))
        s.upload("ls", c.ls)
        s.upload("u", c.u)
        s.upload("v", c.v)
        s.apply_bc("ls", "P")
        init.append({k2: s.download(k2) for k2 in ("ls", "u", "v")})
        dts.append(s.update_dt())
        sessions.append(s)
        params.append(p)
    with api.Batch(params) as b:
        for i, st in enumerate(init):
            for k2, a in st.items():
                b.upload(i, k2, a)
        out = b.step(dts, reinit_mode=api.REINIT_MINRK2, tol=1e-10, maxit=10000)
        assert out["status"] == 0, out
        for i, s in enumerate(sessions):
            r = s.droplet_step(dts[i], reinit_mode=api.REINIT_MINRK2, solver=api.MGPCG, tol=1e-10, maxit=10000)
            assert r["status"] == 0
            assert np.array_equal(b.download(i, "ls"), s.download("ls")), i
            for k2 in ("u", "v", "ps"):
                assert _rel(interior(b.download(i, k2)), interior(s.download(k2))) <= 1e-7, (i, k2)
            assert abs(out["dt_next"][i] - r["dt_next"]) <= 1e-7 * r["dt_next"], i
            s.close()


def test_batch_step_mixed_precision_instances():
    """Mixed-precision instances (FP32 level-set advection and
    reinitialisation) beside FP64 ones in one batch: each gives its
    session's step in the same precision, the level set bit-identical (the
    batched FP32 kernels run the sessions' strip functions), pressure to
    1e-7, velocity to 5e-6; after a second step the level set agrees to 1e-9 (FP64)
    and 1e-6 (mixed: FP32 rounding of the slightly different velocities)."""
    precs = [api.PRECISION_MIXED, api.PRECISION_FP64, api.PRECISION_MIXED, api.PRECISION_MIXED, api.PRECISION_FP64,
             api.PRECISION_MIXED]
    cases, params, init, dts, sessions = [], [], [], [], []
    for k, (nx, ny) in enumerate(SIDES):
        c, g, f = _case(k, nx, ny)
        params.append(params_for(g, f, precision=precs[k]))
        s = api.Session(params_for(g, f, precision=precs[k], solver_flags=api.FLAG_NO_PERSIST_MG))
        s.upload("ls", c.ls)
        s.upload("u", c.u)
        s.upload("v", c.v)
        s.apply_bc("ls", "P")
        init.append({k2: s.download(k2) for k2 in ("ls", "u", "v")})
        dts.append(s.update_dt())
        sessions.append(s)
    with api.Batch(params) as b:
        for i, st in enumerate(init):
            for k2, a in st.items():
                b.upload(i, k2, a)
        out = b.step(dts, reinit_mode=api.REINIT_MINRK2, tol=1e-10, maxit=10000)
        assert out["status"] == 0, out
        nxt = []
        for i, s in enumerate(sessions):
            r = s.droplet_step(dts[i], reinit_mode=api.REINIT_MINRK2, solver=api.MGPCG, tol=1e-10, maxit=10000)
            assert r["status"] == 0
            assert np.array_equal(b.download(i, "ls"), s.download("ls")), i
            # pressure to 1e-7; the velocities of a droplet one step from rest
            # are the small remainder of pressure gradient against surface
            # tension, so the solves' 1e-10 reaches them amplified (measured
            # up to 5.6e-7)
            for k2, bar in (("ps", 1e-7), ("u", 5e-6), ("v", 5e-6)):
                assert _rel(interior(b.download(i, k2)), interior(s.download(k2))) <= bar, (i, k2)
            nxt.append(r["dt_next"])
        out2 = b.step(out["dt_next"], reinit_mode=api.REINIT_MINRK2, tol=1e-10, maxit=10000)
        assert out2["status"] == 0
        for i, s in enumerate(sessions):
            r = s.droplet_step(nxt[i], reinit_mode=api.REINIT_MINRK2, solver=api.MGPCG, tol=1e-10, maxit=10000)
            assert r["status"] == 0
            # the velocities entering step 2 differ by the solves' 1e-10; in
            # FP32 that moves phi by a few ulps (6e-8 relative)
            bar = 1e-6 if precs[i] == api.PRECISION_MIXED else 1e-9
            assert _rel(interior(b.download(i, "ls")), interior(s.download("ls"))) <= bar, i
            s.close()


def test_batch_step_refusals():
    c, g, f = _case(0, 48, 48)
    with api.Batch([params_for(g, f)]) as b:
        with pytest.raises(api.Asd2gError):
            b.step([1e-3], reinit_mode=api.REINIT_FIRSTTIME)
        with pytest.raises(api.Asd2gError):
            b.step([-1.0])
