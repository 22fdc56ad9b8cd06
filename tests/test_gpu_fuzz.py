"""B200: whole droplet steps of asd2g_droplet_step and axisymmetric steps of
asd2g_axi_step against the oracle on drawn configurations (grid sizes, U / V
/ P boundary kinds and constants, axis offsets, fluids, time orders,
reinitialisation modes), with the same strategies the
CPU pins of the oracle against the reference use (tests/test_oracle_fuzz.py).

A randomised sweep kept out of the default GPU suite: it runs with
ASD2G_GPU_FUZZ=1 (ASD2G_GPU_FUZZ_EXAMPLES sets the number of cases).
"""
import os

import numpy as np
import pytest

pytest.importorskip("hypothesis")
from hypothesis import HealthCheck, given, settings  # noqa: E402
from hypothesis import strategies as st  # noqa: E402

from asd2_b200 import api  # noqa: E402
from oracle.pyoracle import GridSpec, Oracle  # noqa: E402
from tests.helpers import assert_bitexact, assert_close, interior, params_for  # noqa: E402
from tests.test_oracle_fuzz import axi_p_sides, consts, drop_fields, fluids, p_sides, sides_uv  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("ASD2G_GPU_FUZZ") != "1", reason="opt-in: ASD2G_GPU_FUZZ=1")]

O = Oracle()
EXAMPLES = int(os.environ.get("ASD2G_GPU_FUZZ_EXAMPLES", "40"))


@settings(max_examples=EXAMPLES, deadline=None, derandomize=True, print_blob=True,
          suppress_health_check=[HealthCheck.too_slow, HealthCheck.data_too_large])
@given(nx=st.integers(8, 32), ny=st.integers(8, 32), bu=sides_uv, bv=sides_uv, bp=p_sides(), cu=consts, cv=consts,
       cp=consts, f=fluids(), mode=st.sampled_from((api.REINIT_ORIGINAL, api.REINIT_SUSSMAN, api.REINIT_MINRK2,
                                                   api.REINIT_MINRK2_SUSSMAN)),
       seed=st.integers(0, 2 ** 31 - 1))
def test_droplet_steps_gpu_fuzz(nx, ny, bu, bv, bp, cu, cv, cp, f, mode, seed):
    """Two steps, pressure to 1e-12: level set bit-identical after the first
    step (within 1e-10 of its max after the second, and with the Sussman
    constraint, whose cos may differ from libm's in the last bit), u, v and
    ps within 1e-8 of their maxima, dt within 1e-9."""
    lx, ly = 1.0, 1.0
    dx, dy = lx / nx, ly / ny
    g = GridSpec(nx, ny, dx, dy, bc_u=bu, bc_v=bv, bc_p=bp, cu=cu, cv=cv, cp=cp)
    ls, u, v = drop_fields(nx, ny, dx, dy, seed)
    O.bc(g, "p", ls)
    st_ = dict(ls=ls.copy(), u=u.copy(), v=v.copy(), kappa=g.zeros(), ps=g.zeros(), p=g.zeros())
    st_["dt"] = dt = O.update_dt(g, f, st_["u"], st_["v"])
    with api.Session(params_for(g, f)) as s:
        for fld in ("ls", "u", "v"):
            s.upload(fld, st_[fld])
        for k in range(2):
            r = s.droplet_step(dt, reinit_mode=mode, tol=1e-12, maxit=200000)
            assert r["status"] == 0, r
            O.droplet_step(g, f, st_, tol=1e-12, reinit_mode=mode)
            gl = s.download("ls")
            if k == 0 and mode not in (api.REINIT_SUSSMAN, api.REINIT_MINRK2_SUSSMAN):  # cos in the constraint
                assert_bitexact(gl, st_["ls"], f"level set after step 0 {bu, bv, bp}")
            else:
                assert_close(gl, st_["ls"], 0.0, 1e-10 * np.abs(st_["ls"]).max(), f"level set step {k}")
            for fld in ("u", "v"):
                ref = st_[fld]
                assert_close(s.download(fld), ref, 0.0, 1e-8 * max(np.abs(ref).max(), 1e-30), f"{fld} step {k}")
            ps_ref = st_["ps"]
            assert_close(interior(s.download("ps")), interior(ps_ref), 0.0,
                         1e-8 * max(np.abs(ps_ref).max(), 1e-30), f"ps step {k}")
            assert abs(r["dt_next"] - st_["dt"]) <= 1e-9 * st_["dt"], (k, r["dt_next"], st_["dt"])
            dt = st_["dt"]


@settings(max_examples=EXAMPLES, deadline=None, derandomize=True, print_blob=True,
          suppress_health_check=[HealthCheck.too_slow, HealthCheck.data_too_large])
@given(nr=st.integers(8, 32), nz=st.integers(8, 40), base=st.sampled_from((0.0, 0.05)), bu=sides_uv, bv=sides_uv,
       bp=axi_p_sides(), cu=consts, cv=consts, cp=consts, f=fluids(axisym=True), seed=st.integers(0, 2 ** 31 - 1))
def test_axisym_steps_gpu_fuzz(nr, nz, base, bu, bv, bp, cu, cv, cp, f, seed):
    """Two axisymmetric driver steps (asd2g_axi_step, level set on the
    reference driver's own kinds: axisym, lsfree x 3) against the oracle's,
    pressure to 1e-12: level set within 1e-10 of max(|phi|, 1), u, v and ps
    within 1e-7 of their maxima, dt within 1e-10."""
    lr, lz = 0.5, 1.0
    dr, dz = lr / nr, lz / nz
    g = GridSpec(nr, nz, dr, dz, bc_u=bu, bc_v=bv, bc_p=bp, cu=cu, cv=cv, cp=cp)
    lg = GridSpec(nr, nz, dr, dz, bc_u=bu, bc_v=bv, bc_p=("axisym", "lsfree", "lsfree", "lsfree"))
    ls, u, v = drop_fields(nr, nz, dr, dz, seed, base_x=base)
    O.bc(lg, "p", ls)
    O.bc(g, "u", u)
    O.bc(g, "v", v)
    st_ = dict(ls=ls, u=u, v=v, kappa=g.zeros())
    st_["dt"] = dt = O.axi_update_dt(g, f, u, v, st_["kappa"])
    with api.Session(params_for(g, f, base_x=base)) as s:
        for fld in ("ls", "u", "v", "kappa"):
            s.upload(fld, st_[fld])
        for k in range(2):
            r = s.axi_step(dt, ls_bc=lg.bc_p, solver=api.PCG, tol=1e-12, maxit=200000)
            assert r["status"] == 0, r
            O.axi_step(g, f, st_, base_r=base, ls_grid=lg, tol=1e-12)
            assert abs(r["dt_next"] - st_["dt"]) <= 1e-10 * st_["dt"], (k, r["dt_next"], st_["dt"])
            dt = st_["dt"]
            for fld in ("ls", "u", "v", "ps"):
                ref = st_[fld]
                err = np.abs(s.download(fld) - ref)[3:-3, 3:-3].max()
                scale = max(np.abs(ref[3:-3, 3:-3]).max(), 1e-30)
                bar = 1e-10 * max(scale, 1.0) if fld == "ls" else 1e-7 * scale
                assert err <= bar, (k, fld, err, scale, bu, bv, bp)
