"""Device-resident multi-step run (asd2g_run_steps): the droplet step as one
CUDA graph per step, the MG-FCG iterations in a device-side WHILE node, dt
handed from step to step on the device, one host synchronisation per run.

The step graph runs the same kernels in the same order as asd2g_droplet_step
with the MG-FCG solver, so the fields after n steps are bit-identical to n
host-driven steps; a failing solve stops the run at that step.
"""
import numpy as np
import pytest

from asd2_b200 import api
from asd2_b200 import workloads as W
from tests.helpers import fluid_from_case, grid_from_case, params_for

pytestmark = pytest.mark.gpu

FIELDS = ("ls", "u", "v", "ps", "p")


def _session(c, precision=api.PRECISION_FP64):
    g, f = grid_from_case(c), fluid_from_case(c)
    s = api.Session(params_for(g, f, precision=precision))
    s.upload("ls", c.ls)
    s.upload("u", c.u)
    s.upload("v", c.v)
    s.apply_bc("ls", "P")
    return s


def _host_steps(s, dt, n, tol, maxit):
    iters, st = 0, 0
    for _ in range(n):
        r = s.droplet_step(dt, solver=api.MGPCG, tol=tol, maxit=maxit)
        iters += r["iters"]
        st = r["status"]
        dt = r["dt_next"]
        if st != 0:
            break
    return dt, iters, st


@pytest.mark.parametrize("precision", [api.PRECISION_FP64, api.PRECISION_MIXED])
def test_run_steps_bit_identical_to_host_steps(precision):
    c = W.droplet(128, seed=4)
    a, b = _session(c, precision), _session(c, precision)
    dt0 = a.update_dt()
    assert b.update_dt() == dt0
    dt_a, iters_a, _ = _host_steps(a, dt0, 3, 1e-10, 10000)
    r = b.run_steps(3, dt0, tol=1e-10, maxit=10000)
    assert r["status"] == 0 and r["steps"] == 3, r
    assert r["dt_next"] == dt_a
    assert r["iters"] == iters_a
    # a second run continues from the device state with the cached graph
    dt_a, iters_a, _ = _host_steps(a, dt_a, 2, 1e-10, 10000)
    r = b.run_steps(2, r["dt_next"], tol=1e-10, maxit=10000)
    assert r["status"] == 0 and r["steps"] == 2 and r["dt_next"] == dt_a and r["iters"] == iters_a
    for f in FIELDS:
        assert np.array_equal(a.download(f), b.download(f)), f
    assert a.last_volume() == b.last_volume()
    a.close()
    b.close()


def test_run_steps_stops_at_failed_solve():
    c = W.droplet(96, seed=8)
    a, b = _session(c), _session(c)
    dt0 = a.update_dt()
    _, _, st = _host_steps(a, dt0, 1, 1e-12, 2)  # two iterations cannot reach 1e-12
    assert st == api.NOT_CONVERGED
    r = b.run_steps(4, dt0, tol=1e-12, maxit=2)
    assert r["status"] == api.NOT_CONVERGED and r["steps"] == 1, r
    for f in FIELDS:  # the later steps were skipped on the device
        assert np.array_equal(a.download(f), b.download(f)), f
    a.close()
    b.close()


def test_run_steps_zero_and_refusals():
    c = W.droplet(64, seed=1)
    s = _session(c)
    dt = s.update_dt()
    r = s.run_steps(0, dt)
    assert r["status"] == 0 and r["steps"] == 0 and r["dt_next"] == dt
    with pytest.raises(api.Asd2gError):
        s.run_steps(1, dt, solver=api.PCG)
    s.close()


def test_checkpoint_restart_continues_bit_identically(tmp_path):
    from asd2_b200 import checkpoint as CK
    c = W.droplet(96, seed=6)
    a = _session(c)
    dt = a.update_dt()
    r = a.run_steps(2, dt, tol=1e-10, maxit=10000)
    path = tmp_path / "run.ck"
    a.checkpoint_save(path, t=0.5, step=2, dt=r["dt_next"])
    fields, meta = CK.read(path)  # the numpy reader sees the same fields
    assert meta["step"] == 2 and np.array_equal(fields["ls"], a.download("ls"))
    b = _session(c)
    b.upload("ls", 0.5 * c.ls)  # another state, replaced by the checkpoint
    info = b.checkpoint_load(path)
    assert info == dict(t=0.5, step=2, dt=r["dt_next"])
    ra = a.run_steps(2, r["dt_next"], tol=1e-10, maxit=10000)
    rb = b.run_steps(2, info["dt"], tol=1e-10, maxit=10000)
    assert ra == rb
    for f in FIELDS:
        assert np.array_equal(a.download(f), b.download(f)), f
    a.close()
    b.close()
