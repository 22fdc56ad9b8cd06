"""Staged copies (asd2g_upload_staged / _download_staged / _join_copies /
_sync_copies): transfers on the session's copy stream, ordered against its
compute work by events.  A loop that uploads step k+1's inputs beside step
k's solve and downloads step k's pressure beside step k+1's assembly gives
the same pressures, bit for bit, as the same solves with plain synchronous
copies; a staged round trip of a field returns it unchanged."""
import numpy as np
import pytest
import torch

from asd2_b200 import api
from asd2_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _systems(n=64, count=3):
    out = []
    for k in range(count):
        c = W.droplet(n, seed=40 + k, rho_ratio=[1000.0, 10.0, 300.0][k])
        with api.Session(api.Params.from_case(c)) as s:
            s.upload("ls", c.ls)
            s.apply_bc("ls", "P")
            s.heaviside()
            s.kappa()
            X = (np.arange(n + 6) - 2.5) / n
            s.upload("div", np.outer(np.sin(3 * X + k), np.cos(2 * X)) * 10.0)
            out.append((c, {f: s.download(f) for f in ("ls", "H", "div")}))
    return out


def _pinned(a):
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t, t.numpy()


def test_staged_round_trip():
    c = W.droplet(48, seed=2)
    with api.Session(api.Params.from_case(c)) as s:
        keep, src = _pinned(c.ls)
        keep2, dst = _pinned(np.zeros_like(c.ls))
        s.upload_staged("ls", src)
        s.join_copies(1)
        s.download_staged("ls", dst)
        s.sync_copies()
        assert np.array_equal(dst, c.ls)


def test_overlapped_solves_match_sequential():
    systems = _systems()
    c0 = systems[0][0]
    dt = 1e-3
    ref = []
    with api.Session(api.Params.from_case(c0)) as s:
        for _, d in systems:
            for f in ("ls", "H", "div"):
                s.upload(f, d[f])
            s.assemble_gfm(dt, recompute_kappa=True)
            r = s.solve_pressure(api.MGPCG, tol=1e-10, maxit=10000, dt=dt)
            assert r["status"] == 0
            ref.append(s.download("ps"))
    pins = [{f: _pinned(d[f]) for f in ("ls", "H", "div")} for _, d in systems]
    outs = [_pinned(np.zeros_like(ref[0])) for _ in systems]
    with api.Session(api.Params.from_case(c0)) as s:
        for f in ("ls", "H", "div"):
            s.upload_staged(f, pins[0][f][1])
        for k in range(len(systems)):
            s.join_copies(1)
            s.assemble_gfm(dt, recompute_kappa=True)
            if k + 1 < len(systems):
                for f in ("ls", "H", "div"):
                    s.upload_staged(f, pins[k + 1][f][1])
            if k > 0:
                s.join_copies(2)
            r = s.solve_pressure(api.MGPCG, tol=1e-10, maxit=10000, dt=dt)
            assert r["status"] == 0
            s.download_staged("ps", outs[k][1])
        s.sync_copies()
    for k in range(len(systems)):
        assert np.array_equal(outs[k][1], ref[k]), k
