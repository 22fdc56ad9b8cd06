"""GPU: the allocation-free pressure solve (asd2g_pcg_solve_static).

Some callers cannot call cudaMalloc -- a host that owns all device memory
through its own pool allocator, a latency-critical loop where an allocation
would synchronise the device, or a process that has reserved the whole GPU.
asd2g_pcg_solve_static serves them with a fixed device-side work space.  This
test calls it through the C ABI on two systems in a row (the second call
reuses the work space the first left behind) and checks each solution
against the session-based entry point (asd2g_solve_pressure) at the
tolerance the other pressure tests use.  The test itself allocates the
system's input and output buffers with torch; the entry point allocates
nothing.

It lives in its own file so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from asd2_b200 import api
from asd2_b200 import workloads as W
from oracle.pyoracle import GridSpec, Oracle
from tests.helpers import assert_close, fluid_from_case, interior, params_for

pytestmark = pytest.mark.gpu
O = Oracle()


def _system(seed, nx, ny):
    c = W.droplet(nx, seed=seed, ny=ny)
    g = GridSpec(c.nx, c.ny, c.dx, c.dy)
    f = fluid_from_case(c)
    ls = c.ls.copy()
    O.bc(g, "p", ls)
    X = (np.arange(g.nx + 6) - 2.5) * g.dx
    Y = (np.arange(g.ny + 6) - 2.5) * g.dy
    div = np.outer(np.sin(3 * X + seed), np.cos(2 * Y)) * 10.0
    return g, f, ls, O.heaviside(g, ls), div


def _to_compact(nat, nx, ny):
    # natural order k = i + nx*j  ->  compact k = j + ny*i
    return np.ascontiguousarray(nat.reshape(ny, nx).T.reshape(-1))


def test_static_solve_matches_session_solve_twice():
    import torch
    L = api.load()
    dt = 1e-3
    for call, (seed, nx, ny) in enumerate([(3, 96, 80), (8, 64, 72)]):
        g, f, ls, H, div = _system(seed, nx, ny)
        with api.Session(params_for(g, f)) as s:
            s.upload("ls", ls)
            s.upload("H", H)
            s.upload("div", div)
            s.assemble_gfm(dt, recompute_kappa=True)
            ref = s.solve_pressure(api.PCG, tol=1e-12, maxit=100000, dt=dt)
            assert ref["status"] == 0
            ps_ref = interior(s.download("ps"))
            sysd = s.get_system()
        dev = torch.device("cuda:0")
        t = {k: torch.from_numpy(_to_compact(sysd[k], g.nx, g.ny)).to(dev) for k in ("diag", "ce", "cn", "rhs")}
        x = torch.full((g.nx * g.ny,), float("nan"), dtype=torch.float64, device=dev)
        it, res = ctypes.c_int(), ctypes.c_double()
        stream = torch.cuda.current_stream().cuda_stream
        rc = L.asd2g_pcg_solve_static(g.nx, g.ny, sysd["pinned"], t["diag"].data_ptr(), t["ce"].data_ptr(),
                                      t["cn"].data_ptr(), t["rhs"].data_ptr(), x.data_ptr(), 1e-12, 100000,
                                      stream, ctypes.byref(it), ctypes.byref(res))
        assert rc == 0, (call, rc, L.asd2g_last_error())
        assert res.value <= 1e-12
        got = x.cpu().numpy().reshape(g.nx, g.ny)  # compact layout is (i, j) row-major
        scale = np.abs(ps_ref).max()
        assert_close(got, ps_ref, 0.0, 1e-9 * scale, f"static solve, call {call + 1}")
        assert abs(it.value - ref["iters"]) <= 2


def test_static_solve_large_maxit():
    """maxit = INT_MAX is a valid cap: the solve stops on convergence, not
    after one chunk of iterations."""
    import torch
    L = api.load()
    g, f, ls, H, div = _system(5, 48, 40)
    with api.Session(params_for(g, f)) as s:
        s.upload("ls", ls)
        s.upload("H", H)
        s.upload("div", div)
        s.assemble_gfm(1e-3, recompute_kappa=True)
        sysd = s.get_system()
    dev = torch.device("cuda:0")
    t = {k: torch.from_numpy(_to_compact(sysd[k], g.nx, g.ny)).to(dev) for k in ("diag", "ce", "cn", "rhs")}
    x = torch.zeros(g.nx * g.ny, dtype=torch.float64, device=dev)
    it, res = ctypes.c_int(), ctypes.c_double()
    rc = L.asd2g_pcg_solve_static(g.nx, g.ny, sysd["pinned"], t["diag"].data_ptr(), t["ce"].data_ptr(),
                                  t["cn"].data_ptr(), t["rhs"].data_ptr(), x.data_ptr(), 1e-10, 2 ** 31 - 1,
                                  torch.cuda.current_stream().cuda_stream, ctypes.byref(it), ctypes.byref(res))
    assert rc == 0, (rc, L.asd2g_last_error())
    assert 64 < it.value < 100000 and res.value <= 1e-10


# Run in a child process: a device reset ends every allocation of the process
# that makes it.  The child allocates its buffers with cudaMalloc through the
# CUDA runtime the library itself uses (same soname, so the same instance).
_RESET_CHILD = r"""
import ctypes, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from asd2_b200 import api
from tests.test_zz_no_alloc import _system, _to_compact
from oracle.pyoracle import Oracle
L = api.load()
rt = ctypes.CDLL("libcudart.so.12")
O = Oracle()
g, f, ls, H, div = _system(4, 40, 32)
sysd = O.gfm_assemble(g, f, 1e-3, ls, O.kappa(g, ls), H, div, recompute_kappa=True)
xref = O.pcg(g, sysd, tol=1e-12, maxit=100000)[0]
n = g.nx * g.ny

def solve():
    ptrs = []
    for k in ("diag", "ce", "cn", "rhs"):
        a = np.ascontiguousarray(_to_compact(sysd[k], g.nx, g.ny))
        p = ctypes.c_void_p()
        assert rt.cudaMalloc(ctypes.byref(p), ctypes.c_size_t(8 * n)) == 0
        assert rt.cudaMemcpy(p, a.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(8 * n), 1) == 0
        ptrs.append(p)
    x = ctypes.c_void_p()
    assert rt.cudaMalloc(ctypes.byref(x), ctypes.c_size_t(8 * n)) == 0
    it, res = ctypes.c_int(), ctypes.c_double()
    rc = L.asd2g_pcg_solve_static(g.nx, g.ny, sysd["pinned"], ptrs[0].value, ptrs[1].value, ptrs[2].value,
                                  ptrs[3].value, x.value, 1e-12, 100000, None, ctypes.byref(it), ctypes.byref(res))
    assert rc == 0, (rc, L.asd2g_last_error())
    out = np.zeros(n)
    assert rt.cudaMemcpy(out.ctypes.data_as(ctypes.c_void_p), x, ctypes.c_size_t(8 * n), 2) == 0
    got = out.reshape(g.nx, g.ny).T.reshape(-1)  # compact (i, j) -> natural k = i + nx*j
    assert np.abs(got - xref).max() <= 1e-9 * np.abs(xref).max(), np.abs(got - xref).max()
    for p in ptrs + [x]:
        rt.cudaFree(p)

solve()
assert rt.cudaDeviceReset() == 0
solve()
print("reset ok")
"""


def test_static_solve_after_device_reset():
    """A cudaDeviceReset between two calls: the second call finds the work
    space's address in the new context (it is looked up again on every call
    whose stream is not capturing) and solves the system correctly."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    p = subprocess.run([sys.executable, "-c", _RESET_CHILD, root], capture_output=True, text=True, timeout=300,
                       cwd=root)
    assert p.returncode == 0 and "reset ok" in p.stdout, p.stdout[-2000:] + p.stderr[-2000:]


def test_static_solve_rejects_oversize():
    L = api.load()
    it, res = ctypes.c_int(), ctypes.c_double()
    rc = L.asd2g_pcg_solve_static(1024, 1024, 1, 1, 1, 1, 1, 1, 1e-8, 10, None, ctypes.byref(it), ctypes.byref(res))
    assert rc == -1
    assert b"262144" in L.asd2g_last_error()
