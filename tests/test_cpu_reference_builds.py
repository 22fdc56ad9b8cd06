"""CPU: the reference's two CPU builds used by the timed baselines.

oracle/_ref/libasd2ref.so is the parity build (serial fixed-order BLAS shim);
oracle/_ref/libasd2ref_blas.so is the same reference sources linked against
OpenBLAS with an OpenMP CSR SpMV, timed beside it as the threaded CPU
baseline.  Its CG must be the same computation: equal to the parity build's
up to the summation order of the BLAS-1 reductions.
"""
import os

import numpy as np
import pytest

from oracle.pyoracle import REF_SO, FluidSpec, GridSpec, Oracle, Reference, have_reference

BLAS_SO = os.path.join(os.path.dirname(REF_SO), "libasd2ref_blas.so")


def _system(n=32, seed=4):
    from asd2_b200 import workloads as W
    c = W.droplet(n, seed=seed)
    g = GridSpec(c.nx, c.ny, c.dx, c.dy, bc_u=c.bc_u, bc_v=c.bc_v, bc_p=("neumann", "neumann", "neumann", "dirichlet"))
    f = FluidSpec(**c.fluid)
    O = Oracle()
    ls = c.ls.copy()
    O.bc(g, "p", ls)
    H = O.heaviside(g, ls)
    kap = O.kappa(g, ls)
    rng = np.random.Generator(np.random.PCG64(seed))
    div = np.ascontiguousarray(rng.standard_normal(g.shape))
    sysd = O.gfm_assemble(g, f, 1.0e-3, ls, kap, H, div, recompute_kappa=True)
    a, ia, ja, b = O.gfm_to_csr(g, sysd)
    rows = len(ia) - 1
    mdiag = np.array([a[ia[r]:ia[r + 1]][ja[ia[r]:ia[r + 1]] == r][0] for r in range(rows)])
    rhs = g.zeros()
    rhs[3:-3, 3:-3] = b.reshape(g.ny, g.nx).T
    return g, f, (a, ia, ja), mdiag, rhs


@pytest.mark.skipif(not (have_reference() and os.path.exists(BLAS_SO)),
                    reason="reference builds (oracle/_ref) not present")
def test_threaded_build_runs_the_same_cg(capfd):
    g, f, csr, mdiag, rhs = _system()
    out = {}
    for name, path in (("serial", REF_SO), ("blas", BLAS_SO)):
        R = Reference(g, f, path=path)
        out[name] = R.cg(rhs, csr, mdiag, 40)[3:-3, 3:-3]
        R.close()
    printed = capfd.readouterr().out
    assert printed.count("CG : 40 40") == 2, printed
    scale = np.abs(out["serial"]).max()
    assert scale > 0
    assert np.abs(out["blas"] - out["serial"]).max() <= 1e-9 * scale


def test_quiet_call_keeps_stdout_clean(capfd):
    """The bench's stdout guard: what a native call prints is returned, not
    written to the process's stdout (which carries the bench's JSON line)."""
    import bench

    def noisy():
        os.write(1, b"CG : 7 7 Err : 0.5\n")
        return 3
    res, text = bench._quiet_call(noisy)
    assert res == 3 and text == "CG : 7 7 Err : 0.5\n"
    assert "CG :" not in capfd.readouterr().out


def test_quiet_call_drains_large_output(capfd):
    """More output than a pipe holds (the reference's GetUHat prints a line
    per grid row) does not block the guard."""
    import bench

    def chatty():
        for _ in range(4096):
            os.write(1, b"x" * 63 + b"\n")
        return 1
    res, text = bench._quiet_call(chatty)
    assert res == 1 and len(text) == 4096 * 64
    assert capfd.readouterr().out == ""


def _raises(payload):
    raise ValueError("planted")


def _dies(payload):
    os._exit(3)


def _sleeps(payload):
    import time
    time.sleep(payload)
    return payload


def test_isolated_worker_never_leaves_the_bench_waiting():
    """The bench's isolated worker returns a result, and turns a raising, a
    dying and an overrunning worker into exceptions (the overrunning one is
    terminated)."""
    import bench
    assert bench._run_isolated(_sleeps, 0, timeout=60) == 0
    with pytest.raises(RuntimeError, match="planted"):
        bench._run_isolated(_raises, None, timeout=60)
    with pytest.raises(RuntimeError, match="died"):
        bench._run_isolated(_dies, None, timeout=60)
    with pytest.raises(TimeoutError):
        bench._run_isolated(_sleeps, 30, timeout=1)
