"""GPU: the MG-FCG solve as one cooperative launch (mg_persist.cu).

Systems up to about 256 x 288 are solved by one kernel launch: one CTA per
16 x 32 tile, grid barriers between the phases, levels from 2 down solved
by every CTA itself.  The method is the multi-kernel MG-FCG's (same
V-cycle, same flexible CG, same FP64 residual replacement); only the
summation order of the dot products differs.  Checks, on square, odd and
rectangular grids with pinned (Neumann) and Dirichlet pressure:

* the one-launch path really ran (asd2g_last_solve_one_launch);
* its pressure equals the multi-kernel solve's (FLAG_NO_PERSIST_MG) to 1e-8
  of max |p| at tol 1e-10, with iteration counts within one;
* it agrees with the oracle's FP64 PCG at 1e-12 to 1e-6 of max |p| (the
  north-star bar) and its true FP64 residual meets the tolerance;
* maxit caps it (NOT_CONVERGED after exactly maxit iterations), and a
  right-hand side of zero returns x = 0 at once;
* grids too large for it fall back to the multi-kernel path.
"""
import numpy as np
import pytest

from asd2_b200 import api
from asd2_b200 import workloads as W
from oracle.pyoracle import GridSpec, Oracle
from tests.helpers import assert_close, fluid_from_case, interior, params_for

pytestmark = pytest.mark.gpu
O = Oracle()


def _case(nx, ny, bc, seed=5):
    c = W.droplet(nx, seed=seed, ny=ny)
    cp = (0.0, 0.5, 0.0, 1.0) if bc == "dirichlet" else (0.0,) * 4
    g = GridSpec(c.nx, c.ny, c.dx, c.dy, bc_p=(bc,) * 4, cp=cp)
    f = fluid_from_case(c)
    ls = c.ls.copy()
    O.bc(g, "p", ls)
    div = W.smooth_field(nx, ny, np.random.default_rng(seed))
    return g, f, ls, div


def _solve(g, f, ls, div, flags, tol=1e-10, maxit=1000, zero_rhs=False):
    with api.Session(params_for(g, f, solver_flags=flags)) as s:
        s.upload("ls", ls)
        s.heaviside()
        if zero_rhs:
            s.fill("div", 0.0)
            s.fill("kappa", 0.0)
            s.assemble_gfm(1e-3, recompute_kappa=False)
        else:
            s.upload("div", div)
            s.assemble_gfm(1e-3, recompute_kappa=True)
        r = s.solve_pressure(api.MGPCG, tol=tol, maxit=maxit, dt=1e-3)
        r["one_launch"] = s.last_solve_one_launch()
        r["true"] = s.true_residual() if not zero_rhs else 0.0
        r["ps"] = interior(s.download("ps"))
        r["sys"] = s.get_system()
    return r


@pytest.mark.parametrize("nx,ny,bc", [(256, 256, "neumann"), (96, 80, "neumann"), (200, 250, "dirichlet"),
                                      (33, 47, "neumann"), (130, 66, "dirichlet"), (48, 40, "neumann"),
                                      (256, 288, "dirichlet")])
def test_one_launch_matches_multi_kernel_and_oracle(nx, ny, bc):
    g, f, ls, div = _case(nx, ny, bc)
    a = _solve(g, f, ls, div, 0)
    b = _solve(g, f, ls, div, api.FLAG_NO_PERSIST_MG)
    assert a["one_launch"] and not b["one_launch"]
    assert a["status"] == 0 and b["status"] == 0, (a["status"], b["status"])
    assert abs(a["iters"] - b["iters"]) <= 1, (a["iters"], b["iters"])
    scale = np.abs(b["ps"]).max()
    assert_close(a["ps"], b["ps"], 0.0, 1e-8 * scale, "one launch vs per-phase kernels")
    assert a["true"] <= 2e-10 and abs(a["true"] - a["resid"]) <= 0.25 * a["true"] + 1e-13, (a["true"], a["resid"])
    x, _, _, _ = O.pcg(g, a["sys"], tol=1e-12, maxit=200000)
    ref = interior(O.scatter(g, x))
    assert_close(a["ps"], ref, 0.0, 1e-6 * np.abs(ref).max(), "one launch vs oracle")


def test_one_launch_maxit_and_zero_rhs():
    g, f, ls, div = _case(96, 80, "neumann")
    r = _solve(g, f, ls, div, 0, tol=1e-14, maxit=3)
    assert r["one_launch"] and r["status"] == 1 and r["iters"] == 3, r["status"]
    z = _solve(g, f, ls, div, 0, zero_rhs=True)
    assert z["one_launch"] and z["status"] == 0 and z["iters"] == 0
    assert np.all(z["ps"] == 0.0)


def test_large_grid_falls_back():
    g, f, ls, div = _case(512, 512, "neumann")
    r = _solve(g, f, ls, div, 0, tol=1e-8)
    assert r["status"] == 0 and not r["one_launch"]


@pytest.mark.parametrize("nx,ny,bc", [(256, 256, "neumann"), (130, 66, "dirichlet"), (33, 47, "neumann")])
def test_one_launch_jacobi_pcg(nx, ny, bc):
    """The FP64 Jacobi-PCG as one cooperative launch (pcg_persist.cu) against
    the per-iteration kernels (FLAG_NO_CLUSTER_PCG) and the oracle: the same
    recurrence, so iteration counts agree to summation-order rounding."""
    g, f, ls, div = _case(nx, ny, bc)

    def run(flags):
        with api.Session(params_for(g, f, solver_flags=flags)) as s:
            s.upload("ls", ls)
            s.heaviside()
            s.upload("div", div)
            s.assemble_gfm(1e-3, recompute_kappa=True)
            r = s.solve_pressure(api.PCG, tol=1e-10, maxit=200000, dt=1e-3)
            return r, s.last_solve_one_launch(), interior(s.download("ps")), s.get_system()
    a, a1, ps_a, sysd = run(0)
    b, b1, ps_b, _ = run(api.FLAG_NO_CLUSTER_PCG)
    assert a1 and not b1
    assert a["status"] == 0 and b["status"] == 0
    assert abs(a["iters"] - b["iters"]) <= max(3, b["iters"] // 50), (a["iters"], b["iters"])
    x, it_ref, _, _ = O.pcg(g, sysd, tol=1e-12, maxit=500000)
    ref = interior(O.scatter(g, x))
    scale = np.abs(ref).max()
    assert_close(ps_a, ref, 0.0, 1e-6 * scale, "one-launch Jacobi-PCG vs oracle")
    assert_close(ps_a, ps_b, 0.0, 1e-6 * scale, "one launch vs per-iteration kernels")
