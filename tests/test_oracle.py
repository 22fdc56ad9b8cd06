"""CPU: the C restatement (oracle/asd2_oracle.c) against the reference.

The golden fixtures were produced by the reference compiled unmodified
(tests/golden/make_golden.py); where the reference build itself is present
(oracle/_ref), the restatement is also compared with it live on fresh seeds.
Everything here is bit-exact: the restatement keeps the reference's operation
order and both are built without FMA contraction.
"""
import math

import numpy as np
import pytest

from oracle.pyoracle import FluidSpec, GridSpec, Oracle, Reference, have_reference
from tests.golden.make_golden import BC_TRIALS
from tests.helpers import GRIDS, assert_bitexact, bc_fixture, golden, ls_grid, mac_grid

O = Oracle()


@pytest.mark.parametrize("name", list(GRIDS))
def test_level_set_golden(name):
    G = golden()
    g = ls_grid(name)
    k = lambda s: G[f"{name}L_{s}"]
    ls, u, v, dt = k("ls"), k("u"), k("v"), float(k("dt"))
    a = ls.copy()
    O.ls_advect(g, a, u, v, dt)
    assert_bitexact(a, k("advect"), "Solve_LevelSet_2D")
    a = ls.copy()
    assert_bitexact(O.ls_weno_rhs(g, a, k("uc"), k("vc")), k("weno_rhs"), "HJWENO5_LS_2D")
    assert_bitexact(a, k("weno_rhs_ls"), "HJWENO5_LS_2D ghost fill of ls")
    for mode in range(5):
        a = k("dist").copy()
        O.reinit(g, mode, a)
        assert_bitexact(a, k(f"reinit{mode}"), f"reinit mode {mode}")
    ls0, ls1 = k("bb_ls0"), k("bb_ls1")
    assert_bitexact(O.subcell_eno_absgrad(g, ls1, ls0), k("subcell"), "SubcellENO_Min_DerivAbsLS_2D")
    assert_bitexact(O.eno_absgrad(g, ls1, ls0), k("eno"), "ENO_DerivAbsLS_2D")
    assert_bitexact(O.heaviside_deriv(g, ls1), k("hd"), "UpdateHeavisideFuncDeriv")
    assert_bitexact(O.sussman_constraint(g, ls1, ls0, k("hd")), k("sussman"), "GetSussmanReinitConstraint")
    assert_bitexact(O.smoothed_sign(g, ls1), k("ssign"), "GetSmoothedSignFunc")


@pytest.mark.parametrize("name", list(GRIDS))
def test_mac_golden(name):
    G = golden()
    g, f = mac_grid(name), FluidSpec()
    k = lambda s: G[f"{name}M_{s}"]
    ls, u, v, dt = k("ls"), k("u"), k("v"), float(k("dt"))
    assert_bitexact(O.kappa(g, ls), k("kappa"), "UpdateKappa")
    assert_bitexact(O.heaviside(g, ls), k("H"), "UpdateHeavisideFunc")
    assert_bitexact(O.smooth_heaviside(g, ls), k("HS"), "UpdateSmoothHeavisideFunc")
    HS, H = k("HS"), k("H")
    assert_bitexact(O.conv_u(g, u, v), k("conv_u"), "AddConvectionFU")
    assert_bitexact(O.conv_v(g, u, v), k("conv_v"), "AddConvectionFV")
    assert_bitexact(O.visc_u(g, f, u, v, ls, HS), k("visc_u"), "AddViscosityFU")
    assert_bitexact(O.visc_v(g, f, u, v, ls, HS), k("visc_v"), "AddViscosityFV")
    assert_bitexact(O.rhs_u(g, f, ls, u, v, HS), k("rhs_u"), "UpdateFU")
    assert_bitexact(O.rhs_v(g, f, ls, u, v, HS), k("rhs_v"), "UpdateFV")
    uh, vh = O.intermediate_vel(g, f, dt, ls, u, v, HS)
    assert_bitexact(uh, k("uhat"), "GetIntermediateVel RK3 u")
    assert_bitexact(vh, k("vhat"), "GetIntermediateVel RK3 v")
    for order in (0, 1):
        a, b = O.intermediate_vel(g, FluidSpec(time_order=order), dt, ls, u, v, HS)
        assert_bitexact(a, k(f"uhat_o{order}"), f"GetIntermediateVel order {order}")
        assert_bitexact(b, k(f"vhat_o{order}"), f"GetIntermediateVel order {order}")
    O.bc(g, "u", uh)
    O.bc(g, "v", vh)
    div = O.divergence(g, uh, vh)
    assert_bitexact(div, k("div"), "GetDivergence")
    kap = k("kappa").copy()
    sysd = O.gfm_assemble(g, f, dt, ls, kap, H, div, recompute_kappa=True)
    assert_bitexact(kap, k("kappa_bc"), "kappa after SolvePoisson's recompute + P fill")
    check_pinned_csr(g, sysd, k("csr_a"), k("csr_ia"), k("csr_ja"), k("csr_b"))
    u2, v2 = u.copy(), v.copy()
    O.update_vel(g, f, dt, u2, v2, uh, vh, k("ps_in"), ls, H, k("kappa_bc"))
    assert_bitexact(u2, k("u_new"), "UpdateVel u")
    assert_bitexact(v2, k("v_new"), "UpdateVel v")
    assert O.update_dt(g, f, u2, v2) == float(k("dt_next"))


def check_pinned_csr(g, sysd, a, ia, ja, b):
    """The reference's all-Neumann CSR (mac2d.cpp:1479-1656) holds, row by row,
    the values S, W, C, E, N of every cell except cell 0, each kept when its
    (shifted) column index is >= 0 -- including zero-valued entries at the W
    and N edges.  Compare the VALUES per row with the restatement's matrix-free
    coefficients (column indices of the reference pin are mis-shifted)."""
    nx, ny = g.nx, g.ny
    assert sysd["pinned"] == 1
    assert len(ia) - 1 == nx * ny - 1
    row = 0
    for j in range(ny):
        for i in range(nx):
            kk = i + nx * j
            if kk == 0:
                continue
            colS = i + (j - 1) * nx - 1 if not (i == 0 and j == 1) else -1
            colW = (i - 1) + j * nx - 1 if not (i == 1 and j == 0) else -1
            colE = (i + 1) + j * nx - 1
            colN = i + (j + 1) * nx - 1
            exp = []
            if colS >= 0:
                exp.append(-sysd["cs"][kk])
            if colW >= 0:
                exp.append(-sysd["cw"][kk])
            exp.append(sysd["diag"][kk])
            if colE >= 0:
                exp.append(-sysd["ce"][kk])
            if colN >= 0:
                exp.append(-sysd["cn"][kk])
            got = a[ia[row]:ia[row + 1]]
            assert len(got) == len(exp), (i, j)
            assert np.array_equal(np.asarray(exp) + 0.0, got + 0.0), (i, j, got, exp)
            row += 1
    assert_bitexact(sysd["rhs"][1:], b, "GFM right-hand side")


def test_dirichlet_reference_solvers_golden():
    """Mode 1 of the oracle's CG/BiCGStab is the reference iteration: on the
    reference-assembled Dirichlet system it reproduces the reference's iterates
    bit for bit (same fixed-order sums as the serial BLAS shim)."""
    G = golden()
    nx, ny, dx, dy = 24, 20, 1.0 / 24, 1.0 / 20
    g = GridSpec(nx, ny, dx, dy, bc_p=("dirichlet",) * 4)
    f = FluidSpec()
    kap = G["D_kappa"].copy()
    sysd = O.gfm_assemble(g, f, float(G["D_dt"]), G["D_ls"], kap, G["D_H"], G["D_div"], recompute_kappa=True)
    a, ia, ja, b = O.gfm_to_csr(g, sysd)
    assert_bitexact(a, G["D_csr_a"], "Dirichlet CSR values")
    assert np.array_equal(ia, G["D_csr_ia"]) and np.array_equal(ja, G["D_csr_ja"])
    assert_bitexact(b, G["D_csr_b"], "Dirichlet rhs")
    for its in (1, 2, 25):
        x, it, _, _ = O.pcg(g, sysd, tol=1e-6, maxit=its, mode=1)
        assert_bitexact(O.scatter(g, x)[3:-3, 3:-3], G[f"D_cg{its}"][3:-3, 3:-3], f"reference CG {its} its")
    for its in (1, 2, 15):
        x, it, _, _ = O.bicgstab(g, sysd, tol=1e-6, maxit=its, mode=1)
        assert_bitexact(O.scatter(g, x)[3:-3, 3:-3], G[f"D_bicg{its}"][3:-3, 3:-3], f"reference BiCGStab {its}")


def laplace_exact(nx, ny):
    """Series solution of Laplace's equation with u = 1 on the top edge and 0
    elsewhere.  The reference's Dirichlet rows move the boundary value into the
    right-hand side with the full 1/dx^2 weight (mac2d.cpp:1521-1528), i.e. the
    value sits at the ghost-cell centre, so the discrete domain spans the ghost
    centres: cell i maps to (i + 1) / (n + 1) of the unit square."""
    x = (np.arange(nx) + 1.0) / (nx + 1)
    y = (np.arange(ny) + 1.0) / (ny + 1)
    X, Y = np.meshgrid(x, y, indexing="ij")
    s = np.zeros_like(X)
    for n in range(1, 400, 2):
        s += 4 / (n * math.pi) * np.sin(n * math.pi * X) * np.exp(n * math.pi * (Y - 1)) * \
            (1 - np.exp(-2 * n * math.pi * Y)) / (1 - np.exp(-2 * n * math.pi))
    return s


def test_laplace_known_answer():
    """The reference's Poisson driver (test_poisson2d_large.cpp:174-323):
    constant coefficients, Dirichlet 0/0/0/1.  The oracle's textbook PCG agrees
    with the reference CG's answer and both approach the series solution."""
    G = golden()
    nx = ny = 32
    g = GridSpec(nx, ny, 1 / 32, 1 / 32, bc_p=("dirichlet",) * 4, cp=(0.0, 0.0, 0.0, 1.0))
    f = FluidSpec(rho_h=1.0, rho_l=1.0, sigma=0.0)
    ls = np.ones(g.shape)
    sysd = O.gfm_assemble(g, f, 1.0, ls, g.zeros(), O.heaviside(g, ls), g.zeros(), recompute_kappa=False)
    a, ia, ja, b = O.gfm_to_csr(g, sysd)
    assert_bitexact(a, G["L_csr_a"], "Laplace CSR")
    x, it, res, tres = O.pcg(g, sysd, tol=1e-12, maxit=10000)
    assert tres < 1e-11
    ref = G["L_ps"][3:-3, 3:-3]
    assert np.abs(O.scatter(g, x)[3:-3, 3:-3] - ref).max() < 1e-5  # the reference stops at 1e-6
    ex = laplace_exact(nx, ny)
    err = np.abs(O.scatter(g, x)[3:-3, 3:-3] - ex)
    # second-order interior error; the top corners carry the data's jump
    assert err[:, : ny // 2].max() < 1e-3 and err.max() < 0.05


@pytest.mark.parametrize("name", list(GRIDS))
def test_ntk_golden(name):
    """UpdateNTK (src/mac2d.cpp:124-219): unit normal where the ENO gradient
    has unit length to 1e-4, other cells left as they were."""
    G = golden()
    g = mac_grid(name)
    for case in ("sdf", "plane"):
        k = lambda s: G[f"{name}M_ntk_{case}_{s}"]
        n0, n1 = O.ntk(g, k("phi"), np.full(g.shape, 7.0), np.full(g.shape, -7.0))
        assert_bitexact(n0, k("nx"), f"UpdateNTK x, {case}")
        assert_bitexact(n1, k("ny"), f"UpdateNTK y, {case}")


@pytest.mark.parametrize("trial", range(BC_TRIALS))
def test_boundary_fills_golden(trial):
    """ApplyBC_{U,V,P}_2D for every kind on every side (periodic, neumann,
    dirichlet, axisym, wall, inlet, outlet; pressure and lsfree on the P
    grid), src/bc2d.cpp:123-934, against the reference's own fills."""
    g, k = bc_fixture(trial)
    for kind in ("U", "V", "P"):
        got = O.bc(g, kind, k(f"{kind}_in").copy())
        assert_bitexact(got, k(f"{kind}_out"), f"{kind} fill {g.bc_u, g.bc_v, g.bc_p}")


@pytest.mark.skipif(not have_reference(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("seed", [1, 2])
def test_against_live_reference(seed):
    """Fresh seeds, run through both the restatement and the reference build."""
    from asd2_b200 import workloads as W
    c = W.perturbed_circle(28, seed=seed)
    g = GridSpec(c.nx, c.ny, c.dx, c.dy, bc_u=c.bc_u, bc_v=c.bc_v, bc_p=c.bc_p)
    R = Reference(g)
    a, b = c.ls.copy(), c.ls.copy()
    for _ in range(3):
        O.ls_advect(g, a, c.u, c.v, c.dt)
        O.reinit(g, 4, a)
        R.ls_advect(b, c.u, c.v, c.dt)
        R.reinit(4, b)
    assert_bitexact(a, b, "3 level-set steps")
    R.close()


def test_masks():
    """Interface-cell and GFM crossing-face masks on a circle."""
    from asd2_b200 import workloads as W
    c = W.droplet(40, seed=3)
    g = GridSpec(c.nx, c.ny, c.dx, c.dy)
    m = O.interface_mask(g, c.ls)
    f = O.ghost_face_mask(g, c.ls)
    assert m.sum() > 0 and (f & 1).sum() > 0 and (f & 2).sum() > 0
    # every crossing face touches an interface cell
    mm = m.reshape(c.ny, c.nx).T
    ff = f.reshape(c.ny, c.nx).T
    for i in range(c.nx):
        for j in range(c.ny):
            if ff[i, j] & 1 and i > 0:
                assert mm[i, j] or mm[i - 1, j]


@pytest.mark.skipif(not have_reference(), reason="reference build (oracle/_ref) not present")
def test_zalesak_against_live_reference():
    """Zalesak's slotted disk (test_levelset2d_large.cpp:1339-1485): the
    initial Reinit_Original_2D and 60 steps of the driver's loop (advect,
    fill, reinitialise, fill) agree bit for bit with the reference."""
    from asd2_b200 import workloads as W
    c = W.zalesak()
    g = GridSpec(c.nx, c.ny, c.dx, c.dy, bc_u=c.bc_u, bc_v=c.bc_v, bc_p=c.bc_p)
    R = Reference(g)
    a, b = c.ls.copy(), c.ls.copy()
    for arr, reinit, bc in ((a, lambda x: O.reinit(g, 0, x), lambda x: O.bc(g, "p", x)),
                            (b, lambda x: R.reinit(0, x), lambda x: R.bc("p", x))):
        reinit(arr)
        bc(arr)
    assert_bitexact(a, b, "initial reinitialisation")
    for _ in range(60):
        O.ls_advect(g, a, c.u, c.v, c.dt)
        O.bc(g, "p", a)
        O.reinit(g, 0, a)
        O.bc(g, "p", a)
        R.ls_advect(b, c.u, c.v, c.dt)
        R.bc("p", b)
        R.reinit(0, b)
        R.bc("p", b)
    assert_bitexact(a, b, "60 steps")
    R.close()


@pytest.mark.skipif(not have_reference(), reason="reference build (oracle/_ref) not present")
def test_reinit_with_kinks_against_live_reference():
    """The reference's kinks driver (test_levelset2d_large.cpp:1042): one
    Reinit_MinRK2_2D over pseudo-time 80 (5120 pseudo-steps) of the union of
    two circles, bit for bit."""
    from tests.helpers import reinit_driver_case
    g, ls, mt = reinit_driver_case("kinks")
    a, b = ls.copy(), ls.copy()
    O.bc(g, "p", a)
    O.reinit(g, 2, a, mt)
    R = Reference(g, ls_max_atime=mt)
    R.bc("p", b)
    R.reinit(2, b)
    assert_bitexact(a, b, "kinks after 5120 pseudo-steps")
    R.close()


@pytest.mark.skipif(not have_reference(), reason="reference build (oracle/_ref) not present")
def test_first_time_reinit_against_live_reference():
    """The reference's first-time reinitialisation driver
    (test_levelset2d_large.cpp:1220): FirstTimeOnlyReinit_Sussman_2D of the
    sign field of the unit circle, bit for bit."""
    from tests.helpers import reinit_driver_case
    g, ls, mt = reinit_driver_case("firsttime")
    a, b = ls.copy(), ls.copy()
    O.bc(g, "p", a)
    O.reinit(g, 3, a, mt)
    R = Reference(g, ls_max_atime=mt)
    R.bc("p", b)
    R.reinit(3, b)
    assert_bitexact(a, b, "first-time reinitialisation")
    R.close()


@pytest.mark.skipif(not have_reference(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("order, mode", [(2, 2), (0, 0), (1, 1), (2, 4)])
def test_droplet_steps_against_live_reference(capfd, order, mode):
    """Whole droplet steps of the reference's MAC driver loop
    (test_mac2d_large.cpp:496-552) run through the reference's own objects
    (LevelSetSolver2D, MACSolver2D with SolvePoisson and its CG) and through
    the oracle's composed step with the reference CG iteration: level set,
    velocities, pressure and dt bit for bit for two steps (time orders Euler,
    RK2, RK3; reinitialisation original, Sussman, MinRK2, MinRK2 with the
    constraint -- both sides call the same libm cos; GFM jumps with surface
    tension; a Dirichlet top so that the reference's own operator is well
    posed, see the all-Neumann pin)."""
    from asd2_b200 import workloads as W
    c = W.droplet(48, seed=5)
    g = GridSpec(c.nx, c.ny, c.dx, c.dy, bc_u=c.bc_u, bc_v=c.bc_v, bc_p=("neumann", "neumann", "neumann", "dirichlet"))
    fl = c.fluid
    f = FluidSpec(rho_h=fl["rho_h"], rho_l=fl["rho_l"], mu_h=fl["mu_h"], mu_l=fl["mu_l"], sigma=fl["sigma"],
                  g=fl["g"], g_axis=fl["g_axis"], fix_gravity=0, time_order=order, cfl=0.5)
    live_droplet_steps(g, f, c.ls, c.u, c.v, mode, steps=2)
    capfd.readouterr()


def live_droplet_steps(g, f, ls0, u0, v0, mode, steps=2, equal=assert_bitexact, len_x=None, len_y=None):
    """`steps` steps of the reference's MAC driver loop through the
    reference's own objects and through the oracle's composed step (reference
    CG iteration to 1e-6); level set, u, v, ps and dt compared with `equal`
    after every step.  len_x / len_y: the domain lengths the reference divides
    by nx / ny for its spacings (default dx * nx, dy * ny)."""
    ls = ls0.copy()
    O.bc(g, "p", ls)
    st = dict(ls=ls.copy(), u=u0.copy(), v=v0.copy(), kappa=g.zeros(), ps=g.zeros(), p=g.zeros())
    st["dt"] = dt = O.update_dt(g, f, st["u"], st["v"])
    R = Reference(g, f, len_x=len_x, len_y=len_y)
    ls_r, u_r, v_r, ps_r = ls.copy(), u0.copy(), v0.copy(), g.zeros()
    for step in range(steps):
        lsB = ls_r.copy()
        R.ls_advect(ls_r, u_r, v_r, dt)
        R.bc("p", ls_r)
        R.reinit(mode, ls_r)
        R.bc("p", ls_r)
        R.set_state(u_r, v_r, ps_r, dt)
        R.kappa(ls_r)
        H, HS = R.heaviside(ls_r)
        uh, vh = R.intermediate_vel(ls_r, u_r, v_r, HS)
        R.bc("u", uh, which=1)
        R.bc("v", vh, which=1)
        ps_r, _ = R.poisson_capture(R.divergence(uh, vh), ls_r, lsB, H, maxiter=100000)
        R.update_vel(uh, vh, ps_r, ls_r, lsB, H)
        got = R.get_state()
        u_r, v_r = got["u"], got["v"]
        dt = R.update_dt(u_r, v_r)
        O.droplet_step(g, f, st, tol=1e-6, maxit=100000, pcg_mode=1, reinit_mode=mode)
        for name, a, b in (("ls", ls_r, st["ls"]), ("u", u_r, st["u"]), ("v", v_r, st["v"]), ("ps", ps_r, st["ps"])):
            equal(b, a, f"step {step} {name}")
        assert dt == st["dt"] or (dt != dt and st["dt"] != st["dt"]), step
    R.close()
