"""CPU: the axisymmetric part of the C restatement (oracle/asd2_oracle.c,
ora_axi_*) against MACSolver2DAxisym (src/mac2dAxisym.cpp).

The golden fixture tests/golden/axisym_golden.npz was produced by the
reference compiled unmodified (tests/golden/make_golden_axisym.py); where the
reference build is present (oracle/_ref) the restatement is also compared with
it live on fresh seeds.  Everything is bit-exact, the curvature included (both
sides call the same libm pow here).
"""
import os

import numpy as np
import pytest

from oracle.pyoracle import AxiReference, Oracle, have_reference
from tests.golden.make_golden_axisym import CASES, case_inputs, smooth_heaviside
from tests.helpers import assert_bitexact
from tests.test_oracle import check_pinned_csr

O = Oracle()
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "axisym_golden.npz"))


def oracle_outputs(g, f, base, ls, u, v, ps, dt):
    """The fixture's pipeline through the restatement."""
    out = {}
    HS = smooth_heaviside(ls, 1.5 * min(g.dx, g.dy))
    H = np.ascontiguousarray((ls >= 0.0).astype(np.float64))
    out["kappa"] = O.axi_kappa(g, base, ls)
    out["dU"], out["dV"] = O.axi_visc(g, f, u, 0.9 * u + 0.01, v, ls, HS)
    out["rhs_u"] = O.axi_rhs_u(g, f, dt, ls, u, v, HS)
    uh = O.axi_uhat(g, f, dt, ls, out["rhs_u"], HS)
    O.bc(g, "u", uh)
    out["uhat"] = uh
    out["rhs_v"] = O.axi_rhs_v(g, f, dt, ls, u, uh, v, HS)
    vh = O.axi_vhat(g, f, dt, ls, out["rhs_v"], HS)
    O.bc(g, "v", vh)
    out["vhat"] = vh
    out["div4p"] = O.axi_div4p(g, base, uh, vh)
    out["div"] = O.axi_divergence(g, base, uh, vh)
    kap = out["kappa"].copy()
    out["sys"] = O.axi_assemble(g, f, base, dt, ls, kap, H, out["div4p"], recompute_kappa=f.sigma != 0.0)
    out["kappa_p"] = kap
    u2, v2 = u.copy(), v.copy()
    O.update_vel(g, f, dt, u2, v2, uh, vh, ps, ls, H, kap)
    out["u_new"], out["v_new"] = u2, v2
    out["dt_next"] = O.axi_update_dt(g, f, u2, v2, kap)
    return out


def compare(g, out, ref, label):
    for k in ("kappa", "dU", "dV", "rhs_u", "uhat", "rhs_v", "vhat", "div4p", "div", "kappa_p", "u_new", "v_new"):
        assert_bitexact(out[k], ref(k), f"{label} {k}")
    sysd = out["sys"]
    a, ia, ja, b = ref("csr_a"), ref("csr_ia"), ref("csr_ja"), ref("csr_b")
    if sysd["pinned"]:
        check_pinned_csr(g, sysd, a, ia, ja, b)
    else:
        a2, ia2, ja2, b2 = O.gfm_to_csr(g, sysd)
        assert np.array_equal(ia2, ia) and np.array_equal(ja2, ja), f"{label} CSR structure"
        assert_bitexact(a2, a, f"{label} CSR values")
        assert_bitexact(b2, b, f"{label} CSR right-hand side")
    assert out["dt_next"] == float(ref("dt_next")[0]), label


@pytest.mark.parametrize("name", list(CASES))
def test_axisym_golden(name):
    g, f, base, ls, u, v, ps = case_inputs(name)
    for k, a in (("ls", ls), ("u", u), ("v", v), ("ps", ps)):
        assert np.array_equal(a, GOLD[f"{name}/{k}"]), f"fixture inputs changed: {k}"
    out = oracle_outputs(g, f, base, ls, u, v, ps, float(GOLD[f"{name}/dt"][0]))
    compare(g, out, lambda k: GOLD[f"{name}/{k}"], name)


def reference_outputs(g, f, base, ls, u, v, ps, dt, **lengths):
    """The fixture's pipeline through the reference's own MACSolver2DAxisym
    (oracle/_ref), in the order the golden script calls it; lengths: len_r /
    len_z for AxiReference."""
    R = AxiReference(g, f, base_r=base, **lengths)
    HS = smooth_heaviside(ls, 1.5 * min(g.dx, g.dy))
    H = np.ascontiguousarray((ls >= 0.0).astype(np.float64))
    ref = {"kappa": R.kappa(ls)}
    R.set_state(u, v, ref["kappa"], dt)
    ref["dU"], ref["dV"] = R.visc(u, 0.9 * u + 0.01, v, ls, HS)
    ref["rhs_u"] = R.rhs_u(ls, u, v, HS)
    ref["uhat"] = R.bc("u", R.uhat(ls, u, ref["rhs_u"], HS))
    ref["rhs_v"] = R.rhs_v(ls, u, ref["uhat"], v, HS)
    ref["vhat"] = R.bc("v", R.vhat(ls, v, ref["rhs_v"], HS))
    ref["div4p"], ref["div"] = R.divergences(ref["uhat"], ref["vhat"])
    _, (ref["csr_a"], ref["csr_ia"], ref["csr_ja"], ref["csr_b"]) = R.poisson_capture(ref["div4p"], ls, ls, H, 0)
    ref["kappa_p"] = R.get_state()["kappa"]
    R.update_vel(ref["uhat"], ref["vhat"], ps, ls, ls, H)
    st = R.get_state()
    ref["u_new"], ref["v_new"] = st["u"], st["v"]
    ref["dt_next"] = np.array([R.update_dt(st["u"], st["v"])])
    R.close()
    return ref


@pytest.mark.skipif(not have_reference(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("name", list(CASES))
def test_axisym_against_live_reference(name, capfd):
    g, f, base, ls, u, v, ps = case_inputs(name, seed=1234)
    dt = 1.5e-3
    ref = reference_outputs(g, f, base, ls, u, v, ps, dt)
    capfd.readouterr()  # GetUHat prints one debug line per z row (mac2dAxisym.cpp:1122-1123)
    out = oracle_outputs(g, f, base, ls, u, v, ps, dt)
    compare(g, out, lambda k: ref[k], f"live {name}")


@pytest.mark.skipif(not have_reference(), reason="reference build (oracle/_ref) not present")
def test_axisym_driver_steps_against_live_reference(capfd):
    """Three whole steps of the reference's axisymmetric driver loop
    (test_mac2d_large.cpp:1264-1306) run through the reference's own objects
    (LevelSetSolver2D with the level set's boundary, MACSolver2DAxisym with
    its CG) and through the oracle's restatement of the step with the
    reference CG iteration: level set, velocities, pressure and dt bit for
    bit, on a bubble with density ratio 816 and surface tension."""
    from oracle.pyoracle import FluidSpec, GridSpec
    nr, nz = 32, 64
    bu = ("axisym", "neumann", "dirichlet", "dirichlet")
    g = GridSpec(nr, nz, 0.5 / nr, 1.0 / nz, bc_u=bu, bc_v=bu, bc_p=("axisym", "pressure", "neumann", "neumann"),
                 cu=(0.0, 1.0, 1.0, 1.0))
    lg = GridSpec(nr, nz, g.dx, g.dy, bc_u=bu, bc_v=bu, bc_p=("axisym", "lsfree", "lsfree", "lsfree"))
    f = FluidSpec(rho_h=1000.0, rho_l=1.226, mu_h=1.137e-3, mu_l=1.78e-5, sigma=0.0728, g=0.0, g_axis=1, cfl=0.3)
    r = (np.arange(nr + 6)[:, None] - 3 + 0.5) * g.dx
    z = (np.arange(nz + 6)[None, :] - 3 + 0.5) * g.dy
    ls = np.ascontiguousarray(np.sqrt(r ** 2 + (z - 0.5) ** 2) - 0.2)
    O.bc(lg, "p", ls)
    O.reinit(lg, 2, ls)
    O.bc(lg, "p", ls)
    u = np.full(ls.shape, 1.0)
    v = g.zeros()
    O.bc(g, "u", u)
    O.bc(g, "v", v)
    live_axi_steps(g, lg, f, ls, u, v, steps=3)
    capfd.readouterr()


def live_axi_steps(g, lg, f, ls, u, v, steps=3, mode=2, base_r=0.0, equal=assert_bitexact, len_r=None,
                   len_z=None):
    """`steps` steps of the reference's axisymmetric driver loop
    (test_mac2d_large.cpp:1264-1306) through the reference's own objects
    (LevelSetSolver2D on the level set's grid lg, MACSolver2DAxisym with its
    CG) and through the oracle's composed step with the reference CG
    iteration; level set, u, v, ps and dt compared with `equal` after every
    step.  len_r / len_z: the lengths the reference divides by nr / nz."""
    from oracle.pyoracle import Reference
    kappa = g.zeros()
    dt = O.axi_update_dt(g, f, u, v, kappa)
    st = dict(ls=ls.copy(), u=u.copy(), v=v.copy(), kappa=kappa.copy(), dt=dt)
    R2 = Reference(lg, f, len_x=len_r, len_y=len_z, base_x=base_r)
    AR = AxiReference(g, f, base_r=base_r, len_r=len_r, len_z=len_z)
    ls_r, u_r, v_r, k_r = ls.copy(), u.copy(), v.copy(), kappa.copy()
    try:
        for step in range(steps):
            lsB = ls_r.copy()
            R2.ls_advect(ls_r, u_r, v_r, dt)
            R2.bc("p", ls_r)
            R2.reinit(mode, ls_r)
            R2.bc("p", ls_r)
            AR.set_state(u_r, v_r, k_r, dt)
            k_r = AR.kappa(ls_r)
            H, HS = R2.heaviside(ls_r)
            uh = AR.bc("u", AR.uhat(ls_r, u_r, AR.rhs_u(ls_r, u_r, v_r, HS), HS))
            vh = AR.bc("v", AR.vhat(ls_r, v_r, AR.rhs_v(ls_r, u_r, uh, v_r, HS), HS))
            d4, _ = AR.divergences(uh, vh)
            R2.bc("p", ls_r)
            ps, _ = AR.poisson_capture(d4, ls_r, lsB, H, maxiter=10000)
            AR.bc("p", ps)
            AR.update_vel(uh, vh, ps, ls_r, lsB, H)
            got = AR.get_state()
            u_r, v_r, k_r = AR.bc("u", got["u"]), AR.bc("v", got["v"]), got["kappa"]
            AR.set_state(u_r, v_r, k_r, dt)
            dt = AR.update_dt(u_r, v_r)
            O.axi_step(g, f, st, base_r=base_r, ls_grid=lg, tol=1e-6, maxit=10000, pcg_mode=1, reinit_mode=mode)
            for name, a, b in (("ls", ls_r, st["ls"]), ("u", u_r, st["u"]), ("v", v_r, st["v"]),
                               ("ps", ps, st["ps"])):
                equal(b, a, f"step {step} {name}")
            assert dt == st["dt"] or (dt != dt and st["dt"] != st["dt"]), step
    finally:
        R2.close()
        AR.close()
