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


@pytest.mark.skipif(not have_reference(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("name", list(CASES))
def test_axisym_against_live_reference(name, capfd):
    g, f, base, ls, u, v, ps = case_inputs(name, seed=1234)
    dt = 1.5e-3
    R = AxiReference(g, f, base_r=base)
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
    capfd.readouterr()  # GetUHat prints one debug line per z row (mac2dAxisym.cpp:1122-1123)
    out = oracle_outputs(g, f, base, ls, u, v, ps, dt)
    compare(g, out, lambda k: ref[k], f"live {name}")
