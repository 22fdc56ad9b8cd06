"""GPU: the axisymmetric MAC step (asd2g_axi_*, asd2_b200/csrc/axisym.cu)
against MACSolver2DAxisym (src/mac2dAxisym.cpp).

* Every function against the reference's own outputs in
  tests/golden/axisym_golden.npz: bit-identical, except the curvature (CUDA's
  pow against libm's: within 1e-13 of max |kappa|).  The assembly is checked
  as the CSR system SolvePoisson hands its CG, from the reference's kappa.
* Whole steps of the reference's axisymmetric driver
  (tests/LargeTests/test_mac2d_large.cpp:1145-1306, 64 x 128 cells) through
  asd2g_axi_step against the oracle's restatement of the same driver: level
  set, velocities, pressure and dt agree within the pressure solve's tolerance
  (both solve to rel. residual 1e-12 with different reduction orders).
"""
import os

import numpy as np
import pytest

from asd2_b200 import api
from oracle.pyoracle import FluidSpec, GridSpec, Oracle
from tests.golden.make_golden_axisym import CASES, case_inputs, smooth_heaviside
from tests.helpers import assert_bitexact, params_for
from tests.test_oracle import check_pinned_csr

pytestmark = pytest.mark.gpu

O = Oracle()
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "axisym_golden.npz"))


def session(g, f, base_r):
    return api.Session(params_for(g, f, base_x=base_r))


@pytest.mark.parametrize("name", list(CASES))
def test_axisym_functions_golden(name):
    g, f, base, ls, u, v, ps = case_inputs(name)
    ref = lambda k: GOLD[f"{name}/{k}"]
    dt = float(ref("dt")[0])
    HS = smooth_heaviside(ls, 1.5 * min(g.dx, g.dy))
    H = np.ascontiguousarray((ls >= 0.0).astype(np.float64))
    with session(g, f, base) as s:
        s.upload("ls", ls)
        s.axi_kappa()
        k = s.download("kappa")
        kr = ref("kappa")
        assert np.abs(k - kr).max() <= 1e-13 * np.abs(kr).max(), np.abs(k - kr).max()
        for fld, a in (("u", u), ("v", v), ("HS", HS), ("H", H)):
            s.upload(fld, a)
        s.axi_rhs_u(dt, out="w0")
        assert_bitexact(s.download("w0"), ref("rhs_u"), f"{name} GetRHSU")
        s.upload("w0", ref("rhs_u"))
        s.axi_hat(0, dt, rhs="w0")
        s.apply_bc("uhat", "U")
        assert_bitexact(s.download("uhat"), ref("uhat"), f"{name} GetUHat")
        s.upload("uhat", ref("uhat"))
        s.axi_rhs_v(dt, out="w1")
        assert_bitexact(s.download("w1"), ref("rhs_v"), f"{name} GetRHSV")
        s.upload("w1", ref("rhs_v"))
        s.axi_hat(1, dt, rhs="w1")
        s.apply_bc("vhat", "V")
        assert_bitexact(s.download("vhat"), ref("vhat"), f"{name} GetVHat")
        s.upload("vhat", ref("vhat"))
        s.axi_divergence(div="div", for_poisson=True)
        assert_bitexact(s.download("div"), ref("div4p"), f"{name} GetDivergence4Poisson")
        s.axi_divergence(div="w2", for_poisson=False)
        assert_bitexact(s.download("w2"), ref("div"), f"{name} GetDivergence")
        # assembly from the reference's own curvature (as SolvePoisson recomputed it)
        s.upload("kappa", ref("kappa_p"))
        s.upload("div", ref("div4p"))
        s.axi_assemble(dt, recompute_kappa=False)
        sysd = s.get_system()
        a, ia, ja, b = ref("csr_a"), ref("csr_ia"), ref("csr_ja"), ref("csr_b")
        if sysd["pinned"]:
            check_pinned_csr(g, sysd, a, ia, ja, b)
        else:
            a2, ia2, ja2, b2 = O.gfm_to_csr(g, sysd)
            assert np.array_equal(ia2, ia) and np.array_equal(ja2, ja)
            assert_bitexact(a2, a, f"{name} CSR values")
            assert_bitexact(b2, b, f"{name} CSR right-hand side")
        # projection (the 2D UpdateVel is the same arithmetic) and UpdateDt
        s.upload("u", u)
        s.upload("v", v)
        s.upload("ps", ps)
        s.update_vel(dt)
        assert_bitexact(s.download("u"), ref("u_new"), f"{name} UpdateVel u")
        assert_bitexact(s.download("v"), ref("v_new"), f"{name} UpdateVel v")
        assert s.axi_update_dt() == float(ref("dt_next")[0])


def _driver_case(kind):
    """The NonSurfaceTension driver (test_mac2d_large.cpp:1145-1230) or a
    stationary bubble with density and viscosity ratios and surface tension
    (after :1346-1420, with valid boundary names), 64 x 128 cells."""
    nr, nz = 64, 128
    if kind == "flow":
        lr, lz, R, zc = 0.5, 1.0, 0.2, 0.5
        bu = ("axisym", "neumann", "dirichlet", "dirichlet")
        g = GridSpec(nr, nz, lr / nr, lz / nz, bc_u=bu, bc_v=bu, bc_p=("axisym", "pressure", "neumann", "neumann"),
                     cu=(0.0, 1.0, 1.0, 1.0))
        f = FluidSpec(rho_h=1.226, rho_l=1.226, mu_h=1.78e-5, mu_l=1.78e-5, sigma=0.0, g=0.0, g_axis=1, cfl=0.3)
        u0, sign = 1.0, 1.0
    else:
        lr, lz, R, zc = 0.02, 0.04, 0.005, 0.02
        bu = ("axisym", "wall", "neumann", "neumann")
        g = GridSpec(nr, nz, lr / nr, lz / nz, bc_u=bu, bc_v=bu, bc_p=("axisym", "wall", "neumann", "outlet"))
        f = FluidSpec(rho_h=1000.0, rho_l=1.226, mu_h=1.137e-3, mu_l=1.78e-5, sigma=0.0728, g=0.0, g_axis=1,
                      cfl=0.5)
        u0, sign = 0.0, 1.0
    lg = GridSpec(nr, nz, g.dx, g.dy, bc_u=g.bc_u, bc_v=g.bc_v, bc_p=("axisym", "lsfree", "lsfree", "lsfree"))
    r = (np.arange(nr + 6)[:, None] - 3 + 0.5) * g.dx
    z = (np.arange(nz + 6)[None, :] - 3 + 0.5) * g.dy
    ls = np.ascontiguousarray(sign * (np.sqrt(r ** 2 + (z - zc) ** 2) - R))
    O.bc(lg, "p", ls)
    O.reinit(lg, 2, ls)
    O.bc(lg, "p", ls)
    u = np.full(ls.shape, u0)
    v = np.zeros(ls.shape)
    O.bc(g, "u", u)
    O.bc(g, "v", v)
    kappa = np.zeros(ls.shape)
    # the driver's first dt: cfl min(dr, dz) / U, then UpdateDt where it is finite (:1242-1244)
    dt = O.axi_update_dt(g, f, u, v, kappa) if u0 else f.cfl * min(g.dx, g.dy) / 1.0
    return g, lg, f, dict(ls=ls, u=u, v=v, kappa=kappa, dt=dt)


@pytest.mark.parametrize("kind", ["flow", "bubble"])
def test_axisym_driver_steps_match_oracle(kind):
    g, lg, f, st = _driver_case(kind)
    steps = 5
    with session(g, f, 0.0) as s:
        for fld in ("ls", "u", "v", "kappa"):
            s.upload(fld, st[fld])
        dt_gpu = st["dt"]
        for k in range(steps):
            r = s.axi_step(dt_gpu, ls_bc=lg.bc_p, solver=api.PCG, tol=1e-12, maxit=200000)
            assert r["status"] == 0, r
            info = O.axi_step(g, f, st, ls_grid=lg, tol=1e-12)
            assert abs(r["dt_next"] - st["dt"]) <= 1e-10 * st["dt"], (k, r["dt_next"], st["dt"])
            dt_gpu = st["dt"]  # both continue with the oracle's dt, so the comparison stays step-for-step
            got = {fld: s.download(fld) for fld in ("ls", "u", "v", "ps")}
            for fld in ("ls", "u", "v", "ps"):
                ref = st[fld]
                err = np.abs(got[fld] - ref)[3:-3, 3:-3].max()
                scale = max(np.abs(ref[3:-3, 3:-3]).max(), 1e-30)
                bar = 1e-10 if fld == "ls" else 1e-7
                assert err <= bar * max(scale, 1.0 if fld == "ls" else scale), (kind, k, fld, err, scale)
            print(f"{kind} step {k}: PCG iterations GPU {r['iters']} / oracle {info['iters']}, dt {st['dt']:.4e}")


def test_axisym_step_mg_solver_and_errors():
    """The multigrid-preconditioned solver gives the same step to its
    tolerance; periodic pressure and mixed precision are refused."""
    g, lg, f, st = _driver_case("bubble")
    outs = []
    for solver in (api.PCG, api.MGPCG):
        with session(g, f, 0.0) as s:
            for fld in ("ls", "u", "v", "kappa"):
                s.upload(fld, st[fld])
            dt = st["dt"]
            for _ in range(3):
                r = s.axi_step(dt, ls_bc=lg.bc_p, solver=solver, tol=1e-12, maxit=200000)
                assert r["status"] == 0, r
                dt = r["dt_next"]
            outs.append({fld: s.download(fld) for fld in ("u", "v", "ps")})
    for fld in ("u", "v", "ps"):
        a, b = outs[0][fld][3:-3, 3:-3], outs[1][fld][3:-3, 3:-3]
        assert np.abs(a - b).max() <= 1e-7 * max(np.abs(a).max(), 1e-30), fld
    gp = GridSpec(g.nx, g.ny, g.dx, g.dy, bc_u=g.bc_u, bc_v=g.bc_v, bc_p=("periodic", "periodic", "neumann", "outlet"))
    with session(gp, f, 0.0) as s:
        with pytest.raises(api.Asd2gError):
            s.axi_assemble(1e-3)
    with api.Session(params_for(g, f, precision=api.PRECISION_MIXED)) as s:
        with pytest.raises(api.Asd2gError):
            s.axi_step(1e-3)


def test_axisym_droplet_collision_driver():
    """The reference's axisymmetric droplet-collision driver
    (test_mac2d_large.cpp:1762-1960): 120 x 320 cells, two spheres of radius
    150 um 3L apart on the axis approaching at +-U/2 (U = 1.4 m/s),
    density 1000 / 1.226, surface tension, all-Neumann pressure (the
    corrected pin), U/V axisym-Dirichlet-Neumann-Neumann, the level set's own
    sides axisym-Neumann; the first MACSolver2DAxisym constructor's
    constants (kRe, kWe finite, no gravity).  Three steps against the
    oracle's restatement of the driver: level set within 1e-10, u, v, ps
    within 1e-7 of their maxima, dt within 1e-10."""
    L, U = 300 * 10e-6, 1.4
    rho_h, mu_h, rho_l, mu_l, sigma = 1000.0, 1.137e-3, 1.226, 1.78e-5, 0.0728
    nr, nz = 120, 320
    lr, lz = L * 3.0, L * 8.0
    base_z = -0.5 * lz
    dr, dz = lr / nr, lz / nz
    bu = ("axisym", "dirichlet", "neumann", "neumann")
    g = GridSpec(nr, nz, dr, dz, bc_u=bu, bc_v=bu, bc_p=("neumann",) * 4)
    lg = GridSpec(nr, nz, dr, dz, bc_u=bu, bc_v=bu, bc_p=("axisym", "neumann", "neumann", "neumann"))
    f = FluidSpec(rho_h=rho_h, rho_l=rho_h * (rho_l / rho_h), mu_h=mu_h, mu_l=mu_h * (mu_l / mu_h), sigma=sigma,
                  g=0.0, g_axis=1, cfl=0.1)
    radius = 150 * 10e-6
    r = (np.arange(nr + 6)[:, None] - 3 + 0.5) * dr
    z = base_z + (np.arange(nz + 6)[None, :] - 3 + 0.5) * dz
    d1 = np.sqrt(r * r + (z - L * 1.5) * (z - L * 1.5)) - radius
    d2 = np.sqrt(r * r + (z + L * 1.5) * (z + L * 1.5)) - radius
    inner = np.zeros((nr + 6, nz + 6), dtype=bool)
    inner[3:-3, 3:-3] = True
    v = np.where(inner & (d1 < 0), -U * 0.5, 0.0)
    v = np.ascontiguousarray(np.where(inner & (d2 < 0), U * 0.5, v))
    ls = np.ascontiguousarray(np.where(inner, np.minimum(d1, d2), 0.0))
    u = g.zeros()
    O.bc(lg, "p", ls)
    O.reinit(lg, 2, ls)
    O.bc(lg, "p", ls)
    O.bc(g, "u", u)
    O.bc(g, "v", v)
    kappa = g.zeros()
    st = dict(ls=ls, u=u, v=v, kappa=kappa, dt=O.axi_update_dt(g, f, u, v, kappa))
    with session(g, f, 0.0) as s:
        for fld in ("ls", "u", "v", "kappa"):
            s.upload(fld, st[fld])
        dt = st["dt"]
        for k in range(3):
            r_ = s.axi_step(dt, ls_bc=lg.bc_p, solver=api.PCG, tol=1e-12, maxit=200000)
            assert r_["status"] == 0, r_
            info = O.axi_step(g, f, st, ls_grid=lg, tol=1e-12)
            assert abs(r_["dt_next"] - st["dt"]) <= 1e-10 * st["dt"], (k, r_["dt_next"], st["dt"])
            for fld in ("ls", "u", "v", "ps"):
                ref = st[fld]
                err = np.abs(s.download(fld) - ref)[3:-3, 3:-3].max()
                scale = max(np.abs(ref[3:-3, 3:-3]).max(), 1e-30)
                bar = 1e-10 * scale if fld == "ls" else 1e-7 * scale
                assert err <= bar, (k, fld, err, scale)
            print(f"collision step {k}: PCG iterations GPU {r_['iters']} / oracle {info['iters']}, "
                  f"dt {st['dt']:.3e}, max |v| {np.abs(st['v'][3:-3, 3:-3]).max():.3f}")
            dt = st["dt"]
