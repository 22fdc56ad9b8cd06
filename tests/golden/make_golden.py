"""Generate the golden fixtures in this directory from the reference itself.

Run from the repository root after ``make -C oracle`` has built
oracle/_ref/libasd2ref.so (the reference's src/*.cpp compiled unmodified):

    python tests/golden/make_golden.py

Every fixture stores seeded inputs and the reference's outputs for them, on
small grids (one non-power-of-two, non-square spacing and one power-of-two
rectangular grid) so that the committed files stay a few hundred KB.  The CPU
tests check the C restatement (oracle/asd2_oracle.c) against these bit for
bit; the GPU tests check the CUDA kernels against them.
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.pyoracle import FluidSpec, GridSpec, Reference  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

GRIDS = {
    # name: (nx, ny, dx, dy)
    "A": (24, 20, 1.0 / 24, 1.0 / 20),
    "B": (32, 16, 1.0 / 32, 1.0 / 32),
}


def centres(nx, ny, dx, dy):
    x = (np.arange(nx + 6) - 3 + 0.5) * dx
    y = (np.arange(ny + 6) - 3 + 0.5) * dy
    return np.meshgrid(x, y, indexing="ij")


def level_set_inputs(nx, ny, dx, dy, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    X, Y = centres(nx, ny, dx, dy)
    lx, ly = nx * dx, ny * dy
    cx, cy = 0.5 * lx, 0.55 * ly
    R = 0.3 * min(lx, ly)
    th = np.arctan2(Y - cy, X - cx)
    a = rng.uniform(-0.02, 0.02, 4) * min(lx, ly)
    psi = rng.uniform(0, 2 * math.pi, 4)
    Rt = R + sum(a[k] * np.cos((k + 2) * th + psi[k]) for k in range(4))
    ls = Rt - np.sqrt((X - cx) ** 2 + (Y - cy) ** 2)
    xf = (np.arange(nx + 6) - 3) * dx
    yf = (np.arange(ny + 6) - 3) * dy
    _, Yc = np.meshgrid(xf, (np.arange(ny + 6) - 3 + 0.5) * dy, indexing="ij")
    Xc, _ = np.meshgrid((np.arange(nx + 6) - 3 + 0.5) * dx, yf, indexing="ij")
    u = -2 * math.pi * (Yc - cy)
    v = 2 * math.pi * (Xc - cx)
    return ls, u, v


def level_set_cases(name, nx, ny, dx, dy):
    tag = "L"
    out = {}
    g = GridSpec(nx, ny, dx, dy, bc_u=("neumann",) * 4, bc_v=("neumann",) * 4, bc_p=("neumann",) * 4)
    R = Reference(g)
    ls, u, v = level_set_inputs(nx, ny, dx, dy, seed=11)
    dt = 0.5 * min(dx, dy) / np.abs(np.concatenate([u.ravel(), v.ravel()])).max()
    out.update(ls=ls, u=u, v=v, dt=np.float64(dt))
    a = ls.copy()
    R.ls_advect(a, u, v, dt)
    out["advect"] = a
    # WENO right-hand side with cell-centred velocities
    uc = 0.5 * (u[:-1, :] + u[1:, :])
    uc = np.vstack([uc, uc[-1:]])
    vc = 0.5 * (v[:, :-1] + v[:, 1:])
    vc = np.hstack([vc, vc[:, -1:]])
    out["uc"], out["vc"] = uc, vc
    a = ls.copy()
    out["weno_rhs"] = R.ls_weno_rhs(a, uc, vc)
    out["weno_rhs_ls"] = a
    # reinitialisation of a distorted field
    X, Y = centres(nx, ny, dx, dy)
    dist = ls * (1.3 + 0.4 * np.sin(3 * X)) + 0.01 * np.cos(5 * Y) * min(dx, dy)
    out["dist"] = dist
    for mode in range(5):
        a = dist.copy()
        R.reinit(mode, a)
        out[f"reinit{mode}"] = a
    # building blocks on (ls1, ls0)
    ls0 = dist.copy()
    R.bc("P", ls0)
    ls1 = ls0 * 0.9 + 0.3 * min(dx, dy) * np.sin(7 * X + 2 * Y)
    out["bb_ls0"], out["bb_ls1"] = ls0, ls1
    out["subcell"] = R.subcell_eno_absgrad(ls1, ls0)
    out["eno"] = R.eno_absgrad(ls1, ls0)
    hd = R.heaviside_deriv(ls1)
    out["hd"] = hd
    out["sussman"] = R.sussman_constraint(ls1, ls0, hd)
    out["ssign"] = R.smoothed_sign(ls1)
    R.close()
    return {f"{name}{tag}_{k}": v for k, v in out.items()}


def droplet_inputs(nx, ny, dx, dy, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    X, Y = centres(nx, ny, dx, dy)
    lx, ly = nx * dx, ny * dy
    r = rng.uniform(0.2, 0.3) * min(lx, ly)
    cx, cy = rng.uniform(0.4, 0.6) * lx, rng.uniform(0.4, 0.6) * ly
    ls = r - np.sqrt((X - cx) ** 2 + (Y - cy) ** 2)
    # a smooth divergence-carrying velocity, then the wall fill
    xf = (np.arange(nx + 6) - 3) * dx
    yf = (np.arange(ny + 6) - 3) * dy
    XU, YU = np.meshgrid(xf, (np.arange(ny + 6) - 3 + 0.5) * dy, indexing="ij")
    XV, YV = np.meshgrid((np.arange(nx + 6) - 3 + 0.5) * dx, yf, indexing="ij")
    u = 0.05 * np.sin(math.pi * XU / lx) * np.cos(math.pi * YU / ly) + 0.01 * rng.standard_normal(XU.shape)
    v = -0.04 * np.cos(math.pi * XV / lx) * np.sin(math.pi * YV / ly) + 0.01 * rng.standard_normal(XV.shape)
    return ls, u, v


def mac_cases(name, nx, ny, dx, dy):
    tag = "M"
    out = {}
    f = FluidSpec()
    g = GridSpec(nx, ny, dx, dy)
    R = Reference(g, f)
    ls, u, v = droplet_inputs(nx, ny, dx, dy, seed=5)
    R.bc("P", ls, which=1)
    R.bc("U", u, which=1)
    R.bc("V", v, which=1)
    out.update(ls=ls, u=u, v=v)
    k = R.kappa(ls)
    out["kappa"] = k
    # UpdateNTK on the droplet's distance field and on a plane whose slope is
    # 1 on the west half and 1.3 on the east half: the normal is stored where
    # |1 - |grad phi|| <= 1e-4 only, so the outputs start from sentinels that
    # mark the cells the reference leaves alone
    Xc, Yc = centres(nx, ny, dx, dy)
    plane = 0.6 * Xc + 0.8 * Yc - 0.4 * (nx * dx)
    plane = np.where(Xc < 0.5 * nx * dx, plane, 1.3 * plane)
    for tag2, phi in (("sdf", ls), ("plane", plane)):
        n0, n1 = np.full(g.shape, 7.0), np.full(g.shape, -7.0)
        R.ntk(phi, n0, n1)
        out[f"ntk_{tag2}_phi"], out[f"ntk_{tag2}_nx"], out[f"ntk_{tag2}_ny"] = phi, n0, n1
    H, HS = R.heaviside(ls)
    out["H"], out["HS"] = H, HS
    cU, cV = R.conv(u, v)
    out["conv_u"], out["conv_v"] = cU, cV
    dU, dV = R.visc(u, v, ls, HS)
    out["visc_u"], out["visc_v"] = dU, dV
    FU, FV = R.rhs(ls, u, v, HS)
    out["rhs_u"], out["rhs_v"] = FU, FV
    dt = 2.0e-4
    out["dt"] = np.float64(dt)
    R.set_state(u, v, g.zeros(), dt)
    uh, vh = R.intermediate_vel(ls, u, v, HS)
    out["uhat"], out["vhat"] = uh.copy(), vh.copy()
    R.bc("U", uh, which=1)
    R.bc("V", vh, which=1)
    div = R.divergence(uh, vh)
    out["div"] = div
    # GFM system as assembled by the reference (captured from its CG call)
    R.set_kappa(k.copy())
    _, (a, ia, ja, b) = R.poisson_capture(div, ls, ls, H, maxiter=0)
    out["csr_a"], out["csr_ia"], out["csr_ja"], out["csr_b"] = a, ia, ja, b
    out["kappa_bc"] = R.get_state()["kappa"]
    # projection with a smooth pseudo-pressure, and the next dt
    X, Y = centres(nx, ny, dx, dy)
    ps = 1e-4 * np.cos(2 * X) * np.sin(3 * Y)
    R.bc("P", ps, which=1)
    out["ps_in"] = ps
    R.set_state(u, v, g.zeros(), dt)
    R.set_kappa(out["kappa_bc"].copy())
    R.update_vel(uh, vh, ps, ls, ls, H)
    st = R.get_state()
    out["u_new"], out["v_new"] = st["u"], st["v"]
    out["dt_next"] = np.float64(R.update_dt(st["u"], st["v"]))
    R.close()
    # time orders 0 and 1 of GetIntermediateVel
    for order in (0, 1):
        R2 = Reference(g, FluidSpec(time_order=order))
        R2.set_state(u, v, g.zeros(), dt)
        a1, b1 = R2.intermediate_vel(ls, u, v, HS)
        out[f"uhat_o{order}"], out[f"vhat_o{order}"] = a1, b1
        R2.close()
    return {f"{name}{tag}_{k}": v for k, v in out.items()}


def dirichlet_cases():
    """Dirichlet-pressure GFM systems solved by the reference's own CG and
    BiCGStab for a fixed number of iterations (the pinned all-Neumann system
    of the reference is mis-indexed and cannot be run meaningfully)."""
    out = {}
    nx, ny, dx, dy = 24, 20, 1.0 / 24, 1.0 / 20
    f = FluidSpec()
    g = GridSpec(nx, ny, dx, dy, bc_p=("dirichlet",) * 4, cp=(0.0, 0.0, 0.0, 0.0))
    R = Reference(g, f)
    ls, u, v = droplet_inputs(nx, ny, dx, dy, seed=9)
    R.bc("P", ls, which=1)
    H, HS = R.heaviside(ls)
    k = R.kappa(ls)
    X, Y = centres(nx, ny, dx, dy)
    div = np.sin(2 * math.pi * X) * np.cos(math.pi * Y)
    dt = 2.0e-4
    R.set_state(u, v, g.zeros(), dt)
    R.set_kappa(k.copy())
    _, (a, ia, ja, b) = R.poisson_capture(div, ls, ls, H, maxiter=0)
    rhs = g.zeros()
    rhs[3:-3, 3:-3] = b.reshape(ny, nx).T
    mdiag = np.array([a[ia[r]:ia[r + 1]][ja[ia[r]:ia[r + 1]] == r][0] for r in range(len(ia) - 1)])
    out.update(ls=ls, div=div, dt=np.float64(dt), kappa=k, H=H, csr_a=a, csr_ia=ia, csr_ja=ja, csr_b=b)
    for its in (1, 2, 25):
        out[f"cg{its}"] = R.cg(rhs, (a, ia, ja), mdiag, its)
    for its in (1, 2, 15):
        out[f"bicg{its}"] = R.bicgstab(rhs, (a, ia, ja), mdiag, its)
    R.close()
    return {f"D_{k}": v for k, v in out.items()}


def laplace_case():
    """The reference's Poisson CG driver (test_poisson2d_large.cpp:174-323) on
    a 32 x 32 grid: constant coefficients, Dirichlet 0 on W/E/S and 1 on N."""
    nx = ny = 32
    dx = dy = 1.0 / 32
    g = GridSpec(nx, ny, dx, dy, bc_p=("dirichlet",) * 4, cp=(0.0, 0.0, 0.0, 1.0))
    f = FluidSpec(rho_h=1.0, rho_l=1.0, sigma=0.0)
    R = Reference(g, f)
    ls = np.ones(g.shape)
    H, _ = R.heaviside(ls)
    div = g.zeros()
    R.set_state(g.zeros(), g.zeros(), g.zeros(), 1.0)
    R.set_kappa(g.zeros())
    _, (a, ia, ja, b) = R.poisson_capture(div, ls, ls, H, maxiter=0)
    rhs = g.zeros()
    rhs[3:-3, 3:-3] = b.reshape(ny, nx).T
    mdiag = np.array([a[ia[r]:ia[r + 1]][ja[ia[r]:ia[r + 1]] == r][0] for r in range(len(ia) - 1)])
    ps = R.cg(rhs, (a, ia, ja), mdiag, 20000)
    R.close()
    return {"L_ps": ps, "L_csr_a": a, "L_csr_b": b}


BC_KINDS_UV = ["periodic", "neumann", "dirichlet", "axisym", "wall", "inlet", "outlet"]
BC_KINDS_P = BC_KINDS_UV + ["pressure", "lsfree"]
BC_TRIALS = 9


def bc_kinds(trial):
    """W/E/S/N kinds of the U/V grids and of the P grid in one trial: over the
    trials every kind meets every side (velocity grids take no "pressure" or
    "lsfree": the reference exits on a constant-pressure velocity side)."""
    uv = tuple(BC_KINDS_UV[(trial + 2 * s) % len(BC_KINDS_UV)] for s in range(4))
    vv = tuple(BC_KINDS_UV[(trial + 3 * s + 1) % len(BC_KINDS_UV)] for s in range(4))
    pp = tuple(BC_KINDS_P[(trial + 2 * s) % len(BC_KINDS_P)] for s in range(4))
    return uv, vv, pp


def bc_cases():
    """Ghost fills of the U, V and P grids (ApplyBC_{U,V,P}_2D,
    src/bc2d.cpp:123-934) for every boundary kind on every side, with random
    boundary constants, on a 13 x 9 grid of unequal spacings."""
    rng = np.random.Generator(np.random.PCG64(21))
    out = {}
    for t in range(BC_TRIALS):
        bu, bv, bp = bc_kinds(t)
        cu, cv, cp = (rng.uniform(-1.0, 1.0, 4) for _ in range(3))
        g = GridSpec(13, 9, 0.1, 0.125, bc_u=bu, bc_v=bv, bc_p=bp, cu=tuple(cu), cv=tuple(cv), cp=tuple(cp))
        R = Reference(g)
        out[f"{t}_consts"] = np.stack([cu, cv, cp])
        for kind in ("U", "V", "P"):
            a = rng.standard_normal(g.shape)
            out[f"{t}_{kind}_in"] = a
            out[f"{t}_{kind}_out"] = R.bc(kind, a.copy(), which=0)
        R.close()
    return {f"BC{k}": v for k, v in out.items()}


def main():
    data = {}
    for name, (nx, ny, dx, dy) in GRIDS.items():
        data.update(level_set_cases(name, nx, ny, dx, dy))
        data.update(mac_cases(name, nx, ny, dx, dy))
    data.update(dirichlet_cases())
    data.update(laplace_case())
    data.update(bc_cases())
    path = os.path.join(OUT, "reference_golden.npz")
    np.savez_compressed(path, **data)
    print(f"wrote {path}: {len(data)} arrays, {os.path.getsize(path) / 1024:.0f} KB")


if __name__ == "__main__":
    main()
