"""Generate axisym_golden.npz in this directory from the reference itself.

Run from the repository root after ``make -C oracle`` has built
oracle/_ref/libasd2ref.so (which includes the reference's src/mac2dAxisym.cpp
compiled unmodified):

    python tests/golden/make_golden_axisym.py

For each case the fixture stores seeded inputs (level set, velocities,
boundary kinds and constants, fluid) and the outputs of MACSolver2DAxisym for
them: UpdateKappa, AddExternalViscosityFU/FV, GetRHSU, GetUHat, GetRHSV,
GetVHat, GetDivergence4Poisson, GetDivergence, the CSR system SolvePoisson
assembles, UpdateVel and UpdateDt.  Grids are small (12 x 16 and 10 x 20
cells) so the file stays a few hundred KB.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.pyoracle import AxiReference, FluidSpec, GridSpec  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "axisym_golden.npz")

# name: (nr, nz, base_r, boundary kinds, gravity axis)
CASES = {
    # the NonSurfaceTension driver's kinds (test_mac2d_large.cpp:1185-1187)
    "drop": (12, 16, 0.0, dict(bc_u=("axisym", "neumann", "dirichlet", "dirichlet"),
                               bc_v=("axisym", "neumann", "dirichlet", "dirichlet"),
                               bc_p=("axisym", "pressure", "neumann", "neumann")), 1),
    # an annulus off the axis with the other kinds the implicit step branches on
    "ring": (10, 20, 0.1, dict(bc_u=("dirichlet", "outlet", "periodic", "periodic"),
                               bc_v=("wall", "inlet", "periodic", "periodic"),
                               bc_p=("neumann", "dirichlet", "neumann", "wall")), 0),
    "wall": (12, 16, 0.05, dict(bc_u=("neumann", "wall", "inlet", "outlet"),
                                bc_v=("neumann", "dirichlet", "wall", "outlet"),
                                bc_p=("wall", "neumann", "neumann", "neumann")), 1),
}


def case_inputs(name, seed=None):
    nr, nz, base, bcs, g_axis = CASES[name]
    seed = sum(map(ord, name)) if seed is None else seed
    rng = np.random.Generator(np.random.PCG64(seed))
    lr, lz = 0.5, 1.0
    dr, dz = lr / nr, lz / nz
    g = GridSpec(nr, nz, dr, dz, cu=tuple(rng.uniform(-1, 1, 4)), cv=tuple(rng.uniform(-1, 1, 4)),
                 cp=tuple(rng.uniform(-1, 1, 4)), **bcs)
    f = FluidSpec(rho_h=1000.0, rho_l=1.226, mu_h=1.0e-3, mu_l=1.78e-5, sigma=0.0728, g=9.8, g_axis=g_axis,
                  fix_gravity=0, cfl=0.3)
    r = base + (np.arange(nr + 6)[:, None] - 3 + 0.5) * dr
    z = (np.arange(nz + 6)[None, :] - 3 + 0.5) * dz
    ls = 0.2 - np.sqrt((r - base) ** 2 + (z - 0.5 * lz) ** 2) + 0.002 * rng.standard_normal((nr + 6, nz + 6))
    u = 0.3 * np.sin(3 * r + 1) * np.cos(2 * z) + 0.01 * rng.standard_normal(ls.shape)
    v = 0.2 * np.cos(2 * r) * np.sin(3 * z + 0.5) + 0.01 * rng.standard_normal(ls.shape)
    ps = 1.0e-3 * rng.standard_normal(ls.shape)
    c = np.ascontiguousarray
    return g, f, base, c(ls), c(u), c(v), c(ps)


def smooth_heaviside(ls, eps):
    H = 0.5 * (1.0 + ls / eps + np.sin(np.pi * ls / eps) / np.pi)
    return np.ascontiguousarray(np.where(ls > eps, 1.0, np.where(ls < -eps, 0.0, H)))


def main():
    out = {}
    dt = 2.0e-3
    for name in CASES:
        g, f, base, ls, u, v, ps = case_inputs(name)
        R = AxiReference(g, f, base_r=base)
        HS = smooth_heaviside(ls, 1.5 * min(g.dx, g.dy))
        H = np.ascontiguousarray((ls >= 0.0).astype(np.float64))
        kappa = R.kappa(ls)
        R.set_state(u, v, kappa, dt)
        dU, dV = R.visc(u, 0.9 * u + 0.01, v, ls, HS)
        rhs_u = R.rhs_u(ls, u, v, HS)
        uhat = R.uhat(ls, u, rhs_u, HS)
        R.bc("u", uhat)
        rhs_v = R.rhs_v(ls, u, uhat, v, HS)
        vhat = R.vhat(ls, v, rhs_v, HS)
        R.bc("v", vhat)
        div4p, div = R.divergences(uhat, vhat)
        _, (a, ia, ja, b) = R.poisson_capture(div4p, ls, ls, H, 0)
        kappa_p = R.get_state()["kappa"]
        R.update_vel(uhat, vhat, ps, ls, ls, H)
        st = R.get_state()
        dt_next = R.update_dt(st["u"], st["v"])
        R.close()
        for k, val in dict(ls=ls, u=u, v=v, ps=ps, HS=HS, H=H, kappa=kappa, dU=dU, dV=dV, rhs_u=rhs_u,
                           uhat=uhat, rhs_v=rhs_v, vhat=vhat, div4p=div4p, div=div, csr_a=a, csr_ia=ia,
                           csr_ja=ja, csr_b=b, kappa_p=kappa_p, u_new=st["u"], v_new=st["v"],
                           dt_next=np.array([dt_next]), dt=np.array([dt])).items():
            out[f"{name}/{k}"] = val
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
