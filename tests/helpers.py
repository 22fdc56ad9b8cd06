"""Shared test helpers: golden fixtures and grid/parameter conversions."""
from __future__ import annotations

import os

import numpy as np

from oracle.pyoracle import FluidSpec, GridSpec

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_golden.npz")
GRIDS = {"A": (24, 20, 1.0 / 24, 1.0 / 20), "B": (32, 16, 1.0 / 32, 1.0 / 32)}

_gold = None


def golden():
    global _gold
    if _gold is None:
        _gold = dict(np.load(GOLDEN))
    return _gold


def ls_grid(name) -> GridSpec:
    nx, ny, dx, dy = GRIDS[name]
    return GridSpec(nx, ny, dx, dy, bc_u=("neumann",) * 4, bc_v=("neumann",) * 4, bc_p=("neumann",) * 4)


def mac_grid(name) -> GridSpec:
    nx, ny, dx, dy = GRIDS[name]
    return GridSpec(nx, ny, dx, dy)


def params_for(g: GridSpec, f: FluidSpec | None = None, **kw):
    from asd2_b200.api import Params
    f = f or FluidSpec()
    return Params(g.nx, g.ny, g.dx, g.dy, bc_u=g.bc_u, bc_v=g.bc_v, bc_p=g.bc_p, bcc_u=g.cu, bcc_v=g.cv,
                  bcc_p=g.cp, rho_h=f.rho_h, rho_l=f.rho_l, mu_h=f.mu_h, mu_l=f.mu_l, sigma=f.sigma, g=f.g,
                  g_axis=f.g_axis, fix_gravity=f.fix_gravity, time_order=f.time_order, cfl=f.cfl, **kw)


def grid_from_case(c) -> GridSpec:
    return GridSpec(c.nx, c.ny, c.dx, c.dy, bc_u=c.bc_u, bc_v=c.bc_v, bc_p=c.bc_p)


def fluid_from_case(c) -> FluidSpec:
    return FluidSpec(**c.fluid) if c.fluid else FluidSpec()


def interior(a):
    return a[3:-3, 3:-3]


def assert_bitexact(a, b, what=""):
    a, b = np.asarray(a), np.asarray(b)
    if not np.array_equal(a, b):
        d = np.abs(a - b)
        idx = np.unravel_index(np.argmax(d), d.shape)
        raise AssertionError(f"{what}: not bit-identical; max |diff| {d.max():.3e} at {idx} "
                             f"({a[idx]!r} vs {b[idx]!r}); {np.count_nonzero(a != b)} cells differ")


def assert_close(a, b, rtol, atol=0.0, what=""):
    a, b = np.asarray(a), np.asarray(b)
    d = np.abs(a - b)
    lim = atol + rtol * np.abs(b)
    if not np.all(d <= lim):
        idx = np.unravel_index(np.argmax(d - lim), d.shape)
        raise AssertionError(f"{what}: max |diff| {d.max():.3e} exceeds tolerance at {idx} "
                             f"({a[idx]!r} vs {b[idx]!r})")


def bc_fixture(trial):
    """The grid of one boundary-fill golden trial (tests/golden/make_golden.py
    bc_cases) and a getter for its arrays."""
    from tests.golden.make_golden import bc_kinds
    G = golden()
    bu, bv, bp = bc_kinds(trial)
    cu, cv, cp = (tuple(float(x) for x in row) for row in G[f"BC{trial}_consts"])
    g = GridSpec(13, 9, 0.1, 0.125, bc_u=bu, bc_v=bv, bc_p=bp, cu=cu, cv=cv, cp=cp)
    return g, (lambda key: G[f"BC{trial}_{key}"])


def reinit_driver_case(name):
    """Initial fields of two of the reference's reinitialisation-only drivers
    (test_levelset2d_large.cpp), 128^2 on [-2, 2]^2 with Neumann sides
    (and "firsttime", :1220, the sign field of the unit circle for the
    first-time Sussman reinitialisation):
    "kinks" (:1042, two overlapping unit circles 1.4 apart, the union's
    distance with its kinks; max pseudo-time 80) and "minrk2_2" (:882, the
    unit circle's distance times (x-1)^2 + (y-1)^2 + 0.1, far from a
    distance function; max pseudo-time 2 max(nx, ny) = 256).  Returns
    (grid, padded phi with zero ghosts, max pseudo-time)."""
    n, L, base = 128, 4.0, -2.0
    dx = L / n
    g = GridSpec(n, n, dx, dx, bc_p=("neumann",) * 4)
    i = np.arange(n + 6)[:, None]
    j = np.arange(n + 6)[None, :]
    x = base + (i - 3 + 0.5) * dx + 0.0 * j
    y = base + (j - 3 + 0.5) * dx + 0.0 * i
    if name == "kinks":
        r, a = 1.0, 0.7
        ls = np.minimum(np.sqrt((x + a) ** 2 + y * y) - r, np.sqrt((x - a) ** 2 + y * y) - r)
        max_atime = 80.0
    elif name == "firsttime":  # :1220, +1 inside / -1 outside the unit circle, FirstTimeOnlyReinit_Sussman_2D
        d = np.sqrt(x * x + y * y) - 1.0
        ls = np.where(d < 0, 1.0, np.where(d > 0, -1.0, 0.0))
        max_atime = 256.0
    else:
        ls = ((x - 1.0) ** 2 + (y - 1.0) ** 2 + 0.1) * (np.sqrt(x * x + y * y) - 1.0)
        max_atime = 256.0
    inner = np.zeros(ls.shape, dtype=bool)
    inner[3:-3, 3:-3] = True
    return g, np.ascontiguousarray(np.where(inner, ls, 0.0)), max_atime
