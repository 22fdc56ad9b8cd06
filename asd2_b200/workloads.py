"""Seeded synthetic inputs for the level-set and droplet workloads.

The reference ships no data sets; its drivers build fields analytically
(tests/LargeTests/test_levelset2d_large.cpp:3-60, test_mac2d_large.cpp:
377-470).  These generators build the same kinds of fields from a seed with
numpy's PCG64 generator, in the padded reference layout
idx(i,j) = j + (ny+6)*i (arrays of shape (nx+6, ny+6)).

* ``perturbed_circle``: signed distance to a circle of radius 0.15 centred at
  (0.5, 0.75) whose radius carries four seeded Fourier modes m = 2..5 with
  sum |a_m| <= 0.01, in a rigid-rotation velocity u = -2 pi (y - 0.5),
  v = 2 pi (x - 0.5) (level-set advection + reinitialisation workload).
* ``droplet``: one heavy droplet of seeded radius in [0.1, 0.2] whose centre
  is at least 0.25 from the walls, fluid at rest, walls all round
  (two-phase step workload).
* ``droplet_batch``: many droplets of uneven grid sizes for batched runs.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

NB = 3


@dataclass
class Case:
    nx: int
    ny: int
    dx: float
    dy: float
    ls: np.ndarray
    u: np.ndarray
    v: np.ndarray
    dt: float = 0.0
    steps: int = 0
    bc_u: tuple = ("dirichlet",) * 4
    bc_v: tuple = ("dirichlet",) * 4
    bc_p: tuple = ("neumann",) * 4
    fluid: dict = field(default_factory=dict)
    meta: dict = field(default_factory=dict)


def _centres(nx, ny, dx, dy):
    x = (np.arange(nx + 2 * NB) - NB + 0.5) * dx
    y = (np.arange(ny + 2 * NB) - NB + 0.5) * dy
    return np.meshgrid(x, y, indexing="ij")


def perturbed_circle(n: int = 128, seed: int = 0, cfl: float = 0.5, revolutions: float = 1.0) -> Case:
    """Level-set workload on [0,1]^2 with n x n cells (Neumann pressure-grid
    boundaries, as the reference's level-set drivers use)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    dx = dy = 1.0 / n
    a = rng.uniform(-0.01, 0.01, size=4)
    s = np.abs(a).sum()
    if s > 0.01:
        a *= 0.01 / s
    psi = rng.uniform(0.0, 2.0 * math.pi, size=4)
    X, Y = _centres(n, n, dx, dy)
    th = np.arctan2(Y - 0.75, X - 0.5)
    R = 0.15 + sum(a[k] * np.cos((k + 2) * th + psi[k]) for k in range(4))
    ls = R - np.sqrt((X - 0.5) ** 2 + (Y - 0.75) ** 2)
    # u on west faces (x = (i-3) dx, y centred), v on south faces.
    xf = (np.arange(n + 2 * NB) - NB) * dx
    yf = (np.arange(n + 2 * NB) - NB) * dy
    _, Yc = np.meshgrid(xf, (np.arange(n + 2 * NB) - NB + 0.5) * dy, indexing="ij")
    Xc, _ = np.meshgrid((np.arange(n + 2 * NB) - NB + 0.5) * dx, yf, indexing="ij")
    u = -2.0 * math.pi * (Yc - 0.5)
    v = 2.0 * math.pi * (Xc - 0.5)
    # dt from the fastest cell-centre speed, rounded to a whole number of
    # steps per revolution (period T = 1).
    sl = slice(NB, -NB)
    speed = np.sqrt((2 * math.pi * (Y[sl, sl] - 0.5)) ** 2 + (2 * math.pi * (X[sl, sl] - 0.5)) ** 2).max()
    steps = int(math.ceil(revolutions / (cfl * dx / speed)))
    dt = revolutions / steps
    return Case(n, n, dx, dy, np.ascontiguousarray(ls), np.ascontiguousarray(u), np.ascontiguousarray(v),
                dt=dt, steps=steps, bc_u=("neumann",) * 4, bc_v=("neumann",) * 4, bc_p=("neumann",) * 4,
                meta=dict(seed=seed, a=a.tolist(), psi=psi.tolist()))


def droplet(n: int = 256, seed: int = 0, rho_ratio: float = 1000.0, mu_ratio: float = 100.0,
            radius=(0.1, 0.2), sigma: float = 0.0728, g: float = 9.8, ny: int | None = None) -> Case:
    """Two-phase droplet on [0,1] x [0, ny/n] with no-slip walls: U/V
    Dirichlet 0, pressure Neumann (the reference's MAC drivers, e.g.
    test_mac2d_large.cpp:423-425).  phi > 0 is the heavy fluid (droplet)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ny = n if ny is None else ny
    dx = dy = 1.0 / n
    lx, ly = 1.0, ny * dy
    r = rng.uniform(*radius)
    cx = rng.uniform(0.25, lx - 0.25)
    cy = rng.uniform(0.25, ly - 0.25) if ly > 0.5 else 0.5 * ly
    X, Y = _centres(n, ny, dx, dy)
    ls = r - np.sqrt((X - cx) ** 2 + (Y - cy) ** 2)
    u = np.zeros_like(ls)
    v = np.zeros_like(ls)
    fluid = dict(rho_h=1000.0, rho_l=1000.0 / rho_ratio, mu_h=1.0e-3, mu_l=1.0e-3 / mu_ratio,
                 sigma=sigma, g=g, g_axis=1, fix_gravity=0, time_order=2, cfl=0.5)
    return Case(n, ny, dx, dy, np.ascontiguousarray(ls), u, v, bc_u=("dirichlet",) * 4,
                bc_v=("dirichlet",) * 4, bc_p=("neumann",) * 4, fluid=fluid,
                meta=dict(seed=seed, radius=r, centre=(cx, cy)))


def zalesak(n: int = 100) -> Case:
    """Zalesak's slotted disk in rigid rotation, the reference's level-set
    driver (test_levelset2d_large.cpp:1339-1485): 100 x 100 cells of size 1,
    disk of radius 15 at (50, 75) with a slot 7.5 wide reaching y = 82.5,
    phi = +2 inside / -2 outside (0 on the circle), sampled at the cell
    corners x = i, y = j; velocity (pi/314)(50 - y, x - 50) at the cell centres
    of the whole padded grid; dt = 1 and 629 steps (one revolution takes
    628); Neumann sides.  The reference reinitialises (Reinit_Original_2D)
    before the first step and after every step."""
    if n != 100:
        raise ValueError("the reference's slotted disk is defined on 100 x 100 unit cells")
    dx = dy = 1.0
    I = np.arange(n + 6)[:, None]
    J = np.arange(n + 6)[None, :]
    xc, yc = (I + 0.5 - 3) * dx, (J + 0.5 - 3) * dy
    u = np.ascontiguousarray(np.broadcast_to((np.pi / 314.0) * (50.0 - yc), (n + 6, n + 6)))
    v = np.ascontiguousarray(np.broadcast_to((np.pi / 314.0) * (xc - 50.0), (n + 6, n + 6)))
    x, y = (I - 3) * dx + 0.0 * J, (J - 3) * dy + 0.0 * I
    d = np.sqrt((x - 50.0) ** 2 + (y - 75.0) ** 2) - 15.0
    ls = np.where(d < 0, 2.0, np.where(d == 0, 0.0, -2.0))
    ls[(x >= 50 - 0.25 * 15.0) & (x <= 50 + 0.25 * 15.0) & (y <= 75 + 7.5)] = -2.0
    inner = np.zeros_like(ls, dtype=bool)
    inner[3:-3, 3:-3] = True
    ls = np.ascontiguousarray(np.where(inner, ls, -2.0))
    return Case(n, n, dx, dy, ls, u, v, dt=1.0, steps=629, bc_u=("neumann",) * 4, bc_v=("neumann",) * 4,
                bc_p=("neumann",) * 4, meta=dict(radius=15.0, centre=(50.0, 75.0), slot=7.5))


def axisym_bubble(nr: int = 64, nz: int = 128) -> Case:
    """An air bubble at rest in water on the axisymmetric (r, z) grid, the
    configuration of the reference's stationary-bubble driver
    (test_mac2d_large.cpp:1346-1420, 0.02 x 0.04 m, R = 5 mm at z = 0.02 m):
    density 1000 / 1.226, viscosity 1.137e-3 / 1.78e-5, sigma 0.0728, no
    gravity; U/V axisym-wall-Neumann-Neumann, pressure axisym-wall-Neumann-
    outlet, the level set's own sides axisym-lsfree-lsfree-lsfree
    (meta["bc_ls"]).  x is r, y is z; phi > 0 is the water (heavy)."""
    lr, lz, R, zc = 0.02, 0.04, 0.005, 0.02
    dr, dz = lr / nr, lz / nz
    r = (np.arange(nr + 6)[:, None] - 3 + 0.5) * dr
    z = (np.arange(nz + 6)[None, :] - 3 + 0.5) * dz
    ls = np.ascontiguousarray(np.sqrt(r ** 2 + (z - zc) ** 2) - R)
    u = np.zeros_like(ls)
    v = np.zeros_like(ls)
    fluid = dict(rho_h=1000.0, rho_l=1.226, mu_h=1.137e-3, mu_l=1.78e-5, sigma=0.0728, g=0.0, g_axis=1,
                 fix_gravity=0, time_order=0, cfl=0.5)
    bu = ("axisym", "wall", "neumann", "neumann")
    # the driver's first dt (cfl min(dr, dz) / U with U = 1; its UpdateDt of a fluid at rest is unbounded)
    return Case(nr, nz, dr, dz, ls, u, v, dt=0.5 * min(dr, dz), bc_u=bu, bc_v=bu,
                bc_p=("axisym", "wall", "neumann", "outlet"), fluid=fluid,
                meta=dict(bc_ls=("axisym", "lsfree", "lsfree", "lsfree"), radius=R, centre=(0.0, zc)))


def droplet_batch(count: int = 256, seed: int = 0, sides=tuple(range(64, 513, 32))) -> list:
    """Uneven batch: per-droplet grid side from ``sides``, radius in
    [0.08, 0.2], density ratio log-uniform in [1, 1000] and viscosity ratio
    log-uniform in [1, 100]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for k in range(count):
        n = int(rng.choice(sides))
        rr = float(10 ** rng.uniform(0.0, 3.0))
        mr = float(10 ** rng.uniform(0.0, 2.0))
        out.append(droplet(n, seed=int(rng.integers(1 << 31)), rho_ratio=rr, mu_ratio=mr, radius=(0.08, 0.2)))
    return out


def multi_droplet(n: int = 256, seed: int = 0, count: int = 3, rho_ratio: float = 1000.0, mu_ratio: float = 100.0,
                  radius=(0.05, 0.15), sigma: float = 0.0728, g: float = 9.8) -> Case:
    """Several droplets on [0,1]^2 (no-slip walls, Neumann pressure): phi is
    the largest of the droplets' signed distances r_k - |x - c_k| (heavy
    inside any droplet); centres at least a radius plus 0.05 from the walls."""
    rng = np.random.Generator(np.random.PCG64(seed))
    dx = dy = 1.0 / n
    X, Y = _centres(n, n, dx, dy)
    ls = np.full_like(X, -np.inf)
    drops = []
    for _ in range(count):
        r = rng.uniform(*radius)
        cx, cy = rng.uniform(r + 0.05, 0.95 - r, size=2)
        ls = np.maximum(ls, r - np.sqrt((X - cx) ** 2 + (Y - cy) ** 2))
        drops.append((r, cx, cy))
    u = np.zeros_like(ls)
    fluid = dict(rho_h=1000.0, rho_l=1000.0 / rho_ratio, mu_h=1.0e-3, mu_l=1.0e-3 / mu_ratio,
                 sigma=sigma, g=g, g_axis=1, fix_gravity=0, time_order=2, cfl=0.5)
    return Case(n, n, dx, dy, np.ascontiguousarray(ls), u, u.copy(), bc_u=("dirichlet",) * 4,
                bc_v=("dirichlet",) * 4, bc_p=("neumann",) * 4, fluid=fluid, meta=dict(seed=seed, drops=drops))


def smooth_field(n: int, ny: int, rng, modes: int = 6, amplitude: float = 10.0) -> np.ndarray:
    """A random smooth padded (n+6) x (ny+6) field: a sum of Fourier modes
    with random wave numbers up to 2*modes, amplitudes decaying with the
    wave number."""
    X = (np.arange(n + 6) - 2.5) / n
    Y = (np.arange(ny + 6) - 2.5) / ny
    f = np.zeros((n + 6, ny + 6))
    for _ in range(modes):
        kx, ky = rng.integers(1, 2 * modes + 1, size=2)
        a = amplitude * rng.normal() / np.hypot(kx, ky)
        px, py = rng.uniform(0, 2 * np.pi, size=2)
        f += a * np.outer(np.cos(np.pi * kx * X + px), np.cos(np.pi * ky * Y + py))
    return f

