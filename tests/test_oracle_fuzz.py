"""CPU: randomised configurations through the C restatement and the reference
compiled unmodified (oracle/_ref), bit for bit.

The golden fixtures and the named live tests pin the restatement on a few
hand-picked boundary sets, grids and fluids.  Here hypothesis draws them:
grid sizes and spacings, the boundary kind of every side of the U, V and P
grids with their constants, the two fluids, gravity, surface tension, the
time order and the reinitialisation mode; each drawn case runs through both
implementations.  The draws are derandomised (the same cases on every run),
so a failure reproduces; hypothesis prints the failing case.

Properties: ghost fills; the building blocks one by one; all five
reinitialisations; the captured GFM system with the reference's CG and
BiCGStab iterates; whole droplet steps; the axisymmetric functions and whole
axisymmetric driver steps; and two properties of the operators the GPU
solvers rely on (the 2D GFM operator is symmetric bit for bit, the
axisymmetric one up to a few ulps at interface-crossing faces).

What the restatement corrects on purpose is kept out of the draws: the
all-Neumann pressure pin (the reference's CSR is mis-indexed), periodic
pressure (the product refuses it) and the V-gravity fix (off, as in the
reference).  The spacings are derived as the reference derives them, length
over cell count.
"""
import numpy as np
import pytest

hyp = pytest.importorskip("hypothesis")
from hypothesis import HealthCheck, given, settings  # noqa: E402
from hypothesis import strategies as st  # noqa: E402

from oracle.pyoracle import AxiReference, FluidSpec, GridSpec, Oracle, Reference, have_reference  # noqa: E402
from tests.helpers import assert_bitexact  # noqa: E402

pytestmark = pytest.mark.skipif(not have_reference(), reason="reference build (oracle/_ref) not present")

O = Oracle()

KINDS_UV = ("periodic", "neumann", "dirichlet", "axisym", "wall", "inlet", "outlet")
KINDS_P = KINDS_UV + ("pressure", "lsfree")
# pressure kinds the GFM assembly accepts; the Dirichlet group holds the
# pressure level where the reference's operator is well posed
P_SOLVED = ("neumann", "dirichlet", "wall", "inlet", "outlet", "pressure")
P_DIRICHLET = ("dirichlet", "inlet", "outlet", "pressure")

FUZZ = settings(max_examples=80, deadline=None, derandomize=True, print_blob=True,
                suppress_health_check=[HealthCheck.too_slow, HealthCheck.data_too_large,
                                       HealthCheck.function_scoped_fixture])


def same(a, b, what):
    """Bit-exact, NaN equal to NaN (ghost cells the reference leaves as 0 / 0
    compare equal when both produce them)."""
    if not np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True):
        assert_bitexact(a, b, what)


consts = st.tuples(*[st.floats(-0.5, 0.5, allow_nan=False, width=64)] * 4)
sides_uv = st.tuples(*[st.sampled_from(KINDS_UV)] * 4)


@st.composite
def p_sides(draw, solved=True):
    """Four pressure kinds; with `solved`, no periodic side and at least one
    side of the Dirichlet group."""
    if not solved:
        return draw(st.tuples(*[st.sampled_from(KINDS_P)] * 4))
    k = list(draw(st.tuples(*[st.sampled_from(P_SOLVED)] * 4)))
    if not any(x in P_DIRICHLET for x in k):
        k[draw(st.integers(0, 3))] = draw(st.sampled_from(P_DIRICHLET))
    return tuple(k)


@st.composite
def fluids(draw, axisym=False):
    rho_h = draw(st.sampled_from((1000.0, 1.0, 10.0)))
    rho_l = draw(st.sampled_from((1.226, 1.0, 100.0)))
    mu_h = draw(st.sampled_from((1.0e-3, 1.0e-2, 1.0)))
    mu_l = draw(st.sampled_from((1.78e-5, 1.0e-3, 1.0)))
    sigma = draw(st.sampled_from((0.0, 0.0728, 1.0)))
    g = draw(st.sampled_from((0.0, 9.8)))
    g_axis = draw(st.integers(0, 1))
    order = 2 if axisym else draw(st.integers(0, 2))
    return FluidSpec(rho_h=rho_h, rho_l=rho_l, mu_h=mu_h, mu_l=mu_l, sigma=sigma, g=g, g_axis=g_axis,
                     fix_gravity=0, time_order=order, cfl=draw(st.sampled_from((0.3, 0.5))))


def drop_fields(nx, ny, dx, dy, seed, base_x=0.0):
    """A perturbed circular drop and a smooth velocity field on the padded
    grid, drawn from `seed`."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lx, ly = nx * dx, ny * dy
    x = base_x + (np.arange(nx + 6)[:, None] - 3 + 0.5) * dx
    y = (np.arange(ny + 6)[None, :] - 3 + 0.5) * dy
    cx = base_x + rng.uniform(0.3, 0.7) * lx
    cy = rng.uniform(0.3, 0.7) * ly
    r = rng.uniform(0.15, 0.3) * min(lx, ly)
    ls = r - np.sqrt((x - cx) ** 2 + (y - cy) ** 2) + 0.01 * r * rng.standard_normal((nx + 6, ny + 6))
    a, b, p, q = rng.uniform(-0.3, 0.3, 4)
    u = a * np.sin(2 * np.pi * y / ly + p) + 0.01 * rng.standard_normal(ls.shape)
    v = b * np.cos(2 * np.pi * x / lx + q) + 0.01 * rng.standard_normal(ls.shape)
    c = np.ascontiguousarray
    return c(ls), c(u), c(v)


@FUZZ
@given(nx=st.integers(4, 18), ny=st.integers(4, 18), bu=sides_uv, bv=sides_uv, bp=p_sides(solved=False),
       cu=consts, cv=consts, cp=consts, seed=st.integers(0, 2 ** 31 - 1))
def test_boundary_fills_fuzz(nx, ny, bu, bv, bp, cu, cv, cp, seed):
    """ApplyBC_{U,V,P}_2D (src/bc2d.cpp:123-934) of any kind on any side, any
    grid from 4 x 4, against the reference's own fills."""
    g = GridSpec(nx, ny, 1.0 / nx, 1.0 / ny, bc_u=bu, bc_v=bv, bc_p=bp, cu=cu, cv=cv, cp=cp)
    R = Reference(g)
    rng = np.random.Generator(np.random.PCG64(seed))
    try:
        for kind in ("u", "v", "p"):
            a = np.ascontiguousarray(rng.standard_normal(g.shape))
            same(O.bc(g, kind, a.copy()), R.bc(kind, a.copy()), f"{kind} fill {bu, bv, bp}")
    finally:
        R.close()


@FUZZ
@given(nx=st.integers(8, 24), ny=st.integers(8, 24), square=st.booleans(), bu=sides_uv, bv=sides_uv,
       bp=p_sides(), cu=consts, cv=consts, cp=consts, f=fluids(), mode=st.sampled_from((0, 1, 2, 4)),
       seed=st.integers(0, 2 ** 31 - 1))
def test_droplet_steps_fuzz(capfd, nx, ny, square, bu, bv, bp, cu, cv, cp, f, mode, seed):
    """Two whole steps of the reference's MAC driver loop
    (test_mac2d_large.cpp:496-552: advection, reinitialisation, curvature,
    Heaviside, intermediate velocity, SolvePoisson with its CG, UpdateVel,
    UpdateDt) through the reference's own objects and through the oracle's
    composed step: level set, u, v, ps and dt bit for bit on drawn grids,
    boundary sets, fluids, time orders and reinitialisation modes."""
    from tests.test_oracle import live_droplet_steps
    # the spacings as the reference derives them: length / cell count
    lx, ly = 1.0, (ny / nx if square else 1.0)
    dx, dy = lx / nx, ly / ny
    g = GridSpec(nx, ny, dx, dy, bc_u=bu, bc_v=bv, bc_p=bp, cu=cu, cv=cv, cp=cp)
    ls, u, v = drop_fields(nx, ny, dx, dy, seed)
    live_droplet_steps(g, f, ls, u, v, mode, steps=2, equal=same, len_x=lx, len_y=ly)
    capfd.readouterr()


AXI_P = ("neumann", "dirichlet", "wall", "inlet", "outlet", "pressure", "axisym")


@FUZZ
@given(nr=st.integers(6, 16), nz=st.integers(8, 20), base=st.sampled_from((0.0, 0.05, 0.1)), bu=sides_uv,
       bv=sides_uv, bp=st.tuples(*[st.sampled_from(AXI_P)] * 4), cu=consts, cv=consts, cp=consts,
       f=fluids(axisym=True), seed=st.integers(0, 2 ** 31 - 1))
def test_axisym_functions_fuzz(capfd, nr, nz, base, bu, bv, bp, cu, cv, cp, f, seed):
    """MACSolver2DAxisym (src/mac2dAxisym.cpp) function by function --
    curvature, viscous terms, right sides, the implicit uhat / vhat (Thomas
    per line), both divergences, the r-weighted GFM system, UpdateVel and
    UpdateDt -- on drawn grids, axis offsets, boundary sets and fluids,
    against the reference's own class."""
    from tests.test_oracle_axisym import compare, oracle_outputs, reference_outputs
    lr, lz = 0.5, 1.0
    dr, dz = lr / nr, lz / nz
    g = GridSpec(nr, nz, dr, dz, bc_u=bu, bc_v=bv, bc_p=bp, cu=cu, cv=cv, cp=cp)
    ls, u, v = drop_fields(nr, nz, dr, dz, seed, base_x=base)
    ps = np.ascontiguousarray(1.0e-3 * np.random.Generator(np.random.PCG64(seed + 1)).standard_normal(ls.shape))
    dt = 1.0e-3
    ref = reference_outputs(g, f, base, ls, u, v, ps, dt, len_r=lr, len_z=lz)
    capfd.readouterr()  # GetUHat's debug line per z row
    out = oracle_outputs(g, f, base, ls, u, v, ps, dt)
    compare(g, out, lambda k: ref[k], f"axisym {bu, bv, bp} base {base}")


@FUZZ
@given(nx=st.integers(6, 20), ny=st.integers(6, 20), bp=p_sides(), cp=consts, f=fluids(),
       its=st.sampled_from((1, 2, 5, 12)), seed=st.integers(0, 2 ** 31 - 1))
def test_gfm_system_and_reference_solvers_fuzz(capfd, nx, ny, bp, cp, f, its, seed):
    """SolvePoisson's GFM system (src/mac2d.cpp:1300-1660, captured before the
    solve) equals the oracle's assembly entry by entry, CSR structure
    included, and the reference's own CG and BiCGStab (src/poisson2d.cpp,
    BiCGStab with its rho_2 that is never updated) equal the oracle's
    reference iterations after `its` iterations, on drawn grids, Dirichlet-
    group pressure boundaries, constants and fluids."""
    lx, ly = 1.0, 1.0
    dx, dy = lx / nx, ly / ny
    g = GridSpec(nx, ny, dx, dy, bc_p=bp, cp=cp)
    ls, u, v = drop_fields(nx, ny, dx, dy, seed)
    rng = np.random.Generator(np.random.PCG64(seed + 7))
    div = np.ascontiguousarray(rng.standard_normal(g.shape))
    dt = 2.0e-4
    R = Reference(g, f, len_x=lx, len_y=ly)
    try:
        R.bc("P", ls, which=1)
        H, _ = R.heaviside(ls)
        k = R.kappa(ls)
        R.set_state(u, v, g.zeros(), dt)
        R.set_kappa(k.copy())
        _, (a, ia, ja, b) = R.poisson_capture(div, ls, ls, H, maxiter=0)
        kap = k.copy()
        sysd = O.gfm_assemble(g, f, dt, ls, kap, H, div, recompute_kappa=True)
        a2, ia2, ja2, b2 = O.gfm_to_csr(g, sysd)
        assert np.array_equal(ia2, ia) and np.array_equal(ja2, ja), "CSR structure"
        same(a2, a, "CSR values")
        same(b2, b, "right-hand side")
        rhs = g.zeros()
        rhs[3:-3, 3:-3] = b.reshape(ny, nx).T
        mdiag = np.array([a[ia[r]:ia[r + 1]][ja[ia[r]:ia[r + 1]] == r][0] for r in range(len(ia) - 1)])
        x, _, _, _ = O.pcg(g, sysd, tol=1e-6, maxit=its, mode=1)
        same(O.scatter(g, x)[3:-3, 3:-3], R.cg(rhs, (a, ia, ja), mdiag, its)[3:-3, 3:-3], f"CG, {its} its")
        x, _, _, _ = O.bicgstab(g, sysd, tol=1e-6, maxit=its, mode=1)
        same(O.scatter(g, x)[3:-3, 3:-3], R.bicgstab(rhs, (a, ia, ja), mdiag, its)[3:-3, 3:-3],
             f"BiCGStab, {its} its")
    finally:
        R.close()
    capfd.readouterr()


@FUZZ
@given(nx=st.integers(6, 28), ny=st.integers(6, 28), bp=st.tuples(*[st.sampled_from(KINDS_P)] * 4),
       mode=st.sampled_from((0, 1, 2, 3, 4)), atime=st.sampled_from((0.0, 1.0, 5.0)),
       shape=st.sampled_from(("drop", "sign", "scaled")), seed=st.integers(0, 2 ** 31 - 1))
def test_reinitialisation_fuzz(nx, ny, bp, mode, atime, shape, seed):
    """Every reinitialisation of LevelSetSolver2D (src/levelset2d.cpp:
    Reinit_Original_2D, Reinit_Sussman_2D, Reinit_MinRK2_2D,
    FirstTimeOnlyReinit_Sussman_2D and MinRK2 with the Sussman constraint)
    over its pseudo-time (the default or a drawn maximum), from a distance
    function, a sign field or a distance far from unit gradient, with every
    P-grid boundary kind on any side, against the reference's own solver."""
    lx, ly = 1.0, 1.0
    dx, dy = lx / nx, ly / ny
    g = GridSpec(nx, ny, dx, dy, bc_p=bp)
    ls, _, _ = drop_fields(nx, ny, dx, dy, seed)
    if shape == "sign":
        ls = np.ascontiguousarray(np.sign(ls))
    elif shape == "scaled":
        x = (np.arange(nx + 6)[:, None] - 3 + 0.5) * dx
        ls = np.ascontiguousarray(ls * ((x - 0.3) ** 2 + 0.1))
    a, b = ls.copy(), ls.copy()
    O.bc(g, "p", a)
    O.reinit(g, mode, a, atime)
    R = Reference(g, len_x=lx, len_y=ly, ls_max_atime=atime)
    try:
        R.bc("p", b)
        R.reinit(mode, b)
    finally:
        R.close()
    same(a, b, f"reinitialisation mode {mode}, {shape}, {bp}")


AXI_P_DIRICHLET = ("dirichlet", "inlet", "outlet", "pressure")


@st.composite
def axi_p_sides(draw):
    """Pressure kinds of the axisymmetric assembly with at least one side of
    its Dirichlet group (no pinned all-Neumann system)."""
    k = list(draw(st.tuples(*[st.sampled_from(AXI_P)] * 4)))
    if not any(x in AXI_P_DIRICHLET for x in k):
        k[draw(st.integers(0, 3))] = draw(st.sampled_from(AXI_P_DIRICHLET))
    return tuple(k)


@FUZZ
@given(nr=st.integers(8, 20), nz=st.integers(8, 24), base=st.sampled_from((0.0, 0.05)), bu=sides_uv, bv=sides_uv,
       bp=axi_p_sides(), bl=st.tuples(*[st.sampled_from(KINDS_P)] * 4), cu=consts, cv=consts, cp=consts,
       f=fluids(axisym=True), mode=st.sampled_from((0, 2, 4)), seed=st.integers(0, 2 ** 31 - 1))
def test_axisym_driver_steps_fuzz(capfd, nr, nz, base, bu, bv, bp, bl, cu, cv, cp, f, mode, seed):
    """Two whole steps of the reference's axisymmetric driver loop (the level
    set on its own P-grid kinds, MACSolver2DAxisym with SolvePoisson's CG)
    against the oracle's composed step, bit for bit, on drawn grids, axis
    offsets, boundary sets of all four grids, fluids and reinitialisations."""
    from tests.test_oracle_axisym import live_axi_steps
    lr, lz = 0.5, 1.0
    dr, dz = lr / nr, lz / nz
    g = GridSpec(nr, nz, dr, dz, bc_u=bu, bc_v=bv, bc_p=bp, cu=cu, cv=cv, cp=cp)
    lg = GridSpec(nr, nz, dr, dz, bc_u=bu, bc_v=bv, bc_p=bl)
    ls, u, v = drop_fields(nr, nz, dr, dz, seed, base_x=base)
    O.bc(lg, "p", ls)
    O.bc(g, "u", u)
    O.bc(g, "v", v)
    live_axi_steps(g, lg, f, ls, u, v, steps=2, mode=mode, base_r=base, equal=same, len_r=lr, len_z=lz)
    capfd.readouterr()


@FUZZ
@given(nx=st.integers(6, 28), ny=st.integers(6, 28), bp=p_sides(), cp=consts, f=fluids(),
       seed=st.integers(0, 2 ** 31 - 1))
def test_gfm_operator_is_symmetric(nx, ny, bp, cp, f, seed):
    """The 2D GFM operator (whose entries equal the reference's bit for bit,
    test_gfm_system_and_reference_solvers_fuzz) is exactly symmetric: the
    west coupling of every cell equals the east coupling of its west
    neighbour and the south coupling the north one, bit for bit.  The GPU
    solvers therefore store each face once (east / north) without changing
    the operator."""
    g = GridSpec(nx, ny, 1.0 / nx, 1.0 / ny, bc_p=bp, cp=cp)
    ls, _, _ = drop_fields(nx, ny, g.dx, g.dy, seed)
    O.bc(g, "p", ls)
    H, kap = O.heaviside(g, ls), O.kappa(g, ls)
    div = np.ascontiguousarray(np.random.Generator(np.random.PCG64(seed)).standard_normal(g.shape))
    s = O.gfm_assemble(g, f, 1.0e-3, ls, kap, H, div, recompute_kappa=True)
    cw, ce, cs, cn = (s[k].reshape(ny, nx) for k in ("cw", "ce", "cs", "cn"))
    assert np.array_equal(cw[:, 1:], ce[:, :-1]), "west/east couplings"
    assert np.array_equal(cs[1:, :], cn[:-1, :]), "south/north couplings"


@FUZZ
@given(nr=st.integers(6, 28), nz=st.integers(6, 28), base=st.sampled_from((0.0, 0.05, 0.1)), bp=axi_p_sides(),
       cp=consts, sigma=st.sampled_from((0.0, 0.0728, 1.0)), seed=st.integers(0, 2 ** 31 - 1))
def test_axisym_operator_asymmetry_is_rounding_at_crossing_faces(nr, nz, base, bp, cp, sigma, seed):
    """The r-weighted GFM operator of MACSolver2DAxisym (entries equal to the
    reference's, test_axisym_functions_fuzz) is symmetric except at faces the
    interface crosses, where the two cells interpolate the face radius in
    different orders: there the two couplings differ by at most a few ulps
    (relative 1e-15).  That is the whole difference between the reference's
    operator and the once-per-face storage of the GPU solvers."""
    g = GridSpec(nr, nz, 0.5 / nr, 1.0 / nz, bc_p=bp, cp=cp)
    f = FluidSpec(rho_h=1000.0, rho_l=1.226, sigma=sigma)
    ls, _, _ = drop_fields(nr, nz, g.dx, g.dy, seed, base_x=base)
    O.bc(g, "p", ls)
    H = np.ascontiguousarray((ls >= 0.0).astype(np.float64))
    kap = O.axi_kappa(g, base, ls)
    div = np.ascontiguousarray(np.random.Generator(np.random.PCG64(seed)).standard_normal(g.shape))
    s = O.axi_assemble(g, f, base, 1.0e-3, ls, kap, H, div, recompute_kappa=True)
    cw, ce, cs, cn = (s[k].reshape(nz, nr) for k in ("cw", "ce", "cs", "cn"))
    heavy = ls[3:-3, 3:-3].T >= 0.0  # (z, r)
    for d, ref, cross in ((cw[:, 1:] - ce[:, :-1], ce[:, :-1], heavy[:, 1:] != heavy[:, :-1]),
                          (cs[1:, :] - cn[:-1, :], cn[:-1, :], heavy[1:, :] != heavy[:-1, :])):
        assert not np.any((d != 0) & ~cross), "asymmetry away from the interface"
        assert np.all(np.abs(d) <= 1e-15 * np.abs(ref)), float(np.max(np.abs(d) / np.maximum(np.abs(ref), 1e-300)))


@FUZZ
@given(nx=st.integers(5, 26), ny=st.integers(5, 26), bp=st.tuples(*[st.sampled_from(KINDS_P)] * 4),
       bu=sides_uv, bv=sides_uv, f=fluids(), shape=st.sampled_from(("drop", "sign", "noise")),
       seed=st.integers(0, 2 ** 31 - 1))
def test_building_blocks_fuzz(capfd, nx, ny, bp, bu, bv, f, shape, seed):
    """The building blocks one by one on drawn grids, boundary sets and fields
    (a drop, a sign field with its ties, plain noise): the WENO5 right side
    and its 1D kernel (levelset2d.cpp:88-262), the subcell and plain ENO
    Godunov gradients (:560-785), the Sussman constraint and the Heaviside
    derivative (:27-41, :787-893), the smoothed sign (:914-923), the
    curvature and UpdateNTK (mac2d.cpp:124-252), both Heavisides (:87-122),
    convection and viscosity (:308-1041), the divergence (:1729-1738) and
    UpdateDt (:1851-1880), against the reference's own classes."""
    lx, ly = 1.0, 1.0
    dx, dy = lx / nx, ly / ny
    g = GridSpec(nx, ny, dx, dy, bc_u=bu, bc_v=bv, bc_p=bp)
    ls, u, v = drop_fields(nx, ny, dx, dy, seed)
    rng = np.random.Generator(np.random.PCG64(seed + 3))
    if shape == "sign":
        ls = np.ascontiguousarray(np.sign(ls))
    elif shape == "noise":
        ls = np.ascontiguousarray(rng.standard_normal(ls.shape))
    ls0 = np.ascontiguousarray(ls + 0.01 * rng.standard_normal(ls.shape))
    R = Reference(g, f, len_x=lx, len_y=ly)
    try:
        # every call gets its own copies: the functions fill ghost cells of
        # their inputs in place, and some fills are not idempotent
        k = lambda a: a.copy()
        same(O.ls_weno_rhs(g, k(ls), u, v), R.ls_weno_rhs(k(ls), u, v), "HJWENO5_LS_2D")
        F = rng.standard_normal(nx + 6)
        for a, b in zip(O.unit_weno5(F, dx, nx), R.unit_weno5(F, dx, nx)):
            same(a, b, "UnitHJWENO5")
        same(O.subcell_eno_absgrad(g, k(ls), k(ls0)), R.subcell_eno_absgrad(k(ls), k(ls0)), "SubcellENO_Min_DerivAbsLS_2D")
        same(O.eno_absgrad(g, k(ls), k(ls0)), R.eno_absgrad(k(ls), k(ls0)), "ENO_DerivAbsLS_2D")
        hd = O.heaviside_deriv(g, k(ls0))
        same(hd, R.heaviside_deriv(k(ls0)), "UpdateHeavisideFuncDeriv")
        same(O.sussman_constraint(g, k(ls), k(ls0), k(hd)), R.sussman_constraint(k(ls), k(ls0), k(hd)), "GetSussmanReinitConstraint")
        same(O.smoothed_sign(g, k(ls0)), R.smoothed_sign(k(ls0)), "GetSmoothedSignFunc")
        same(O.kappa(g, k(ls)), R.kappa(k(ls)), "UpdateKappa")
        a = O.ntk(g, k(ls), np.full(g.shape, 7.0), np.full(g.shape, -7.0))
        b = R.ntk(k(ls), np.full(g.shape, 7.0), np.full(g.shape, -7.0))
        same(a[0], b[0], "UpdateNTK x")
        same(a[1], b[1], "UpdateNTK y")
        H, HS = R.heaviside(k(ls))
        same(O.heaviside(g, k(ls)), H, "UpdateHeavisideFunc")
        same(O.smooth_heaviside(g, k(ls)), HS, "UpdateSmoothHeavisideFunc")
        cu, cv = R.conv(k(u), k(v))
        same(O.conv_u(g, k(u), k(v)), cu, "AddConvectionFU")
        same(O.conv_v(g, k(u), k(v)), cv, "AddConvectionFV")
        du, dv = R.visc(k(u), k(v), k(ls), k(HS))
        same(O.visc_u(g, f, k(u), k(v), k(ls), k(HS)), du, "AddViscosityFU")
        same(O.visc_v(g, f, k(u), k(v), k(ls), k(HS)), dv, "AddViscosityFV")
        same(O.divergence(g, k(u), k(v)), R.divergence(k(u), k(v)), "GetDivergence")
        assert O.update_dt(g, f, k(u), k(v)) == R.update_dt(k(u), k(v)), "UpdateDt"
    finally:
        R.close()
    capfd.readouterr()
