/* asd2g: B200 (sm_100a) implementation of the 2D two-phase droplet step of
 * appleparan/ASD2, behind a C ABI.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, returns an
 * int status (0 ok, > 0 not converged, < 0 error; see ASD2G_E*) and never
 * throws.  A session owns one grid's device fields; all work is enqueued on
 * the session's CUDA stream.  Fields use the reference layout: a padded
 * (nx+6) x (ny+6) array of doubles, idx(i,j) = j + (ny+6)*i, three ghost
 * layers, u on west faces and v on south faces (levelset2d.cpp:1048-1050).
 *
 * Reference interfaces replaced (appleparan/ASD2, file:line):
 *   LevelSetSolver2D   include/levelset2d.h:17-87
 *   MACSolver2D        include/mac2d.h:31-168
 *   PoissonSolver2D    include/poisson2d.h:31-61
 *   BoundaryCondition2D include/bc2d.h:20-127
 *   MACSolver2DAxisym  include/mac2dAxisym.h:31-168 (the asd2g_axi_* functions)
 * The C++ classes with those exact signatures live in asd2_b200/dropin/ and
 * are implemented on top of these functions.
 */
#ifndef ASD2G_H_INCLUDED
#define ASD2G_H_INCLUDED
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ASD2G_VERSION 1

/* ---- status codes ---- */
#define ASD2G_OK 0
#define ASD2G_NOT_CONVERGED 1     /* iterative solve hit maxit */
#define ASD2G_E_ARG (-1)          /* invalid argument (size, enum, null) */
#define ASD2G_E_CUDA (-2)         /* CUDA runtime error */
#define ASD2G_E_NOMEM (-3)        /* device (or host) allocation failed */
#define ASD2G_E_UNSUPPORTED (-4)  /* configuration outside the implemented path */
#define ASD2G_E_NONFINITE (-5)    /* NaN/Inf detected (the reference exit(1)s) */
#define ASD2G_E_BREAKDOWN (-6)    /* Krylov breakdown (zero denominator) */
#define ASD2G_E_IO (-7)           /* checkpoint file: open/read/write failed, or not a valid checkpoint */
#define ASD2G_E_INTERNAL (-8)     /* a C++ exception inside the library, caught at the entry point */

/* ---- boundary kinds: same values as enum class BC2D (include/common.h:4) ---- */
enum asd2g_bc {
    ASD2G_BC_PERIODIC = 0, ASD2G_BC_NEUMANN, ASD2G_BC_DIRICHLET, ASD2G_BC_AXISYM, ASD2G_BC_WALL,
    ASD2G_BC_INLET, ASD2G_BC_OUTLET, ASD2G_BC_PRESSURE, ASD2G_BC_LSFREE, ASD2G_BC_CUSTOM
};

/* ---- device fields of a session ---- */
enum asd2g_field {
    ASD2G_LS = 0,   /* level set phi (cell centres; > 0 heavy fluid) */
    ASD2G_U,        /* u on west faces */
    ASD2G_V,        /* v on south faces */
    ASD2G_PS,       /* pseudo pressure ps = p * dt (cell centres) */
    ASD2G_P,        /* pressure p = ps / dt */
    ASD2G_KAPPA,    /* curvature */
    ASD2G_H,        /* sharp Heaviside of phi */
    ASD2G_HS,       /* smoothed Heaviside of phi */
    ASD2G_DIV,      /* divergence of (uhat, vhat) */
    ASD2G_UHAT,     /* intermediate velocity */
    ASD2G_VHAT,
    ASD2G_LSB,      /* phi at the start of the step */
    ASD2G_LS0,      /* phi at the start of reinitialisation (lsInit) */
    ASD2G_W0,       /* general work arrays (padded) usable by callers */
    ASD2G_W1,
    ASD2G_W2,
    ASD2G_W3,
    ASD2G_NFIELDS
};

/* ---- reinitialisation modes ---- */
enum asd2g_reinit {
    ASD2G_REINIT_ORIGINAL = 0,      /* Reinit_Original_2D        levelset2d.cpp:264 */
    ASD2G_REINIT_SUSSMAN = 1,       /* Reinit_Sussman_2D         levelset2d.cpp:318 */
    ASD2G_REINIT_MINRK2 = 2,        /* Reinit_MinRK2_2D          levelset2d.cpp:433 */
    ASD2G_REINIT_FIRSTTIME = 3,     /* FirstTimeOnlyReinit_Sussman_2D levelset2d.cpp:377 */
    ASD2G_REINIT_MINRK2_SUSSMAN = 4 /* MinRK2 subcell steps + Sussman constraint after each */
};

/* ---- pressure solvers ---- */
enum asd2g_solver {
    ASD2G_SOLVER_PCG = 0,          /* Jacobi-PCG, textbook recurrence            */
    ASD2G_SOLVER_PCG_REFERENCE = 1,/* the reference iteration, poisson2d.cpp:285  */
    ASD2G_SOLVER_BICGSTAB = 2,     /* right-Jacobi BiCGStab (rho_2 carried)       */
    ASD2G_SOLVER_BICGSTAB_REFERENCE = 3, /* poisson2d.cpp:403 as written (rho_2 = 1) */
    ASD2G_SOLVER_MGPCG = 4,        /* FP64 flexible CG preconditioned by an FP32 multigrid V-cycle */
    ASD2G_SOLVER_UNET = 5          /* FP64 flexible CG preconditioned by the V-cycle plus a learned
                                      correction (asd2g_set_preconditioner_net), Jacobi-PCG fallback */
};

/* solver_flags bits */
#define ASD2G_FLAG_NO_CLUSTER_PCG 1 /* Jacobi-PCG always as per-iteration kernels (no one-launch or cluster solver) */
#define ASD2G_FLAG_NO_PERSIST_MG 2  /* MG-FCG always as per-phase kernels (no one-launch solve) */

/* precision (no reference counterpart: the reference is FP64 throughout) */
#define ASD2G_PRECISION_FP64 0  /* every field and kernel in FP64 (the drop-in) */
#define ASD2G_PRECISION_MIXED 1 /* level-set advection + reinitialisation in FP32 (FP64 fields stay
                                   the interface); momentum, GFM assembly and projection in FP64;
                                   pressure with ASD2G_SOLVER_MGPCG is FP32 inside, FP64 outside.
                                   Needs Neumann/Dirichlet pressure on all sides and reinit mode
                                   0, 2 or 4. */

/* Curvature of the level set (asd2g_params.curvature).
 * ASD2G_CURVATURE_REFERENCE: UpdateKappa (mac2d.cpp:221-252), the expanded
 *   (phi_x^2 phi_yy - 2 phi_x phi_y phi_xy + phi_y^2 phi_xx) / |grad phi|^3
 *   with central differences (the cross term from differenced phi_x).
 * ASD2G_CURVATURE_DIVERGENCE: kappa = div(grad phi / |grad phi|) in
 *   conservative form: normals on the four cell faces (the normal component
 *   from the two cells beside the face, the tangential one from the four
 *   cells around it), differenced across the cell; the same limiter
 *   |kappa| <= 1 / min(dx, dy).  The reference lists better curvature
 *   discretisations as future work (README.md:73). */
enum { ASD2G_CURVATURE_REFERENCE = 0, ASD2G_CURVATURE_DIVERGENCE = 1 };

typedef struct asd2g_params {
    int32_t nx, ny;          /* interior cells (>= 4 each) */
    int32_t nbc;             /* ghost layers: must be 3 (WENO5) */
    int32_t precision;       /* ASD2G_PRECISION_FP64 (the drop-in) or ASD2G_PRECISION_MIXED */
    double base_x, base_y;   /* lower-left corner (base_x is kBaseR of the asd2g_axi_* functions) */
    double dx, dy;           /* cell sizes */
    int32_t bc_u[4], bc_v[4], bc_p[4];      /* asd2g_bc per side, order W, E, S, N */
    double bcc_u[4], bcc_v[4], bcc_p[4];    /* Dirichlet constants per side */
    double rho_h, rho_l, mu_h, mu_l;        /* heavy (phi > 0) and light fluid */
    double sigma, gravity;                  /* surface tension, gravity constant */
    int32_t g_axis;          /* GAXISENUM2D: 0 X, 1 Y */
    int32_t fix_gravity;     /* 0: reproduce mac2d.cpp:294 (V takes AddGravityFU) */
    int32_t time_order;      /* TIMEORDERENUM: 0 Euler, 1 RK2, 2 RK3 */
    int32_t solver_flags;    /* ASD2G_FLAG_* bits (0 = defaults) */
    double cfl;
    double ls_max_atime;     /* reinit pseudo-time; <= 0: 1.5*kThickness (levelset2d.cpp:10) */
    int32_t numbers_given;   /* 1: use re/we/fr below; 0: kRe = rho_h/mu_h, kWe = rho_h/sigma,
                                kFr = 1/gravity (the second MACSolver2D constructor with L = U = 1) */
    int32_t curvature;       /* ASD2G_CURVATURE_*: 0 UpdateKappa's formula (mac2d.cpp:221), 1 the
                                divergence of face normals (no reference counterpart) */
    double re, we, fr;       /* kRe, kWe, kFr of MACSolver2D (mac2d.h:37): viscosity is skipped when
                                kRe <= 0, the curvature is recomputed in the solve when kWe is finite and
                                nonzero, gravity needs kFr finite (mac2d.cpp:598, :1307, :1047) */
} asd2g_params;

typedef struct asd2g_session asd2g_session;

/* Version of this ABI (ASD2G_VERSION). */
int asd2g_version(void);
/* Human-readable text for the last error on this thread. */
const char *asd2g_last_error(void);

/* Create a session on the current CUDA device.  stream: a cudaStream_t, or
 * NULL for a stream owned by the session.  Replaces the constructors
 * LevelSetSolver2D(...) levelset2d.h:19-22, MACSolver2D(...) mac2d.h:75-84,
 * PoissonSolver2D(nx, ny, nbc) poisson2d.h:33. */
int asd2g_create(const asd2g_params *params, void *stream, asd2g_session **out);
int asd2g_destroy(asd2g_session *s);
int asd2g_sync(asd2g_session *s);

/* Device pointer of a field ((nx+6)*(ny+6) doubles). */
int asd2g_field_ptr(asd2g_session *s, int field, double **dptr);
/* Host <-> device copies of a whole padded field (synchronous). */
int asd2g_upload(asd2g_session *s, int field, const double *host);
int asd2g_download(asd2g_session *s, int field, double *host);
/* The same upload queued on the session's stream without waiting for it (no
 * reference counterpart: the reference keeps its fields on the host).  The
 * host buffer must stay valid and unchanged until the session next
 * synchronises (asd2g_sync, a pressure solve, a download); from pinned host
 * memory the copy overlaps the host's next calls. */
int asd2g_upload_async(asd2g_session *s, int field, const double *host);
/* Staged copies on the session's own copy stream, for callers that overlap
 * the transfers of one step with the computation of another (no reference
 * counterpart).  Each staged copy first waits for the compute work enqueued
 * on the session so far (so it never overwrites a field an earlier call
 * still reads, nor reads one an earlier call still writes) and then runs
 * beside later compute calls.  asd2g_join_copies(s, which) makes the compute
 * work enqueued after it wait for the staged uploads (which = 1), downloads
 * (2) or both (3) issued so far; call it before the first call that reads an
 * uploaded field or writes a downloaded one.  asd2g_sync_copies waits on the
 * host for every staged copy.  Host buffers: pinned for a truly
 * asynchronous copy, untouched until the copy is known complete. */
int asd2g_upload_staged(asd2g_session *s, int field, const double *host);
int asd2g_download_staged(asd2g_session *s, int field, double *host);
int asd2g_join_copies(asd2g_session *s, int which);
int asd2g_sync_copies(asd2g_session *s);
int asd2g_copy_field(asd2g_session *s, int dst, int src);
int asd2g_fill_field(asd2g_session *s, int field, double value);

/* Ghost fill of one field as a U, V or P grid (kind 'U', 'V', 'P').
 * BoundaryCondition2D::ApplyBC_{U,V,P}_2D, bc2d.cpp:123,239,346. */
int asd2g_apply_bc(asd2g_session *s, int field, char kind);
/* One side (0 W, 1 E, 2 S, 3 N) of that fill.  fill = ASD2G_FILL_CONFIGURED
 * applies the session's boundary kind for that side (BC_UW ... BC_PN,
 * bc2d.cpp:355-573); the other values force one rule (BC_PeriodicUW,
 * BC_NeumannUW, BC_DirichletUW, BC_LSFreeBoundaryPW, ... :575-934) with the
 * session's Dirichlet constant for that side. */
enum asd2g_fill {
    ASD2G_FILL_CONFIGURED = -1, ASD2G_FILL_PERIODIC = 1, ASD2G_FILL_NEUMANN = 2, ASD2G_FILL_DIRICHLET = 3,
    ASD2G_FILL_LSFREE = 4
};
int asd2g_apply_bc_side(asd2g_session *s, int field, char kind, int side, int fill);

/* ---- level set (levelset2d.cpp) ---- */
/* Solve_LevelSet_2D(LS, U, V, dt): TVD-RK3 + HJ-WENO5, levelset2d.cpp:43. */
int asd2g_ls_advect(asd2g_session *s, double dt);
/* HJWENO5_LS_2D(ls, uc, vc) -> out (cell-centred velocities), :88.  Applies
 * the P boundary to ls first, as the reference does. */
int asd2g_ls_weno_rhs(asd2g_session *s, int ls, int uc, int vc, int out);
/* Reinitialise LS in place (asd2g_reinit mode). */
int asd2g_reinit(asd2g_session *s, int mode);
/* Building blocks: SubcellENO_Min_DerivAbsLS_2D :616, ENO_DerivAbsLS_2D :560,
 * GetSussmanReinitConstraint :787, UpdateHeavisideFuncDeriv :27,
 * GetSmoothedSignFunc :914.  All write every cell of out the reference writes
 * and zero the rest (fresh-vector semantics). */
int asd2g_subcell_eno(asd2g_session *s, int ls, int ls0, int out);
int asd2g_eno(asd2g_session *s, int ls, int ls0, int out);
int asd2g_sussman_constraint(asd2g_session *s, int ls, int ls0, int hd, int out);
int asd2g_heaviside_deriv(asd2g_session *s, int ls, int out);
int asd2g_smoothed_sign(asd2g_session *s, int ls, int out);
/* Level-set step: advect (dt) then reinitialise (mode).  In a mixed-precision
 * session both run in FP32 on an FP32 copy of LS (LS is read and written in
 * FP64, ghosts included). */
int asd2g_ls_step(asd2g_session *s, double dt, int reinit_mode);
/* FP64 volume check (no reference counterpart; the reference's tests print
 * the area of phi >= 0, test_levelset2d_large.cpp:106-130): recomputes H and
 * HS from LS and returns sum(H) dx dy and sum(HS) dx dy over the interior. */
int asd2g_volume(asd2g_session *s, double *sharp, double *smooth);
/* The same two integrals for the level set of the last asd2g_droplet_step. */
int asd2g_last_volume(asd2g_session *s, double *sharp, double *smooth);
/* UnitHJWENO5(F, FP, FM, d, n), levelset2d.cpp:159 / mac2d.cpp:465: WENO5
 * one-sided derivatives of the line F[0 .. n+5] (host arrays), written to
 * FP[3 .. n+2] and FM[3 .. n+2].  n + 6 must not exceed (nx+6)*(ny+6). */
int asd2g_weno5_line(asd2g_session *s, const double *F, double *FP, double *FM, double d, int n);
/* HJWENO5_DerivAbsLS_2D(ls, ls0) -> out, levelset2d.cpp:488. */
int asd2g_weno_absgrad(asd2g_session *s, int ls, int ls0, int out);

/* ---- MAC momentum (mac2d.cpp) ---- */
/* UpdateKappa(LS) -> KAPPA interior, mac2d.cpp:221. */
int asd2g_kappa(asd2g_session *s);
/* UpdateHeavisideFunc / UpdateSmoothHeavisideFunc(LS) -> H, HS, :87, :103. */
int asd2g_heaviside(asd2g_session *s);
/* AddConvectionFU/FV(u, v) -> cu, cv (:308, :389). */
int asd2g_convection(asd2g_session *s, int u, int v, int cu, int cv);
/* AddViscosityFU/FV(u, v, ls, h) -> du, dv (:570, :811). */
int asd2g_viscosity(asd2g_session *s, int u, int v, int ls, int h, int du, int dv);
/* UpdateFU/FV(ls, u, v, h) -> fu, fv (:254, :281). */
int asd2g_momentum_rhs(asd2g_session *s, int ls, int u, int v, int h, int fu, int fv);
/* GetIntermediateVel(LS, U, V, UHAT, VHAT, h) with time step dt, :1081.
 * Writes the interior faces of UHAT and VHAT only, as the reference does. */
int asd2g_intermediate_vel(asd2g_session *s, double dt, int h);
/* GetDivergence(u, v) -> div, :1729. */
int asd2g_divergence(asd2g_session *s, int u, int v, int div);
/* UpdateVel(U, V, UHAT, VHAT, PS, LS, H) with KAPPA, :1740; then the U/V
 * boundary fill the reference applies at its end. */
int asd2g_update_vel(asd2g_session *s, double dt);
/* UpdateDt(U, V), :1851. */
int asd2g_update_dt(asd2g_session *s, double *dt);
/* UpdateNTK (mac2d.cpp:124-219) as far as the reference implements it: the
 * unit normal (central differences) at cells where |1 - |grad phi|| <= 1e-4
 * (ENO gradient), written into fields nxf and nyf; other cells untouched. */
int asd2g_update_ntk(asd2g_session *s, int ls, int nxf, int nyf);

/* ---- axisymmetric MAC solver (MACSolver2DAxisym, mac2dAxisym.cpp) ----
 * The session's grid is read as (r, z): x is r (nx = kNr, dx = kDr, base_x =
 * kBaseR), y is z.  Gravity axis 0 is R, 1 is Z (GAXISENUM2DAXISYM).  The
 * convection term, Heaviside, UpdateVel and the pressure solvers are the 2D
 * entry points (the reference's axisymmetric versions are the same
 * arithmetic; asd2g_heaviside, asd2g_update_vel, asd2g_solve_pressure). */
/* UpdateKappa(LS) -> KAPPA interior, mac2dAxisym.cpp:222 (the hoop term
 * uses r = base_x + (i + 1/2) dr). */
int asd2g_axi_kappa(asd2g_session *s);
/* GetRHSU(ls, u, v, h) with time step dt -> out (whole padded array, U ghost
 * fill applied), :264.  Viscosity is skipped when kRe <= 0. */
int asd2g_axi_rhs_u(asd2g_session *s, double dt, int ls, int u, int v, int h, int out);
/* GetRHSV(ls, u, uhat, v, h) -> out (V ghost fill applied), :294. */
int asd2g_axi_rhs_v(asd2g_session *s, double dt, int ls, int u, int uhat, int v, int h, int out);
/* AddExternalViscosityFU(u, v, ls, h) -> du and AddExternalViscosityFV(u,
 * uhat, v, ls, h) -> dv (:590, :755), whole padded arrays (0 off the
 * interior faces, and everywhere when kRe <= 0). */
int asd2g_axi_viscosity(asd2g_session *s, int ls, int u, int uhat, int v, int h, int du, int dv);
/* GetUHat (comp 0, :950) / GetVHat (comp 1, :1231)(ls, rhs, h) with time step
 * dt -> out: the implicit viscous step, one tridiagonal solve per r line and
 * per z line; only the interior faces of out are written (the rest 0, no
 * ghost fill). */
int asd2g_axi_hat(asd2g_session *s, int comp, double dt, int ls, int rhs, int h, int out);
/* GetDivergence4Poisson (for_poisson = 1, :1980) or GetDivergence (0,
 * :1996) of (u, v) -> div (0 outside the interior). */
int asd2g_axi_divergence(asd2g_session *s, int u, int v, int div, int for_poisson);
/* SolvePoisson's assembly (:1488-1916) from LS, KAPPA, H, DIV with time step
 * dt into the session's system (then asd2g_solve_pressure solves it).
 * recompute_kappa: the axisymmetric curvature and its P ghosts first (what
 * SolvePoisson does when kWe is finite and nonzero).  Pressure sides:
 * Neumann, axisym, wall (zero flux), Dirichlet, inlet, outlet, pressure (the
 * constant); periodic is ASD2G_E_UNSUPPORTED.  The Krylov solvers store each
 * face coefficient once (from its east / north cell); the reference's west
 * and south entries of a face crossed by the interface differ from those by
 * rounding (the two cells interpolate the face radius in different orders). */
int asd2g_axi_assemble(asd2g_session *s, double dt, int recompute_kappa);
/* UpdateDt(U, V) with max |KAPPA| in the surface-tension bound, :2104. */
int asd2g_axi_update_dt(asd2g_session *s, double *dt);
/* One step of the axisymmetric driver (tests/LargeTests/test_mac2d_large.cpp
 * :1264-1306): lsB = LS; advect and reinitialise LS (reinit_mode) with the
 * level-set solver's own P-grid kinds ls_bc[4] and constants ls_bcc[4] (NULL:
 * the session's pressure kinds); curvature; H, HS; rhs_u, uhat (U fill);
 * rhs_v, vhat (V fill); the r-weighted divergence; assembly; pressure solve
 * (solver ASD2G_SOLVER_PCG .. ASD2G_SOLVER_MGPCG); projection; next dt.  FP64
 * sessions only.  *dt is the step's dt and receives the next one. */
int asd2g_axi_step(asd2g_session *s, double *dt, int reinit_mode, const int32_t *ls_bc, const double *ls_bcc,
                   int solver, double tol, int maxit, int *iters, double *rel_resid);

/* ---- GFM pressure (mac2d.cpp:1249-1727, poisson2d.cpp) ---- */
/* Assemble the matrix-free GFM system from LS, KAPPA, H, DIV with time step
 * dt.  recompute_kappa: recompute KAPPA from LS and fill its P ghosts first
 * (what SolvePoisson does when kWe is finite and nonzero, :1307-1310). */
int asd2g_assemble_gfm(asd2g_session *s, double dt, int recompute_kappa);
/* Copy the assembled system to the host in the reference's natural order
 * k = i + nx*j: diagonal, west/east/south/north coupling magnitudes (the
 * off-diagonal entries are their negatives) and right-hand side.  Any pointer
 * may be NULL.  *pinned = 1 when cell 0 is held at 0 (all-Neumann pressure). */
int asd2g_get_system(asd2g_session *s, double *diag, double *cw, double *ce, double *cs, double *cn,
                     double *rhs, int *pinned);
/* Solve the assembled system into PS (interior; P ghosts filled), and set
 * P = PS / dt.  tol is on ||b - A x|| / ||b||.  Returns ASD2G_NOT_CONVERGED
 * when maxit is reached.  iters and rel_resid may be NULL; rel_resid is the
 * recurrence residual, except for ASD2G_SOLVER_MGPCG, which confirms
 * convergence by recomputing b - A x in FP64 (restarting if it is above tol)
 * and reports that residual; if it stagnates at FP64 rounding level above
 * tol, the solve ends there with ASD2G_OK and rel_resid > tol. */
int asd2g_solve_pressure(asd2g_session *s, int solver, double tol, int maxit, double dt, int *iters,
                         double *rel_resid);
/* ||b - A x|| / ||b|| of the current PS against the assembled system, in FP64. */
int asd2g_true_residual(asd2g_session *s, double *rel);
/* PoissonSolver2D's CSR interface (poisson2d.cpp:230-575): solve A x = b for
 * a caller-assembled CSR matrix (0-based, host arrays: ia[rows+1], ja/a[nnz])
 * with the Jacobi preconditioner diag (one value per row), from x = 0.
 * solver: ASD2G_SOLVER_PCG, _PCG_REFERENCE, _BICGSTAB or _BICGSTAB_REFERENCE.
 * Column indices outside [0, rows) are skipped.  rows must not exceed nx*ny
 * of the session.  x (host, rows values) receives the solution. */
int asd2g_csr_solve(asd2g_session *s, int solver, int rows, const int *ia, const int *ja, const double *a,
                    const double *diag, const double *b, double *x, double tol, int maxit, int *iters,
                    double *rel_resid);

/* ---- batched GFM pressure solves (no reference counterpart) ----
 * Many independent droplets of uneven grid sizes: each phase of assembly and
 * of the mixed-precision multigrid-preconditioned flexible CG is one kernel
 * launch for the whole batch; every instance has its own solver scalars and
 * stops on its own (same rules as ASD2G_SOLVER_MGPCG).  Instances need
 * Neumann or Dirichlet pressure on all four sides. */
typedef struct asd2g_batch asd2g_batch;
/* params[0 .. count-1]: one per instance (grid, fluid, BCs as for a session). */
int asd2g_batch_create(const asd2g_params *params, int count, void *stream, asd2g_batch **out);
int asd2g_batch_destroy(asd2g_batch *b);
/* Padded (nx+6)*(ny+6) arrays of instance inst: LS, KAPPA, H, DIV (inputs of
 * the assembly), PS, P (outputs of the solve), and for asd2g_batch_step U, V,
 * HS, UHAT, VHAT, LSB, LS0. */
int asd2g_batch_upload(asd2g_batch *b, int inst, int field, const double *host);
int asd2g_batch_download(asd2g_batch *b, int inst, int field, double *host);
/* Device arena of a field (all instances, instance i at offset(i) doubles). */
int asd2g_batch_field_ptr(asd2g_batch *b, int field, void **dptr, size_t *stride_doubles);
int asd2g_batch_offset(asd2g_batch *b, int inst, size_t *offset_doubles);
/* GFM assembly of every instance (KAPPA as uploaded), dt[count]. */
int asd2g_batch_assemble(asd2g_batch *b, const double *dt);
/* Solve every assembled system to the FP64-verified rel. residual tol; PS and
 * P written (P = PS / dt).  iters[count], rel_resid[count] may be NULL.
 * ASD2G_NOT_CONVERGED if any instance reached maxit. */
int asd2g_batch_solve(asd2g_batch *b, double tol, int maxit, int *iters, double *rel_resid);
int asd2g_batch_sync(asd2g_batch *b);
/* The full droplet step of every instance (what asd2g_droplet_step does for
 * one session, with the MG-FCG pressure solve), one kernel launch per phase
 * for the whole batch: level-set advection, reinitialisation (reinit_mode 0,
 * 1, 2 or 4; 1 and 4 with FP64 instances only), curvature, Heaviside, FP64
 * volume check, intermediate velocity,
 * divergence, GFM assembly, batched MG-FCG to tol, projection, next dt.
 * Instances: FP64 or mixed precision (the level-set advection and
 * reinitialisation in FP32, as asd2g_droplet_step of a mixed session does);
 * each keeps its own time order (0, 1, 2) and its own
 * reinitialisation step count (ls_max_atime), the phases running up to the
 * largest and the instances without a phase skipping it.
 * dt[count]: each instance's step dt, replaced by its next dt.  Fields LS, U,
 * V (and the others) are uploaded/downloaded with asd2g_batch_upload/download
 * (LS, U, V, PS, P, KAPPA, H, HS, DIV, UHAT, VHAT, LSB, LS0). */
int asd2g_batch_step(asd2g_batch *b, double *dt, int reinit_mode, double tol, int maxit, int *iters,
                     double *rel_resid);
/* Multigrid tile shape the batch uses (rows x cols cells per tile).  The
 * first asd2g_batch_solve / asd2g_batch_step times four FCG iterations with
 * each candidate shape (16x32, 32x32, 16x64) on the batch's own hierarchy
 * and keeps the fastest; trial_ms[3] (may be NULL) receives those times (0
 * before tuning or when the environment variable ASD2G_MG_TILE=0|1|2 fixes
 * the shape). */
int asd2g_batch_tile_shape(asd2g_batch *b, int *rows, int *cols, float *trial_ms);
/* Volume check of the last batch step per instance: sum H dx dy, sum HS dx dy. */
int asd2g_batch_volume(asd2g_batch *b, double *sharp, double *smooth);

/* ---- learned preconditioner building blocks (no reference counterpart) ----
 * 3x3 "same" convolution on the tcgen05 tensor cores: BF16 NHWC activations
 * (cin a multiple of 16), BF16 packed weights, FP32 accumulation, FP32 bias,
 * optional ReLU; out: BF16 NHWC with cout channels (16, 32, 48, 64, 96, 128 or
 * 192), out32:
 * channel 0 in FP32 (either may be NULL).  All pointers are device memory;
 * err (device int, may be NULL) is set if a tensor-core wait timed out. */
size_t asd2g_conv_wpack_bytes(int cout_pad, int cin_pad);
/* w[cout][cin][3][3] FP32 (device) -> packed BF16 weights, zero-padded. */
int asd2g_conv_pack_weights(const float *w, int cout, int cin, int cout_pad, int cin_pad, void *wpack, void *stream);
int asd2g_conv3x3_bf16(const void *in, int n, int h, int w, int cin, const void *wpack, const float *bias, int cout,
                       void *out, float *out32, int relu, int *err, void *stream);

/* ---- the learned preconditioner (no reference counterpart) ----
 * A 4-level U-Net (16/32/64/128 channels, 15 3x3 convolutions, ReLU, 2x2
 * average pooling, nearest upsampling + skip concatenation); forward and
 * input-gradient convolutions and the weight gradients on the tcgen05
 * tensor cores (BF16, FP32 accumulation), Adam on FP32 master weights.
 * Images: H x W, both multiples of 8.  A forward pass takes B images with
 * B * H * W <= max_batch * max_h * max_w; a training step B <= max_batch
 * images of H * W <= max_h * max_w.
 * feats: device FP32 [B][H][W][4] (vector / RMS, diag / s, ce / s, cn / s);
 * out and target: device FP32 [B][H][W]. */
typedef struct asd2g_unet asd2g_unet;
int asd2g_unet_create(int max_batch, int max_h, int max_w, void *stream, asd2g_unet **out);
int asd2g_unet_destroy(asd2g_unet *u);
size_t asd2g_unet_nparams(asd2g_unet *u);
int asd2g_unet_init(asd2g_unet *u, unsigned long long seed);
/* FP32 host arrays of asd2g_unet_nparams() values (layer by layer: W[cout][cin][3][3], b[cout padded to 16]). */
int asd2g_unet_set_params(asd2g_unet *u, const float *host);
int asd2g_unet_get_params(asd2g_unet *u, float *host);
/* Gradients of the last train step (same layout). */
int asd2g_unet_get_grads(asd2g_unet *u, float *host);
int asd2g_unet_forward(asd2g_unet *u, int B, int H, int W, const float *feats, float *out);
/* One Adam step; *loss_mean = mean over the batch of |out - target|^2 / |target|^2 (may be NULL). */
int asd2g_unet_train_step(asd2g_unet *u, int B, int H, int W, const float *feats, const float *target, float lr,
                          float *loss_mean);
/* One Adam step on the residual loss, mean over samples of 1 - (a.r)^2 /
 * (|a|^2 |r|^2) with r = feats channel 0, a = A out and A the symmetric
 * 5-point operator of feats channels 1..3 (diag, coupling to the next image
 * row, coupling to the next column): the squared relative residual that the
 * best scalar multiple of out leaves.  No target is needed. */
int asd2g_unet_train_step_residual(asd2g_unet *u, int B, int H, int W, const float *feats, float lr,
                                   float *loss_mean);
/* One Adam step on the energy loss, mean over samples of 1 - (out' A t)^2 /
 * ((out' A out)(t' A t)) with t = target and A as above: the squared relative
 * A-norm error that the best scalar multiple of out leaves. */
int asd2g_unet_train_step_energy(asd2g_unet *u, int B, int H, int W, const float *feats, const float *target,
                                 float lr, float *loss_mean);
/* 1 if a tensor-core wait of any launch so far timed out. */
int asd2g_unet_error_flag(asd2g_unet *u, int *flag);
/* Run the network's launches on this stream from now on (NULL: the stream it
 * was created with). */
int asd2g_unet_set_stream(asd2g_unet *u, void *stream);
/* Attach (or detach with NULL) the network used by ASD2G_SOLVER_UNET: nx and
 * ny multiples of 8 and within the network's maximum image size; keep the
 * network alive while attached.  The solve is flexible CG in FP64 with a
 * two-level preconditioner: z_mg = one FP32 V-cycle of r (the multigrid of
 * ASD2G_SOLVER_MGPCG), r1 = r - A z_mg, u = network(features of r1) (BF16 /
 * FP32 inside), z = z_mg + omega u with omega = (u . r1) / (u . Au) in
 * FP64; the network runs on the first application and on every 8th
 * iteration, the V-cycle alone otherwise and after a residual replacement
 * (each new direction is A-orthogonalised against the three before it).
 * Convergence is verified on the FP64 residual as for
 * ASD2G_SOLVER_MGPCG; if it does not converge within min(maxit, 500)
 * iterations the system is solved again by Jacobi-PCG and
 * asd2g_last_fallback reports 1. */
int asd2g_set_preconditioner_net(asd2g_session *s, asd2g_unet *net);
int asd2g_last_fallback(asd2g_session *s, int *used);
/* The same learned preconditioner for a batch (no reference counterpart):
 * the batch copies the network's weights (later changes to net are not seen
 * until it is attached again) and groups its instances by grid size, one
 * network pass per group; every instance needs nx and ny multiples of 8.
 * asd2g_batch_solve_with(b, ASD2G_SOLVER_UNET, ...) then runs the truncated
 * flexible CG above for every instance, each phase one launch for the whole
 * batch, each instance stopping on its own; if any instance has not
 * converged within min(maxit, 500) iterations, the whole batch is solved
 * again by the batched MG-FCG and asd2g_batch_last_fallback reports 1.
 * solver ASD2G_SOLVER_MGPCG is asd2g_batch_solve. */
int asd2g_batch_set_preconditioner_net(asd2g_batch *b, asd2g_unet *net);
int asd2g_batch_solve_with(asd2g_batch *b, int solver, double tol, int maxit, int *iters, double *rel_resid);
int asd2g_batch_last_fallback(asd2g_batch *b, int *used);
/* How the session's last pressure solve ran: *one_launch = 1 when the whole
 * solve was one kernel launch (the thread-block-cluster Jacobi-PCG or the
 * cooperative MG-FCG of systems up to about 256 x 256), 0 when it ran as
 * per-phase kernels.  No reference counterpart (solver introspection). */
int asd2g_last_solve_one_launch(asd2g_session *s, int *one_launch);
/* Training pair of the network from the session's last assembled and solved
 * system (solution x): z = V-cycle(b), r1 = b - A z, e = x - z; feats (device
 * FP32 [nx][ny][4]) = (r1 / rms(r1), diag / s, ce / s, cn / s), target
 * (device FP32 [nx][ny]) = e / rms(e), s = max diag (omega makes the
 * output's scale irrelevant).  The session's solution is left in place. */
int asd2g_pc_training_pair(asd2g_session *s, void *feats, void *target);
/* The same at a later Krylov iterate: x0 = the MG-FCG iterate after `iters`
 * (0..1000) iterations from 0, r = b - A x0 (recurrence), z = V-cycle(r), r1 =
 * r - A z, e = x - x0 - z.  iters = 0 is asd2g_pc_training_pair. */
int asd2g_pc_training_pair_at(asd2g_session *s, int iters, void *feats, void *target);

/* ---- whole step (test_mac2d_large.cpp:496-552) ----
 * lsB = LS; advect; reinit (reinit_mode); kappa; H, HS; intermediate velocity
 * with HS; U/V fill; divergence; GFM assembly; pressure solve; projection;
 * new dt.  *dt is read as the step's dt and receives the next one. */
int asd2g_droplet_step(asd2g_session *s, double *dt, int reinit_mode, int solver, double tol, int maxit,
                       int *iters, double *rel_resid);

/* ---- device-resident multi-step run (no reference counterpart: the
 * driver loop of test_mac2d_large.cpp:496-552 without host round trips) ----
 * nsteps droplet steps as one CUDA graph per step, launched back to back
 * with a single synchronisation at the end: the MG-FCG iterations run in a
 * device-side WHILE loop (graph conditional node) and dt passes from one step
 * to the next on the device.  solver must be ASD2G_SOLVER_MGPCG.  *dt is the
 * first step's dt and receives the next one.  A step whose solve fails (or
 * whose next dt is not positive and finite) ends the run: later steps are
 * skipped on the device, *steps_done counts the steps executed including the
 * failed one, and the status is that step's (ASD2G_NOT_CONVERGED,
 * ASD2G_E_NONFINITE, ASD2G_E_BREAKDOWN).  iters_total / max_resid (may be
 * NULL): iterations summed over the steps, largest final relative residual.
 * The step's results are bit-identical to asd2g_droplet_step with the same
 * arguments. */
int asd2g_run_steps(asd2g_session *s, int nsteps, double *dt, int reinit_mode, int solver, double tol, int maxit,
                    int *steps_done, long long *iters_total, double *max_resid);

/* ---- checkpoint / restart (no reference counterpart: the reference writes
 * Tecplot output only) ----
 * A raw binary file: a 128-byte little-endian header
 *   char magic[8] = "ASD2GCK1"; u32 version = 2; u32 header_bytes = 128;
 *   i32 nx, ny, nbc (= 3), precision; f64 t, dt; i64 step;
 *   u32 nfields, field_bits (bit f set for each field id stored);
 *   u64 payload_bytes; u64 checksum; zero padding
 * then the fields LS, U, V, PS, P in that order, each the padded
 * (nx+6) x (ny+6) FP64 array of the session layout.  checksum = sum of
 * w_i (2 i + 1) mod 2^64 over the little-endian 64-bit words w_i of the
 * header (its checksum field read as 0; words 0-15) followed by the payload
 * (words 16 on): any changed word, header included, changes it.  Enough to restart a
 * run (with t, step and the next dt) and to hand fields between processes.
 * save: writes the session's current fields.  load: checks magic, version,
 * sizes (nx, ny must match the session) and checksum, then replaces the
 * fields.  info: reads and verifies a file without a session (no GPU needed). */
int asd2g_checkpoint_save(asd2g_session *s, const char *path, double t, long long step, double dt);
int asd2g_checkpoint_load(asd2g_session *s, const char *path, double *t, long long *step, double *dt);
int asd2g_checkpoint_info(const char *path, int *nx, int *ny, double *t, long long *step, double *dt);

/* ---- allocation-free solve (no counterpart in the reference) ----
 * Jacobi-PCG (textbook recurrence, FP64) on a system the caller has already
 * assembled, for callers that cannot call cudaMalloc: a host that owns all
 * device memory through its own pool and hands out only pre-registered
 * buffers, a latency-critical loop where cudaMalloc/cudaFree would implicitly
 * synchronise the device, or a process that has reserved the whole GPU.  It
 * allocates nothing: its work space is a fixed file-scope device array of
 * ASD2G_STATIC_MAX_UNKNOWNS unknowns (about 10 MiB, held on every GPU that
 * loads the library until exit); larger systems are rejected with
 * ASD2G_E_ARG.  The system is given in the compact interior layout
 * k = j + ny*i (0-based interior indices, y fastest), as device arrays of
 * nx*ny doubles: diag, and the east/north couplings ce, cn (the matrix
 * entries are -ce and -cn; west/south couplings are the neighbours' ce/cn).
 * pinned = 1 holds cell 0 at 0 (b[0] must then be 0).  x receives the
 * solution.  All work runs on `stream` (a cudaStream_t, NULL = legacy
 * stream) and the call returns when the solve has finished.
 * The first call on a device looks up the array's address (with that device
 * current) and caches it; make that first call before any stream capture.
 * Later calls look the address up again unless their stream is capturing,
 * so the cache follows a cudaDeviceReset or another context made current on
 * the device.  An error pending before the call is reported as ASD2G_E_CUDA
 * without launching anything.  At most maxit iterations (rounded up to
 * even) are launched.
 * Every call shares the array, which keeps the last call's contents; each
 * call resets what it reads first, and calls that overlap on the GPU race. */
#define ASD2G_STATIC_MAX_UNKNOWNS (512 * 512)
int asd2g_pcg_solve_static(int nx, int ny, int pinned, const double *diag, const double *ce, const double *cn,
                           const double *b, double *x, double tol, int maxit, void *stream, int *iters,
                           double *rel_resid);

#ifdef __cplusplus
}
#endif
#endif
