/* CPU oracle for the 2D two-phase droplet step of appleparan/ASD2.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm, used by tests/, by __graft_entry__.smoke() and by bench.py's CPU
 * baseline leg as the checker.  The product (asd2_b200/) never links or calls
 * it.  Each function names the reference file:line it follows; the restated
 * arithmetic keeps the reference's operation order so that results can be
 * compared bit for bit where no transcendental function is involved.
 *
 * Pinning: the restatement is checked against the reference sources compiled
 * unmodified (oracle/_ref/libasd2ref.so, built by oracle/Makefile) and against
 * golden vectors generated from that build (tests/golden/).
 *
 * Layout: every field is a padded (nx+6)*(ny+6) array of doubles with
 * idx(i,j) = j + (ny+6)*i (levelset2d.cpp:1048-1050); interior cells are
 * i in [3, nx+3), j in [3, ny+3).  u lives on west faces, v on south faces.
 */
#ifndef ASD2_ORACLE_H
#define ASD2_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Boundary kinds, same order as enum class BC2D (include/common.h:4). */
enum { ORA_PERIODIC = 0, ORA_NEUMANN, ORA_DIRICHLET, ORA_AXISYM, ORA_WALL, ORA_INLET,
       ORA_OUTLET, ORA_PRESSURE, ORA_LSFREE, ORA_CUSTOM };

typedef struct {
    int32_t nx, ny;
    double dx, dy;
    int32_t bc_u[4], bc_v[4], bc_p[4]; /* W, E, S, N */
    double cu[4], cv[4], cp[4];        /* Dirichlet constants W, E, S, N */
} ora_grid;

typedef struct {
    double rho_h, rho_l, mu_h, mu_l;
    double sigma, g;
    int32_t g_axis;      /* GAXISENUM2D: 0 X, 1 Y */
    int32_t fix_gravity; /* 0: V takes its gravity from AddGravityFU (mac2d.cpp:294) */
    int32_t time_order;  /* TIMEORDERENUM: 0 Euler, 1 RK2, 2 RK3 */
    double cfl;
} ora_fluid;

/* ---- boundary ghost fill (bc2d.cpp:123,239,346 and :575-934) ---- */
void ora_bc_u(const ora_grid *g, double *a);
void ora_bc_v(const ora_grid *g, double *a);
void ora_bc_p(const ora_grid *g, double *a);

/* ---- level set (levelset2d.cpp) ---- */
void ora_unit_weno5(const double *F, double *FP, double *FM, double d, int n);
void ora_ls_weno_rhs(const ora_grid *g, double *ls, const double *u, const double *v, double *L);
void ora_ls_advect(const ora_grid *g, double *ls, const double *u, const double *v, double dt);
void ora_smoothed_sign(const ora_grid *g, const double *ls, double *out);
void ora_heaviside_deriv(const ora_grid *g, const double *ls, double *out);
void ora_eno_absgrad(const ora_grid *g, const double *ls, const double *ls0, double *out);
void ora_subcell_eno_absgrad(const ora_grid *g, const double *ls, const double *ls0, double *out);
void ora_sussman_constraint(const ora_grid *g, const double *ls, const double *ls0, const double *hd,
                            double *out);
int ora_reinit_steps(const ora_grid *g, double max_atime);
/* mode: 0 original, 1 Sussman, 2 MinRK2, 3 first-time-only Sussman,
 *       4 MinRK2 + Sussman area constraint after every pseudo-step.
 * max_atime <= 0 selects the default 1.5 * kThickness. */
void ora_reinit(const ora_grid *g, int mode, double max_atime, double *ls);

/* ---- MAC momentum (mac2d.cpp) ---- */
void ora_kappa(const ora_grid *g, const double *ls, double *kappa);
void ora_ntk(const ora_grid *g, const double *ls, double *nxo, double *nyo);
void ora_heaviside(const ora_grid *g, const double *ls, double *H);
void ora_smooth_heaviside(const ora_grid *g, const double *ls, double *HS);
void ora_conv_u(const ora_grid *g, const double *u, const double *v, double *cU);
void ora_conv_v(const ora_grid *g, const double *u, const double *v, double *cV);
void ora_visc_u(const ora_grid *g, const ora_fluid *f, const double *u, const double *v, const double *ls,
                const double *H, double *dU);
void ora_visc_v(const ora_grid *g, const ora_fluid *f, const double *u, const double *v, const double *ls,
                const double *H, double *dV);
void ora_rhs_u(const ora_grid *g, const ora_fluid *f, const double *ls, const double *u, const double *v,
               const double *H, double *FU);
void ora_rhs_v(const ora_grid *g, const ora_fluid *f, const double *ls, const double *u, const double *v,
               const double *H, double *FV);
void ora_intermediate_vel(const ora_grid *g, const ora_fluid *f, double dt, const double *ls, const double *u,
                          const double *v, double *uhat, double *vhat, const double *H);
void ora_divergence(const ora_grid *g, const double *u, const double *v, double *div);
void ora_update_vel(const ora_grid *g, const ora_fluid *f, double dt, double *u, double *v, const double *us,
                    const double *vs, const double *ps, const double *ls, const double *H,
                    const double *kappa);
double ora_update_dt(const ora_grid *g, const ora_fluid *f, const double *u, const double *v);

/* ---- GFM Poisson assembly (mac2d.cpp:1249-1656) ----
 * Matrix-free form over the nx*ny interior cells, natural order k = i + nx*j
 * (0-based interior indices):
 *   (A x)_k = diag_k x_k - cw_k x_W - ce_k x_E - cs_k x_S - cn_k x_N
 * where a face coefficient is 0 when the reference drops that entry.  rhs is
 * the reference right-hand side.  pinned = 1 when all four pressure sides are
 * Neumann/axisym/wall: cell 0 is then held at 0 and its row and column are
 * removed (the corrected form of the reference pin, mac2d.cpp:1585-1607).
 * kappa must already hold the curvature used by the reference (it recomputes
 * it when kWe is finite and nonzero, mac2d.cpp:1307-1310; ora_gfm_assemble
 * does the same when recompute_kappa is set, and writes it back). */
int ora_gfm_assemble(const ora_grid *g, const ora_fluid *f, double dt, const double *ls, double *kappa,
                     const double *H, const double *div, int recompute_kappa, double *diag, double *cw,
                     double *ce, double *cs, double *cn, double *rhs);
/* The same system as CSR in the reference's row order (S, W, C, E, N), with
 * the pin applied consistently.  Arrays must hold nx*ny+1 / 5*nx*ny entries.
 * Returns the number of rows. */
int ora_gfm_to_csr(const ora_grid *g, const double *diag, const double *cw, const double *ce, const double *cs,
                   const double *cn, const double *rhs, int pinned, double *a, int32_t *ia, int32_t *ja,
                   double *b);

/* Apply the matrix-free operator (natural order, pinned row/col forced to 0). */
void ora_gfm_apply(int nx, int ny, const double *diag, const double *cw, const double *ce, const double *cs,
                   const double *cn, int pinned, const double *x, double *y);

/* Jacobi-preconditioned CG on the matrix-free system.
 * mode 0: textbook PCG (x0 = 0, stop at ||b-Ax||/||b|| <= tol).
 * mode 1: the reference iteration (poisson2d.cpp:285-401) including its
 *         first-iteration direction and the err_tol^2 term in alpha, with tol
 *         as the stopping threshold.
 * Returns iterations; *resid receives the recurrence residual ratio and
 * *true_resid the recomputed ||b - A x|| / ||b||. */
int ora_pcg(int nx, int ny, const double *diag, const double *cw, const double *ce, const double *cs,
            const double *cn, int pinned, const double *b, double *x, double tol, int maxit, int mode,
            double *resid, double *true_resid);
/* Right-Jacobi BiCGStab in the reference's form (poisson2d.cpp:403-575).
 * mode 1 reproduces the reference exactly (rho_2 is never updated and stays
 * 1.0); mode 0 is the IML++ recurrence. */
int ora_bicgstab(int nx, int ny, const double *diag, const double *cw, const double *ce, const double *cs,
                 const double *cn, int pinned, const double *b, double *x, double tol, int maxit, int mode,
                 double *resid, double *true_resid);

/* ---- axisymmetric MAC solver (MACSolver2DAxisym, mac2dAxisym.cpp) ----
 * The grid's x is r (index i, kNr = nx, kDr = dx) and y is z (j).  base_r is
 * kBaseR; the reference uses it in the curvature, the divergence and the
 * assembly but not in the viscous terms (which take r = (i + 1/2) dr). */
void ora_axi_kappa(const ora_grid *g, double base_r, const double *ls, double *kappa);
void ora_axi_visc_u(const ora_grid *g, const ora_fluid *f, const double *u, const double *v, const double *ls,
                    const double *H, double *dU);
void ora_axi_visc_v(const ora_grid *g, const ora_fluid *f, const double *u, const double *uhat, const double *v,
                    const double *ls, const double *H, double *dV);
/* GetRHSU / GetRHSV with time step dt, including their U / V ghost fill. */
void ora_axi_rhs_u(const ora_grid *g, const ora_fluid *f, double dt, const double *ls, const double *u,
                   const double *v, const double *H, double *rhs);
void ora_axi_rhs_v(const ora_grid *g, const ora_fluid *f, double dt, const double *ls, const double *u,
                   const double *uhat, const double *v, const double *H, double *rhs);
/* GetUHat / GetVHat: the implicit viscous step (no ghost fill). */
void ora_axi_uhat(const ora_grid *g, const ora_fluid *f, double dt, const double *ls, const double *rhs,
                  const double *H, double *uhat);
void ora_axi_vhat(const ora_grid *g, const ora_fluid *f, double dt, const double *ls, const double *rhs,
                  const double *H, double *vhat);
/* GetDivergence4Poisson (r-weighted) and GetDivergence. */
void ora_axi_div4p(const ora_grid *g, double base_r, const double *u, const double *v, double *div);
void ora_axi_divergence(const ora_grid *g, double base_r, const double *u, const double *v, double *div);
/* SolvePoisson's assembly (mac2dAxisym.cpp:1488-1916) in the matrix-free
 * form of ora_gfm_assemble. */
int ora_axi_assemble(const ora_grid *g, const ora_fluid *f, double base_r, double dt, const double *ls,
                     double *kappa, const double *H, const double *div, int recompute_kappa, double *diag,
                     double *cw, double *ce, double *cs, double *cn, double *rhs);
double ora_axi_update_dt(const ora_grid *g, const ora_fluid *f, const double *u, const double *v,
                         const double *kappa);

/* Scatter/gather between natural-order vectors and padded cell arrays. */
void ora_gather(const ora_grid *g, const double *padded, double *nat);
void ora_scatter(const ora_grid *g, const double *nat, double *padded);

/* Masks (bit-exact checks): interface cells (levelset2d.cpp:655,686,723,745)
 * and GFM crossing faces (mac2d.cpp:1351-1443), one byte per interior cell,
 * natural order.  face_mask bit 0: west face crosses, bit 1: south face. */
void ora_interface_mask(const ora_grid *g, const double *ls0, uint8_t *mask);
void ora_ghost_face_mask(const ora_grid *g, const double *ls, uint8_t *mask);

#ifdef __cplusplus
}
#endif
#endif
