/* CPU oracle: plain-C restatement of the reference's 2D droplet hot path.
 * TEST INFRASTRUCTURE ONLY (see asd2_oracle.h).  Citations are file:line in
 * the appleparan/ASD2 tree.  Operation order follows the reference so that
 * results built with -ffp-contract=off agree with it bit for bit wherever no
 * libm transcendental (cos, sin, pow with a non-2 exponent) is involved.
 * std::pow(x, 2.0) in the reference compiles to x*x (g++ folds it), and is
 * written that way here. */
#include "asd2_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NB 3
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static inline long IX(const ora_grid *g, int i, int j) { return (long)j + (long)(g->ny + 2 * NB) * i; }
static inline long ASZ(const ora_grid *g) { return (long)(g->nx + 2 * NB) * (g->ny + 2 * NB); }
static inline double sq(double x) { return x * x; }
static double *zalloc(long n) { return (double *)calloc((size_t)n, sizeof(double)); }
static inline int isgn(double v) { return (v > 0) - (v < 0); }
/* std::max / std::min semantics: max(a,b) = (a < b) ? b : a. */
static inline double smax(double a, double b) { return (a < b) ? b : a; }
static inline double smin(double a, double b) { return (b < a) ? b : a; }

/* LevelSetSolver2D::MinMod, levelset2d.cpp:1036-1046 */
static inline double minmod(double a, double b) {
    if ((fabs(a) <= fabs(b)) && (a * b > 0)) return a;
    if ((fabs(a) > fabs(b)) && (a * b > 0)) return b;
    if (a * b <= 0) return 0.0;
    return NAN;
}

/* ======================================================================= */
/* Boundary conditions, bc2d.cpp.  Sides are applied W, E, S, N in order    */
/* (ApplyBC_*_2D, :123-128, :239-244, :346-353).                            */
/* ======================================================================= */
enum { K_NONE = 0, K_PER, K_NEU, K_DIR, K_LSF };

/* Dispatch tables BC_UW..BC_PN (bc2d.cpp:355-573). side: 0 W, 1 E, 2 S, 3 N */
static int kind_u(int side, int bc) {
    switch (bc) {
    case ORA_PERIODIC: return K_PER;
    case ORA_NEUMANN: return K_NEU;
    case ORA_AXISYM: return side < 2 ? K_DIR : K_NEU;
    case ORA_WALL: case ORA_DIRICHLET: case ORA_INLET: return K_DIR;
    case ORA_OUTLET: return K_NEU;
    default: return K_NONE;
    }
}
static int kind_v(int side, int bc) {
    switch (bc) {
    case ORA_PERIODIC: return K_PER;
    case ORA_NEUMANN: return K_NEU;
    case ORA_AXISYM: return side < 2 ? K_NEU : K_DIR;
    case ORA_WALL: case ORA_DIRICHLET: case ORA_INLET: return K_DIR;
    case ORA_OUTLET: return K_NEU;
    default: return K_NONE;
    }
}
static int kind_p(int bc) {
    switch (bc) {
    case ORA_PERIODIC: return K_PER;
    case ORA_NEUMANN: case ORA_AXISYM: case ORA_WALL: return K_NEU;
    case ORA_DIRICHLET: case ORA_INLET: case ORA_OUTLET: case ORA_PRESSURE: return K_DIR;
    case ORA_LSFREE: return K_LSF;
    default: return K_NONE;
    }
}

void ora_bc_u(const ora_grid *g, double *a) {
    const int nx = g->nx, ny = g->ny;
    int k;
    /* W: :575-579 periodic, :599-606 Neumann, :631-640 Dirichlet */
    k = kind_u(0, g->bc_u[0]);
    if (k == K_PER) {
        for (int i = 0; i <= NB; i++)
            for (int j = NB; j < ny + NB; j++) a[IX(g, i, j)] = a[IX(g, nx - 1 + i, j)];
    } else if (k == K_NEU) {
        for (int j = 0; j < ny + 2 * NB; j++) a[IX(g, NB, j)] = a[IX(g, NB + 1, j)];
        for (int i = 0; i < NB; i++)
            for (int j = NB; j <= ny + NB; j++) a[IX(g, i, j)] = a[IX(g, 2 * NB - i, j)];
    } else if (k == K_DIR) {
        const double c = g->cu[0];
        for (int j = 0; j < ny + 2 * NB; j++) a[IX(g, NB, j)] = c;
        for (int i = 0; i < NB; i++)
            for (int j = NB; j < ny + NB; j++) a[IX(g, i, j)] = -a[IX(g, 2 * NB - i, j)] + 2.0 * c;
    }
    /* E: :581-585, :608-615, :642-650 */
    k = kind_u(1, g->bc_u[1]);
    if (k == K_PER) {
        for (int i = 0; i < NB; i++)
            for (int j = NB; j < ny + NB; j++) a[IX(g, nx + i + NB, j)] = a[IX(g, i + NB, j)];
    } else if (k == K_NEU) {
        for (int j = 0; j < ny + 2 * NB; j++) a[IX(g, nx + NB, j)] = a[IX(g, nx + NB - 1, j)];
        for (int i = 1; i < NB; i++)
            for (int j = NB; j <= ny + NB; j++) a[IX(g, nx + 2 * NB - i, j)] = a[IX(g, nx + i, j)];
    } else if (k == K_DIR) {
        const double c = g->cu[1];
        for (int j = 0; j < ny + 2 * NB; j++) a[IX(g, nx + NB, j)] = c;
        for (int i = 1; i < NB; i++)
            for (int j = NB; j < ny + NB; j++) a[IX(g, nx + 2 * NB - i, j)] = -a[IX(g, nx + i, j)] + 2.0 * c;
    }
    /* S: :587-591, :617-621, :652-657 */
    k = kind_u(2, g->bc_u[2]);
    if (k == K_PER) {
        for (int i = NB + 1; i < nx + NB; i++)
            for (int j = 0; j < NB; j++) a[IX(g, i, j)] = a[IX(g, i, ny + j)];
    } else if (k == K_NEU) {
        for (int i = NB + 1; i < nx + NB; i++)
            for (int j = 0; j < NB; j++) a[IX(g, i, j)] = a[IX(g, i, 2 * NB - j - 1)];
    } else if (k == K_DIR) {
        const double c = g->cu[2];
        for (int i = NB; i < nx + NB; i++)
            for (int j = 0; j < NB; j++) a[IX(g, i, j)] = -a[IX(g, i, 2 * NB - j - 1)] + 2.0 * c;
    }
    /* N: :593-597, :623-627, :659-664 */
    k = kind_u(3, g->bc_u[3]);
    if (k == K_PER) {
        for (int i = NB + 1; i < nx + NB; i++)
            for (int j = 0; j < NB; j++) a[IX(g, i, ny + j + NB)] = a[IX(g, i, j + NB)];
    } else if (k == K_NEU) {
        for (int i = NB + 1; i < nx + NB; i++)
            for (int j = 0; j < NB; j++) a[IX(g, i, ny + 2 * NB - j - 1)] = a[IX(g, i, ny + j)];
    } else if (k == K_DIR) {
        const double c = g->cu[3];
        for (int i = NB; i < nx + NB; i++)
            for (int j = 0; j < NB; j++) a[IX(g, i, ny + 2 * NB - j - 1)] = -a[IX(g, i, ny + j)] + 2.0 * c;
    }
}

void ora_bc_v(const ora_grid *g, double *a) {
    const int nx = g->nx, ny = g->ny;
    int k;
    /* W: :666-670 periodic, :690-694 Neumann, :730-735 Dirichlet */
    k = kind_v(0, g->bc_v[0]);
    if (k == K_PER) {
        for (int i = 0; i < NB; i++)
            for (int j = NB + 1; j < ny + NB; j++) a[IX(g, i, j)] = a[IX(g, nx + i, j)];
    } else if (k == K_NEU) {
        for (int i = 0; i < NB; i++)
            for (int j = NB + 1; j < ny + NB; j++) a[IX(g, i, j)] = a[IX(g, 2 * NB - i - 1, j)];
    } else if (k == K_DIR) {
        const double c = g->cv[0];
        for (int i = 0; i < NB; i++)
            for (int j = NB + 1; j < ny + NB; j++) a[IX(g, i, j)] = -a[IX(g, 2 * NB - i - 1, j)] + 2.0 * c;
    }
    /* E: :672-676, :696-700, :737-742 */
    k = kind_v(1, g->bc_v[1]);
    if (k == K_PER) {
        for (int i = 0; i < NB; i++)
            for (int j = NB + 1; j < ny + NB; j++) a[IX(g, nx + i + NB, j)] = a[IX(g, i + NB, j)];
    } else if (k == K_NEU) {
        for (int i = 0; i < NB; i++)
            for (int j = NB + 1; j < ny + NB; j++) a[IX(g, nx + 2 * NB - i - 1, j)] = a[IX(g, nx + i, j)];
    } else if (k == K_DIR) {
        const double c = g->cv[1];
        for (int i = 0; i < NB; i++)
            for (int j = NB + 1; j < ny + NB; j++) a[IX(g, nx + 2 * NB - i - 1, j)] = -a[IX(g, nx + i, j)] + 2.0 * c;
    }
    /* S: :678-682, :702-709, :744-752 */
    k = kind_v(2, g->bc_v[2]);
    if (k == K_PER) {
        for (int i = NB; i < nx + NB; i++)
            for (int j = 0; j <= NB; j++) a[IX(g, i, j)] = a[IX(g, i, ny - 1 + j)];
    } else if (k == K_NEU) {
        for (int i = 0; i < nx + 2 * NB; i++) a[IX(g, i, NB)] = a[IX(g, i, NB + 1)];
        for (int i = NB; i < nx + NB; i++)
            for (int j = 0; j < NB; j++) a[IX(g, i, j)] = a[IX(g, i, 2 * NB - j)];
    } else if (k == K_DIR) {
        const double c = g->cv[2];
        for (int i = 0; i < nx + 2 * NB; i++) a[IX(g, i, NB)] = c;
        for (int i = NB; i < nx + NB; i++)
            for (int j = 0; j < NB; j++) a[IX(g, i, j)] = -a[IX(g, i, 2 * NB - j)] + 2.0 * c;
    }
    /* N: :684-688, :711-718, :754-762 */
    k = kind_v(3, g->bc_v[3]);
    if (k == K_PER) {
        for (int i = NB; i < nx + NB; i++)
            for (int j = 0; j < NB; j++) a[IX(g, i, ny + j + NB)] = a[IX(g, i, j + NB)];
    } else if (k == K_NEU) {
        for (int i = 0; i < nx + 2 * NB; i++) a[IX(g, i, ny + NB)] = a[IX(g, i, ny + NB - 1)];
        for (int i = NB; i < nx + NB; i++)
            for (int j = 1; j < NB; j++) a[IX(g, i, ny + 2 * NB - j)] = a[IX(g, i, ny + j)];
    } else if (k == K_DIR) {
        const double c = g->cv[3];
        for (int i = 0; i < nx + 2 * NB; i++) a[IX(g, i, ny + NB)] = c;
        for (int i = NB; i < nx + NB; i++)
            for (int j = 1; j < NB; j++) a[IX(g, i, ny + 2 * NB - j)] = -a[IX(g, i, ny + j)] + 2.0 * c;
    }
}

void ora_bc_p(const ora_grid *g, double *a) {
    const int nx = g->nx, ny = g->ny;
    const double dx = g->dx, dy = g->dy;
    int k;
    /* W: :764-768 periodic, :788-792 Neumann, :835-840 Dirichlet, :863-870 LS free */
    k = kind_p(g->bc_p[0]);
    if (k == K_PER) {
        for (int i = 0; i < NB; i++)
            for (int j = NB; j < ny + NB; j++) a[IX(g, i, j)] = a[IX(g, nx + i, j)];
    } else if (k == K_NEU) {
        for (int i = 0; i < NB; i++)
            for (int j = NB; j < ny + NB; j++) a[IX(g, i, j)] = a[IX(g, 2 * NB - i - 1, j)];
    } else if (k == K_DIR) {
        const double c = g->cp[0];
        for (int i = 0; i < NB; i++)
            for (int j = NB; j < ny + NB; j++) a[IX(g, i, j)] = -a[IX(g, 2 * NB - i - 1, j)] + 2.0 * c;
    } else if (k == K_LSF) {
        for (int i = NB - 1; i >= 0; i--)
            for (int j = NB; j < ny + NB; j++)
                a[IX(g, i, j)] = a[IX(g, i + 1, j)] + dx * (a[IX(g, i + 1, j)] - a[IX(g, i + 2, j)]) / dx;
    }
    /* E: :770-774 (writes interior columns nx..nx+2, as the reference does),
     * :794-798, :842-847, :872-880 */
    k = kind_p(g->bc_p[1]);
    if (k == K_PER) {
        for (int i = 0; i < NB; i++)
            for (int j = NB; j < ny + NB; j++) a[IX(g, nx + i, j)] = a[IX(g, i + NB, j)];
    } else if (k == K_NEU) {
        for (int i = 0; i < NB; i++)
            for (int j = NB; j < ny + NB; j++) a[IX(g, nx + 2 * NB - i - 1, j)] = a[IX(g, nx + i, j)];
    } else if (k == K_DIR) {
        const double c = g->cp[1];
        for (int i = 0; i < NB; i++)
            for (int j = NB; j < ny + NB; j++) a[IX(g, nx + 2 * NB - i - 1, j)] = -a[IX(g, nx + i, j)] + 2.0 * c;
    } else if (k == K_LSF) {
        for (int i = 0; i < NB; i++)
            for (int j = NB; j < ny + NB; j++)
                a[IX(g, nx + NB + i, j)] = a[IX(g, nx + NB + i - 1, j)] +
                    dx * (a[IX(g, nx + NB + i - 1, j)] - a[IX(g, nx + NB + i - 2, j)]) / dx;
    }
    /* S: :776-780, :800-804, :849-854, :882-890 */
    k = kind_p(g->bc_p[2]);
    if (k == K_PER) {
        for (int i = NB; i < nx + NB; i++)
            for (int j = 0; j < NB; j++) a[IX(g, i, j)] = a[IX(g, i, ny + j)];
    } else if (k == K_NEU) {
        for (int i = NB; i < nx + NB; i++)
            for (int j = 0; j < NB; j++) a[IX(g, i, j)] = a[IX(g, i, 2 * NB - j - 1)];
    } else if (k == K_DIR) {
        const double c = g->cp[2];
        for (int i = NB; i < nx + NB; i++)
            for (int j = 0; j < NB; j++) a[IX(g, i, j)] = -a[IX(g, i, 2 * NB - j - 1)] + 2.0 * c;
    } else if (k == K_LSF) {
        for (int i = NB; i < nx + NB; i++)
            for (int j = NB - 1; j >= 0; j--)
                a[IX(g, i, j)] = a[IX(g, i, j + 1)] + dy * (a[IX(g, i, j + 1)] - a[IX(g, i, j + 2)]) / dy;
    }
    /* N: :782-786, :806-810, :856-861, :892-900 */
    k = kind_p(g->bc_p[3]);
    if (k == K_PER) {
        for (int i = NB; i < nx + NB; i++)
            for (int j = 0; j < NB; j++) a[IX(g, i, ny + j + NB)] = a[IX(g, i, j + NB)];
    } else if (k == K_NEU) {
        for (int i = NB; i < nx + NB; i++)
            for (int j = 0; j < NB; j++) a[IX(g, i, ny + 2 * NB - j - 1)] = a[IX(g, i, ny + j)];
    } else if (k == K_DIR) {
        const double c = g->cp[3];
        for (int i = NB; i < nx + NB; i++)
            for (int j = 0; j < NB; j++) a[IX(g, i, ny + 2 * NB - j - 1)] = -a[IX(g, i, ny + j)] + 2.0 * c;
    } else if (k == K_LSF) {
        for (int i = NB; i < nx + NB; i++)
            for (int j = 0; j < NB; j++)
                a[IX(g, i, ny + NB + j)] = a[IX(g, i, ny + NB + j - 1)] +
                    dy * (a[IX(g, i, ny + NB + j - 1)] - a[IX(g, i, ny + NB + j - 2)]) / dy;
    }
}

/* ======================================================================= */
/* WENO5 (LevelSetSolver2D::UnitHJWENO5, levelset2d.cpp:159-262; the same   */
/* code is MACSolver2D::UnitHJWENO5, mac2d.cpp:465-568).  F has n+6 points. */
/* ======================================================================= */
void ora_unit_weno5(const double *F, double *FP, double *FM, double d, int n) {
    const double eps = 1e-6;
    const int m = n + 2 * NB;
    double *D = zalloc(m);
    for (int i = 0; i < m - 1; i++) D[i] = F[i + 1] - F[i];
    for (int i = NB; i < n + NB; i++) {
        /* phi^- (:181-219) */
        double is0 = 13.0 / 12.0 * sq((D[i - 3] - 2.0 * D[i - 2] + D[i - 1]) / d) +
                     1.0 / 4.0 * sq((D[i - 3] - 4.0 * D[i - 2] + 3.0 * D[i - 1]) / d);
        double is1 = 13.0 / 12.0 * sq((D[i - 2] - 2.0 * D[i - 1] + D[i]) / d) + 1.0 / 4.0 * sq((D[i - 2] - D[i]) / d);
        double is2 = 13.0 / 12.0 * sq((D[i - 1] - 2.0 * D[i] + D[i + 1]) / d) +
                     1.0 / 4.0 * sq((3.0 * D[i - 1] - 4.0 * D[i] + D[i + 1]) / d);
        double a0 = 0.1 / sq(eps + is0), a1 = 0.6 / sq(eps + is1), a2 = 0.3 / sq(eps + is2);
        double w0 = a0 / (a0 + a1 + a2), w1 = a1 / (a0 + a1 + a2), w2 = a2 / (a0 + a1 + a2);
        FM[i] = w0 * (1.0 / 3.0 * D[i - 3] - 7.0 / 6.0 * D[i - 2] + 11.0 / 6.0 * D[i - 1]) / d +
                w1 * (-1.0 / 6.0 * D[i - 2] + 5.0 / 6.0 * D[i - 1] + 1.0 / 3.0 * D[i]) / d +
                w2 * (1.0 / 3.0 * D[i - 1] + 5.0 / 6.0 * D[i] - 1.0 / 6.0 * D[i + 1]) / d;
        /* phi^+ (:221-259) */
        is0 = 13.0 / 12.0 * sq((D[i + 2] - 2.0 * D[i + 1] + D[i]) / d) +
              1.0 / 4.0 * sq((D[i + 2] - 4.0 * D[i + 1] + 3.0 * D[i]) / d);
        is1 = 13.0 / 12.0 * sq((D[i + 1] - 2.0 * D[i] + D[i - 1]) / d) + 1.0 / 4.0 * sq((D[i + 1] - D[i - 1]) / d);
        is2 = 13.0 / 12.0 * sq((D[i] - 2.0 * D[i - 1] + D[i - 2]) / d) +
              1.0 / 4.0 * sq((3.0 * D[i] - 4.0 * D[i - 1] + D[i - 2]) / d);
        a0 = 0.1 / sq(eps + is0);
        a1 = 0.6 / sq(eps + is1);
        a2 = 0.3 / sq(eps + is2);
        w0 = a0 / (a0 + a1 + a2);
        w1 = a1 / (a0 + a1 + a2);
        w2 = a2 / (a0 + a1 + a2);
        FP[i] = w0 * (1.0 / 3.0 * D[i + 2] - 7.0 / 6.0 * D[i + 1] + 11.0 / 6.0 * D[i]) / d +
                w1 * (-1.0 / 6.0 * D[i + 1] + 5.0 / 6.0 * D[i] + 1.0 / 3.0 * D[i - 1]) / d +
                w2 * (1.0 / 3.0 * D[i] + 5.0 / 6.0 * D[i - 1] - 1.0 / 6.0 * D[i - 2]) / d;
    }
    free(D);
}

/* WENO sweep of a product field along x (rows j) or y (columns i) and the
 * signed-velocity blend, shared by HJWENO5_LS_2D (levelset2d.cpp:88-157) and
 * AddConvectionFU/FV (mac2d.cpp:308-463).
 * Fx[i,j] is the x-flux, Fy the y-flux; ax, ay the blend velocities. */
static void weno_blend(const ora_grid *g, const double *Fx, const double *Fy, const double *ax, const double *ay,
                       int i0, int j0, double *out) {
    const int nx = g->nx, ny = g->ny, mx = nx + 2 * NB, my = ny + 2 * NB;
    const long n = ASZ(g);
    double *LXP = zalloc(n), *LXM = zalloc(n), *LYP = zalloc(n), *LYM = zalloc(n);
    double *f = zalloc(mx > my ? mx : my), *fp = zalloc(mx > my ? mx : my), *fm = zalloc(mx > my ? mx : my);
    for (int j = NB; j < ny + NB; j++) {
        for (int i = 0; i < mx; i++) f[i] = Fx[IX(g, i, j)];
        memset(fp, 0, sizeof(double) * mx);
        memset(fm, 0, sizeof(double) * mx);
        ora_unit_weno5(f, fp, fm, g->dx, nx);
        for (int i = 0; i < mx; i++) { LXP[IX(g, i, j)] = fp[i]; LXM[IX(g, i, j)] = fm[i]; }
    }
    for (int i = NB; i < nx + NB; i++) {
        for (int j = 0; j < my; j++) f[j] = Fy[IX(g, i, j)];
        memset(fp, 0, sizeof(double) * my);
        memset(fm, 0, sizeof(double) * my);
        ora_unit_weno5(f, fp, fm, g->dy, ny);
        for (int j = 0; j < my; j++) { LYP[IX(g, i, j)] = fp[j]; LYM[IX(g, i, j)] = fm[j]; }
    }
    for (int i = i0; i < nx + NB; i++)
        for (int j = j0; j < ny + NB; j++) {
            const long k = IX(g, i, j);
            out[k] = 0.5 * (LXP[k] + LXM[k]) + 0.5 * (LYP[k] + LYM[k]) - ax[k] * (0.5 * (LXP[k] - LXM[k])) -
                     ay[k] * (0.5 * (LYP[k] - LYM[k]));
        }
    free(LXP); free(LXM); free(LYP); free(LYM); free(f); free(fp); free(fm);
}

/* HJWENO5_LS_2D, levelset2d.cpp:88-157.  Applies the P boundary to ls first
 * (:99), as the reference does. */
void ora_ls_weno_rhs(const ora_grid *g, double *ls, const double *u, const double *v, double *L) {
    const long n = ASZ(g);
    ora_bc_p(g, ls);
    double *Fx = zalloc(n), *Fy = zalloc(n);
    for (long k = 0; k < n; k++) { Fx[k] = ls[k] * u[k]; Fy[k] = ls[k] * v[k]; }
    memset(L, 0, sizeof(double) * n);
    weno_blend(g, Fx, Fy, u, v, NB, NB, L);
    free(Fx); free(Fy);
}

/* Solve_LevelSet_2D, levelset2d.cpp:43-86 (TVD-RK3). */
void ora_ls_advect(const ora_grid *g, double *ls, const double *u, const double *v, double dt) {
    const int nx = g->nx, ny = g->ny;
    const long n = ASZ(g);
    double *tu = zalloc(n), *tv = zalloc(n), *L = zalloc(n), *LS1 = zalloc(n), *LS2 = zalloc(n);
    for (int i = NB; i < nx + NB; i++)
        for (int j = NB; j < ny + NB; j++) {
            tu[IX(g, i, j)] = (u[IX(g, i, j)] + u[IX(g, i + 1, j)]) * 0.5;
            tv[IX(g, i, j)] = (v[IX(g, i, j)] + v[IX(g, i, j + 1)]) * 0.5;
        }
    ora_bc_p(g, tu);
    ora_bc_p(g, tv);
    ora_ls_weno_rhs(g, ls, tu, tv, L);
    for (int i = NB; i < nx + NB; i++)
        for (int j = NB; j < ny + NB; j++) LS1[IX(g, i, j)] = ls[IX(g, i, j)] - dt * L[IX(g, i, j)];
    ora_bc_p(g, LS1);
    ora_ls_weno_rhs(g, LS1, tu, tv, L);
    for (int i = NB; i < nx + NB; i++)
        for (int j = NB; j < ny + NB; j++) {
            const long k = IX(g, i, j);
            LS2[k] = 0.75 * ls[k] + 0.25 * LS1[k] - 0.25 * dt * L[k];
        }
    ora_bc_p(g, LS2);
    ora_ls_weno_rhs(g, LS2, tu, tv, L);
    for (int i = NB; i < nx + NB; i++)
        for (int j = NB; j < ny + NB; j++) {
            const long k = IX(g, i, j);
            ls[k] = 1.0 / 3.0 * ls[k] + 2.0 / 3.0 * LS2[k] - 2.0 / 3.0 * dt * L[k];
        }
    ora_bc_p(g, ls);
    free(tu); free(tv); free(L); free(LS1); free(LS2);
}

/* ======================================================================= */
/* Reinitialisation                                                         */
/* ======================================================================= */
static double ls_eps(const ora_grid *g) { return g->dx < g->dy ? g->dx : g->dy; } /* kEps = min(dx,dy) :4 */

/* GetSmoothedSignFunc, levelset2d.cpp:914-923 (all cells) */
void ora_smoothed_sign(const ora_grid *g, const double *ls, double *out) {
    const double e = ls_eps(g);
    const long n = ASZ(g);
    for (long k = 0; k < n; k++) out[k] = ls[k] / sqrt(ls[k] * ls[k] + e * e);
}

/* UpdateHeavisideFuncDeriv, levelset2d.cpp:27-41 (all cells) */
void ora_heaviside_deriv(const ora_grid *g, const double *ls, double *out) {
    const double e = ls_eps(g);
    const long n = ASZ(g);
    for (long k = 0; k < n; k++) out[k] = fabs(ls[k]) > e ? 0.0 : 0.5 * (1.0 / e + cos(M_PI * ls[k] / e));
}

/* Second-order ENO one-sided derivatives with a minmod limiter
 * (ENO_DerivAbsLS_2D :567-594 and SubcellENO_Min_DerivAbsLS_2D :635-644). */
static inline void eno_x(const ora_grid *g, const double *ls, int i, int j, double *dP, double *dM) {
    const double dx = g->dx;
    const double lm2 = ls[IX(g, i - 2, j)], lm1 = ls[IX(g, i - 1, j)], l0 = ls[IX(g, i, j)],
                 lp1 = ls[IX(g, i + 1, j)], lp2 = ls[IX(g, i + 2, j)];
    *dP = (lp1 - l0) / dx - dx * 0.5 * minmod((lm1 - 2.0 * l0 + lp1) / (dx * dx), (l0 - 2.0 * lp1 + lp2) / (dx * dx));
    *dM = (l0 - lm1) / dx + dx * 0.5 * minmod((lm1 - 2.0 * l0 + lp1) / (dx * dx), (lm2 - 2.0 * lm1 + l0) / (dx * dx));
}
static inline void eno_y(const ora_grid *g, const double *ls, int i, int j, double *dP, double *dM) {
    const double dy = g->dy;
    const double lm2 = ls[IX(g, i, j - 2)], lm1 = ls[IX(g, i, j - 1)], l0 = ls[IX(g, i, j)],
                 lp1 = ls[IX(g, i, j + 1)], lp2 = ls[IX(g, i, j + 2)];
    *dP = (lp1 - l0) / dy - dy * 0.5 * minmod((lm1 - 2.0 * l0 + lp1) / (dy * dy), (l0 - 2.0 * lp1 + lp2) / (dy * dy));
    *dM = (l0 - lm1) / dy + dy * 0.5 * minmod((lm1 - 2.0 * l0 + lp1) / (dy * dy), (lm2 - 2.0 * lm1 + l0) / (dy * dy));
}

/* Godunov |grad phi| (:596-610, :770-782) */
static inline double godunov(double s0, double dPX, double dMX, double dPY, double dMY) {
    if (s0 >= 0)
        return sqrt(smax(sq(smin(dPX, 0.0)), sq(smax(dMX, 0.0))) + smax(sq(smin(dPY, 0.0)), sq(smax(dMY, 0.0))));
    return sqrt(smax(sq(smax(dPX, 0.0)), sq(smin(dMX, 0.0))) + smax(sq(smax(dPY, 0.0)), sq(smin(dMY, 0.0))));
}

/* ENO_DerivAbsLS_2D, levelset2d.cpp:560-613 (interior cells; others 0) */
void ora_eno_absgrad(const ora_grid *g, const double *ls, const double *ls0, double *out) {
    memset(out, 0, sizeof(double) * ASZ(g));
    for (int i = NB; i < g->nx + NB; i++)
        for (int j = NB; j < g->ny + NB; j++) {
            double dPX, dMX, dPY, dMY;
            eno_x(g, ls, i, j, &dPX, &dMX);
            eno_y(g, ls, i, j, &dPY, &dMY);
            out[IX(g, i, j)] = godunov(ls0[IX(g, i, j)], dPX, dMX, dPY, dMY);
        }
}

/* Min-Gibou subcell one-sided derivatives at cells whose neighbour has the
 * other sign in ls0: SubcellENO_Min_DerivAbsLS_2D, levelset2d.cpp:655-681
 * (plus side) and :686-711 (minus side).  h is dx or dy; l0.. are ls0 values
 * along the axis; c is ls at the cell. */
static inline double subcell_plus(double h, double c, double i0m1, double i00, double i0p1, double i0p2, double dflt) {
    const double kSmall = 1.0e-10;
    double DD = minmod((i0m1 - 2.0 * i00 + i0p1) / (h * h), (i00 - 2.0 * i0p1 + i0p2) / (h * h));
    double c2 = 0.5 * DD;
    double c1 = (i0p1 - i00) / h;
    double c0 = (i0p1 + i00) * 0.5 - c2 * h * h * 0.25;
    double nd;
    (void)dflt;
    if (fabs(c2) > kSmall)
        nd = 0.5 * h + (-c1 - isgn(i00) * sqrt(c1 * c1 - 4.0 * c2 * c0)) / (2.0 * c2);
    else
        nd = 0.5 * h - c0 / c1;
    double d = -c / nd - 0.5 * nd * DD;
    if (fabs(nd) < h * 0.01) d = -0.5 * nd * DD;
    return d;
}
static inline double subcell_minus(double h, double c, double i0m2, double i0m1, double i00, double i0p1) {
    const double kSmall = 1.0e-10;
    double DD = minmod((i0m1 - 2.0 * i00 + i0p1) / (h * h), (i0m2 - 2.0 * i0m1 + i00) / (h * h));
    double c2 = 0.5 * DD;
    double c1 = (i00 - i0m1) / h;
    double c0 = (i00 + i0m1) * 0.5 - c2 * h * h * 0.25;
    double nd;
    if (fabs(c2) > kSmall)
        nd = 0.5 * h - (-c1 + isgn(i00) * sqrt(c1 * c1 - 4.0 * c2 * c0)) / (2.0 * c2);
    else
        nd = 0.5 * h + c0 / c1;
    double d = c / nd + 0.5 * nd * DD;
    if (fabs(nd) < h * 0.01) d = 0.5 * nd * DD;
    return d;
}

/* SubcellENO_Min_DerivAbsLS_2D, levelset2d.cpp:616-785 */
void ora_subcell_eno_absgrad(const ora_grid *g, const double *ls, const double *ls0, double *out) {
    memset(out, 0, sizeof(double) * ASZ(g));
    for (int i = NB; i < g->nx + NB; i++)
        for (int j = NB; j < g->ny + NB; j++) {
            double dPX, dMX, dPY, dMY;
            const double c = ls[IX(g, i, j)];
            eno_x(g, ls, i, j, &dPX, &dMX);
            const double xm2 = ls0[IX(g, i - 2, j)], xm1 = ls0[IX(g, i - 1, j)], x0 = ls0[IX(g, i, j)],
                         xp1 = ls0[IX(g, i + 1, j)], xp2 = ls0[IX(g, i + 2, j)];
            if (x0 * xp1 < 0) dPX = subcell_plus(g->dx, c, xm1, x0, xp1, xp2, dPX);
            if (x0 * xm1 < 0) dMX = subcell_minus(g->dx, c, xm2, xm1, x0, xp1);
            eno_y(g, ls, i, j, &dPY, &dMY);
            const double ym2 = ls0[IX(g, i, j - 2)], ym1 = ls0[IX(g, i, j - 1)], yp1 = ls0[IX(g, i, j + 1)],
                         yp2 = ls0[IX(g, i, j + 2)];
            if (x0 * yp1 < 0) dPY = subcell_plus(g->dy, c, ym1, x0, yp1, yp2, dPY);
            if (x0 * ym1 < 0) dMY = subcell_minus(g->dy, c, ym2, ym1, x0, yp1);
            out[IX(g, i, j)] = godunov(x0, dPX, dMX, dPY, dMY);
        }
}

/* GetSussmanReinitConstraint, levelset2d.cpp:787-893 */
void ora_sussman_constraint(const ora_grid *g, const double *ls, const double *ls0, const double *hd,
                            double *out) {
    const double kEps = ls_eps(g), kThick = 1.5 * kEps, kAdt = kEps * 0.5;
    const double dx = g->dx, dy = g->dy;
    memset(out, 0, sizeof(double) * ASZ(g));
    for (int i = NB; i < g->nx + NB; i++)
        for (int j = NB; j < g->ny + NB; j++) {
            if (hd[IX(g, i, j)] == 0.0) continue;
#define L_(a, b) ls[IX(g, i + (a), j + (b))]
#define I_(a, b) ls0[IX(g, i + (a), j + (b))]
            double lf[3][3], lif[3][3], Hp[3][3], L[3][3], dA[3][3], f[3][3];
            lf[0][0] = 0.25 * (L_(0, 0) + L_(-1, 0) + L_(-1, -1) + L_(0, -1));
            lf[0][1] = 0.5 * (L_(0, -1) + L_(0, 0));
            lf[0][2] = 0.25 * (L_(0, 0) + L_(-1, 0) + L_(-1, 1) + L_(0, 1));
            lf[1][0] = 0.5 * (L_(0, -1) + L_(0, 0));
            lf[1][1] = L_(0, 0);
            lf[1][2] = 0.5 * (L_(0, 0) + L_(0, 1));
            lf[2][0] = 0.25 * (L_(0, 0) + L_(1, 0) + L_(1, -1) + L_(0, -1));
            lf[2][1] = 0.5 * (L_(0, 0) + L_(1, 0));
            lf[2][2] = 0.25 * (L_(0, 0) + L_(1, 0) + L_(1, 1) + L_(0, 1));
            lif[0][0] = 0.25 * (I_(0, 0) + I_(-1, 0) + I_(-1, -1) + I_(0, -1));
            lif[0][1] = 0.5 * (I_(0, -1) + I_(0, 0));
            lif[0][2] = 0.25 * (I_(0, 0) + I_(-1, 0) + I_(-1, 1) + I_(0, 1));
            lif[1][0] = 0.5 * (I_(0, -1) + I_(0, 0));
            lif[1][1] = I_(0, 0);
            lif[1][2] = 0.5 * (I_(0, 0) + I_(0, 1));
            lif[2][0] = 0.25 * (I_(0, 0) + I_(1, 0) + I_(1, -1) + I_(0, -1));
            lif[2][1] = 0.5 * (I_(0, 0) + I_(1, 0));
            lif[2][2] = 0.25 * (I_(0, 0) + I_(1, 0) + I_(1, 1) + I_(0, 1));
            /* |grad phi0| at the nine sub-points (:840-873), including the
             * reference's "- -0.5" at [0][2] and the 2*dx at [2][1]. */
            dA[0][0] = sqrt(sq(((I_(0, 0) + I_(0, -1)) * 0.5 - 0.5 * (I_(-1, 0) + I_(-1, -1))) / dx) +
                            sq((lif[0][1] - 0.5 * (I_(0, -1) + I_(-1, -1))) / dy));
            dA[0][1] = sqrt(sq((lif[1][1] - I_(-1, 0)) / dx) + sq((lif[2][0] - lif[0][0]) / dy));
            dA[0][2] = sqrt(sq((lif[1][2] - -0.5 * (I_(-1, 0) + I_(-1, 1))) / dx) +
                            sq((0.5 * (I_(-1, 1) + I_(0, 1)) - lif[0][1]) / dy));
            dA[1][0] = sqrt(sq((lif[2][0] - lif[0][0]) / dx) + sq((lif[1][1] - 0.5 * (I_(0, -1) + I_(0, 0))) / dy));
            dA[1][1] = sqrt(sq((lif[2][1] - lif[0][1]) / dx) + sq((lif[1][2] - lif[1][0]) / dy));
            dA[1][2] = sqrt(sq((lif[2][2] - lif[0][2]) / dx) + sq((I_(0, 1) - lif[1][1]) / dy));
            dA[2][0] = sqrt(sq((0.5 * (I_(1, 0) + I_(1, -1)) - lif[1][0]) / dx) +
                            sq((lif[2][1] - 0.5 * (I_(0, -1) + I_(1, -1))) / dy));
            dA[2][1] = sqrt(sq((I_(1, 0) - lif[1][1]) / (2.0 * dx)) + sq((lif[2][2] - lif[2][0]) / dy));
            dA[2][2] = sqrt(sq((0.5 * (I_(1, 0) + I_(1, 1)) - lif[1][1]) / dx) +
                            sq((0.5 * (I_(0, 1) + I_(1, 1)) - lif[2][1]) / dy));
#undef L_
#undef I_
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    if (fabs(lf[a][b]) > kThick)
                        Hp[a][b] = 0.0;
                    else
                        Hp[a][b] = 0.5 / kEps + 0.5 / kEps * cos(M_PI * lf[a][b] / kEps);
                    L[a][b] = (lf[a][b] - lif[a][b]) / kAdt;
                    f[a][b] = Hp[a][b] * dA[a][b];
                }
            double s1 = 0.0, s2 = 0.0;
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    s1 += Hp[a][b] * L[a][b];
                    s2 += Hp[a][b] * f[a][b];
                }
            s1 += 15.0 * Hp[1][1] * L[1][1];
            s2 += 15.0 * Hp[1][1] * f[1][1];
            out[IX(g, i, j)] -= kAdt * f[1][1] * s1 / s2;
        }
}

/* Pseudo-step count of `while (m_atime < kMaxATime) m_atime += kAdt;`
 * (levelset2d.cpp:274-275 and the other reinit loops). */
int ora_reinit_steps(const ora_grid *g, double max_atime) {
    const double e = ls_eps(g), adt = e * 0.5;
    const double mt = max_atime > 0.0 ? max_atime : 1.5 * (1.5 * e);
    double t = 0.0;
    int n = 0;
    while (t < mt) { t += adt; n++; }
    return n;
}

void ora_reinit(const ora_grid *g, int mode, double max_atime, double *ls) {
    const int nx = g->nx, ny = g->ny;
    const long n = ASZ(g);
    const double e = ls_eps(g), adt = e * 0.5;
    double *ls0 = zalloc(n), *a1 = zalloc(n), *a2 = zalloc(n), *LS1 = zalloc(n), *LS2 = zalloc(n),
           *tmp = zalloc(n), *hd = zalloc(n), *sc = zalloc(n), *S = zalloc(n);
    if (mode == 3) {
        /* FirstTimeOnlyReinit_Sussman_2D, levelset2d.cpp:377-431 */
        memcpy(ls0, ls, sizeof(double) * n);
        ora_eno_absgrad(g, ls0, ls0, a1);
        for (int i = NB; i < nx + NB; i++)
            for (int j = NB; j < ny + NB; j++)
                if (a1[IX(g, i, j)] > 0.0) ls0[IX(g, i, j)] = ls0[IX(g, i, j)] / a1[IX(g, i, j)];
        ora_bc_p(g, ls0);
        const double lx = g->dx * nx, ly = g->dy * ny, mt = lx > ly ? lx : ly;
        double t = 0.0;
        while (t < mt) {
            t += adt;
            ora_bc_p(g, ls);
            ora_eno_absgrad(g, ls, ls0, a1);
            for (int i = NB; i < nx + NB; i++)
                for (int j = NB; j < ny + NB; j++) {
                    const long k = IX(g, i, j);
                    LS1[k] = ls[k] - adt * isgn(ls0[k]) * (a1[k] - 1.0);
                }
            ora_bc_p(g, LS1);
            ora_eno_absgrad(g, LS1, ls0, a2);
            for (int i = NB; i < nx + NB; i++)
                for (int j = NB; j < ny + NB; j++) {
                    const long k = IX(g, i, j);
                    LS2[k] = ls[k] - adt * isgn(ls0[k]) * (a2[k] - 1.0);
                }
            ora_bc_p(g, LS2);
            for (int i = NB; i < nx + NB; i++)
                for (int j = NB; j < ny + NB; j++) {
                    const long k = IX(g, i, j);
                    ls[k] = 0.5 * (ls[k] + LS2[k]);
                }
        }
        ora_bc_p(g, ls);
        goto done;
    }
    {
        const int steps = ora_reinit_steps(g, max_atime);
        if (mode == 2 || mode == 4) ora_bc_p(g, ls); /* Reinit_MinRK2_2D :435 */
        memcpy(ls0, ls, sizeof(double) * n);
        if (mode == 2 || mode == 4) ora_smoothed_sign(g, ls0, S);
        for (int s = 0; s < steps; s++) {
            ora_bc_p(g, ls);
            if (mode == 0) {
                /* Reinit_Original_2D, levelset2d.cpp:264-316 */
                ora_eno_absgrad(g, ls, ls0, a1);
                for (int i = NB; i < nx + NB; i++)
                    for (int j = NB; j < ny + NB; j++) {
                        const long k = IX(g, i, j);
                        LS1[k] = ls[k] - adt * isgn(ls0[k]) * (a1[k] - 1.0);
                    }
                ora_bc_p(g, LS1);
                ora_eno_absgrad(g, LS1, ls0, a2);
                for (int i = NB; i < nx + NB; i++)
                    for (int j = NB; j < ny + NB; j++) {
                        const long k = IX(g, i, j);
                        LS2[k] = LS1[k] - adt * isgn(ls0[k]) * (a2[k] - 1.0);
                    }
                ora_bc_p(g, LS2);
                for (int i = NB; i < nx + NB; i++)
                    for (int j = NB; j < ny + NB; j++) tmp[IX(g, i, j)] = 0.5 * (ls[IX(g, i, j)] + LS2[IX(g, i, j)]);
                ora_bc_p(g, tmp);
                for (int i = NB; i < nx + NB; i++)
                    for (int j = NB; j < ny + NB; j++) ls[IX(g, i, j)] = tmp[IX(g, i, j)];
            } else if (mode == 1) {
                /* Reinit_Sussman_2D, levelset2d.cpp:318-375.  No boundary
                 * fill on LS1/LS2 (their ghosts stay 0) and ls only receives
                 * the constraint, as in the reference. */
                ora_eno_absgrad(g, ls, ls0, a1);
                for (int i = NB; i < nx + NB; i++)
                    for (int j = NB; j < ny + NB; j++) {
                        const long k = IX(g, i, j);
                        LS1[k] = ls[k] - adt * isgn(ls0[k]) * (a1[k] - 1.0);
                    }
                ora_eno_absgrad(g, LS1, ls0, a2);
                for (int i = NB; i < nx + NB; i++)
                    for (int j = NB; j < ny + NB; j++) {
                        const long k = IX(g, i, j);
                        LS2[k] = LS1[k] - adt * isgn(ls0[k]) * (a2[k] - 1.0);
                    }
                for (int i = NB; i < nx + NB; i++)
                    for (int j = NB; j < ny + NB; j++) tmp[IX(g, i, j)] = 0.5 * (ls[IX(g, i, j)] + LS2[IX(g, i, j)]);
                ora_bc_p(g, tmp);
                ora_heaviside_deriv(g, tmp, hd);
                ora_sussman_constraint(g, tmp, ls0, hd, sc);
                for (int i = NB; i < nx + NB; i++)
                    for (int j = NB; j < ny + NB; j++) ls[IX(g, i, j)] += sc[IX(g, i, j)];
            } else {
                /* Reinit_MinRK2_2D, levelset2d.cpp:433-486; mode 4 adds the
                 * Sussman constraint where the reference comments it out (:474). */
                ora_subcell_eno_absgrad(g, ls, ls0, a1);
                for (int i = NB; i < nx + NB; i++)
                    for (int j = NB; j < ny + NB; j++) {
                        const long k = IX(g, i, j);
                        LS1[k] = ls[k] - adt * S[k] * (a1[k] - 1.0);
                    }
                ora_bc_p(g, LS1);
                ora_subcell_eno_absgrad(g, LS1, ls0, a2);
                for (int i = NB; i < nx + NB; i++)
                    for (int j = NB; j < ny + NB; j++) {
                        const long k = IX(g, i, j);
                        LS2[k] = LS1[k] - adt * S[k] * (a2[k] - 1.0);
                    }
                ora_bc_p(g, LS2);
                for (int i = NB; i < nx + NB; i++)
                    for (int j = NB; j < ny + NB; j++) tmp[IX(g, i, j)] = 0.5 * (ls[IX(g, i, j)] + LS2[IX(g, i, j)]);
                ora_bc_p(g, tmp);
                if (mode == 4) {
                    ora_heaviside_deriv(g, tmp, hd);
                    ora_sussman_constraint(g, tmp, ls0, hd, sc);
                    for (int i = NB; i < nx + NB; i++)
                        for (int j = NB; j < ny + NB; j++) ls[IX(g, i, j)] = tmp[IX(g, i, j)] + sc[IX(g, i, j)];
                } else {
                    for (int i = NB; i < nx + NB; i++)
                        for (int j = NB; j < ny + NB; j++) ls[IX(g, i, j)] = tmp[IX(g, i, j)];
                }
            }
        }
        ora_bc_p(g, ls);
    }
done:
    free(ls0); free(a1); free(a2); free(LS1); free(LS2); free(tmp); free(hd); free(sc); free(S);
}

/* ======================================================================= */
/* MAC solver                                                               */
/* ======================================================================= */
/* UpdateKappa, mac2d.cpp:221-252 (interior cells written). */
void ora_kappa(const ora_grid *g, const double *ls, double *kappa) {
    const int nx = g->nx, ny = g->ny;
    const long n = ASZ(g);
    const double dx = g->dx, dy = g->dy, eps = 1.0e-100;
    double *gx = zalloc(n), *gy = zalloc(n), *sz = zalloc(n);
    for (int i = NB; i < nx + NB; i++)
        for (int j = NB; j < ny + NB; j++) {
            const long k = IX(g, i, j);
            gx[k] = (ls[IX(g, i + 1, j)] - ls[IX(g, i - 1, j)]) / (2.0 * dx);
            gy[k] = (ls[IX(g, i, j + 1)] - ls[IX(g, i, j - 1)]) / (2.0 * dy);
            sz[k] = sqrt(gx[k] * gx[k] + gy[k] * gy[k] + eps);
        }
    const double lim = 1.0 / (dx < dy ? dx : dy);
    for (int i = NB; i < nx + NB; i++)
        for (int j = NB; j < ny + NB; j++) {
            const long k = IX(g, i, j);
            double kap = (gx[k] * gx[k] * (ls[IX(g, i, j - 1)] - 2.0 * ls[k] + ls[IX(g, i, j + 1)]) / (dy * dy) -
                          2.0 * gx[k] * gy[k] * (gx[IX(g, i, j + 1)] - gx[IX(g, i, j - 1)]) / (2.0 * dy) +
                          gy[k] * gy[k] * (ls[IX(g, i - 1, j)] - 2.0 * ls[k] + ls[IX(g, i + 1, j)]) / (dx * dx)) /
                         pow(sz[k], 3.0);
            kappa[k] = isgn(kap) * fabs(smin(fabs(kap), lim));
        }
    free(gx); free(gy); free(sz);
}

/* MACSolver2D::UpdateNTK, mac2d.cpp:124-219, as far as the reference goes.
 * Q = |1 - |grad phi|| with the ENO gradient ENO_DerivAbsLS_2D(phi, phi)
 * (:138-145).  Where Q <= 1e-4 the unit normal from central differences is
 * stored (:204-209).  Where Q > 1e-4 the reference picks one-sided
 * derivatives but its curve-fitting branch is empty, so nothing is stored
 * (:150-201).  Cells not stored keep what nxo / nyo held on entry. */
void ora_ntk(const ora_grid *g, const double *ls, double *nxo, double *nyo) {
    const double eta = 0.0001, eps = 1.0e-100;
    double *ab = zalloc(ASZ(g));
    ora_eno_absgrad(g, ls, ls, ab);
    for (int i = NB; i < g->nx + NB; i++)
        for (int j = NB; j < g->ny + NB; j++) {
            const long k = IX(g, i, j);
            if (fabs(1.0 - ab[k]) > eta) continue;
            const double gx = (ls[IX(g, i + 1, j)] - ls[IX(g, i - 1, j)]) / (2.0 * g->dx);
            const double gy = (ls[IX(g, i, j + 1)] - ls[IX(g, i, j - 1)]) / (2.0 * g->dy);
            nxo[k] = 1.0 / sqrt(gx * gx + gy * gy + eps) * gx;
            nyo[k] = 1.0 / sqrt(gx * gx + gy * gy + eps) * gy;
        }
    free(ab);
}

/* UpdateHeavisideFunc, mac2d.cpp:87-101 (all cells) */
void ora_heaviside(const ora_grid *g, const double *ls, double *H) {
    const long n = ASZ(g);
    for (long k = 0; k < n; k++) H[k] = ls[k] >= 0.0 ? 1.0 : 0.0;
}

/* UpdateSmoothHeavisideFunc, mac2d.cpp:103-122 (all cells) */
void ora_smooth_heaviside(const ora_grid *g, const double *ls, double *HS) {
    const long n = ASZ(g);
    const double eps = (g->dx < g->dy ? g->dx : g->dy) * 1.5;
    for (long k = 0; k < n; k++) {
        if (ls[k] > eps)
            HS[k] = 1.0;
        else if (ls[k] < -eps)
            HS[k] = 0.0;
        else
            HS[k] = 0.5 * (1.0 + ls[k] / eps + 1.0 / M_PI * sin(M_PI * ls[k] / eps));
    }
}

/* AddConvectionFU, mac2d.cpp:308-387.  tmpV is 0 outside the u-interior. */
void ora_conv_u(const ora_grid *g, const double *u, const double *v, double *cU) {
    const int nx = g->nx, ny = g->ny;
    const long n = ASZ(g);
    double *tv = zalloc(n), *Fx = zalloc(n), *Fy = zalloc(n);
    for (int j = NB; j < ny + NB; j++)
        for (int i = NB + 1; i < nx + NB; i++)
            tv[IX(g, i, j)] = (v[IX(g, i, j)] + v[IX(g, i - 1, j)] + v[IX(g, i - 1, j + 1)] + v[IX(g, i, j + 1)]) * 0.25;
    for (long k = 0; k < n; k++) { Fx[k] = u[k] * u[k]; Fy[k] = u[k] * tv[k]; }
    memset(cU, 0, sizeof(double) * n);
    weno_blend(g, Fx, Fy, u, tv, NB + 1, NB, cU);
    free(tv); free(Fx); free(Fy);
}

/* AddConvectionFV, mac2d.cpp:389-463.  tmpU is 0 outside the v-interior. */
void ora_conv_v(const ora_grid *g, const double *u, const double *v, double *cV) {
    const int nx = g->nx, ny = g->ny;
    const long n = ASZ(g);
    double *tu = zalloc(n), *Fx = zalloc(n), *Fy = zalloc(n);
    for (int j = NB + 1; j < ny + NB; j++)
        for (int i = NB; i < nx + NB; i++)
            tu[IX(g, i, j)] = (u[IX(g, i, j)] + u[IX(g, i, j - 1)] + u[IX(g, i + 1, j - 1)] + u[IX(g, i + 1, j)]) * 0.25;
    for (long k = 0; k < n; k++) { Fx[k] = v[k] * tu[k]; Fy[k] = v[k] * v[k]; }
    memset(cV, 0, sizeof(double) * n);
    weno_blend(g, Fx, Fy, tu, v, NB, NB + 1, cV);
    free(tu); free(Fx); free(Fy);
}

static inline double re_positive(const ora_fluid *f) {
    /* kRe = rhoH * L * U / muH with L = U = 1 (mac2d.cpp:33); viscosity is
     * skipped when kRe <= 0 (:598, :838). */
    return f->rho_h / f->mu_h;
}

/* AddViscosityFU, mac2d.cpp:570-809 */
void ora_visc_u(const ora_grid *g, const ora_fluid *f, const double *u, const double *v, const double *ls,
                const double *H, double *dU) {
    const int nx = g->nx, ny = g->ny;
    const long n = ASZ(g);
    const double dx = g->dx, dy = g->dy, rH = f->rho_h, rL = f->rho_l;
    memset(dU, 0, sizeof(double) * n);
    if (!(re_positive(f) > 0.0)) return;
    double *mu = zalloc(n);
    for (int i = NB; i < nx + NB; i++)
        for (int j = NB; j < ny + NB; j++) mu[IX(g, i, j)] = f->mu_l + (f->mu_h - f->mu_l) * H[IX(g, i, j)];
#define LS(a, b) ls[IX(g, i + (a), j + (b))]
#define MU(a, b) mu[IX(g, i + (a), j + (b))]
    for (int i = NB + 1; i < nx + NB; i++)
        for (int j = NB; j < ny + NB; j++) {
            const double uM = u[IX(g, i, j)], uW = u[IX(g, i - 1, j)], uE = u[IX(g, i + 1, j)],
                         uS = u[IX(g, i, j - 1)], uN = u[IX(g, i, j + 1)];
            const double vW = v[IX(g, i - 1, j)], vW_N = v[IX(g, i - 1, j + 1)], vM = v[IX(g, i, j)],
                         vN = v[IX(g, i, j + 1)];
            const double lsW = LS(-1, 0), lsM = LS(0, 0);
            const double lsUNHalf = 0.25 * (LS(0, 0) + LS(-1, 0) + LS(-1, 1) + LS(0, 1));
            const double lsUSHalf = 0.25 * (LS(0, 0) + LS(-1, 0) + LS(-1, -1) + LS(0, -1));
            double th, iWE = 0.0, iSN = 0.0;
            /* :687-714 */
            if (lsW >= 0 && lsM >= 0) iWE = 1.0 / rH;
            else if (lsW <= 0 && lsM <= 0) iWE = 1.0 / rL;
            else if (lsW > 0 && lsM <= 0) {
                th = fabs(lsW) / (fabs(lsW) + fabs(lsM));
                iWE = 1.0 / (rL * rH) / (1.0 / rL * th + 1.0 / rH * (1.0 - th));
            } else if (lsW <= 0 && lsM > 0) {
                th = fabs(lsW) / (fabs(lsW) + fabs(lsM));
                iWE = 1.0 / (rH * rL) / (1.0 / rH * th + 1.0 / rL * (1.0 - th));
            }
            /* :716-743 */
            if (lsUSHalf >= 0 && lsUNHalf >= 0) iSN = 1.0 / rH;
            else if (lsUSHalf <= 0 && lsUNHalf <= 0) iSN = 1.0 / rL;
            else if (lsUSHalf > 0 && lsUNHalf <= 0) {
                th = fabs(lsUSHalf) / (fabs(lsUSHalf) + fabs(lsUNHalf));
                iSN = 1.0 / (rL * rH) / (1.0 / rL * th + 1.0 / rH * (1.0 - th));
            } else if (lsUSHalf <= 0 && lsUNHalf > 0) {
                th = fabs(lsUSHalf) / (fabs(lsUSHalf) + fabs(lsUNHalf));
                iSN = 1.0 / (rH * rL) / (1.0 / rH * th + 1.0 / rL * (1.0 - th));
            }
            /* :745-760 */
            const double muU_X_W = MU(-1, 0) * (uM - uW) / dx;
            const double muU_X_E = MU(0, 0) * (uE - uM) / dx;
            const double muU_Y_S = 0.25 * (MU(0, 0) + MU(-1, 0) + MU(-1, -1) + MU(0, -1)) * (uM - uS) / dy;
            const double muU_Y_N = 0.25 * (MU(0, 0) + MU(-1, 0) + MU(-1, 1) + MU(0, 1)) * (uN - uM) / dy;
            const double muV_X_S = 0.25 * (MU(0, 0) + MU(-1, 0) + MU(-1, -1) + MU(0, -1)) * (vM - vW) / dx;
            const double muV_X_N = 0.25 * (MU(0, 0) + MU(-1, 0) + MU(-1, 1) + MU(0, 1)) * (vN - vW_N) / dx;
            const double visX = 2.0 * (muU_X_E - muU_X_W) / dx;
            const double visY = (muU_Y_N - muU_Y_S) / dy + (muV_X_N - muV_X_S) / dy;
            dU[IX(g, i, j)] = visX * iWE + visY * iSN;
        }
#undef LS
#undef MU
    free(mu);
}

/* AddViscosityFV, mac2d.cpp:811-1041 (harmonic 1/rho overwritten by the
 * arithmetic 1/rhoEff at :1000-1001, as the reference does). */
void ora_visc_v(const ora_grid *g, const ora_fluid *f, const double *u, const double *v, const double *ls,
                const double *H, double *dV) {
    const int nx = g->nx, ny = g->ny;
    const long n = ASZ(g);
    const double dx = g->dx, dy = g->dy, rH = f->rho_h, rL = f->rho_l;
    memset(dV, 0, sizeof(double) * n);
    if (!(re_positive(f) > 0.0)) return;
    double *mu = zalloc(n);
    for (int i = NB; i < nx + NB; i++)
        for (int j = NB; j < ny + NB; j++) mu[IX(g, i, j)] = f->mu_l + (f->mu_h - f->mu_l) * H[IX(g, i, j)];
#define LS(a, b) ls[IX(g, i + (a), j + (b))]
#define MU(a, b) mu[IX(g, i + (a), j + (b))]
    for (int i = NB; i < nx + NB; i++)
        for (int j = NB + 1; j < ny + NB; j++) {
            const double vW = v[IX(g, i - 1, j)], vE = v[IX(g, i + 1, j)], vS = v[IX(g, i, j - 1)],
                         vN = v[IX(g, i, j + 1)], vM = v[IX(g, i, j)];
            const double uM = u[IX(g, i, j)], uE = u[IX(g, i + 1, j)], uS = u[IX(g, i, j - 1)],
                         uE_S = u[IX(g, i + 1, j - 1)];
            const double lsVWHalf = 0.25 * (LS(0, 0) + LS(-1, 0) + LS(-1, -1) + LS(0, -1));
            const double lsVEHalf = 0.25 * (LS(0, 0) + LS(1, 0) + LS(1, -1) + LS(0, -1));
            const double lsM = LS(0, 0), lsS = LS(0, -1);
            double th, rWE = 0.0, rSN = 0.0;
            /* :939-966 */
            if (lsVWHalf >= 0 && lsVEHalf >= 0) rWE = rH;
            else if (lsVWHalf <= 0 && lsVEHalf <= 0) rWE = rL;
            else if (lsVWHalf > 0 && lsVEHalf <= 0) {
                th = fabs(lsVWHalf) / (fabs(lsVWHalf) + fabs(lsVEHalf));
                rWE = rH * th + rL * (1.0 - th);
            } else if (lsVWHalf <= 0 && lsVEHalf > 0) {
                th = fabs(lsVWHalf) / (fabs(lsVWHalf) + fabs(lsVEHalf));
                rWE = rL * th + rH * (1.0 - th);
            }
            /* :968-995 */
            if (lsS >= 0 && lsM >= 0) rSN = rH;
            else if (lsS <= 0 && lsM <= 0) rSN = rL;
            else if (lsS > 0 && lsM <= 0) {
                th = fabs(lsS) / (fabs(lsS) + fabs(lsM));
                rSN = rH * th + rL * (1.0 - th);
            } else if (lsS <= 0 && lsM > 0) {
                th = fabs(lsS) / (fabs(lsS) + fabs(lsM));
                rSN = rL * th + rH * (1.0 - th);
            }
            const double iWE = 1.0 / rWE, iSN = 1.0 / rSN;
            /* :1002-1023 */
            const double muU_Y_W = 0.25 * (MU(0, 0) + MU(-1, 0) + MU(-1, -1) + MU(0, -1)) * (uM - uS) / dy;
            const double muU_Y_E = 0.25 * (MU(0, 0) + MU(1, 0) + MU(1, -1) + MU(0, -1)) * (uE - uE_S) / dy;
            const double muV_X_W = 0.25 * (MU(0, 0) + MU(-1, 0) + MU(-1, -1) + MU(0, -1)) * (vM - vW) / dx;
            const double muV_X_E = 0.25 * (MU(0, 0) + MU(1, 0) + MU(1, -1) + MU(0, -1)) * (vE - vM) / dx;
            const double muV_Y_S = MU(0, -1) * (vM - vS) / dy;
            const double muV_Y_N = MU(0, 0) * (vN - vM) / dy;
            const double visX = (muU_Y_E - muU_Y_W) / dx + (muV_X_E - muV_X_W) / dx;
            const double visY = 2.0 * (muV_Y_N - muV_Y_S) / dy;
            dV[IX(g, i, j)] = visX * iWE + visY * iSN;
        }
#undef LS
#undef MU
    free(mu);
}

/* Gravity (AddGravityFU/FV, mac2d.cpp:1043-1079).  kG = g, kFr = 1/g with
 * L = U = 1 (mac2d.cpp:33-35).  UpdateFV takes AddGravityFU (:294) unless
 * fix_gravity is set. */
static int gravity_on(const ora_fluid *f, int axis) {
    const double fr = 1.0 / f->g;
    return (fr != 0 || f->g != 0.0) && !isnan(fr) && !isinf(fr) && f->g_axis == axis;
}

/* UpdateFU, mac2d.cpp:254-279 */
void ora_rhs_u(const ora_grid *g, const ora_fluid *f, const double *ls, const double *u, const double *v,
               const double *H, double *FU) {
    const long n = ASZ(g);
    double *cU = zalloc(n), *vU = zalloc(n);
    ora_conv_u(g, u, v, cU);
    ora_visc_u(g, f, u, v, ls, H, vU);
    const double gU = gravity_on(f, 0) ? -f->g : 0.0;
    memset(FU, 0, sizeof(double) * n);
    for (int i = NB + 1; i < g->nx + NB; i++)
        for (int j = NB; j < g->ny + NB; j++) {
            const long k = IX(g, i, j);
            FU[k] = -cU[k] + vU[k] + gU;
        }
    free(cU); free(vU);
}

/* UpdateFV, mac2d.cpp:281-306 */
void ora_rhs_v(const ora_grid *g, const ora_fluid *f, const double *ls, const double *u, const double *v,
               const double *H, double *FV) {
    const long n = ASZ(g);
    double *cV = zalloc(n), *vV = zalloc(n);
    ora_conv_v(g, u, v, cV);
    ora_visc_v(g, f, u, v, ls, H, vV);
    memset(FV, 0, sizeof(double) * n);
    for (int i = NB; i < g->nx + NB; i++)
        for (int j = NB + 1; j < g->ny + NB; j++) {
            const long k = IX(g, i, j);
            double gV;
            if (f->fix_gravity)
                gV = gravity_on(f, 1) ? -f->g : 0.0;
            else /* the AddGravityFU pattern: nonzero for i >= 4 only */
                gV = (gravity_on(f, 0) && i >= NB + 1) ? -f->g : 0.0;
            FV[k] = -cV[k] + vV[k] + gV;
        }
    free(cV); free(vV);
}

/* GetIntermediateVel, mac2d.cpp:1081-1239 */
void ora_intermediate_vel(const ora_grid *g, const ora_fluid *f, double dt, const double *ls, const double *u,
                          const double *v, double *uhat, double *vhat, const double *H) {
    const int nx = g->nx, ny = g->ny;
    const long n = ASZ(g);
    double *FU1 = zalloc(n), *FV1 = zalloc(n), *FU2 = zalloc(n), *FV2 = zalloc(n);
#define ULOOP for (int i = NB + 1; i < nx + NB; i++) for (int j = NB; j < ny + NB; j++)
#define VLOOP for (int i = NB; i < nx + NB; i++) for (int j = NB + 1; j < ny + NB; j++)
    if (f->time_order == 0) {
        ora_rhs_u(g, f, ls, u, v, H, FU1);
        ora_rhs_v(g, f, ls, u, v, H, FV1);
        ULOOP uhat[IX(g, i, j)] = u[IX(g, i, j)] + dt * FU1[IX(g, i, j)];
        VLOOP vhat[IX(g, i, j)] = v[IX(g, i, j)] + dt * FV1[IX(g, i, j)];
    } else if (f->time_order == 1) {
        ora_rhs_u(g, f, ls, u, v, H, FU1);
        ora_rhs_v(g, f, ls, u, v, H, FV1);
        ULOOP FU2[IX(g, i, j)] = u[IX(g, i, j)] + dt * FU1[IX(g, i, j)];
        VLOOP FV2[IX(g, i, j)] = v[IX(g, i, j)] + dt * FV1[IX(g, i, j)];
        ora_bc_u(g, FU2);
        ora_bc_v(g, FV2);
        ora_rhs_u(g, f, ls, FU2, FV2, H, FU1);
        ora_rhs_v(g, f, ls, FU2, FV2, H, FV1);
        ULOOP FU2[IX(g, i, j)] = FU2[IX(g, i, j)] + dt * FU1[IX(g, i, j)];
        VLOOP FV2[IX(g, i, j)] = FV2[IX(g, i, j)] + dt * FV1[IX(g, i, j)];
        ULOOP uhat[IX(g, i, j)] = 0.5 * u[IX(g, i, j)] + 0.5 * FU2[IX(g, i, j)];
        VLOOP vhat[IX(g, i, j)] = 0.5 * v[IX(g, i, j)] + 0.5 * FV2[IX(g, i, j)];
    } else {
        /* RK3, :1145-1220 */
        ora_rhs_u(g, f, ls, u, v, H, FU1);
        ora_rhs_v(g, f, ls, u, v, H, FV1);
        ULOOP FU2[IX(g, i, j)] = u[IX(g, i, j)] + dt * FU1[IX(g, i, j)];
        VLOOP FV2[IX(g, i, j)] = v[IX(g, i, j)] + dt * FV1[IX(g, i, j)];
        ora_bc_u(g, FU2);
        ora_bc_v(g, FV2);
        ora_rhs_u(g, f, ls, FU2, FV2, H, FU1);
        ora_rhs_v(g, f, ls, FU2, FV2, H, FV1);
        ULOOP FU2[IX(g, i, j)] = FU2[IX(g, i, j)] + dt * FU1[IX(g, i, j)];
        VLOOP FV2[IX(g, i, j)] = FV2[IX(g, i, j)] + dt * FV1[IX(g, i, j)];
        memset(FU1, 0, sizeof(double) * n);
        memset(FV1, 0, sizeof(double) * n);
        ULOOP FU1[IX(g, i, j)] = 0.75 * u[IX(g, i, j)] + 0.25 * FU2[IX(g, i, j)];
        VLOOP FV1[IX(g, i, j)] = 0.75 * v[IX(g, i, j)] + 0.25 * FV2[IX(g, i, j)];
        ora_bc_u(g, FU1);
        ora_bc_v(g, FV1);
        ora_rhs_u(g, f, ls, FU1, FV1, H, FU2);
        ora_rhs_v(g, f, ls, FU1, FV1, H, FV2);
        ULOOP FU1[IX(g, i, j)] = FU1[IX(g, i, j)] + dt * FU2[IX(g, i, j)];
        VLOOP FV1[IX(g, i, j)] = FV1[IX(g, i, j)] + dt * FV2[IX(g, i, j)];
        ULOOP uhat[IX(g, i, j)] = 1.0 / 3.0 * u[IX(g, i, j)] + 2.0 / 3.0 * FU1[IX(g, i, j)];
        VLOOP vhat[IX(g, i, j)] = 1.0 / 3.0 * v[IX(g, i, j)] + 2.0 / 3.0 * FV1[IX(g, i, j)];
    }
#undef ULOOP
#undef VLOOP
    free(FU1); free(FV1); free(FU2); free(FV2);
}

/* GetDivergence, mac2d.cpp:1729-1738 */
void ora_divergence(const ora_grid *g, const double *u, const double *v, double *div) {
    memset(div, 0, sizeof(double) * ASZ(g));
    for (int i = NB; i < g->nx + NB; i++)
        for (int j = NB; j < g->ny + NB; j++)
            div[IX(g, i, j)] = (u[IX(g, i + 1, j)] - u[IX(g, i, j)]) / g->dx + (v[IX(g, i, j + 1)] - v[IX(g, i, j)]) / g->dy;
}

/* Face theta rule of the GFM (mac2d.cpp:1341-1358 and the three copies that
 * follow; UpdateVel :1770-1786).  a is the "first" cell of the pair as the
 * reference orders it, b the second; heavy = fraction of the face on the
 * heavy side, th = the kappa interpolation weight. */
static inline void gfm_theta_first(double lsA, double lsB, double *thH, double *th) {
    /* pair (W, M) or (S, M): thetaH weights lsM when lsW < 0 */
    if (lsA >= 0.0 && lsB >= 0.0) { *thH = 1.0; *th = 0.0; }
    else if (lsA < 0.0 && lsB < 0.0) { *thH = 0.0; *th = 0.0; }
    else if (lsA >= 0.0 && lsB < 0.0) {
        *thH = fabs(lsA) / (fabs(lsA) + fabs(lsB));
        *th = fabs(lsA) / (fabs(lsA) + fabs(lsB));
    } else {
        *thH = fabs(lsB) / (fabs(lsA) + fabs(lsB));
        *th = fabs(lsA) / (fabs(lsA) + fabs(lsB));
    }
}
static inline void gfm_theta_second(double lsM, double lsE, double *thH, double *th) {
    /* pair (M, E) or (M, N), mac2d.cpp:1372-1388 */
    if (lsM >= 0.0 && lsE >= 0.0) { *thH = 1.0; *th = 0.0; }
    else if (lsM < 0.0 && lsE < 0.0) { *thH = 0.0; *th = 0.0; }
    else if (lsM >= 0.0 && lsE < 0.0) {
        *thH = fabs(lsM) / (fabs(lsM) + fabs(lsE));
        *th = fabs(lsE) / (fabs(lsM) + fabs(lsE));
    } else {
        *thH = fabs(lsE) / (fabs(lsM) + fabs(lsE));
        *th = fabs(lsE) / (fabs(lsM) + fabs(lsE));
    }
}

static int p_all_neumann(const ora_grid *g) {
    for (int s = 0; s < 4; s++) {
        const int b = g->bc_p[s];
        if (!(b == ORA_NEUMANN || b == ORA_AXISYM || b == ORA_WALL)) return 0;
    }
    return 1;
}
static int p_dirichlet_like(int b) {
    /* assembly's Dirichlet branch includes WALL (mac2d.cpp:1521-1523) */
    return b == ORA_DIRICHLET || b == ORA_INLET || b == ORA_OUTLET || b == ORA_PRESSURE || b == ORA_WALL;
}

int ora_gfm_assemble(const ora_grid *g, const ora_fluid *f, double dt, const double *ls, double *kappa,
                     const double *H, const double *div, int recompute_kappa, double *diag, double *cw,
                     double *ce, double *cs, double *cn, double *rhs) {
    const int nx = g->nx, ny = g->ny;
    const double dx = g->dx, dy = g->dy, rH = f->rho_h, rL = f->rho_l, sig = f->sigma;
    if (recompute_kappa) {
        ora_kappa(g, ls, kappa);
        ora_bc_p(g, kappa);
    }
    const int pin = p_all_neumann(g);
    for (int j = NB; j < ny + NB; j++)
        for (int i = NB; i < nx + NB; i++) {
            const long c = IX(g, i, j);
            const int k = (i - NB) + nx * (j - NB);
            const double lsW = ls[IX(g, i - 1, j)], lsE = ls[IX(g, i + 1, j)], lsM = ls[c], lsS = ls[IX(g, i, j - 1)],
                         lsN = ls[IX(g, i, j + 1)];
            double thH, th, rhoEff, kEff;
            /* west face, :1341-1367 */
            gfm_theta_first(lsW, lsM, &thH, &th);
            rhoEff = rH * thH + rL * (1.0 - thH);
            double iW = 1.0 / rhoEff;
            kEff = kappa[c] * th + kappa[IX(g, i - 1, j)] * (1.0 - th);
            double FW = -dt * (-sig * kEff) * (H[c] - H[IX(g, i - 1, j)]);
            FW *= iW / (dx * dx);
            /* east face, :1372-1395 */
            gfm_theta_second(lsM, lsE, &thH, &th);
            rhoEff = rH * thH + rL * (1.0 - thH);
            double iE = 1.0 / rhoEff;
            kEff = kappa[c] * th + kappa[IX(g, i + 1, j)] * (1.0 - th);
            double FE = dt * (-sig * kEff) * (H[IX(g, i + 1, j)] - H[c]);
            FE *= iE / (dx * dx);
            /* south face, :1398-1422 */
            gfm_theta_first(lsS, lsM, &thH, &th);
            rhoEff = rH * thH + rL * (1.0 - thH);
            double iS = 1.0 / rhoEff;
            kEff = kappa[c] * th + kappa[IX(g, i, j - 1)] * (1.0 - th);
            double FS = -dt * (-sig * kEff) * (H[c] - H[IX(g, i, j - 1)]);
            FS *= iS / (dy * dy);
            /* north face, :1425-1448 */
            gfm_theta_second(lsM, lsN, &thH, &th);
            rhoEff = rH * thH + rL * (1.0 - thH);
            double iN = 1.0 / rhoEff;
            kEff = kappa[c] * th + kappa[IX(g, i, j + 1)] * (1.0 - th);
            double FN = dt * (-sig * kEff) * (H[IX(g, i, j + 1)] - H[c]);
            FN *= iN / (dy * dy);
            double r = 0.0;
            r -= FW + FE + FS + FN; /* :1454 */
            r -= div[c];            /* :1468-1470 */
            /* Row values (:1497-1513): coefficients are negated 1/rho. */
            iS *= -1.0; iW *= -1.0; iE *= -1.0; iN *= -1.0;
            double aS = iS / (dy * dy), aW = iW / (dx * dx), aE = iE / (dx * dx), aN = iN / (dy * dy);
            double aC = -(iW + iE) / (dx * dx) - (iS + iN) / (dy * dy);
            /* boundary edits, :1515-1583 */
            if (i == NB && g->bc_p[0] == ORA_NEUMANN) { aW = 0.0; aC += iW / (dx * dx); }
            else if (i == NB && p_dirichlet_like(g->bc_p[0])) { aW = 0.0; r -= iW / (dx * dx) * (g->cp[0]); }
            if (i == NB + nx - 1 && g->bc_p[1] == ORA_NEUMANN) { aE = 0.0; aC += iE / (dx * dx); }
            else if (i == NB + nx - 1 && p_dirichlet_like(g->bc_p[1])) { aE = 0.0; r -= iE / (dx * dx) * (g->cp[1]); }
            if (j == NB && g->bc_p[2] == ORA_NEUMANN) { aS = 0.0; aC += iS / (dy * dy); }
            else if (j == NB && p_dirichlet_like(g->bc_p[2])) { aS = 0.0; r -= iS / (dy * dy) * (g->cp[2]); }
            if (j == NB + ny - 1 && g->bc_p[3] == ORA_NEUMANN) { aN = 0.0; aC += iN / (dy * dy); }
            else if (j == NB + ny - 1 && p_dirichlet_like(g->bc_p[3])) { aN = 0.0; r -= iN / (dy * dy) * (g->cp[3]); }
            /* (periodic pressure, :1530-1582, is out of scope and rejected by
             * the product; here it simply keeps the interior coefficients.) */
            diag[k] = aC;
            cw[k] = -aW;
            ce[k] = -aE;
            cs[k] = -aS;
            cn[k] = -aN;
            rhs[k] = r;
        }
    if (pin) {
        /* corrected pin: cell 0 held at ps = 0 (the reference zeroes ps before
         * assembly, :1324-1328, so its rhs correction terms are 0). */
        rhs[0] = 0.0;
        if (nx > 1) cw[1] = 0.0;
        if (ny > 1) cs[nx] = 0.0;
    }
    return pin;
}

int ora_gfm_to_csr(const ora_grid *g, const double *diag, const double *cw, const double *ce, const double *cs,
                   const double *cn, const double *rhs, int pinned, double *a, int32_t *ia, int32_t *ja,
                   double *b) {
    const int nx = g->nx, ny = g->ny;
    int row = 0, nnz = 0;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const int k = i + nx * j;
            if (pinned && k == 0) continue;
            const int sh = pinned ? 1 : 0;
            ia[row] = nnz;
            if (j > 0 && cs[k] != 0.0 && !(pinned && k - nx == 0)) { a[nnz] = -cs[k]; ja[nnz++] = k - nx - sh; }
            if (i > 0 && cw[k] != 0.0 && !(pinned && k - 1 == 0)) { a[nnz] = -cw[k]; ja[nnz++] = k - 1 - sh; }
            a[nnz] = diag[k]; ja[nnz++] = k - sh;
            if (i < nx - 1 && ce[k] != 0.0) { a[nnz] = -ce[k]; ja[nnz++] = k + 1 - sh; }
            if (j < ny - 1 && cn[k] != 0.0) { a[nnz] = -cn[k]; ja[nnz++] = k + nx - sh; }
            b[row] = rhs[k];
            row++;
        }
    ia[row] = nnz;
    return row;
}

void ora_gfm_apply(int nx, int ny, const double *diag, const double *cw, const double *ce, const double *cs,
                   const double *cn, int pinned, const double *x, double *y) {
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const int k = i + nx * j;
            if (pinned && k == 0) { y[k] = 0.0; continue; }
            /* row order S, W, C, E, N as in the reference CSR */
            double s = 0.0;
            if (j > 0) s += -cs[k] * x[k - nx];
            if (i > 0) s += -cw[k] * x[k - 1];
            s += diag[k] * x[k];
            if (i < nx - 1) s += -ce[k] * x[k + 1];
            if (j < ny - 1) s += -cn[k] * x[k + nx];
            y[k] = s;
        }
}

static double dotn(long n, const double *a, const double *b) {
    double s = 0.0;
    for (long k = 0; k < n; k++) s += a[k] * b[k];
    return s;
}

static double true_residual(int nx, int ny, const double *diag, const double *cw, const double *ce,
                            const double *cs, const double *cn, int pinned, const double *b, const double *x) {
    const long n = (long)nx * ny;
    double *Ax = zalloc(n);
    ora_gfm_apply(nx, ny, diag, cw, ce, cs, cn, pinned, x, Ax);
    double rr = 0.0, bb = 0.0;
    for (long k = 0; k < n; k++) {
        if (pinned && k == 0) continue;
        rr += (b[k] - Ax[k]) * (b[k] - Ax[k]);
        bb += b[k] * b[k];
    }
    free(Ax);
    if (bb == 0.0) bb = 1.0;
    return sqrt(rr) / sqrt(bb);
}

int ora_pcg(int nx, int ny, const double *diag, const double *cw, const double *ce, const double *cs,
            const double *cn, int pinned, const double *b, double *x, double tol, int maxit, int mode,
            double *resid, double *true_resid) {
    const long n = (long)nx * ny;
    double *r = zalloc(n), *z = zalloc(n), *p = zalloc(n), *q = zalloc(n), *Minv = zalloc(n);
    for (long k = 0; k < n; k++) {
        x[k] = 0.0;
        Minv[k] = (pinned && k == 0) ? 0.0 : 1.0 / diag[k]; /* InvertMatrixDiagonal :577-585 */
        r[k] = (pinned && k == 0) ? 0.0 : b[k];
    }
    double bn = sqrt(dotn(n, r, r));
    if (bn == 0.0) bn = 1.0; /* :336-337 */
    double rn = sqrt(dotn(n, r, r)), res = rn / bn;
    int it = 0;
    const double ett = (mode == 1) ? tol * tol : 0.0;
    if (mode == 1) {
        /* reference iteration, poisson2d.cpp:331-394 */
        memcpy(p, r, sizeof(double) * n);
        double rho1 = 1.0;
        int conv = res <= tol;
        while (it < maxit && !conv) {
            for (long k = 0; k < n; k++) z[k] = Minv[k] * r[k];
            const double rho = dotn(n, r, z);
            if (it == 1) memcpy(p, z, sizeof(double) * n);
            else {
                const double beta = rho / rho1;
                for (long k = 0; k < n; k++) p[k] *= beta;
                for (long k = 0; k < n; k++) p[k] += 1.0 * z[k];
            }
            ora_gfm_apply(nx, ny, diag, cw, ce, cs, cn, pinned, p, q);
            const double alpha = rho / (dotn(n, p, q) + ett);
            for (long k = 0; k < n; k++) x[k] += alpha * p[k];
            for (long k = 0; k < n; k++) r[k] += -alpha * q[k];
            rn = sqrt(dotn(n, r, r));
            res = rn / bn;
            if (res <= tol) conv = 1;
            rho1 = rho;
            it++;
        }
    } else {
        double rho_old = 0.0;
        while (it < maxit && res > tol) {
            for (long k = 0; k < n; k++) z[k] = Minv[k] * r[k];
            const double rho = dotn(n, r, z);
            if (it == 0) memcpy(p, z, sizeof(double) * n);
            else {
                const double beta = rho / rho_old;
                for (long k = 0; k < n; k++) p[k] = z[k] + beta * p[k];
            }
            ora_gfm_apply(nx, ny, diag, cw, ce, cs, cn, pinned, p, q);
            const double alpha = rho / dotn(n, p, q);
            for (long k = 0; k < n; k++) { x[k] += alpha * p[k]; r[k] -= alpha * q[k]; }
            rho_old = rho;
            res = sqrt(dotn(n, r, r)) / bn;
            it++;
        }
    }
    if (resid) *resid = res;
    if (true_resid) *true_resid = true_residual(nx, ny, diag, cw, ce, cs, cn, pinned, b, x);
    free(r); free(z); free(p); free(q); free(Minv);
    return it;
}

int ora_bicgstab(int nx, int ny, const double *diag, const double *cw, const double *ce, const double *cs,
                 const double *cn, int pinned, const double *b, double *x, double tol, int maxit, int mode,
                 double *resid, double *true_resid) {
    /* poisson2d.cpp:403-575 (right Jacobi preconditioning, IML++ form).
     * mode 1 keeps the reference's rho_2 = 1 for every iteration (the loop
     * never assigns it); mode 0 carries rho_2 = rho_1 as IML++ does. */
    const long n = (long)nx * ny;
    double *r = zalloc(n), *rt = zalloc(n), *v = zalloc(n), *p = zalloc(n), *ph = zalloc(n), *s = zalloc(n),
           *sh = zalloc(n), *t = zalloc(n), *Minv = zalloc(n);
    for (long k = 0; k < n; k++) {
        x[k] = 0.0;
        Minv[k] = (pinned && k == 0) ? 0.0 : 1.0 / diag[k];
        r[k] = (pinned && k == 0) ? 0.0 : b[k];
    }
    memcpy(rt, r, sizeof(double) * n);
    double bn = sqrt(dotn(n, r, r));
    if (bn == 0.0) bn = 1.0;
    double rn = sqrt(dotn(n, r, r)), res = rn / bn;
    double alpha = 1.0, omega = 1.0, rho1 = 1.0, rho2 = 1.0;
    int it = 0, conv = res <= tol;
    while (it < maxit && !conv) {
        rho1 = dotn(n, rt, r);
        if (rho1 == 0.0) break;
        if (it == 1) memcpy(p, r, sizeof(double) * n);
        else {
            const double beta = (rho1 / rho2) * (alpha / omega);
            for (long k = 0; k < n; k++) p[k] += -omega * v[k];
            for (long k = 0; k < n; k++) p[k] *= beta;
            for (long k = 0; k < n; k++) p[k] += 1.0 * r[k];
        }
        for (long k = 0; k < n; k++) ph[k] = Minv[k] * p[k];
        ora_gfm_apply(nx, ny, diag, cw, ce, cs, cn, pinned, ph, v);
        alpha = rho1 / dotn(n, rt, v);
        for (long k = 0; k < n; k++) s[k] = r[k] - alpha * v[k];
        res = sqrt(dotn(n, s, s)) / bn;
        if (res < tol) {
            for (long k = 0; k < n; k++) x[k] += alpha * ph[k];
            conv = 1;
            break;
        }
        for (long k = 0; k < n; k++) sh[k] = Minv[k] * s[k];
        ora_gfm_apply(nx, ny, diag, cw, ce, cs, cn, pinned, sh, t);
        omega = dotn(n, t, s) / dotn(n, t, t);
        for (long k = 0; k < n; k++) x[k] += alpha * ph[k];
        for (long k = 0; k < n; k++) x[k] += omega * sh[k];
        for (long k = 0; k < n; k++) r[k] = s[k] - omega * t[k];
        rn = sqrt(dotn(n, r, r));
        res = rn / bn;
        if (res <= tol) conv = 1;
        if (mode == 0) rho2 = rho1;
        it++;
    }
    if (resid) *resid = res;
    if (true_resid) *true_resid = true_residual(nx, ny, diag, cw, ce, cs, cn, pinned, b, x);
    free(r); free(rt); free(v); free(p); free(ph); free(s); free(sh); free(t); free(Minv);
    return it;
}

/* UpdateVel, mac2d.cpp:1740-1849 (u = uhat - grad ps / rho + GFM jump term) */
void ora_update_vel(const ora_grid *g, const ora_fluid *f, double dt, double *u, double *v, const double *us,
                    const double *vs, const double *ps, const double *ls, const double *H,
                    const double *kappa) {
    const int nx = g->nx, ny = g->ny;
    const double dx = g->dx, dy = g->dy, rH = f->rho_h, rL = f->rho_l, sig = f->sigma;
    for (int i = NB + 1; i < nx + NB; i++)
        for (int j = NB; j < ny + NB; j++) {
            const long c = IX(g, i, j), w = IX(g, i - 1, j);
            double thH, th;
            gfm_theta_first(ls[w], ls[c], &thH, &th);
            const double rhoEff = rH * thH + rL * (1.0 - thH);
            const double iR = 1.0 / rhoEff;
            const double kEff = kappa[c] * th + kappa[w] * (1.0 - th);
            double val = dt * (-sig * kEff) * (H[c] - H[w]);
            val *= iR / dx;
            val += us[c] - iR * (ps[c] - ps[w]) / dx;
            u[c] = val;
        }
    for (int i = NB; i < nx + NB; i++)
        for (int j = NB + 1; j < ny + NB; j++) {
            const long c = IX(g, i, j), s = IX(g, i, j - 1);
            double thH, th;
            gfm_theta_first(ls[s], ls[c], &thH, &th);
            const double rhoEff = rH * thH + rL * (1.0 - thH);
            const double iR = 1.0 / rhoEff;
            const double kEff = kappa[c] * th + kappa[s] * (1.0 - th);
            double val = dt * (-sig * kEff) * (H[c] - H[s]);
            val *= iR / dy;
            val += vs[c] - iR * (ps[c] - ps[s]) / dy;
            v[c] = val;
        }
    ora_bc_u(g, u);
    ora_bc_v(g, v);
}

/* UpdateDt, mac2d.cpp:1851-1880 (product u[i+1]*u[i], max(muH,muL)). */
double ora_update_dt(const ora_grid *g, const ora_fluid *f, const double *u, const double *v) {
    const double dx = g->dx, dy = g->dy;
    double uA = 0.0, vA = 0.0;
    for (int i = NB; i < g->nx + NB; i++)
        for (int j = NB; j < g->ny + NB; j++) {
            uA = smax(uA, fabs((u[IX(g, i + 1, j)] * u[IX(g, i, j)]) * 0.5));
            vA = smax(vA, fabs((v[IX(g, i, j + 1)] * v[IX(g, i, j)]) * 0.5));
        }
    const double C = uA / dx + vA / dy;
    const double V = smax(f->mu_h, f->mu_l) * (2.0 / (dx * dx + dy * dy));
    const double G = smax(sqrt(fabs(f->g) / dy), sqrt(fabs(f->g) / dx));
    const double hmin = smin(dx, dy);
    const double S = sqrt((f->sigma / hmin) / (smin(f->rho_h, f->rho_l) * (hmin * hmin)));
    double dt = 1.79769313486231570815e+308;
    dt = smin(dt, f->cfl / (0.5 * (C + V + sqrt((C + V) * (C + V) + 4.0 * G * G + 4.0 * S * S))));
    return dt;
}

/* ======================================================================= */
/* Axisymmetric MAC solver: MACSolver2DAxisym, mac2dAxisym.cpp             */
/* x is r (i, nx = kNr, dx = kDr), y is z (j, ny = kNz, dy = kDz).          */
/* ======================================================================= */
static inline double axi_mu(const ora_fluid *f, const double *H, long c) { return f->mu_l + (f->mu_h - f->mu_l) * H[c]; }
static inline double axi_q(const double *a, long c0, long c1, long c2, long c3) {
    /* 0.25 * (a0 + a1 + a2 + a3), summed left to right as the reference writes it */
    return 0.25 * (a[c0] + a[c1] + a[c2] + a[c3]);
}
/* Heavy fraction of a face between level-set values a and b, the rule of the
 * implicit viscous step (mac2dAxisym.cpp:1027-1043): both >= 0 heavy, both
 * <= 0 light, else the fraction on the heavy side. */
static inline double axi_heavy(double a, double b) {
    if (a >= 0.0 && b >= 0.0) return 1.0;
    if (a <= 0.0 && b <= 0.0) return 0.0;
    if (a >= 0.0 && b < 0.0) return fabs(a) / (fabs(a) + fabs(b));
    return fabs(b) / (fabs(a) + fabs(b));
}
/* Effective density of the explicit viscous terms (mac2dAxisym.cpp:682-736):
 * the pure cases take the fluid density itself. */
static inline double axi_rho_face(const ora_fluid *f, double a, double b) {
    if (a >= 0.0 && b >= 0.0) return f->rho_h;
    if (a <= 0.0 && b <= 0.0) return f->rho_l;
    const double t = (a >= 0.0) ? fabs(a) / (fabs(a) + fabs(b)) : fabs(b) / (fabs(a) + fabs(b));
    return f->rho_h * t + f->rho_l * (1.0 - t);
}

/* UpdateKappa, mac2dAxisym.cpp:222-262.  The r-derivative is one-sided in the
 * first column (the axis); dphi/dz of a neighbour column outside the
 * interior is 0 (never computed there); r = kBaseR + (i + 1/2) dr. */
void ora_axi_kappa(const ora_grid *g, double base_r, const double *ls, double *kappa) {
    const int nx = g->nx, ny = g->ny;
    const long n = ASZ(g);
    const double dr = g->dx, dz = g->dy, eps = 1.0e-100;
    double *gr = zalloc(n), *gz = zalloc(n), *sz = zalloc(n);
    for (int i = NB; i < nx + NB; i++)
        for (int j = NB; j < ny + NB; j++) {
            const long k = IX(g, i, j);
            gr[k] = (ls[IX(g, i + 1, j)] - ls[IX(g, i - 1, j)]) / (2.0 * dr);
            gz[k] = (ls[IX(g, i, j + 1)] - ls[IX(g, i, j - 1)]) / (2.0 * dz);
            if (i == NB) gr[k] = (ls[IX(g, i + 1, j)] - ls[k]) / dr;
            sz[k] = sqrt(gr[k] * gr[k] + gz[k] * gz[k] + eps);
        }
    const double lim = 1.0 / smin(dr, dz);
    for (int i = NB; i < nx + NB; i++)
        for (int j = NB; j < ny + NB; j++) {
            const long k = IX(g, i, j);
            const double r = base_r + (i + 0.5 - NB) * dr;
            const double dR = gr[k], dZ = gz[k], s = sz[k];
            double kap = ((ls[IX(g, i - 1, j)] - 2.0 * ls[k] + ls[IX(g, i + 1, j)]) / (dr * dr) * dZ * dZ -
                          2.0 * (gz[IX(g, i + 1, j)] - gz[IX(g, i - 1, j)]) / (2.0 * dr) * dR * dZ +
                          (ls[IX(g, i, j - 1)] - 2.0 * ls[k] + ls[IX(g, i, j + 1)]) / (dz * dz) * dR * dR +
                          dR * (s * s) / r) /
                         pow(s, 3.0);
            kappa[k] = isgn(kap) * fabs(smin(fabs(kap), lim));
        }
    free(gr); free(gz); free(sz);
}

/* AddExternalViscosityFU, mac2dAxisym.cpp:590-753: the z-part of the viscous
 * stress on u faces, over the density of the face's z-neighbourhood. */
void ora_axi_visc_u(const ora_grid *g, const ora_fluid *f, const double *u, const double *v, const double *ls,
                    const double *H, double *dU) {
    (void)u;
    const int nx = g->nx, ny = g->ny;
    const double dr = g->dx, dz = g->dy;
    memset(dU, 0, sizeof(double) * ASZ(g));
    if (!(re_positive(f) > 0.0)) return;
    for (int i = NB + 1; i < nx + NB; i++)
        for (int j = NB; j < ny + NB; j++) {
            const long M = IX(g, i, j), W = IX(g, i - 1, j), Nn = IX(g, i, j + 1), WN = IX(g, i - 1, j + 1),
                       S = IX(g, i, j - 1), WS = IX(g, i - 1, j - 1);
            const double lsN = axi_q(ls, M, W, WN, Nn), lsS = axi_q(ls, M, W, WS, S);
            const double muN = 0.25 * (axi_mu(f, H, M) + axi_mu(f, H, W) + axi_mu(f, H, WN) + axi_mu(f, H, Nn));
            const double muS = 0.25 * (axi_mu(f, H, M) + axi_mu(f, H, W) + axi_mu(f, H, WS) + axi_mu(f, H, S));
            const double rhoSN = axi_rho_face(f, lsS, lsN);
            const double visZ = (muN * (v[Nn] - v[WN]) / dr - muS * (v[M] - v[W]) / dr) / dz;
            dU[M] = visZ / rhoSN;
        }
}

/* AddExternalViscosityFV, mac2dAxisym.cpp:755-910: the r-part on v faces plus
 * the hoop term built from the new uhat, r = (i + 1/2) dr (no kBaseR). */
void ora_axi_visc_v(const ora_grid *g, const ora_fluid *f, const double *u, const double *uhat, const double *v,
                    const double *ls, const double *H, double *dV) {
    (void)v;
    const int nx = g->nx, ny = g->ny;
    const double dr = g->dx, dz = g->dy;
    memset(dV, 0, sizeof(double) * ASZ(g));
    if (!(re_positive(f) > 0.0)) return;
    for (int i = NB; i < nx + NB; i++)
        for (int j = NB + 1; j < ny + NB; j++) {
            const long M = IX(g, i, j), W = IX(g, i - 1, j), E = IX(g, i + 1, j), S = IX(g, i, j - 1),
                       WS = IX(g, i - 1, j - 1), ES = IX(g, i + 1, j - 1);
            const double r = (i + 0.5 - NB) * dr;
            const double lsVW = axi_q(ls, M, W, WS, S), lsVE = axi_q(ls, M, E, ES, S);
            const double muVW = 0.25 * (axi_mu(f, H, M) + axi_mu(f, H, W) + axi_mu(f, H, WS) + axi_mu(f, H, S));
            const double muVE = 0.25 * (axi_mu(f, H, M) + axi_mu(f, H, E) + axi_mu(f, H, ES) + axi_mu(f, H, S));
            const double rhoWE = axi_rho_face(f, lsVW, lsVE);
            const double rhoSN = axi_rho_face(f, ls[S], ls[M]);
            const double visR = (muVE * (u[E] - u[ES]) / dz - muVW * (u[M] - u[S]) / dz) / dr;
            const double visZ = 0.5 * (axi_mu(f, H, M) + axi_mu(f, H, S)) / r *
                                (0.5 * (uhat[M] + uhat[E]) - 0.5 * (uhat[S] + uhat[ES])) / dz;
            dV[M] = visR / rhoWE + visZ / rhoSN;
        }
}

/* GetRHSU, mac2dAxisym.cpp:264-292: u + dt (-conv + gravity + viscous) on the
 * interior u faces, zero elsewhere, then the U ghost fill. */
void ora_axi_rhs_u(const ora_grid *g, const ora_fluid *f, double dt, const double *ls, const double *u,
                   const double *v, const double *H, double *rhs) {
    const long n = ASZ(g);
    double *cU = zalloc(n), *vU = zalloc(n);
    ora_conv_u(g, u, v, cU);
    ora_axi_visc_u(g, f, u, v, ls, H, vU);
    const double gU = gravity_on(f, 0) ? -f->g : 0.0; /* AddGravityFU, :912-929 (axis R) */
    memset(rhs, 0, sizeof(double) * n);
    for (int i = NB + 1; i < g->nx + NB; i++)
        for (int j = NB; j < g->ny + NB; j++) {
            const long k = IX(g, i, j);
            rhs[k] = u[k] + dt * (-cU[k] + gU + vU[k]);
        }
    ora_bc_u(g, rhs);
    free(cU); free(vU);
}

/* GetRHSV, mac2dAxisym.cpp:294-322.  Its gravity is AddGravityFU() (:306),
 * nonzero only where the U pattern is (i >= 4, axis R), unless fix_gravity
 * selects AddGravityFV (axis Z). */
void ora_axi_rhs_v(const ora_grid *g, const ora_fluid *f, double dt, const double *ls, const double *u,
                   const double *uhat, const double *v, const double *H, double *rhs) {
    const long n = ASZ(g);
    double *cV = zalloc(n), *vV = zalloc(n);
    ora_conv_v(g, u, v, cV);
    ora_axi_visc_v(g, f, u, uhat, v, ls, H, vV);
    memset(rhs, 0, sizeof(double) * n);
    for (int i = NB; i < g->nx + NB; i++)
        for (int j = NB + 1; j < g->ny + NB; j++) {
            const long k = IX(g, i, j);
            double gV;
            if (f->fix_gravity) gV = gravity_on(f, 1) ? -f->g : 0.0;
            else gV = (gravity_on(f, 0) && i >= NB + 1) ? -f->g : 0.0;
            rhs[k] = v[k] + dt * (-cV[k] + gV + vV[k]);
        }
    ora_bc_v(g, rhs);
    free(cV); free(vV);
}

/* The Thomas algorithm for lo[k] x[k-1] + di[k] x[k] + up[k] x[k+1] = x[k],
 * k = 0..n-1 (n >= 2), in the elimination order of SolveTDMA
 * (mac2dAxisym.cpp:2255-2306): up and x are overwritten, x holds the result. */
static void axi_thomas(int n, const double *lo, const double *di, double *up, double *x) {
    up[0] = up[0] / di[0];
    x[0] = x[0] / di[0];
    for (int k = 1; k < n; k++) {
        const double piv = di[k] - lo[k] * up[k - 1];
        if (k < n - 1) up[k] = up[k] / piv;
        x[k] = (x[k] - lo[k] * x[k - 1]) / piv;
    }
    for (int k = n - 2; k >= 0; k--) x[k] = x[k] - up[k] * x[k + 1];
}

/* GetUHat, mac2dAxisym.cpp:950-1229: the u faces i = 4 .. nx+2 solved
 * implicitly for the viscous r- and z-terms, one Thomas sweep per z row
 * (r-direction, the (1/r) d/dr (r mu du/dr) stencil) and then one per r
 * column (z-direction), and finally divided by 1 + dt/rho (mu_W + mu_M)/r^2.
 * Raw U kinds and constants pick the end rows (:1047-1086, :1138-1177). */
void ora_axi_uhat(const ora_grid *g, const ora_fluid *f, double dt, const double *ls, const double *rhs,
                  const double *H, double *uhat) {
    const int nr = g->nx, nz = g->ny, m = nr - 1;
    const double dr = g->dx, dz = g->dy, rH = f->rho_h, rL = f->rho_l;
    const int bW = g->bc_u[0], bE = g->bc_u[1], bS = g->bc_u[2], bN = g->bc_u[3];
    const int L = (m > nz ? m : nz);
    double *lo = zalloc(L), *di = zalloc(L), *up = zalloc(L), *x = zalloc(L);
    double *s2 = zalloc((long)m * nz), *s1 = zalloc((long)m * nz);
    memset(uhat, 0, sizeof(double) * ASZ(g));
    for (int jj = 0; jj < nz; jj++) { /* r lines */
        const int J = jj + NB;
        for (int k = 0; k < m; k++) {
            const int I = k + NB + 1;
            const double rUM = (k + 1.0) * dr, rPW = (k + 0.5) * dr, rPM = (k + 1.5) * dr;
            const double muW = axi_mu(f, H, IX(g, I - 1, J)), muM = axi_mu(f, H, IX(g, I, J));
            const double thH = axi_heavy(ls[IX(g, I - 1, J)], ls[IX(g, I, J)]);
            const double rho = rH * thH + rL * (1.0 - thH);
            x[k] = rhs[IX(g, I, J)];
            lo[k] = -dt / (rho * rUM) * (2.0 * rPW * muW) / (dr * dr);
            di[k] = 1.0 + dt / (rho * rUM) * 2.0 * (rPW * muW + rPM * muM) / (dr * dr);
            up[k] = -dt / (rho * rUM) * (2.0 * rPM * muM) / (dr * dr);
            if (k == 0) {
                if (bW == ORA_NEUMANN || bW == ORA_OUTLET) { di[k] += lo[k]; lo[k] = 0.0; }
                else if (bW == ORA_DIRICHLET || bW == ORA_AXISYM || bW == ORA_INLET || bW == ORA_WALL) { x[k] -= lo[k] * g->cu[0]; lo[k] = 0.0; }
                else if (bW == ORA_PERIODIC) { x[k] -= lo[k] * rhs[IX(g, m - 1 + NB + 1, J)]; lo[k] = 0.0; }
            }
            if (k == m - 1) {
                if (bE == ORA_NEUMANN || bE == ORA_OUTLET) { di[k] += up[k]; up[k] = 0.0; }
                else if (bE == ORA_DIRICHLET || bE == ORA_AXISYM || bE == ORA_INLET || bE == ORA_WALL) { x[k] -= up[k] * g->cu[1]; up[k] = 0.0; }
                else if (bE == ORA_PERIODIC) { x[k] -= up[k] * rhs[IX(g, NB + 1, J)]; up[k] = 0.0; }
            }
        }
        axi_thomas(m, lo, di, up, x);
        for (int k = 0; k < m; k++) s2[jj + (long)nz * k] = x[k];
    }
    for (int k = 0; k < m; k++) { /* z lines */
        const int I = k + NB + 1;
        for (int jj = 0; jj < nz; jj++) {
            const int J = jj + NB;
            const long M = IX(g, I, J), W = IX(g, I - 1, J), S = IX(g, I, J - 1), WS = IX(g, I - 1, J - 1),
                       Nn = IX(g, I, J + 1), WN = IX(g, I - 1, J + 1);
            const double lsS = axi_q(ls, M, W, WS, S), lsN = axi_q(ls, M, W, WN, Nn);
            const double muS = 0.25 * (axi_mu(f, H, M) + axi_mu(f, H, W) + axi_mu(f, H, WS) + axi_mu(f, H, S));
            const double muN = 0.25 * (axi_mu(f, H, M) + axi_mu(f, H, W) + axi_mu(f, H, WN) + axi_mu(f, H, Nn));
            const double thH = axi_heavy(lsS, lsN);
            const double rho = rH * thH + rL * (1.0 - thH);
            x[jj] = s2[jj + (long)nz * k];
            lo[jj] = -dt / rho * muS / (dz * dz);
            di[jj] = 1.0 + dt / rho * (muS + muN) / (dz * dz);
            up[jj] = -dt / rho * muN / (dz * dz);
            if (jj == 0) {
                if (bS == ORA_NEUMANN || bS == ORA_AXISYM || bS == ORA_OUTLET) { di[jj] += lo[jj]; lo[jj] = 0.0; }
                else if (bS == ORA_DIRICHLET || bS == ORA_INLET || bS == ORA_WALL) { x[jj] -= lo[jj] * 2.0 * g->cu[2]; lo[jj] = 0.0; }
                else if (bS == ORA_PERIODIC) { x[jj] -= lo[jj] * s2[(nz - 1) + (long)nz * k]; lo[jj] = 0.0; }
            }
            if (jj == nz - 1) {
                if (bN == ORA_NEUMANN || bN == ORA_AXISYM || bN == ORA_OUTLET) { di[jj] += up[jj]; up[jj] = 0.0; }
                else if (bN == ORA_DIRICHLET || bN == ORA_INLET || bN == ORA_WALL) { x[jj] -= up[jj] * 2.0 * g->cu[3]; up[jj] = 0.0; }
                else if (bN == ORA_PERIODIC) { x[jj] -= up[jj] * s2[0 + (long)nz * k]; up[jj] = 0.0; }
            }
        }
        axi_thomas(nz, lo, di, up, x);
        for (int jj = 0; jj < nz; jj++) s1[jj + (long)nz * k] = x[jj];
    }
    for (int k = 0; k < m; k++) {
        const int I = k + NB + 1;
        const double rUM = (I - NB) * dr;
        for (int jj = 0; jj < nz; jj++) {
            const int J = jj + NB;
            const long M = IX(g, I, J), W = IX(g, I - 1, J);
            const double thH = axi_heavy(ls[W], ls[M]);
            const double rho = rH * thH + rL * (1.0 - thH);
            uhat[M] = s1[jj + (long)nz * k] / (1.0 + dt / rho * (axi_mu(f, H, W) + axi_mu(f, H, M)) / (rUM * rUM));
        }
    }
    free(lo); free(di); free(up); free(x); free(s1); free(s2);
}

/* GetVHat, mac2dAxisym.cpp:1231-1478: the v faces j = 4 .. ny+2, r lines over
 * all nx cells (the (1/r) d/dr (r mu dv/dr) stencil) then z lines. */
void ora_axi_vhat(const ora_grid *g, const ora_fluid *f, double dt, const double *ls, const double *rhs,
                  const double *H, double *vhat) {
    const int nr = g->nx, nz = g->ny, m = nz - 1;
    const double dr = g->dx, dz = g->dy, rH = f->rho_h, rL = f->rho_l;
    const int bW = g->bc_v[0], bE = g->bc_v[1], bS = g->bc_v[2], bN = g->bc_v[3];
    const int L = (nr > m ? nr : m);
    double *lo = zalloc(L), *di = zalloc(L), *up = zalloc(L), *x = zalloc(L);
    double *s1 = zalloc((long)nr * m);
    memset(vhat, 0, sizeof(double) * ASZ(g));
    for (int jj = 0; jj < m; jj++) { /* r lines */
        const int J = jj + NB + 1;
        for (int k = 0; k < nr; k++) {
            const int I = k + NB;
            const long M = IX(g, I, J), W = IX(g, I - 1, J), E = IX(g, I + 1, J), S = IX(g, I, J - 1),
                       WS = IX(g, I - 1, J - 1), ES = IX(g, I + 1, J - 1);
            const double rVM = (k + 0.5) * dr, rVW = k * dr, rVE = (k + 1.0) * dr;
            const double lsVW = axi_q(ls, M, W, S, WS), lsVE = axi_q(ls, M, E, S, ES);
            const double muVW = 0.25 * (axi_mu(f, H, M) + axi_mu(f, H, W) + axi_mu(f, H, S) + axi_mu(f, H, WS));
            const double muVE = 0.25 * (axi_mu(f, H, M) + axi_mu(f, H, E) + axi_mu(f, H, S) + axi_mu(f, H, ES));
            const double thH = axi_heavy(lsVW, lsVE);
            const double rho = rH * thH + rL * (1.0 - thH);
            x[k] = rhs[M];
            lo[k] = -dt / (rho * rVM) * rVW * muVW / (dr * dr);
            di[k] = 1.0 + dt / (rho * rVM) * (rVW * muVW + rVE * muVE) / (dr * dr);
            up[k] = -dt / (rho * rVM) * rVE * muVE / (dr * dr);
            if (k == 0) {
                if (bW == ORA_NEUMANN || bW == ORA_AXISYM || bW == ORA_OUTLET) { di[k] += lo[k]; lo[k] = 0.0; }
                else if (bW == ORA_DIRICHLET || bW == ORA_INLET || bW == ORA_WALL) { x[k] -= lo[k] * 2.0 * g->cv[0]; lo[k] = 0.0; }
                else if (bW == ORA_PERIODIC) { x[k] -= lo[k] * rhs[IX(g, nr - 1 + NB, J)]; lo[k] = 0.0; }
            }
            if (k == nr - 1) {
                if (bE == ORA_NEUMANN || bE == ORA_AXISYM || bE == ORA_OUTLET) { di[k] += up[k]; up[k] = 0.0; }
                else if (bE == ORA_DIRICHLET || bE == ORA_INLET || bE == ORA_WALL) { x[k] -= up[k] * 2.0 * g->cv[1]; up[k] = 0.0; }
                else if (bE == ORA_PERIODIC) { x[k] -= up[k] * rhs[IX(g, NB, J)]; up[k] = 0.0; }
            }
        }
        axi_thomas(nr, lo, di, up, x);
        for (int k = 0; k < nr; k++) s1[jj + (long)m * k] = x[k];
    }
    for (int k = 0; k < nr; k++) { /* z lines */
        const int I = k + NB;
        for (int jj = 0; jj < m; jj++) {
            const int J = jj + NB + 1;
            const long M = IX(g, I, J), S = IX(g, I, J - 1);
            const double muS = axi_mu(f, H, S), muM = axi_mu(f, H, M);
            const double thH = axi_heavy(ls[S], ls[M]);
            const double rho = rH * thH + rL * (1.0 - thH);
            x[jj] = s1[jj + (long)m * k];
            lo[jj] = -dt / rho * (2.0 * muS) / (dz * dz);
            di[jj] = 1.0 + dt / rho * 2.0 * (muS + muM) / (dz * dz);
            up[jj] = -dt / rho * (2.0 * muM) / (dz * dz);
            if (jj == 0) {
                if (bS == ORA_NEUMANN || bS == ORA_OUTLET) { di[jj] += lo[jj]; lo[jj] = 0.0; }
                else if (bS == ORA_DIRICHLET || bS == ORA_AXISYM || bS == ORA_INLET || bS == ORA_WALL) { x[jj] -= lo[jj] * g->cv[2]; lo[jj] = 0.0; }
                else if (bS == ORA_PERIODIC) { x[jj] -= lo[jj] * s1[(m - 1) + (long)m * k]; lo[jj] = 0.0; }
            }
            if (jj == m - 1) {
                if (bN == ORA_NEUMANN || bN == ORA_OUTLET) { di[jj] += up[jj]; up[jj] = 0.0; }
                else if (bN == ORA_DIRICHLET || bN == ORA_AXISYM || bN == ORA_INLET || bN == ORA_WALL) { x[jj] -= up[jj] * g->cv[3]; up[jj] = 0.0; }
                else if (bN == ORA_PERIODIC) { x[jj] -= up[jj] * s1[0 + (long)m * k]; up[jj] = 0.0; }
            }
        }
        axi_thomas(m, lo, di, up, x);
        for (int jj = 0; jj < m; jj++) vhat[IX(g, I, jj + NB + 1)] = x[jj];
    }
    free(lo); free(di); free(up); free(x); free(s1);
}

/* GetDivergence4Poisson, mac2dAxisym.cpp:1980-1994: r times the divergence,
 * (r_e u_e - r_w u_w) / dr + r_c (v_n - v_s) / dz. */
void ora_axi_div4p(const ora_grid *g, double base_r, const double *u, const double *v, double *div) {
    const double dr = g->dx, dz = g->dy;
    memset(div, 0, sizeof(double) * ASZ(g));
    for (int i = NB; i < g->nx + NB; i++)
        for (int j = NB; j < g->ny + NB; j++) {
            const double rc = base_r + (i + 0.5 - NB) * dr, re = base_r + (i + 1.0 - NB) * dr,
                         rw = base_r + (i - NB) * dr;
            div[IX(g, i, j)] = (re * u[IX(g, i + 1, j)] - rw * u[IX(g, i, j)]) / dr +
                               rc * (v[IX(g, i, j + 1)] - v[IX(g, i, j)]) / dz;
        }
}

/* GetDivergence, mac2dAxisym.cpp:1996-2008: u/r + du/dr + dv/dz at centres. */
void ora_axi_divergence(const ora_grid *g, double base_r, const double *u, const double *v, double *div) {
    const double dr = g->dx, dz = g->dy;
    memset(div, 0, sizeof(double) * ASZ(g));
    for (int i = NB; i < g->nx + NB; i++)
        for (int j = NB; j < g->ny + NB; j++) {
            const double rc = base_r + (i + 0.5 - NB) * dr;
            const double uw = u[IX(g, i, j)], ue = u[IX(g, i + 1, j)];
            div[IX(g, i, j)] = 0.5 * (uw + ue) / rc + (ue - uw) / dr + (v[IX(g, i, j + 1)] - v[IX(g, i, j)]) / dz;
        }
}

static int axi_p_neumann(int b) { return b == ORA_NEUMANN || b == ORA_AXISYM || b == ORA_WALL; }
static int axi_p_dirichlet(int b) {
    return b == ORA_DIRICHLET || b == ORA_INLET || b == ORA_OUTLET || b == ORA_PRESSURE;
}

/* SolvePoisson's assembly, mac2dAxisym.cpp:1488-1916: the r-weighted GFM
 * operator.  West/east faces carry r at the face, or (across the interface)
 * r interpolated between the two centres with the kappa weight theta (the
 * west one clamped at 0); south/north faces carry the centre's r.  Neumann
 * group: Neumann, axisym, wall; Dirichlet group: Dirichlet, inlet, outlet,
 * pressure (with the 2 * constant of :1797-1801).  ps is zeroed before the
 * assembly (:1558-1562), which makes the -ps terms -0. */
int ora_axi_assemble(const ora_grid *g, const ora_fluid *f, double base_r, double dt, const double *ls,
                     double *kappa, const double *H, const double *div, int recompute_kappa, double *diag,
                     double *cw, double *ce, double *cs, double *cn, double *rhs) {
    const int nx = g->nx, ny = g->ny;
    const double dr = g->dx, dz = g->dy, rH = f->rho_h, rL = f->rho_l, sig = f->sigma;
    if (recompute_kappa) {
        ora_axi_kappa(g, base_r, ls, kappa);
        ora_bc_p(g, kappa);
    }
    int pin = 1;
    for (int s = 0; s < 4; s++) pin &= axi_p_neumann(g->bc_p[s]);
    for (int j = NB; j < ny + NB; j++)
        for (int i = NB; i < nx + NB; i++) {
            const long c = IX(g, i, j), w = IX(g, i - 1, j), e = IX(g, i + 1, j), s = IX(g, i, j - 1),
                       nn = IX(g, i, j + 1);
            const int k = (i - NB) + nx * (j - NB);
            const double lsW = ls[w], lsE = ls[e], lsM = ls[c], lsS = ls[s], lsN = ls[nn];
            const double rPW = base_r + (i - 0.5 - NB) * dr, rPM = base_r + (i + 0.5 - NB) * dr,
                         rPE = base_r + (i + 1.5 - NB) * dr, rWf = base_r + (i - NB) * dr,
                         rEf = base_r + (i + 1.0 - NB) * dr;
            double thH, th, rEff, rho, kEff;
            /* west face (:1579-1611) */
            if (lsW >= 0.0 && lsM >= 0.0) { thH = 1.0; th = 0.0; rEff = rWf; }
            else if (lsW < 0.0 && lsM < 0.0) { thH = 0.0; th = 0.0; rEff = rWf; }
            else {
                gfm_theta_first(lsW, lsM, &thH, &th);
                rEff = smax(rPM * th + rPW * (1.0 - th), 0.0);
            }
            rho = rH * thH + rL * (1.0 - thH);
            kEff = kappa[c] * th + kappa[w] * (1.0 - th);
            double pW = rEff / rho;
            double FW = -dt * (-sig * kEff) * (H[c] - H[w]);
            FW *= pW / (dr * dr);
            /* east face (:1614-1644), not clamped */
            if (lsM >= 0.0 && lsE >= 0.0) { thH = 1.0; th = 0.0; rEff = rEf; }
            else if (lsM < 0.0 && lsE < 0.0) { thH = 0.0; th = 0.0; rEff = rEf; }
            else {
                gfm_theta_second(lsM, lsE, &thH, &th);
                rEff = rPM * th + rPE * (1.0 - th);
            }
            rho = rH * thH + rL * (1.0 - thH);
            kEff = kappa[c] * th + kappa[e] * (1.0 - th);
            double pE = rEff / rho;
            double FE = dt * (-sig * kEff) * (H[e] - H[c]);
            FE *= pE / (dr * dr);
            /* south and north faces (:1646-1700): the centre's r */
            gfm_theta_first(lsS, lsM, &thH, &th);
            rho = rH * thH + rL * (1.0 - thH);
            kEff = kappa[c] * th + kappa[s] * (1.0 - th);
            double pS = rPM / rho;
            double FS = -dt * (-sig * kEff) * (H[c] - H[s]);
            FS *= pS / (dz * dz);
            gfm_theta_second(lsM, lsN, &thH, &th);
            rho = rH * thH + rL * (1.0 - thH);
            kEff = kappa[c] * th + kappa[nn] * (1.0 - th);
            double pN = rPM / rho;
            double FN = dt * (-sig * kEff) * (H[nn] - H[c]);
            FN *= pN / (dz * dz);
            double r = 0.0;
            r -= FW + FE + FS + FN;
            r -= div[c];
            pS *= -1.0; pW *= -1.0; pE *= -1.0; pN *= -1.0;
            double aS = pS / (dz * dz), aW = pW / (dr * dr), aE = pE / (dr * dr), aN = pN / (dz * dz);
            double aC = -(pW + pE) / (dr * dr) - (pS + pN) / (dz * dz);
            if (i == NB && axi_p_neumann(g->bc_p[0])) { aW = 0.0; aC += pW / (dr * dr); }
            else if (i == NB && axi_p_dirichlet(g->bc_p[0])) { aW = 0.0; r -= pW / (dr * dr) * (-0.0 + 2.0 * g->cp[0]); }
            if (i == NB + nx - 1 && axi_p_neumann(g->bc_p[1])) { aE = 0.0; aC += pE / (dr * dr); }
            else if (i == NB + nx - 1 && axi_p_dirichlet(g->bc_p[1])) { aE = 0.0; r -= pE / (dr * dr) * (-0.0 + 2.0 * g->cp[1]); }
            if (j == NB && axi_p_neumann(g->bc_p[2])) { aS = 0.0; aC += pS / (dz * dz); }
            else if (j == NB && axi_p_dirichlet(g->bc_p[2])) { aS = 0.0; r -= pS / (dz * dz) * (-0.0 + 2.0 * g->cp[2]); }
            if (j == NB + ny - 1 && axi_p_neumann(g->bc_p[3])) { aN = 0.0; aC += pN / (dz * dz); }
            else if (j == NB + ny - 1 && axi_p_dirichlet(g->bc_p[3])) { aN = 0.0; r -= pN / (dz * dz) * (-0.0 + 2.0 * g->cp[3]); }
            diag[k] = aC;
            cw[k] = -aW;
            ce[k] = -aE;
            cs[k] = -aS;
            cn[k] = -aN;
            rhs[k] = r;
        }
    if (pin) { /* the corrected pin of ora_gfm_assemble (cell 0 held at 0) */
        rhs[0] = 0.0;
        if (nx > 1) cw[1] = 0.0;
        if (ny > 1) cs[nx] = 0.0;
    }
    return pin;
}

/* UpdateDt, mac2dAxisym.cpp:2104-2133: the CFL bound of the convective,
 * gravity and surface-tension speeds (the viscous one is computed there but
 * not used); the surface-tension speed uses max |kappa|. */
double ora_axi_update_dt(const ora_grid *g, const ora_fluid *f, const double *u, const double *v,
                         const double *kappa) {
    const double dr = g->dx, dz = g->dy;
    double uA = 0.0, vA = 0.0, kA = 0.0;
    for (int i = NB; i < g->nx + NB; i++)
        for (int j = NB; j < g->ny + NB; j++) {
            uA = smax(uA, fabs((u[IX(g, i + 1, j)] * u[IX(g, i, j)]) * 0.5));
            vA = smax(vA, fabs((v[IX(g, i, j + 1)] * v[IX(g, i, j)]) * 0.5));
            kA = smax(kA, fabs(kappa[IX(g, i, j)]));
        }
    const double C = uA / dr + vA / dz;
    const double G = smax(sqrt(fabs(f->g) / dz), sqrt(fabs(f->g) / dr));
    const double h = smin(dr, dz);
    const double S = sqrt((f->sigma * kA) / (smin(f->rho_h, f->rho_l) * (h * h)));
    double dt = 1.79769313486231570815e+308;
    dt = smin(dt, f->cfl / (0.5 * (C + sqrt(C * C + 4.0 * (G * G) + 4.0 * (S * S)))));
    return dt;
}

void ora_gather(const ora_grid *g, const double *padded, double *nat) {
    for (int j = 0; j < g->ny; j++)
        for (int i = 0; i < g->nx; i++) nat[i + g->nx * j] = padded[IX(g, i + NB, j + NB)];
}
void ora_scatter(const ora_grid *g, const double *nat, double *padded) {
    for (int j = 0; j < g->ny; j++)
        for (int i = 0; i < g->nx; i++) padded[IX(g, i + NB, j + NB)] = nat[i + g->nx * j];
}

void ora_interface_mask(const ora_grid *g, const double *ls0, uint8_t *mask) {
    for (int j = NB; j < g->ny + NB; j++)
        for (int i = NB; i < g->nx + NB; i++) {
            const double c = ls0[IX(g, i, j)];
            const int m = (c * ls0[IX(g, i + 1, j)] < 0) || (c * ls0[IX(g, i - 1, j)] < 0) ||
                          (c * ls0[IX(g, i, j + 1)] < 0) || (c * ls0[IX(g, i, j - 1)] < 0);
            mask[(i - NB) + g->nx * (j - NB)] = (uint8_t)m;
        }
}

void ora_ghost_face_mask(const ora_grid *g, const double *ls, uint8_t *mask) {
    for (int j = NB; j < g->ny + NB; j++)
        for (int i = NB; i < g->nx + NB; i++) {
            const int c = ls[IX(g, i, j)] >= 0.0;
            const int w = ls[IX(g, i - 1, j)] >= 0.0;
            const int s = ls[IX(g, i, j - 1)] >= 0.0;
            mask[(i - NB) + g->nx * (j - NB)] = (uint8_t)((c != w) | ((c != s) << 1));
        }
}
