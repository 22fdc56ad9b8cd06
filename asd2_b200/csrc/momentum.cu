// MAC momentum kernels (mac2d.cpp): curvature, Heaviside functions, the
// WENO5 convection + variable-viscosity + gravity right-hand side fused with
// the Runge-Kutta stage update, divergence, projection and the CFL time step.
#include <type_traits>

#include "batch.cuh"
#include "lsmath.cuh"
#include "momentum.cuh"

namespace asd2g {

// ---------------------------------------------------------------- kappa --
// UpdateKappa, mac2d.cpp:221-252.  dLSdX is only defined on interior cells
// (zero elsewhere), which matters for the cross term at j = 3 and ny+2.
// Cell kernels are tile functions of the TJ x TI interior tile (bx, by),
// wrapped by one-grid kernels here and by batched kernels (work lists of
// instance tiles) at the end of this file.
__device__ __forceinline__ void kappa_tile(const Grid &g, const DivH &d2x, const DivH &d2y, const DivH &dxx,
                                           const DivH &dyy, double lim, const double *__restrict__ ls,
                                           double *__restrict__ kappa, int bx, int by) {
    const int j = NB + bx * TJ + threadIdx.x, i = NB + by * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    auto gx = [&](int jj) -> double {
        if (jj < NB || jj >= g.ny + NB) return 0.0;
        return d2x(ls[IX(g, i + 1, jj)] - ls[IX(g, i - 1, jj)]);
    };
    const double c = ls[IX(g, i, j)];
    const double gxc = gx(j);
    const double gyc = d2y(ls[IX(g, i, j + 1)] - ls[IX(g, i, j - 1)]);
    const double sz = sqrt(gxc * gxc + gyc * gyc + 1.0e-100);
    double k = (dyy(gxc * gxc * (ls[IX(g, i, j - 1)] - 2.0 * c + ls[IX(g, i, j + 1)])) -
                d2y(2.0 * gxc * gyc * (gx(j + 1) - gx(j - 1))) +
                dxx(gyc * gyc * (ls[IX(g, i - 1, j)] - 2.0 * c + ls[IX(g, i + 1, j)]))) /
               pow(sz, 3.0);
    k = isgn(k) * fabs(smin(fabs(k), lim));
    kappa[IX(g, i, j)] = k;
}

// ASD2G_CURVATURE_DIVERGENCE: kappa = div(n), n = grad phi / |grad phi| on
// the cell faces.  x face (i+1/2, j): phi_x = (phi(i+1,j) - phi(i,j)) / dx,
// phi_y = (phi(i,j+1) + phi(i+1,j+1) - phi(i,j-1) - phi(i+1,j-1)) / (4 dy);
// y faces alike; kappa = (nx(i+1/2) - nx(i-1/2)) / dx + (ny(j+1/2) -
// ny(j-1/2)) / dy, limited as UpdateKappa limits it.  Reads phi on the
// 3 x 3 block around each face pair (ghost cells included).
__device__ __forceinline__ void kappa_div_tile(const Grid &g, double lim, const double *__restrict__ ls,
                                               double *__restrict__ kappa, int bx, int by) {
    const int j = NB + bx * TJ + threadIdx.x, i = NB + by * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    const double dx = g.dx, dy = g.dy;
    auto L = [&](int a, int b) { return ls[IX(g, i + a, j + b)]; };
    auto nx = [&](int a) {  // x face between cells i + a and i + a + 1
        const double px = (L(a + 1, 0) - L(a, 0)) / dx;
        const double py = (L(a, 1) + L(a + 1, 1) - L(a, -1) - L(a + 1, -1)) / (4.0 * dy);
        return px / sqrt(px * px + py * py + 1.0e-100);
    };
    auto ny = [&](int b) {  // y face between cells j + b and j + b + 1
        const double py = (L(0, b + 1) - L(0, b)) / dy;
        const double px = (L(1, b) + L(1, b + 1) - L(-1, b) - L(-1, b + 1)) / (4.0 * dx);
        return py / sqrt(px * px + py * py + 1.0e-100);
    };
    double k = (nx(0) - nx(-1)) / dx + (ny(0) - ny(-1)) / dy;
    k = isgn(k) * fabs(smin(fabs(k), lim));
    kappa[IX(g, i, j)] = k;
}
__global__ void k_kappa(Grid g, DivH d2x, DivH d2y, DivH dxx, DivH dyy, double lim, const double *__restrict__ ls,
                        double *__restrict__ kappa) {
    if (g.kappa_mode == 1) kappa_div_tile(g, lim, ls, kappa, blockIdx.x, blockIdx.y);
    else kappa_tile(g, d2x, d2y, dxx, dyy, lim, ls, kappa, blockIdx.x, blockIdx.y);
}

// ------------------------------------------------------------ Heaviside --
// UpdateHeavisideFunc / UpdateSmoothHeavisideFunc over every cell
// (mac2d.cpp:87-122).
__device__ __forceinline__ void heaviside_cell(double eps, const double *__restrict__ ls, double *__restrict__ H,
                                               double *__restrict__ HS, int64_t k) {
    const double l = ls[k];
    H[k] = l >= 0.0 ? 1.0 : 0.0;
    double hs;
    if (l > eps) hs = 1.0;
    else if (l < -eps) hs = 0.0;
    else hs = 0.5 * (1.0 + l / eps + 1.0 / kPi * sin(kPi * l / eps));
    HS[k] = hs;
}
__global__ void k_heaviside(int64_t n, double eps, const double *__restrict__ ls, double *__restrict__ H,
                            double *__restrict__ HS) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        heaviside_cell(eps, ls, H, HS, k);
}

// ------------------------------------------------------- momentum terms --
// tmpV of AddConvectionFU (mac2d.cpp:314-316): defined on the U interior.
__device__ __forceinline__ double tv_at(const Grid &g, const double *v, int i, int jj) {
    if (jj < NB || jj >= g.ny + NB || i < NB + 1 || i >= g.nx + NB) return 0.0;
    return (v[IX(g, i, jj)] + v[IX(g, i - 1, jj)] + v[IX(g, i - 1, jj + 1)] + v[IX(g, i, jj + 1)]) * 0.25;
}
// tmpU of AddConvectionFV (:395-397): defined on the V interior.
__device__ __forceinline__ double tu_at(const Grid &g, const double *u, int ii, int j) {
    if (j < NB + 1 || j >= g.ny + NB || ii < NB || ii >= g.nx + NB) return 0.0;
    return (u[IX(g, ii, j)] + u[IX(g, ii, j - 1)] + u[IX(g, ii + 1, j - 1)] + u[IX(g, ii + 1, j)]) * 0.25;
}
// mu on interior cells, 0 elsewhere (:603-605)
__device__ __forceinline__ double mu_at(const Grid &g, const MomConst &M, const double *H, int i, int j) {
    if (i < NB || i >= g.nx + NB || j < NB || j >= g.ny + NB) return 0.0;
    return M.mu_l + (M.mu_h - M.mu_l) * H[IX(g, i, j)];
}

// AddConvectionFU at u-face (i,j), i >= 4 (mac2d.cpp:308-387)
__device__ double conv_u(const Grid &g, const MomConst &M, const double *u, const double *v, int i, int j) {
    double D[6], xp, xm, yp, ym;
    double F[7];
#pragma unroll
    for (int k = 0; k < 7; k++) {
        const double a = u[IX(g, i - 3 + k, j)];
        F[k] = a * a;
    }
#pragma unroll
    for (int k = 0; k < 6; k++) D[k] = F[k + 1] - F[k];
    weno5_point(D, M.ddx, xp, xm);
#pragma unroll
    for (int k = 0; k < 7; k++) F[k] = u[IX(g, i, j - 3 + k)] * tv_at(g, v, i, j - 3 + k);
#pragma unroll
    for (int k = 0; k < 6; k++) D[k] = F[k + 1] - F[k];
    weno5_point(D, M.ddy, yp, ym);
    return weno_blend(xp, xm, yp, ym, u[IX(g, i, j)], tv_at(g, v, i, j));
}

// AddConvectionFV at v-face (i,j), j >= 4 (:389-463)
__device__ double conv_v(const Grid &g, const MomConst &M, const double *u, const double *v, int i, int j) {
    double D[6], xp, xm, yp, ym;
    double F[7];
#pragma unroll
    for (int k = 0; k < 7; k++) F[k] = v[IX(g, i - 3 + k, j)] * tu_at(g, u, i - 3 + k, j);
#pragma unroll
    for (int k = 0; k < 6; k++) D[k] = F[k + 1] - F[k];
    weno5_point(D, M.ddx, xp, xm);
#pragma unroll
    for (int k = 0; k < 7; k++) {
        const double a = v[IX(g, i, j - 3 + k)];
        F[k] = a * a;
    }
#pragma unroll
    for (int k = 0; k < 6; k++) D[k] = F[k + 1] - F[k];
    weno5_point(D, M.ddy, yp, ym);
    return weno_blend(xp, xm, yp, ym, tu_at(g, u, i, j), v[IX(g, i, j)]);
}

// Inverse effective density for viscosity U (harmonic form, :687-743).
__device__ __forceinline__ double visc_irho_harm(double a, double b, double rH, double rL) {
    if (a >= 0 && b >= 0) return 1.0 / rH;
    if (a <= 0 && b <= 0) return 1.0 / rL;
    if (a > 0 && b <= 0) {
        const double th = fabs(a) / (fabs(a) + fabs(b));
        return 1.0 / (rL * rH) / (1.0 / rL * th + 1.0 / rH * (1.0 - th));
    }
    if (a <= 0 && b > 0) {
        const double th = fabs(a) / (fabs(a) + fabs(b));
        return 1.0 / (rH * rL) / (1.0 / rH * th + 1.0 / rL * (1.0 - th));
    }
    return 0.0;
}
// Effective density for viscosity V (arithmetic form, :939-995).
__device__ __forceinline__ double visc_rho_arith(double a, double b, double rH, double rL) {
    if (a >= 0 && b >= 0) return rH;
    if (a <= 0 && b <= 0) return rL;
    if (a > 0 && b <= 0) {
        const double th = fabs(a) / (fabs(a) + fabs(b));
        return rH * th + rL * (1.0 - th);
    }
    if (a <= 0 && b > 0) {
        const double th = fabs(a) / (fabs(a) + fabs(b));
        return rL * th + rH * (1.0 - th);
    }
    return 0.0;
}

// AddViscosityFU at u-face (i,j) (:570-809)
__device__ double visc_u(const Grid &g, const MomConst &M, const double *u, const double *v, const double *ls,
                         const double *H, int i, int j) {
#define LS(a, b) ls[IX(g, i + (a), j + (b))]
#define MU(a, b) mu_at(g, M, H, i + (a), j + (b))
    const double uM = u[IX(g, i, j)], uW = u[IX(g, i - 1, j)], uE = u[IX(g, i + 1, j)], uS = u[IX(g, i, j - 1)],
                 uN = u[IX(g, i, j + 1)];
    const double vW = v[IX(g, i - 1, j)], vW_N = v[IX(g, i - 1, j + 1)], vM = v[IX(g, i, j)], vN = v[IX(g, i, j + 1)];
    const double lsUNHalf = 0.25 * (LS(0, 0) + LS(-1, 0) + LS(-1, 1) + LS(0, 1));
    const double lsUSHalf = 0.25 * (LS(0, 0) + LS(-1, 0) + LS(-1, -1) + LS(0, -1));
    const double iWE = visc_irho_harm(LS(-1, 0), LS(0, 0), M.rho_h, M.rho_l);
    const double iSN = visc_irho_harm(lsUSHalf, lsUNHalf, M.rho_h, M.rho_l);
    const double mSs = 0.25 * (MU(0, 0) + MU(-1, 0) + MU(-1, -1) + MU(0, -1));
    const double mNs = 0.25 * (MU(0, 0) + MU(-1, 0) + MU(-1, 1) + MU(0, 1));
    const double muU_X_W = M.ddx(MU(-1, 0) * (uM - uW));
    const double muU_X_E = M.ddx(MU(0, 0) * (uE - uM));
    const double muU_Y_S = M.ddy(mSs * (uM - uS));
    const double muU_Y_N = M.ddy(mNs * (uN - uM));
    const double muV_X_S = M.ddx(mSs * (vM - vW));
    const double muV_X_N = M.ddx(mNs * (vN - vW_N));
    const double visX = M.ddx(2.0 * (muU_X_E - muU_X_W));
    const double visY = M.ddy(muU_Y_N - muU_Y_S) + M.ddy(muV_X_N - muV_X_S);
    return visX * iWE + visY * iSN;
#undef LS
#undef MU
}

// AddViscosityFV at v-face (i,j) (:811-1041)
__device__ double visc_v(const Grid &g, const MomConst &M, const double *u, const double *v, const double *ls,
                         const double *H, int i, int j) {
#define LS(a, b) ls[IX(g, i + (a), j + (b))]
#define MU(a, b) mu_at(g, M, H, i + (a), j + (b))
    const double vW = v[IX(g, i - 1, j)], vE = v[IX(g, i + 1, j)], vS = v[IX(g, i, j - 1)], vN = v[IX(g, i, j + 1)],
                 vM = v[IX(g, i, j)];
    const double uM = u[IX(g, i, j)], uE = u[IX(g, i + 1, j)], uS = u[IX(g, i, j - 1)], uE_S = u[IX(g, i + 1, j - 1)];
    const double lsVWHalf = 0.25 * (LS(0, 0) + LS(-1, 0) + LS(-1, -1) + LS(0, -1));
    const double lsVEHalf = 0.25 * (LS(0, 0) + LS(1, 0) + LS(1, -1) + LS(0, -1));
    const double iWE = 1.0 / visc_rho_arith(lsVWHalf, lsVEHalf, M.rho_h, M.rho_l);
    const double iSN = 1.0 / visc_rho_arith(LS(0, -1), LS(0, 0), M.rho_h, M.rho_l);
    const double mW = 0.25 * (MU(0, 0) + MU(-1, 0) + MU(-1, -1) + MU(0, -1));
    const double mE = 0.25 * (MU(0, 0) + MU(1, 0) + MU(1, -1) + MU(0, -1));
    const double muU_Y_W = M.ddy(mW * (uM - uS));
    const double muU_Y_E = M.ddy(mE * (uE - uE_S));
    const double muV_X_W = M.ddx(mW * (vM - vW));
    const double muV_X_E = M.ddx(mE * (vE - vM));
    const double muV_Y_S = M.ddy(MU(0, -1) * (vM - vS));
    const double muV_Y_N = M.ddy(MU(0, 0) * (vN - vM));
    const double visX = M.ddx(muU_Y_E - muU_Y_W) + M.ddx(muV_X_E - muV_X_W);
    const double visY = M.ddy(2.0 * (muV_Y_N - muV_Y_S));
    return visX * iWE + visY * iSN;
#undef LS
#undef MU
}

// UpdateFU / UpdateFV (:254-306) fused with the Runge-Kutta stage of
// GetIntermediateVel (:1081-1239).  in = stage input (with ghosts filled),
// base = u^n.  KIND: 0 out = in + dt F(in); 1 out = 0.75 base + 0.25 (in + dt F);
// 2 out = 1/3 base + 2/3 (in + dt F); 3 out = 0.5 base + 0.5 (in + dt F);
// 4 out = F(in); 5 out = convection; 6 out = viscosity.
template <int KIND>
__device__ __forceinline__ void mom_stage_tile(const Grid &g, const MomConst &M, const double *__restrict__ ls,
                                               const double *__restrict__ H, const double *__restrict__ uin,
                                               const double *__restrict__ vin, const double *__restrict__ ub,
                                               const double *__restrict__ vb, double *__restrict__ uout,
                                               double *__restrict__ vout, const double *__restrict__ dtp, int bx,
                                               int by) {
    const int j = NB + bx * TJ + threadIdx.x, i = NB + by * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    const double dt = (KIND <= 3) ? *dtp : 0.0;
    if (i >= NB + 1) {  // u interior faces i = 4 .. nx+2
        double F;
        if (KIND == 5) F = conv_u(g, M, uin, vin, i, j);
        else if (KIND == 6) F = M.visc ? visc_u(g, M, uin, vin, ls, H, i, j) : 0.0;
        else F = -conv_u(g, M, uin, vin, i, j) + (M.visc ? visc_u(g, M, uin, vin, ls, H, i, j) : 0.0) + M.gu;
        const int64_t c = IX(g, i, j);
        double o;
        if (KIND == 0) o = uin[c] + dt * F;
        else if (KIND == 1) o = 0.75 * ub[c] + 0.25 * (uin[c] + dt * F);
        else if (KIND == 2) o = 1.0 / 3.0 * ub[c] + 2.0 / 3.0 * (uin[c] + dt * F);
        else if (KIND == 3) o = 0.5 * ub[c] + 0.5 * (uin[c] + dt * F);
        else o = F;
        uout[c] = o;
    }
    if (j >= NB + 1) {  // v interior faces j = 4 .. ny+2
        double F;
        if (KIND == 5) F = conv_v(g, M, uin, vin, i, j);
        else if (KIND == 6) F = M.visc ? visc_v(g, M, uin, vin, ls, H, i, j) : 0.0;
        else {
            const double gv = (M.gv_from_u && i < NB + 1) ? 0.0 : M.gv;
            F = -conv_v(g, M, uin, vin, i, j) + (M.visc ? visc_v(g, M, uin, vin, ls, H, i, j) : 0.0) + gv;
        }
        const int64_t c = IX(g, i, j);
        double o;
        if (KIND == 0) o = vin[c] + dt * F;
        else if (KIND == 1) o = 0.75 * vb[c] + 0.25 * (vin[c] + dt * F);
        else if (KIND == 2) o = 1.0 / 3.0 * vb[c] + 2.0 / 3.0 * (vin[c] + dt * F);
        else if (KIND == 3) o = 0.5 * vb[c] + 0.5 * (vin[c] + dt * F);
        else o = F;
        vout[c] = o;
    }
}
template <int KIND>
__global__ void __launch_bounds__(TJ *TI) k_mom_stage(Grid g, MomConst M, const double *__restrict__ ls,
                                                        const double *__restrict__ H, const double *__restrict__ uin,
                                                        const double *__restrict__ vin, const double *__restrict__ ub,
                                                        const double *__restrict__ vb, double *__restrict__ uout,
                                                        double *__restrict__ vout, const double *__restrict__ dtp) {
    mom_stage_tile<KIND>(g, M, ls, H, uin, vin, ub, vb, uout, vout, dtp, blockIdx.x, blockIdx.y);
}

// ------------------------------------------------------------ divergence --
// GetDivergence, mac2d.cpp:1729-1738
__device__ __forceinline__ void divergence_tile(const Grid &g, const DivH &ddx, const DivH &ddy,
                                                const double *__restrict__ u, const double *__restrict__ v,
                                                double *__restrict__ div, int bx, int by) {
    const int j = NB + bx * TJ + threadIdx.x, i = NB + by * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    div[IX(g, i, j)] = ddx(u[IX(g, i + 1, j)] - u[IX(g, i, j)]) + ddy(v[IX(g, i, j + 1)] - v[IX(g, i, j)]);
}
__global__ void k_divergence(Grid g, DivH ddx, DivH ddy, const double *__restrict__ u, const double *__restrict__ v,
                             double *__restrict__ div) {
    divergence_tile(g, ddx, ddy, u, v, div, blockIdx.x, blockIdx.y);
}

// ------------------------------------------------------------ projection --
// Face theta rule of the GFM (mac2d.cpp:1341-1358; UpdateVel :1770-1786)
__device__ __forceinline__ void gfm_theta_first(double a, double b, double &thH, double &th) {
    if (a >= 0.0 && b >= 0.0) { thH = 1.0; th = 0.0; }
    else if (a < 0.0 && b < 0.0) { thH = 0.0; th = 0.0; }
    else if (a >= 0.0 && b < 0.0) { thH = fabs(a) / (fabs(a) + fabs(b)); th = fabs(a) / (fabs(a) + fabs(b)); }
    else { thH = fabs(b) / (fabs(a) + fabs(b)); th = fabs(a) / (fabs(a) + fabs(b)); }
}

// UpdateVel, mac2d.cpp:1740-1849
__device__ __forceinline__ void update_vel_tile(const Grid &g, const MomConst &M, const DivH &ddx, const DivH &ddy,
                                                const double *__restrict__ us, const double *__restrict__ vs,
                                                const double *__restrict__ ps, const double *__restrict__ ls,
                                                const double *__restrict__ H, const double *__restrict__ kappa,
                                                double *__restrict__ u, double *__restrict__ v,
                                                const double *__restrict__ dtp, int bx, int by) {
    const int j = NB + bx * TJ + threadIdx.x, i = NB + by * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    const double dt = *dtp;
    const int64_t c = IX(g, i, j);
    if (i >= NB + 1) {
        const int64_t w = IX(g, i - 1, j);
        double thH, th;
        gfm_theta_first(ls[w], ls[c], thH, th);
        const double iR = 1.0 / (M.rho_h * thH + M.rho_l * (1.0 - thH));
        const double kEff = kappa[c] * th + kappa[w] * (1.0 - th);
        double val = dt * (-M.sigma * kEff) * (H[c] - H[w]);
        val *= M.dx_pow2 ? iR * M.inv_dx : iR / g.dx;
        val += us[c] - ddx(iR * (ps[c] - ps[w]));
        u[c] = val;
    }
    if (j >= NB + 1) {
        const int64_t s = IX(g, i, j - 1);
        double thH, th;
        gfm_theta_first(ls[s], ls[c], thH, th);
        const double iR = 1.0 / (M.rho_h * thH + M.rho_l * (1.0 - thH));
        const double kEff = kappa[c] * th + kappa[s] * (1.0 - th);
        double val = dt * (-M.sigma * kEff) * (H[c] - H[s]);
        val *= M.dy_pow2 ? iR * M.inv_dy : iR / g.dy;
        val += vs[c] - ddy(iR * (ps[c] - ps[s]));
        v[c] = val;
    }
}
__global__ void k_update_vel(Grid g, MomConst M, DivH ddx, DivH ddy, const double *__restrict__ us,
                             const double *__restrict__ vs, const double *__restrict__ ps, const double *__restrict__ ls,
                             const double *__restrict__ H, const double *__restrict__ kappa, double *__restrict__ u,
                             double *__restrict__ v, const double *__restrict__ dtp) {
    update_vel_tile(g, M, ddx, ddy, us, vs, ps, ls, H, kappa, u, v, dtp, blockIdx.x, blockIdx.y);
}

// --------------------------------------------------------------- UpdateDt --
// mac2d.cpp:1851-1880.  max over interior of |u[i+1]*u[i]*0.5| and the v
// analogue (max is order-free, so the GPU value is the reference's).  The
// last block to finish computes dt.
// The CFL time step from the largest |u u| / 2 (a) and |v v| / 2 (b).
__device__ __forceinline__ double cfl_dt(const Grid &g, const MomConst &M, double a, double b) {
    const double dx = g.dx, dy = g.dy;
    const double C = a / dx + b / dy;
    const double V = smax(M.mu_h, M.mu_l) * (2.0 / (dx * dx + dy * dy));
    const double G = smax(sqrt(fabs(M.g) / dy), sqrt(fabs(M.g) / dx));
    const double hmin = smin(dx, dy);
    const double S = sqrt((M.sigma / hmin) / (smin(M.rho_h, M.rho_l) * (hmin * hmin)));
    double dt = 1.79769313486231570815e+308;
    dt = smin(dt, M.cfl / (0.5 * (C + V + sqrt((C + V) * (C + V) + 4.0 * G * G + 4.0 * S * S))));
    return dt;
}

__global__ void k_update_dt(Grid g, MomConst M, const double *__restrict__ u, const double *__restrict__ v,
                            double *__restrict__ partial, unsigned *__restrict__ counter, double *__restrict__ dt_out) {
    double ua = 0.0, va = 0.0;
    const int64_t n = (int64_t)g.nx * g.ny;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int i = NB + (int)(t / g.ny), j = NB + (int)(t % g.ny);
        ua = smax(ua, fabs((u[IX(g, i + 1, j)] * u[IX(g, i, j)]) * 0.5));
        va = smax(va, fabs((v[IX(g, i, j + 1)] * v[IX(g, i, j)]) * 0.5));
    }
    __shared__ double su[32], sv[32];
    for (int o = 16; o > 0; o >>= 1) {
        ua = smax(ua, __shfl_down_sync(0xffffffffu, ua, o));
        va = smax(va, __shfl_down_sync(0xffffffffu, va, o));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { su[wid] = ua; sv[wid] = va; }
    __syncthreads();
    __shared__ bool last;
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) { a = smax(a, su[w]); b = smax(b, sv[w]); }
        partial[2 * blockIdx.x] = a;
        partial[2 * blockIdx.x + 1] = b;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double a = 0.0, b = 0.0;
        for (unsigned k = 0; k < gridDim.x; k++) {
            a = smax(a, ((volatile double *)partial)[2 * k]);
            b = smax(b, ((volatile double *)partial)[2 * k + 1]);
        }
        *dt_out = cfl_dt(g, M, a, b);
        *counter = 0u;
    }
}

// ------------------------------------------------------------- UpdateNTK --
// MACSolver2D::UpdateNTK (mac2d.cpp:124-219) as far as the reference goes:
// Q = |1 - |grad phi|_ENO(phi, phi)|; where Q <= 1e-4 the unit normal from
// central differences is written; elsewhere (its curve-fitting branch is
// empty) nothing is written.  absg holds ENO_DerivAbsLS_2D(phi, phi).
__global__ void k_ntk(Grid g, DivH d2x, DivH d2y, const double *__restrict__ ls, const double *__restrict__ absg,
                      double *__restrict__ nxo, double *__restrict__ nyo) {
    const int j = NB + blockIdx.x * TJ + threadIdx.x, i = NB + blockIdx.y * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    const double Q = fabs(1.0 - absg[IX(g, i, j)]);
    if (Q > 0.0001) return;
    const double gx = d2x(ls[IX(g, i + 1, j)] - ls[IX(g, i - 1, j)]);
    const double gy = d2y(ls[IX(g, i, j + 1)] - ls[IX(g, i, j - 1)]);
    nxo[IX(g, i, j)] = 1.0 / sqrt(gx * gx + gy * gy + 1.0e-100) * gx;
    nyo[IX(g, i, j)] = 1.0 / sqrt(gx * gx + gy * gy + 1.0e-100) * gy;
}

void launch_ntk(const Grid &g, const double *ls, const double *absg, double *nxo, double *nyo, cudaStream_t st) {
    k_ntk<<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, make_divh(2.0 * g.dx), make_divh(2.0 * g.dy), ls, absg, nxo, nyo);
}

// ------------------------------------------------------------------ host --
MomConst make_momconst(const Grid &g, const MomParams &p) {
    MomConst M;
    M.ddx = make_divh(g.dx);
    M.ddy = make_divh(g.dy);
    M.rho_h = p.rho_h;
    M.rho_l = p.rho_l;
    M.mu_h = p.mu_h;
    M.mu_l = p.mu_l;
    M.sigma = p.sigma;
    M.g = p.g;
    M.cfl = p.cfl;
    // kRe = rhoH L U / muH with L = U = 1 (mac2d.cpp:33) unless given; no
    // viscosity when kRe <= 0 (:598).
    const double re = p.numbers_given ? p.re : p.rho_h / p.mu_h;
    M.visc = !(re <= 0.0);
    // Gravity (AddGravityFU/FV :1043-1079): kG = g, kFr = U^2 / (g L) (:35).
    const double fr = p.numbers_given ? p.fr : 1.0 / p.g;
    auto on = [&](int axis) { return (fr != 0 || p.g != 0.0) && !std::isnan(fr) && !std::isinf(fr) && p.g_axis == axis; };
    M.gu = on(0) ? -p.g : 0.0;
    if (p.fix_gravity) {
        M.gv = on(1) ? -p.g : 0.0;
        M.gv_from_u = 0;
    } else {
        // UpdateFV adds AddGravityFU() (:294): -g where the U pattern is
        // nonzero, i.e. columns i >= 4, when the axis is X.
        M.gv = on(0) ? -p.g : 0.0;
        M.gv_from_u = 1;
    }
    const DivH hx = make_divh(g.dx), hy = make_divh(g.dy);
    M.dx_pow2 = hx.pow2;
    M.dy_pow2 = hy.pow2;
    M.inv_dx = hx.inv;
    M.inv_dy = hy.inv;
    return M;
}

void launch_kappa(const Grid &g, const double *ls, double *kappa, cudaStream_t st) {
    const double lim = 1.0 / (g.dx < g.dy ? g.dx : g.dy);
    k_kappa<<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, make_divh(2.0 * g.dx), make_divh(2.0 * g.dy),
                                                   make_divh(g.dx * g.dx), make_divh(g.dy * g.dy), lim, ls, kappa);
}

void launch_heaviside(const Grid &g, const double *ls, double *H, double *HS, cudaStream_t st) {
    const int64_t n = (int64_t)g.sx * g.sy;
    const double eps = (g.dx < g.dy ? g.dx : g.dy) * 1.5;
    k_heaviside<<<(int)((n + 255) / 256), 256, 0, st>>>(n, eps, ls, H, HS);
}

void launch_mom_stage(int kind, const Grid &g, const MomConst &M, const double *ls, const double *H, const double *uin,
                      const double *vin, const double *ub, const double *vb, double *uout, double *vout,
                      const double *dtp, cudaStream_t st) {
    const dim3 grd = cell_grid(g), blk(TJ, TI);
#define MK(K) k_mom_stage<K><<<grd, blk, 0, st>>>(g, M, ls, H, uin, vin, ub, vb, uout, vout, dtp)
    switch (kind) {
    case 0: MK(0); break;
    case 1: MK(1); break;
    case 2: MK(2); break;
    case 3: MK(3); break;
    case 4: MK(4); break;
    case 5: MK(5); break;
    default: MK(6); break;
    }
#undef MK
}

void launch_divergence(const Grid &g, const double *u, const double *v, double *div, cudaStream_t st) {
    k_divergence<<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, make_divh(g.dx), make_divh(g.dy), u, v, div);
}

void launch_update_vel(const Grid &g, const MomConst &M, const double *us, const double *vs, const double *ps,
                       const double *ls, const double *H, const double *kappa, double *u, double *v,
                       const double *dtp, cudaStream_t st) {
    k_update_vel<<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, M, make_divh(g.dx), make_divh(g.dy), us, vs, ps, ls, H,
                                                        kappa, u, v, dtp);
    launch_fill_uv(g, u, v, st);
}

void launch_update_dt(const Grid &g, const MomConst &M, const double *u, const double *v, double *partial,
                      unsigned *counter, double *dt_out, cudaStream_t st) {
    k_update_dt<<<DT_BLOCKS, 256, 0, st>>>(g, M, u, v, partial, counter, dt_out);
}

// ------------------------------------------------------------------------
// Batched full step (asd2g_batch_step): the tile functions above over the
// (instance, tile) work list, one launch per phase for the whole batch.
__global__ void k_bkappa(const BInst *__restrict__ insts, const BTile *__restrict__ tiles) {
    const BTile t = tiles[blockIdx.x];
    const BInst &I = insts[t.inst];
    if (I.g.kappa_mode == 1) kappa_div_tile(I.g, I.kappa_lim, bslot(I, BS_LS), bslot(I, BS_KAPPA), t.bx, t.by);
    else kappa_tile(I.g, I.d2x, I.d2y, I.dxx, I.dyy, I.kappa_lim, bslot(I, BS_LS), bslot(I, BS_KAPPA), t.bx, t.by);
}

__global__ void k_bheaviside(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    const int64_t n = (int64_t)I.g.sx * I.g.sy, k0 = (int64_t)w.c * BSTEP_PAD_CHUNK;
    for (int t = threadIdx.x; t < BSTEP_PAD_CHUNK; t += blockDim.x)
        if (k0 + t < n) heaviside_cell(I.hs_eps, bslot(I, BS_LS), bslot(I, BS_H), bslot(I, BS_HS), k0 + t);
}

template <int SLOT>
__global__ void __launch_bounds__(TJ *TI) k_bmom_slot(const BInst *__restrict__ insts, const BTile *__restrict__ tiles) {
    const BTile t = tiles[blockIdx.x];
    const BInst &I = insts[t.inst];
    const int o = I.order;
    auto stage = [&](auto kind, int in_u, int in_v, int base_u, int base_v, int out_u, int out_v) {
        mom_stage_tile<decltype(kind)::value>(I.g, I.M, bslot(I, BS_LS), bslot(I, BS_HS), bslot(I, in_u),
                                              bslot(I, in_v), base_u >= 0 ? bslot(I, base_u) : nullptr,
                                              base_v >= 0 ? bslot(I, base_v) : nullptr, bslot(I, out_u),
                                              bslot(I, out_v), I.sc, t.bx, t.by);
    };
    using K0 = std::integral_constant<int, 0>;
    using K1 = std::integral_constant<int, 1>;
    using K2 = std::integral_constant<int, 2>;
    using K3 = std::integral_constant<int, 3>;
    if (SLOT == 0) {
        if (o == 0) stage(K0{}, BS_U, BS_V, -1, -1, BS_UHAT, BS_VHAT);
        else stage(K0{}, BS_U, BS_V, -1, -1, BS_UA, BS_VA);
    } else if (SLOT == 1) {
        if (o == 1) stage(K3{}, BS_UA, BS_VA, BS_U, BS_V, BS_UHAT, BS_VHAT);
        else if (o == 2) stage(K1{}, BS_UA, BS_VA, BS_U, BS_V, BS_UB, BS_VB);
    } else {
        if (o == 2) stage(K2{}, BS_UB, BS_VB, BS_U, BS_V, BS_UHAT, BS_VHAT);
    }
}

__global__ void k_bdivergence(const BInst *__restrict__ insts, const BTile *__restrict__ tiles) {
    const BTile t = tiles[blockIdx.x];
    const BInst &I = insts[t.inst];
    divergence_tile(I.g, I.ddx, I.ddy, bslot(I, BS_UHAT), bslot(I, BS_VHAT), bslot(I, BS_DIV), t.bx, t.by);
}

__global__ void k_bupdate_vel(const BInst *__restrict__ insts, const BTile *__restrict__ tiles) {
    const BTile t = tiles[blockIdx.x];
    const BInst &I = insts[t.inst];
    update_vel_tile(I.g, I.M, I.ddx, I.ddy, bslot(I, BS_UHAT), bslot(I, BS_VHAT), bslot(I, BS_PS), bslot(I, BS_LS),
                    bslot(I, BS_H), bslot(I, BS_KAPPA), bslot(I, BS_U), bslot(I, BS_V), I.sc, t.bx, t.by);
}

// Per-instance two-value reduction over the instance's FCG chunks (block c of
// I.chunks): MAX or SUM; the instance's last block gets the totals.
template <bool MAX>
__device__ __forceinline__ bool binst_reduce2(const BInst &I, int c, double a, double b, double &ta, double &tb) {
    __shared__ double sa[32], sb[32];
    __shared__ bool last;
    for (int o = 16; o > 0; o >>= 1) {
        const double oa = __shfl_down_sync(0xffffffffu, a, o), ob = __shfl_down_sync(0xffffffffu, b, o);
        a = MAX ? smax(a, oa) : a + oa;
        b = MAX ? smax(b, ob) : b + ob;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sa[wid] = a;
        sb[wid] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0.0, y = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            x = MAX ? smax(x, sa[w]) : x + sa[w];
            y = MAX ? smax(y, sb[w]) : y + sb[w];
        }
        I.partial[2 * c] = x;
        I.partial[2 * c + 1] = y;
        __threadfence();
        last = atomicAdd(&I.ks->counter, 1u) == (unsigned)I.chunks - 1u;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return false;
    __threadfence();
    double x = 0.0, y = 0.0;
    for (int k = 0; k < I.chunks; k++) {
        const double pa = __ldcg(I.partial + 2 * k), pb = __ldcg(I.partial + 2 * k + 1);
        x = MAX ? smax(x, pa) : x + pa;
        y = MAX ? smax(y, pb) : y + pb;
    }
    ta = x;
    tb = y;
    I.ks->counter = 0u;
    return true;
}

__global__ void __launch_bounds__(256) k_bupdate_dt(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    const Grid &g = I.g;
    const double *u = bslot(I, BS_U), *v = bslot(I, BS_V);
    double ua = 0.0, va = 0.0;
    const int64_t k0 = (int64_t)w.c * FCG_CHUNK;
    for (int t = threadIdx.x; t < FCG_CHUNK; t += blockDim.x) {
        const int64_t k = k0 + t;
        if (k >= I.n) break;
        const int i = NB + (int)(k / g.ny), j = NB + (int)(k % g.ny);
        ua = smax(ua, fabs((u[IX(g, i + 1, j)] * u[IX(g, i, j)]) * 0.5));
        va = smax(va, fabs((v[IX(g, i, j + 1)] * v[IX(g, i, j)]) * 0.5));
    }
    double a, b;
    if (binst_reduce2<true>(I, w.c, ua, va, a, b)) I.sc[1] = cfl_dt(g, I.M, a, b);
}

__global__ void __launch_bounds__(256) k_bvolume(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    const Grid &g = I.g;
    const double *H = bslot(I, BS_H), *HS = bslot(I, BS_HS);
    double sa = 0.0, sb = 0.0;
    const int64_t k0 = (int64_t)w.c * FCG_CHUNK;
    for (int t = threadIdx.x; t < FCG_CHUNK; t += blockDim.x) {
        const int64_t k = k0 + t;
        if (k >= I.n) break;
        const int64_t c = IX(g, NB + (int)(k / g.ny), NB + (int)(k % g.ny));
        sa += H[c];
        sb += HS[c];
    }
    double a, b;
    if (binst_reduce2<false>(I, w.c, sa, sb, a, b)) {
        I.sc[2] = a * g.dx * g.dy;
        I.sc[3] = b * g.dx * g.dy;
    }
}

void launch_bstep_kappa(const BStepPlan &P, cudaStream_t st) {
    k_bkappa<<<P.ntiles, dim3(TJ, TI), 0, st>>>(P.insts, P.tiles);
}
void launch_bstep_heaviside(const BStepPlan &P, cudaStream_t st) {
    k_bheaviside<<<P.npad, 256, 0, st>>>(P.insts, P.pad_chunks);
}
void launch_bstep_volume(const BStepPlan &P, cudaStream_t st) {
    k_bvolume<<<P.nchunks, 256, 0, st>>>(P.insts, P.chunks);
}
void launch_bstep_mom_slot(const BStepPlan &P, int slot, cudaStream_t st) {
    const dim3 blk(TJ, TI);
    if (slot == 0) k_bmom_slot<0><<<P.ntiles, blk, 0, st>>>(P.insts, P.tiles);
    else if (slot == 1) k_bmom_slot<1><<<P.ntiles, blk, 0, st>>>(P.insts, P.tiles);
    else k_bmom_slot<2><<<P.ntiles, blk, 0, st>>>(P.insts, P.tiles);
}
void launch_bstep_divergence(const BStepPlan &P, cudaStream_t st) {
    k_bdivergence<<<P.ntiles, dim3(TJ, TI), 0, st>>>(P.insts, P.tiles);
}
void launch_bstep_update_vel(const BStepPlan &P, cudaStream_t st) {
    k_bupdate_vel<<<P.ntiles, dim3(TJ, TI), 0, st>>>(P.insts, P.tiles);
    launch_bstep_fill_uv(P, BS_U, BS_V, st);
}
void launch_bstep_update_dt(const BStepPlan &P, cudaStream_t st) {
    k_bupdate_dt<<<P.nchunks, 256, 0, st>>>(P.insts, P.chunks);
}

}  // namespace asd2g
