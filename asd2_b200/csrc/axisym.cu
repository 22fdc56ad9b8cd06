// The axisymmetric MAC step (MACSolver2DAxisym, mac2dAxisym.cpp) on the
// padded (r, z) grid: x is r (index i, dx = dr), y is z (index j, the
// contiguous one).  Convection, Heaviside and the projection are the 2D
// solver's kernels (the reference's axisymmetric versions are the same
// arithmetic); this unit holds what differs: the curvature with its hoop term,
// the viscous terms, the implicit viscous step of uhat and vhat (one Thomas
// solve per grid line, r lines then z lines), the r-weighted divergence, the
// r-weighted GFM assembly and the time-step bound.
//
// Built with -fmad=false and IEEE division, in the reference's operation
// order: every kernel except the curvature (CUDA's pow in place of libm's) is
// bit-identical to the reference.
#include "lsmath.cuh"
#include "momentum.cuh"
#include "pressure.cuh"

namespace asd2g {

namespace {

__device__ __forceinline__ double mu_of(const MomConst &M, const double *__restrict__ H, int64_t c) {
    return M.mu_l + (M.mu_h - M.mu_l) * H[c];
}
// 0.25 * (a0 + a1 + a2 + a3), summed left to right.
__device__ __forceinline__ double quarter(const double *__restrict__ a, int64_t c0, int64_t c1, int64_t c2,
                                          int64_t c3) {
    return 0.25 * (a[c0] + a[c1] + a[c2] + a[c3]);
}
__device__ __forceinline__ double quarter_mu(const MomConst &M, const double *__restrict__ H, int64_t c0, int64_t c1,
                                             int64_t c2, int64_t c3) {
    return 0.25 * (mu_of(M, H, c0) + mu_of(M, H, c1) + mu_of(M, H, c2) + mu_of(M, H, c3));
}
// Heavy fraction of a face between level-set values a, b (the implicit
// step's rule, mac2dAxisym.cpp:1027-1043): both >= 0 heavy, both <= 0 light.
__device__ __forceinline__ double heavy_frac(double a, double b) {
    if (a >= 0.0 && b >= 0.0) return 1.0;
    if (a <= 0.0 && b <= 0.0) return 0.0;
    if (a >= 0.0 && b < 0.0) return fabs(a) / (fabs(a) + fabs(b));
    return fabs(b) / (fabs(a) + fabs(b));
}
__device__ __forceinline__ double rho_mix(const MomConst &M, double thH) {
    return M.rho_h * thH + M.rho_l * (1.0 - thH);
}
// Density of the explicit viscous terms (mac2dAxisym.cpp:682-736): the pure
// cases take the fluid's own density.
__device__ __forceinline__ double rho_face(const MomConst &M, double a, double b) {
    if (a >= 0.0 && b >= 0.0) return M.rho_h;
    if (a <= 0.0 && b <= 0.0) return M.rho_l;
    return rho_mix(M, (a >= 0.0) ? fabs(a) / (fabs(a) + fabs(b)) : fabs(b) / (fabs(a) + fabs(b)));
}

// Face fractions of the GFM assembly (mac2dAxisym.cpp:1579-1700; the same
// rules as the 2D assembly): thH the heavy fraction, th the curvature weight.
// first: pair (W, M) or (S, M); second: pair (M, E) or (M, N).
__device__ __forceinline__ void face_first(double a, double b, double &thH, double &th) {
    if (a >= 0.0 && b >= 0.0) { thH = 1.0; th = 0.0; }
    else if (a < 0.0 && b < 0.0) { thH = 0.0; th = 0.0; }
    else if (a >= 0.0 && b < 0.0) { thH = fabs(a) / (fabs(a) + fabs(b)); th = fabs(a) / (fabs(a) + fabs(b)); }
    else { thH = fabs(b) / (fabs(a) + fabs(b)); th = fabs(a) / (fabs(a) + fabs(b)); }
}
__device__ __forceinline__ void face_second(double m, double e, double &thH, double &th) {
    if (m >= 0.0 && e >= 0.0) { thH = 1.0; th = 0.0; }
    else if (m < 0.0 && e < 0.0) { thH = 0.0; th = 0.0; }
    else if (m >= 0.0 && e < 0.0) { thH = fabs(m) / (fabs(m) + fabs(e)); th = fabs(e) / (fabs(m) + fabs(e)); }
    else { thH = fabs(e) / (fabs(m) + fabs(e)); th = fabs(e) / (fabs(m) + fabs(e)); }
}

// ---------------------------------------------------------------- kappa --
// UpdateKappa, mac2dAxisym.cpp:222-262: the 2D curvature expression plus the
// hoop term dphi/dr |grad phi|^2 / r; one-sided dphi/dr in the axis column;
// dphi/dz of a column outside the interior reads as 0.
__global__ void k_axi_kappa(Grid g, double base_r, double lim, const double *__restrict__ ls,
                            double *__restrict__ kappa) {
    const int j = NB + blockIdx.x * TJ + threadIdx.x, i = NB + blockIdx.y * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    const double dr = g.dx, dz = g.dy;
    const int64_t c = IX(g, i, j);
    auto gz = [&](int ii) -> double {
        if (ii < NB || ii >= g.nx + NB) return 0.0;
        return (ls[IX(g, ii, j + 1)] - ls[IX(g, ii, j - 1)]) / (2.0 * dz);
    };
    double dR = (ls[IX(g, i + 1, j)] - ls[IX(g, i - 1, j)]) / (2.0 * dr);
    if (i == NB) dR = (ls[IX(g, i + 1, j)] - ls[c]) / dr;
    const double dZ = gz(i);
    const double s = sqrt(dR * dR + dZ * dZ + 1.0e-100);
    const double r = base_r + (i + 0.5 - NB) * dr;
    double k = ((ls[IX(g, i - 1, j)] - 2.0 * ls[c] + ls[IX(g, i + 1, j)]) / (dr * dr) * dZ * dZ -
                2.0 * (gz(i + 1) - gz(i - 1)) / (2.0 * dr) * dR * dZ +
                (ls[IX(g, i, j - 1)] - 2.0 * ls[c] + ls[IX(g, i, j + 1)]) / (dz * dz) * dR * dR + dR * (s * s) / r) /
               pow(s, 3.0);
    kappa[c] = isgn(k) * fabs(smin(fabs(k), lim));
}

// ----------------------------------------------------------- right sides --
// GetRHSU (mac2dAxisym.cpp:264-292) over the whole padded array: interior u
// faces get u + dt (-cU + gU + vU) with the viscous term of
// AddExternalViscosityFU (:590-753) computed here, every other entry 0
// (visc_only: the viscous term alone, AddExternalViscosityFU itself).
__global__ void k_axi_rhs_u(Grid g, MomConst M, const double *__restrict__ ls, const double *__restrict__ u,
                            const double *__restrict__ v, const double *__restrict__ H,
                            const double *__restrict__ cU, const double *__restrict__ dtp, int visc_only,
                            double *__restrict__ out) {
    const int j = blockIdx.x * TJ + threadIdx.x, i = blockIdx.y * TI + threadIdx.y;
    if (i >= g.sx || j >= g.sy) return;
    const int64_t c = IX(g, i, j);
    if (!(i >= NB + 1 && i < g.nx + NB && j >= NB && j < g.ny + NB)) {
        out[c] = 0.0;
        return;
    }
    double vU = 0.0;
    if (M.visc) {
        const int64_t W = IX(g, i - 1, j), Nn = IX(g, i, j + 1), WN = IX(g, i - 1, j + 1), S = IX(g, i, j - 1),
                      WS = IX(g, i - 1, j - 1);
        const double lsN = quarter(ls, c, W, WN, Nn), lsS = quarter(ls, c, W, WS, S);
        const double muN = quarter_mu(M, H, c, W, WN, Nn), muS = quarter_mu(M, H, c, W, WS, S);
        const double visZ = (muN * (v[Nn] - v[WN]) / g.dx - muS * (v[c] - v[W]) / g.dx) / g.dy;
        vU = visZ / rho_face(M, lsS, lsN);
    }
    out[c] = visc_only ? vU : u[c] + *dtp * (-cU[c] + M.gu + vU);
}

// GetRHSV (mac2dAxisym.cpp:294-322) with AddExternalViscosityFV (:755-910):
// the r-part of the stress plus the hoop term from the new uhat, r = (i +
// 1/2) dr without kBaseR as the reference has it.  Gravity follows the U
// pattern (AddGravityFU, :306) unless the session fixes it.
__global__ void k_axi_rhs_v(Grid g, MomConst M, const double *__restrict__ ls, const double *__restrict__ u,
                            const double *__restrict__ uhat, const double *__restrict__ v,
                            const double *__restrict__ H, const double *__restrict__ cV,
                            const double *__restrict__ dtp, int visc_only, double *__restrict__ out) {
    const int j = blockIdx.x * TJ + threadIdx.x, i = blockIdx.y * TI + threadIdx.y;
    if (i >= g.sx || j >= g.sy) return;
    const int64_t c = IX(g, i, j);
    if (!(i >= NB && i < g.nx + NB && j >= NB + 1 && j < g.ny + NB)) {
        out[c] = 0.0;
        return;
    }
    double vV = 0.0;
    if (M.visc) {
        const int64_t W = IX(g, i - 1, j), E = IX(g, i + 1, j), S = IX(g, i, j - 1), WS = IX(g, i - 1, j - 1),
                      ES = IX(g, i + 1, j - 1);
        const double r = (i + 0.5 - NB) * g.dx;
        const double lsVW = quarter(ls, c, W, WS, S), lsVE = quarter(ls, c, E, ES, S);
        const double muVW = quarter_mu(M, H, c, W, WS, S), muVE = quarter_mu(M, H, c, E, ES, S);
        const double visR = (muVE * (u[E] - u[ES]) / g.dy - muVW * (u[c] - u[S]) / g.dy) / g.dx;
        const double visZ = 0.5 * (mu_of(M, H, c) + mu_of(M, H, S)) / r *
                            (0.5 * (uhat[c] + uhat[E]) - 0.5 * (uhat[S] + uhat[ES])) / g.dy;
        vV = visR / rho_face(M, lsVW, lsVE) + visZ / rho_face(M, ls[S], ls[c]);
    }
    const double gV = (M.gv_from_u && i < NB + 1) ? 0.0 : M.gv;
    out[c] = visc_only ? vV : v[c] + *dtp * (-cV[c] + gV + vV);
}

// ------------------------------------------------------ implicit viscous --
// GetUHat / GetVHat (mac2dAxisym.cpp:950-1229, :1231-1478): per grid line a
// tridiagonal system lo x[k-1] + di x[k] + up x[k+1] = d, solved in the
// elimination order of SolveTDMA (:2255-2306): scale the first row, pivot
// di - lo up', back-substitute.  Bit-exact parity needs that serial
// recurrence per line, so the work is split: fully parallel kernels compute
// every row's coefficients and end-row edits (raw U / V kinds, Grid bu / bv)
// into line-ordered arrays, then one thread per line runs only the
// recurrence, streaming its four arrays with the next row prefetched.  The
// r lines use the padded layout (line = j, consecutive threads read
// consecutive j); the z lines a transposed copy (element (i, j) at i + sx j)
// so that their reads are coalesced too.
struct Tri {
    double lo, di, up, d;
};

// End-row edits of a line: first = the first row (lo dropped), else the last
// (up dropped).  neu: the kind folds the dropped entry into the diagonal;
// dir: it moves scale * constant to the right side; per: the other end's
// right side value.
__device__ __forceinline__ void end_row(Tri &t, bool first, bool neu, bool dir, bool per, double scale, double cst,
                                        double other) {
    double &e = first ? t.lo : t.up;
    if (neu) {
        t.di += e;
        e = 0.0;
    } else if (dir) {
        t.d -= scale == 1.0 ? e * cst : e * scale * cst;
        e = 0.0;
    } else if (per) {
        t.d -= e * other;
        e = 0.0;
    }
}

__device__ __forceinline__ bool k_neu2(int b) { return b == 1 /*NEUMANN*/ || b == 6 /*OUTLET*/; }
__device__ __forceinline__ bool k_neu3(int b) { return b == 1 || b == 3 /*AXISYM*/ || b == 6; }
__device__ __forceinline__ bool k_dir3(int b) { return b == 2 /*DIRICHLET*/ || b == 5 /*INLET*/ || b == 4 /*WALL*/; }
__device__ __forceinline__ bool k_dir4(int b) { return k_dir3(b) || b == 3; }

// transposed (z-line) position of cell (i, j)
__device__ __forceinline__ int64_t TX(const Grid &g, int i, int j) { return (int64_t)i + (int64_t)g.sx * j; }

__device__ __forceinline__ void store_tri(const Tri &t, int64_t a, double *lo, double *di, double *up, double *d) {
    lo[a] = t.lo;
    di[a] = t.di;
    up[a] = t.up;
    d[a] = t.d;
}

// u, r lines: faces i = 4 .. nx+2 of every row j (k = i - 4, m = nx - 1 rows).
__global__ void k_axi_coef_u_r(Grid g, MomConst M, const double *__restrict__ ls, const double *__restrict__ rhs,
                               const double *__restrict__ H, const double *__restrict__ dtp, double *lo, double *di,
                               double *up, double *d) {
    const int J = NB + blockIdx.x * TJ + threadIdx.x, I = NB + 1 + blockIdx.y * TI + threadIdx.y;
    if (J >= g.ny + NB || I >= g.nx + NB) return;
    const int k = I - NB - 1, m = g.nx - 1;
    const double dr = g.dx, dt = *dtp;
    const int64_t c = IX(g, I, J), w = IX(g, I - 1, J);
    const double rUM = (k + 1.0) * dr, rPW = (k + 0.5) * dr, rPM = (k + 1.5) * dr;
    const double muW = mu_of(M, H, w), muM = mu_of(M, H, c);
    const double rho = rho_mix(M, heavy_frac(ls[w], ls[c]));
    Tri t;
    t.d = rhs[c];
    t.lo = -dt / (rho * rUM) * (2.0 * rPW * muW) / (dr * dr);
    t.di = 1.0 + dt / (rho * rUM) * 2.0 * (rPW * muW + rPM * muM) / (dr * dr);
    t.up = -dt / (rho * rUM) * (2.0 * rPM * muM) / (dr * dr);
    if (k == 0)
        end_row(t, true, k_neu2(g.bu[0]), k_dir4(g.bu[0]), g.bu[0] == 0, 1.0, g.cu[0], rhs[IX(g, m + NB, J)]);
    if (k == m - 1)
        end_row(t, false, k_neu2(g.bu[1]), k_dir4(g.bu[1]), g.bu[1] == 0, 1.0, g.cu[1], rhs[IX(g, NB + 1, J)]);
    store_tri(t, c, lo, di, up, d);
}

// u, z lines of every column i (rows j = 3 .. ny+2) from the r-solved field
// xr, transposed; den = 1 + dt / rho (mu_W + mu_M) / r^2, the 1/r^2 term.
__global__ void k_axi_coef_u_z(Grid g, MomConst M, const double *__restrict__ ls, const double *__restrict__ H,
                               const double *__restrict__ dtp, const double *__restrict__ xr, double *lo, double *di,
                               double *up, double *d, double *den) {
    const int J = NB + blockIdx.x * TJ + threadIdx.x, I = NB + 1 + blockIdx.y * TI + threadIdx.y;
    if (J >= g.ny + NB || I >= g.nx + NB) return;
    const int jj = J - NB, n = g.ny;
    const double dz = g.dy, dt = *dtp;
    const int64_t c = IX(g, I, J), W = IX(g, I - 1, J), S = IX(g, I, J - 1), WS = IX(g, I - 1, J - 1),
                  Nn = IX(g, I, J + 1), WN = IX(g, I - 1, J + 1);
    const double lsS = quarter(ls, c, W, WS, S), lsN = quarter(ls, c, W, WN, Nn);
    const double muS = quarter_mu(M, H, c, W, WS, S), muN = quarter_mu(M, H, c, W, WN, Nn);
    const double rho = rho_mix(M, heavy_frac(lsS, lsN));
    Tri t;
    t.d = xr[c];
    t.lo = -dt / rho * muS / (dz * dz);
    t.di = 1.0 + dt / rho * (muS + muN) / (dz * dz);
    t.up = -dt / rho * muN / (dz * dz);
    if (jj == 0)
        end_row(t, true, k_neu3(g.bu[2]), k_dir3(g.bu[2]), g.bu[2] == 0, 2.0, g.cu[2], xr[IX(g, I, n - 1 + NB)]);
    if (jj == n - 1)
        end_row(t, false, k_neu3(g.bu[3]), k_dir3(g.bu[3]), g.bu[3] == 0, 2.0, g.cu[3], xr[IX(g, I, NB)]);
    const int64_t a = TX(g, I, J);
    store_tri(t, a, lo, di, up, d);
    const double rUM = (I - NB) * g.dx;
    const double rhoWE = rho_mix(M, heavy_frac(ls[W], ls[c]));
    den[a] = 1.0 + dt / rhoWE * (mu_of(M, H, W) + mu_of(M, H, c)) / (rUM * rUM);
}

// v, r lines: cells i = 3 .. nx+2 of v-row j (j = 4 .. ny+2).
__global__ void k_axi_coef_v_r(Grid g, MomConst M, const double *__restrict__ ls, const double *__restrict__ rhs,
                               const double *__restrict__ H, const double *__restrict__ dtp, double *lo, double *di,
                               double *up, double *d) {
    const int J = NB + 1 + blockIdx.x * TJ + threadIdx.x, I = NB + blockIdx.y * TI + threadIdx.y;
    if (J >= g.ny + NB || I >= g.nx + NB) return;
    const int k = I - NB, n = g.nx;
    const double dr = g.dx, dt = *dtp;
    const int64_t c = IX(g, I, J), W = IX(g, I - 1, J), E = IX(g, I + 1, J), S = IX(g, I, J - 1),
                  WS = IX(g, I - 1, J - 1), ES = IX(g, I + 1, J - 1);
    const double rVM = (k + 0.5) * dr, rVW = k * dr, rVE = (k + 1.0) * dr;
    const double lsVW = quarter(ls, c, W, S, WS), lsVE = quarter(ls, c, E, S, ES);
    const double muVW = quarter_mu(M, H, c, W, S, WS), muVE = quarter_mu(M, H, c, E, S, ES);
    const double rho = rho_mix(M, heavy_frac(lsVW, lsVE));
    Tri t;
    t.d = rhs[c];
    t.lo = -dt / (rho * rVM) * rVW * muVW / (dr * dr);
    t.di = 1.0 + dt / (rho * rVM) * (rVW * muVW + rVE * muVE) / (dr * dr);
    t.up = -dt / (rho * rVM) * rVE * muVE / (dr * dr);
    if (k == 0)
        end_row(t, true, k_neu3(g.bv[0]), k_dir3(g.bv[0]), g.bv[0] == 0, 2.0, g.cv[0], rhs[IX(g, n - 1 + NB, J)]);
    if (k == n - 1)
        end_row(t, false, k_neu3(g.bv[1]), k_dir3(g.bv[1]), g.bv[1] == 0, 2.0, g.cv[1], rhs[IX(g, NB, J)]);
    store_tri(t, c, lo, di, up, d);
}

// v, z lines of every column i (v faces j = 4 .. ny+2), transposed.
__global__ void k_axi_coef_v_z(Grid g, MomConst M, const double *__restrict__ ls, const double *__restrict__ H,
                               const double *__restrict__ dtp, const double *__restrict__ xr, double *lo, double *di,
                               double *up, double *d) {
    const int J = NB + 1 + blockIdx.x * TJ + threadIdx.x, I = NB + blockIdx.y * TI + threadIdx.y;
    if (J >= g.ny + NB || I >= g.nx + NB) return;
    const int jj = J - NB - 1, n = g.ny - 1;
    const double dz = g.dy, dt = *dtp;
    const int64_t c = IX(g, I, J), S = IX(g, I, J - 1);
    const double muS = mu_of(M, H, S), muM = mu_of(M, H, c);
    const double rho = rho_mix(M, heavy_frac(ls[S], ls[c]));
    Tri t;
    t.d = xr[c];
    t.lo = -dt / rho * (2.0 * muS) / (dz * dz);
    t.di = 1.0 + dt / rho * 2.0 * (muS + muM) / (dz * dz);
    t.up = -dt / rho * (2.0 * muM) / (dz * dz);
    if (jj == 0)
        end_row(t, true, k_neu2(g.bv[2]), k_dir4(g.bv[2]), g.bv[2] == 0, 1.0, g.cv[2], xr[IX(g, I, n - 1 + NB + 1)]);
    if (jj == n - 1)
        end_row(t, false, k_neu2(g.bv[3]), k_dir4(g.bv[3]), g.bv[3] == 0, 1.0, g.cv[3], xr[IX(g, I, NB + 1)]);
    store_tri(t, TX(g, I, J), lo, di, up, d);
}

// Element (line l, row k) of a line-ordered array: base + l * ls + k * ks.
struct LineMap {
    int64_t base, ls, ks;
};

// The recurrence of one line per thread (n >= 2 rows): the forward sweep
// overwrites up with the scaled upper diagonal and d with the scaled right
// side, the back substitution leaves the solution in d, or, with out, writes
// it there through O (divided by den when den is given).  The rows are read
// TP ahead into a register ring (the loads of row k + TP are issued before row
// k's divisions), since one row's dependent chain is far shorter than a load
// from L2 or HBM.
constexpr int TP = 8;

// Rows further ahead than the register ring are pulled into L1 with a
// prefetch hint PF rows ahead (the ring alone covers 8 rows of the dependent
// chain, less than an L2 round trip).  Build-time tunable.
#ifndef ASD2G_AXI_THOMAS_PF
#define ASD2G_AXI_THOMAS_PF 32
#endif
constexpr int PF = ASD2G_AXI_THOMAS_PF;

// Lines per CTA.  A sweep has one thread per grid line and no more (1023 to
// 2048 threads at 1024 x 2048), so the CTAs are kept small to spread the
// lines over all the SMs: each SM's L1 keeps a bounded number of misses in
// flight, and the rows' loads bound the sweep.  8 adjacent lines read 64
// contiguous bytes per row and array (two full sectors).  Wider CTAs only
// once there are lines for several CTAs per SM.  Build-time override:
// ASD2G_AXI_THOMAS_LINES.
inline int thomas_lines_per_cta(int nlines) {
#ifdef ASD2G_AXI_THOMAS_LINES
    (void)nlines;
    return ASD2G_AXI_THOMAS_LINES;
#else
    return nlines <= 4 * 148 * 8 ? 8 : nlines <= 4 * 148 * 32 ? 32 : 64;
#endif
}
__device__ __forceinline__ void pf_l1(const void *p) { asm volatile("prefetch.L1 [%0];" ::"l"(p)); }

// a / b with the IEEE result, taking the quotient of a zero numerator as the
// product (a signed zero, sign(a) xor sign(b), for finite nonzero b): where
// the fluid is at rest most right sides are exactly 0, and the division
// sequence leaves its fast path for a zero quotient.
__device__ __forceinline__ double qdiv(double a, double b) { return a == 0.0 ? a * b : a / b; }

__global__ void __launch_bounds__(64) k_axi_thomas(int nlines, int n, LineMap A, const double *__restrict__ lo,
                                                   const double *__restrict__ di, double *__restrict__ up,
                                                   double *__restrict__ d, LineMap O, double *__restrict__ out,
                                                   const double *__restrict__ den) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nlines) return;
    const int64_t a0 = A.base + (int64_t)l * A.ls, ks = A.ks;
    double rlo[TP], rdi[TP], rup[TP], rd[TP];
#pragma unroll
    for (int q = 0; q < TP; q++)
        if (q < n) {
            const int64_t a = a0 + (int64_t)q * ks;
            rlo[q] = lo[a];
            rdi[q] = di[a];
            rup[q] = up[a];
            rd[q] = d[a];
        }
    double up_prev = 0.0, x_prev = 0.0;
    for (int k0 = 0; k0 < n; k0 += TP) {
#pragma unroll
        for (int q = 0; q < TP; q++) {
            const int k = k0 + q;
            if (k < n) {
                const double clo = rlo[q], cdi = rdi[q], cup = rup[q], cd = rd[q];
                if (k + TP < n) {
                    const int64_t a = a0 + (int64_t)(k + TP) * ks;
                    rlo[q] = lo[a];
                    rdi[q] = di[a];
                    rup[q] = up[a];
                    rd[q] = d[a];
                }
                if (k + PF < n) {
                    const int64_t a = a0 + (int64_t)(k + PF) * ks;
                    pf_l1(lo + a);
                    pf_l1(di + a);
                    pf_l1(up + a);
                    pf_l1(d + a);
                }
                if (k == 0) {
                    up_prev = qdiv(cup, cdi);
                    x_prev = qdiv(cd, cdi);
                } else {
                    const double piv = cdi - clo * up_prev;
                    up_prev = (k < n - 1) ? qdiv(cup, piv) : cup;
                    x_prev = qdiv(cd - clo * x_prev, piv);
                }
                const int64_t a = a0 + (int64_t)k * ks;
                up[a] = up_prev;
                d[a] = x_prev;
            }
        }
    }
    // back substitution, rows n-2 .. 0, again TP rows ahead
    const int64_t o0 = out ? O.base + (int64_t)l * O.ls : 0;
    auto emit = [&](int k, int64_t a, double x) {
        if (out) out[o0 + (int64_t)k * O.ks] = den ? qdiv(x, den[a]) : x;
        else d[a] = x;
    };
    emit(n - 1, a0 + (int64_t)(n - 1) * ks, x_prev);
    double bup[TP], bd[TP];
#pragma unroll
    for (int q = 0; q < TP; q++) {
        const int k = n - 2 - q;
        if (k >= 0) {
            const int64_t a = a0 + (int64_t)k * ks;
            bup[q] = up[a];
            bd[q] = d[a];
        }
    }
    for (int k0 = n - 2; k0 >= 0; k0 -= TP) {
#pragma unroll
        for (int q = 0; q < TP; q++) {
            const int k = k0 - q;
            if (k >= 0) {
                const double cup = bup[q], cd = bd[q];
                if (k - TP >= 0) {
                    const int64_t a = a0 + (int64_t)(k - TP) * ks;
                    bup[q] = up[a];
                    bd[q] = d[a];
                }
                if (k - PF >= 0) {
                    const int64_t a = a0 + (int64_t)(k - PF) * ks;
                    pf_l1(up + a);
                    pf_l1(d + a);
                    if (den) pf_l1(den + a);
                }
                x_prev = cd - cup * x_prev;
                emit(k, a0 + (int64_t)k * ks, x_prev);
            }
        }
    }
}

// ------------------------------------------------------------ divergence --
// GetDivergence4Poisson (mac2dAxisym.cpp:1980-1994, for_poisson = 1):
// (r_e u_e - r_w u_w) / dr + r_c (v_n - v_s) / dz; GetDivergence (:1996-2008):
// u/r + du/dr + dv/dz.  Every entry outside the interior is 0.
__global__ void k_axi_div(Grid g, double base_r, int for_poisson, const double *__restrict__ u,
                          const double *__restrict__ v, double *__restrict__ div) {
    const int j = blockIdx.x * TJ + threadIdx.x, i = blockIdx.y * TI + threadIdx.y;
    if (i >= g.sx || j >= g.sy) return;
    const int64_t c = IX(g, i, j);
    if (!(i >= NB && i < g.nx + NB && j >= NB && j < g.ny + NB)) {
        div[c] = 0.0;
        return;
    }
    const double dr = g.dx, dz = g.dy;
    const double rc = base_r + (i + 0.5 - NB) * dr;
    const double uw = u[c], ue = u[IX(g, i + 1, j)], dv = v[IX(g, i, j + 1)] - v[c];
    if (for_poisson) {
        const double re = base_r + (i + 1.0 - NB) * dr, rw = base_r + (i - NB) * dr;
        div[c] = (re * ue - rw * uw) / dr + rc * dv / dz;
    } else {
        div[c] = 0.5 * (uw + ue) / rc + (ue - uw) / dr + dv / dz;
    }
}

// -------------------------------------------------------------- assembly --
__device__ __forceinline__ bool p_neu(int b) { return b == 1 || b == 3 || b == 4; }  // NEUMANN, AXISYM, WALL
__device__ __forceinline__ bool p_dir(int b) { return b == 2 || b == 5 || b == 6 || b == 7; }  // DIRICHLET, INLET, OUTLET, PRESSURE

// One interior cell of SolvePoisson's system (mac2dAxisym.cpp:1563-1916) in
// the matrix-free form of the 2D assembly.  West/east coefficients carry r at
// the face, or across the interface r interpolated between the centres with
// the curvature weight theta (the west one clamped at 0); south/north carry
// the centre's r.  ps is zero during the reference's assembly, so its -ps
// terms are -0.
__global__ void k_axi_assemble(Grid g, MomConst M, double base_r, const double *__restrict__ ls,
                               const double *__restrict__ kappa, const double *__restrict__ H,
                               const double *__restrict__ div, const double *__restrict__ dtp, Sys S) {
    const int j = NB + blockIdx.x * TJ + threadIdx.x, i = NB + blockIdx.y * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    const double dt = *dtp, dr = g.dx, dz = g.dy, sig = M.sigma;
    const int64_t c = IX(g, i, j), w = IX(g, i - 1, j), e = IX(g, i + 1, j), s = IX(g, i, j - 1),
                  n = IX(g, i, j + 1);
    const double lsW = ls[w], lsE = ls[e], lsM = ls[c], lsS = ls[s], lsN = ls[n];
    const double rPW = base_r + (i - 0.5 - NB) * dr, rPM = base_r + (i + 0.5 - NB) * dr,
                 rPE = base_r + (i + 1.5 - NB) * dr, rWf = base_r + (i - NB) * dr, rEf = base_r + (i + 1.0 - NB) * dr;
    double thH, th, rEff, kEff;
    // west face
    if (lsW >= 0.0 && lsM >= 0.0) { thH = 1.0; th = 0.0; rEff = rWf; }
    else if (lsW < 0.0 && lsM < 0.0) { thH = 0.0; th = 0.0; rEff = rWf; }
    else {
        face_first(lsW, lsM, thH, th);
        rEff = smax(rPM * th + rPW * (1.0 - th), 0.0);
    }
    kEff = kappa[c] * th + kappa[w] * (1.0 - th);
    double pW = rEff / rho_mix(M, thH);
    double FW = -dt * (-sig * kEff) * (H[c] - H[w]);
    FW *= pW / (dr * dr);
    // east face
    if (lsM >= 0.0 && lsE >= 0.0) { thH = 1.0; th = 0.0; rEff = rEf; }
    else if (lsM < 0.0 && lsE < 0.0) { thH = 0.0; th = 0.0; rEff = rEf; }
    else {
        face_second(lsM, lsE, thH, th);
        rEff = rPM * th + rPE * (1.0 - th);
    }
    kEff = kappa[c] * th + kappa[e] * (1.0 - th);
    double pE = rEff / rho_mix(M, thH);
    double FE = dt * (-sig * kEff) * (H[e] - H[c]);
    FE *= pE / (dr * dr);
    // south and north faces
    face_first(lsS, lsM, thH, th);
    kEff = kappa[c] * th + kappa[s] * (1.0 - th);
    double pS = rPM / rho_mix(M, thH);
    double FS = -dt * (-sig * kEff) * (H[c] - H[s]);
    FS *= pS / (dz * dz);
    face_second(lsM, lsN, thH, th);
    kEff = kappa[c] * th + kappa[n] * (1.0 - th);
    double pN = rPM / rho_mix(M, thH);
    double FN = dt * (-sig * kEff) * (H[n] - H[c]);
    FN *= pN / (dz * dz);
    double r = 0.0;
    r -= FW + FE + FS + FN;
    r -= div[c];
    pS *= -1.0; pW *= -1.0; pE *= -1.0; pN *= -1.0;
    double aS = pS / (dz * dz), aW = pW / (dr * dr), aE = pE / (dr * dr), aN = pN / (dz * dz);
    double aC = -(pW + pE) / (dr * dr) - (pS + pN) / (dz * dz);
    const int nx = g.nx, ny = g.ny;
    if (i == NB && p_neu(g.bp[0])) { aW = 0.0; aC += pW / (dr * dr); }
    else if (i == NB && p_dir(g.bp[0])) { aW = 0.0; r -= pW / (dr * dr) * (-0.0 + 2.0 * g.cp[0]); }
    if (i == NB + nx - 1 && p_neu(g.bp[1])) { aE = 0.0; aC += pE / (dr * dr); }
    else if (i == NB + nx - 1 && p_dir(g.bp[1])) { aE = 0.0; r -= pE / (dr * dr) * (-0.0 + 2.0 * g.cp[1]); }
    if (j == NB && p_neu(g.bp[2])) { aS = 0.0; aC += pS / (dz * dz); }
    else if (j == NB && p_dir(g.bp[2])) { aS = 0.0; r -= pS / (dz * dz) * (-0.0 + 2.0 * g.cp[2]); }
    if (j == NB + ny - 1 && p_neu(g.bp[3])) { aN = 0.0; aC += pN / (dz * dz); }
    else if (j == NB + ny - 1 && p_dir(g.bp[3])) { aN = 0.0; r -= pN / (dz * dz) * (-0.0 + 2.0 * g.cp[3]); }
    const int ii = i - NB, jj = j - NB;
    const int64_t k = (int64_t)jj + (int64_t)ny * ii;
    const bool pin0 = S.pinned && ii == 0 && jj == 0;
    S.diag[k] = aC;
    S.cw[k] = (S.pinned && ii == 1 && jj == 0) ? 0.0 : -aW;
    S.ce[k] = -aE;
    S.cs[k] = (S.pinned && ii == 0 && jj == 1) ? 0.0 : -aS;
    S.cn[k] = -aN;
    S.b[k] = pin0 ? 0.0 : r;
    S.minv[k] = pin0 ? 0.0 : 1.0 / aC;
}

// --------------------------------------------------------------- UpdateDt --
// mac2dAxisym.cpp:2104-2133: maxima of |u_e u_w| / 2, |v_n v_s| / 2 and
// |kappa| (block partials, the last block to finish combines them; max is
// order-independent), then dt = cfl / (C/2 + sqrt(C^2 + 4 G^2 + 4 S^2)/2).
__global__ void k_axi_update_dt(Grid g, MomConst M, const double *__restrict__ u, const double *__restrict__ v,
                                const double *__restrict__ kappa, double *__restrict__ partial,
                                unsigned *__restrict__ counter, double *__restrict__ dt_out) {
    double a[3] = {0.0, 0.0, 0.0};
    const int64_t n = (int64_t)g.nx * g.ny;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int i = NB + (int)(t / g.ny), j = NB + (int)(t % g.ny);
        a[0] = smax(a[0], fabs((u[IX(g, i + 1, j)] * u[IX(g, i, j)]) * 0.5));
        a[1] = smax(a[1], fabs((v[IX(g, i, j + 1)] * v[IX(g, i, j)]) * 0.5));
        a[2] = smax(a[2], fabs(kappa[IX(g, i, j)]));
    }
    __shared__ double sm[3][32];
    __shared__ bool last;
#pragma unroll
    for (int q = 0; q < 3; q++)
        for (int o = 16; o > 0; o >>= 1) a[q] = smax(a[q], __shfl_down_sync(0xffffffffu, a[q], o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0)
        for (int q = 0; q < 3; q++) sm[q][wid] = a[q];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q < 3; q++) {
            double m = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = smax(m, sm[q][w]);
            partial[3 * blockIdx.x + q] = m;
        }
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!(last && threadIdx.x == 0)) return;
    __threadfence();
    double m[3] = {0.0, 0.0, 0.0};
    for (unsigned b = 0; b < gridDim.x; b++)
        for (int q = 0; q < 3; q++) m[q] = smax(m[q], __ldcg(partial + 3 * b + q));
    *counter = 0u;
    const double dr = g.dx, dz = g.dy;
    const double C = m[0] / dr + m[1] / dz;
    const double G = smax(sqrt(fabs(M.g) / dz), sqrt(fabs(M.g) / dr));
    const double h = smin(dr, dz);
    const double Sv = sqrt((M.sigma * m[2]) / (smin(M.rho_h, M.rho_l) * (h * h)));
    double dt = 1.79769313486231570815e+308;
    dt = smin(dt, M.cfl / (0.5 * (C + sqrt(C * C + 4.0 * (G * G) + 4.0 * (Sv * Sv)))));
    *dt_out = dt;
}

}  // namespace

// ------------------------------------------------------------------ host --
void launch_axi_kappa(const Grid &g, const double *ls, double *kappa, cudaStream_t st) {
    const double lim = 1.0 / (g.dy < g.dx ? g.dy : g.dx);
    k_axi_kappa<<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, g.base_x, lim, ls, kappa);
}

static dim3 padded_grid(const Grid &g) { return dim3((g.sy + TJ - 1) / TJ, (g.sx + TI - 1) / TI); }

void launch_axi_rhs_u(const Grid &g, const MomConst &M, const double *ls, const double *u, const double *v,
                      const double *H, const double *cU, const double *dtp, double *out, cudaStream_t st,
                      int visc_only) {
    k_axi_rhs_u<<<padded_grid(g), dim3(TJ, TI), 0, st>>>(g, M, ls, u, v, H, cU, dtp, visc_only, out);
}

void launch_axi_rhs_v(const Grid &g, const MomConst &M, const double *ls, const double *u, const double *uhat,
                      const double *v, const double *H, const double *cV, const double *dtp, double *out,
                      cudaStream_t st, int visc_only) {
    k_axi_rhs_v<<<padded_grid(g), dim3(TJ, TI), 0, st>>>(g, M, ls, u, uhat, v, H, cV, dtp, visc_only, out);
}

// The implicit step of one velocity component into out (zeroed first: only
// its interior faces are written, as in the reference).  w[0..5]: six padded
// scratch arrays (coefficients lo, di, up, the r-line right sides and
// solution, the z-line right sides, the 1/r^2 denominators).
void launch_axi_hat(const Grid &g, const MomConst &M, int comp, const double *ls, const double *rhs,
                    const double *H, const double *dtp, double *out, double *const w[6], cudaStream_t st) {
    double *lo = w[0], *di = w[1], *up = w[2], *dr = w[3], *dz = w[4], *den = w[5];
    const int64_t sx = g.sx, sy = g.sy;
    cudaMemsetAsync(out, 0, sizeof(double) * (size_t)sx * sy, st);
    const dim3 blk(TJ, TI);
    if (comp == 0) {
        const int m = g.nx - 1;
        k_axi_coef_u_r<<<dim3((g.ny + TJ - 1) / TJ, (m + TI - 1) / TI), blk, 0, st>>>(g, M, ls, rhs, H, dtp, lo, di,
                                                                                       up, dr);
        int T = thomas_lines_per_cta(g.ny);
        k_axi_thomas<<<(g.ny + T - 1) / T, T, 0, st>>>(g.ny, m, LineMap{NB + sy * (NB + 1), 1, sy}, lo, di, up, dr,
                                                       LineMap{0, 0, 0}, nullptr, nullptr);
        k_axi_coef_u_z<<<dim3((g.ny + TJ - 1) / TJ, (m + TI - 1) / TI), blk, 0, st>>>(g, M, ls, H, dtp, dr, lo, di,
                                                                                       up, dz, den);
        T = thomas_lines_per_cta(m);
        k_axi_thomas<<<(m + T - 1) / T, T, 0, st>>>(m, g.ny, LineMap{(NB + 1) + sx * NB, 1, sx}, lo, di, up, dz,
                                                    LineMap{NB + sy * (NB + 1), sy, 1}, out, den);
    } else {
        const int m = g.ny - 1;
        k_axi_coef_v_r<<<dim3((m + TJ - 1) / TJ, (g.nx + TI - 1) / TI), blk, 0, st>>>(g, M, ls, rhs, H, dtp, lo, di,
                                                                                        up, dr);
        int T = thomas_lines_per_cta(m);
        k_axi_thomas<<<(m + T - 1) / T, T, 0, st>>>(m, g.nx, LineMap{(NB + 1) + sy * NB, 1, sy}, lo, di, up, dr,
                                                    LineMap{0, 0, 0}, nullptr, nullptr);
        k_axi_coef_v_z<<<dim3((m + TJ - 1) / TJ, (g.nx + TI - 1) / TI), blk, 0, st>>>(g, M, ls, H, dtp, dr, lo, di,
                                                                                        up, dz);
        T = thomas_lines_per_cta(g.nx);
        k_axi_thomas<<<(g.nx + T - 1) / T, T, 0, st>>>(g.nx, m, LineMap{NB + sx * (NB + 1), 1, sx}, lo, di, up, dz,
                                                       LineMap{(NB + 1) + sy * NB, sy, 1}, out, nullptr);
    }
}

void launch_axi_div(const Grid &g, int for_poisson, const double *u, const double *v, double *div, cudaStream_t st) {
    k_axi_div<<<padded_grid(g), dim3(TJ, TI), 0, st>>>(g, g.base_x, for_poisson, u, v, div);
}

void launch_axi_assemble(const Grid &g, const MomConst &M, const double *ls, const double *kappa, const double *H,
                         const double *div, const double *dtp, const Sys &S, cudaStream_t st) {
    k_axi_assemble<<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, M, g.base_x, ls, kappa, H, div, dtp, S);
}

void launch_axi_update_dt(const Grid &g, const MomConst &M, const double *u, const double *v, const double *kappa,
                          double *partial, unsigned *counter, double *dt_out, cudaStream_t st) {
    k_axi_update_dt<<<DT_BLOCKS, 256, 0, st>>>(g, M, u, v, kappa, partial, counter, dt_out);
}

}  // namespace asd2g
