// Level-set kernels: HJ-WENO5 + TVD-RK3 advection (Solve_LevelSet_2D,
// levelset2d.cpp:43-157) and the reinitialisation passes (:264-486, :560-893).
//
// Each kernel computes final interior values and, when the pressure-grid
// boundary is Neumann/Dirichlet on all sides, also writes the ghost mirrors
// of the cells it owns (p_mirror_store), which is what the reference's
// ApplyBC_P_2D after the loop would produce.  Otherwise the host runs the
// P fill after the kernel.
#include "lsmath.cuh"

namespace asd2g {

// ------------------------------------------------------------------------
// Velocity centring (levelset2d.cpp:50-54).
__global__ void k_center_vel(Grid g, const double *__restrict__ u, const double *__restrict__ v,
                             double *__restrict__ tu, double *__restrict__ tv) {
    const int j = NB + blockIdx.x * TJ + threadIdx.x, i = NB + blockIdx.y * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    const double a = (u[IX(g, i, j)] + u[IX(g, i + 1, j)]) * 0.5;
    const double b = (v[IX(g, i, j)] + v[IX(g, i, j + 1)]) * 0.5;
    tu[IX(g, i, j)] = a;
    tv[IX(g, i, j)] = b;
    if (g.p_mirror) {
        p_mirror_store(g, tu, i, j, a);
        p_mirror_store(g, tv, i, j, b);
    }
}

// ------------------------------------------------------------------------
// One TVD-RK3 stage.  L = HJWENO5_LS_2D(phi_in, tu, tv) at each interior
// cell, then
//   STAGE 1: out = phi_n - dt L                                      (:68)
//   STAGE 2: out = 0.75 phi_n + 0.25 phi_in - 0.25 dt L              (:75)
//   STAGE 3: out = 1/3 phi_n + 2/3 phi_in - 2/3 dt L                 (:82)
//   STAGE 0: out = L (HJWENO5_LS_2D itself)
// The fluxes F = phi*u (x) and phi*v (y) of a 8 x 32 cell tile plus its
// three-cell halo along each axis are staged in shared memory; every cell
// then differences its own 7-point windows, so each interior value is
// computed exactly as the reference's per-row/per-column sweep computes it.
// out may alias phi_n (stage 3 writes phi in place): each thread reads
// phi_n only at its own cell before writing it.
template <int STAGE>
__global__ void __launch_bounds__(TJ *TI) k_ls_stage(Grid g, DivH ddx, DivH ddy, const double *__restrict__ phi_in,
                                                       const double *__restrict__ tu, const double *__restrict__ tv,
                                                       const double *phi_n, double *out,
                                                       const double *__restrict__ dtp) {
    __shared__ double sFx[TI + 2 * NB][TJ];      // rows i0-3 .. i0+TI+2, cols j0 .. j0+TJ-1
    __shared__ double sFy[TI][TJ + 2 * NB + 1];  // rows i0 .. i0+TI-1, cols j0-3 .. j0+TJ+2
    const int j0 = NB + blockIdx.x * TJ, i0 = NB + blockIdx.y * TI;
    const int tid = threadIdx.y * TJ + threadIdx.x;
    for (int t = tid; t < (TI + 2 * NB) * TJ; t += TJ * TI) {
        const int r = t / TJ, c = t % TJ;
        const int i = i0 - NB + r, j = j0 + c;
        double f = 0.0;
        if (i < g.sx && j < g.ny + NB) f = phi_in[IX(g, i, j)] * tu[IX(g, i, j)];
        sFx[r][c] = f;
    }
    for (int t = tid; t < TI * (TJ + 2 * NB); t += TJ * TI) {
        const int r = t / (TJ + 2 * NB), c = t % (TJ + 2 * NB);
        const int i = i0 + r, j = j0 - NB + c;
        double f = 0.0;
        if (i < g.nx + NB && j < g.sy) f = phi_in[IX(g, i, j)] * tv[IX(g, i, j)];
        sFy[r][c] = f;
    }
    __syncthreads();
    const int ti = threadIdx.y, tj = threadIdx.x;
    const int i = i0 + ti, j = j0 + tj;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    double D[6], xp, xm, yp, ym;
#pragma unroll
    for (int k = 0; k < 6; k++) D[k] = sFx[ti + k + 1][tj] - sFx[ti + k][tj];
    weno5_point(D, ddx, xp, xm);
#pragma unroll
    for (int k = 0; k < 6; k++) D[k] = sFy[ti][tj + k + 1] - sFy[ti][tj + k];
    weno5_point(D, ddy, yp, ym);
    const int64_t c = IX(g, i, j);
    const double L = weno_blend(xp, xm, yp, ym, tu[c], tv[c]);
    const double dt = STAGE == 0 ? 0.0 : *dtp;
    double val;
    if (STAGE == 0) val = L;
    else if (STAGE == 1) val = phi_n[c] - dt * L;
    else if (STAGE == 2) val = 0.75 * phi_n[c] + 0.25 * phi_in[c] - 0.25 * dt * L;
    else val = 1.0 / 3.0 * phi_n[c] + 2.0 / 3.0 * phi_in[c] - 2.0 / 3.0 * dt * L;
    out[c] = val;
    if (STAGE != 0 && g.p_mirror) p_mirror_store(g, out, i, j, val);
}

// ------------------------------------------------------------------------
// Reinitialisation passes.  Every pass reads its stencil input from buffers
// other than the one it writes, except for the cell-local reads of `base`,
// so in-place use of `out == base` is safe.
enum { RM_ORIG = 0, RM_SUSS = 1, RM_MINRK2 = 2, RM_FIRST = 3, RM_MINRK2_SUSS = 4 };

__device__ __forceinline__ double reinit_sign(int mode, double l0, double eps) {
    // MinRK2 uses the smoothed sign of phi0 (levelset2d.cpp:445,456); the
    // other modes use sign(phi0) (:284).
    return (mode == RM_MINRK2 || mode == RM_MINRK2_SUSS) ? smoothed_sign(l0, eps) : (double)isgn(l0);
}

// Pass A: out = src - adt * S * (|grad src| - 1)   (LS1 of every mode)
template <int MODE>
__global__ void k_reinit_a(Grid g, LsConst K, const double *__restrict__ src, const double *__restrict__ ls0,
                           double *__restrict__ out, int mirror) {
    const int j = NB + blockIdx.x * TJ + threadIdx.x, i = NB + blockIdx.y * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    constexpr bool SUB = (MODE == RM_MINRK2 || MODE == RM_MINRK2_SUSS);
    const int64_t c = IX(g, i, j);
    const double a = absgrad<SUB>(g, K, src, ls0, i, j);
    const double S = reinit_sign(MODE, ls0[c], K.eps);
    double val;
    if (SUB) val = src[c] - K.adt * S * (a - 1.0);
    else val = src[c] - K.adt * (double)isgn(ls0[c]) * (a - 1.0);
    out[c] = val;
    if (mirror) p_mirror_store(g, out, i, j, val);
}

// Pass B: LS2 = step_base - adt * S * (|grad ls1| - 1); out = 0.5 * (base + LS2)
// step_base is ls1 itself except for the first-time mode, which steps from
// phi again (levelset2d.cpp:413-416).
template <int MODE>
__global__ void k_reinit_b(Grid g, LsConst K, const double *__restrict__ ls1, const double *__restrict__ ls0,
                           const double *base, double *out, int mirror) {
    const int j = NB + blockIdx.x * TJ + threadIdx.x, i = NB + blockIdx.y * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    constexpr bool SUB = (MODE == RM_MINRK2 || MODE == RM_MINRK2_SUSS);
    const int64_t c = IX(g, i, j);
    const double a = absgrad<SUB>(g, K, ls1, ls0, i, j);
    const double b = base[c];
    double ls2;
    if (SUB) ls2 = ls1[c] - K.adt * reinit_sign(MODE, ls0[c], K.eps) * (a - 1.0);
    else if (MODE == RM_FIRST) ls2 = b - K.adt * (double)isgn(ls0[c]) * (a - 1.0);
    else ls2 = ls1[c] - K.adt * (double)isgn(ls0[c]) * (a - 1.0);
    const double val = 0.5 * (b + ls2);
    out[c] = val;
    if (mirror) p_mirror_store(g, out, i, j, val);
}

// Pass C (Sussman constraint, :787-893): out = base + constraint(tmp, ls0)
// with hd = UpdateHeavisideFuncDeriv(tmp).  Sussman mode: base = phi
// (levelset2d.cpp:368-372); MinRK2+Sussman: base = tmp.
__global__ void k_reinit_c(Grid g, LsConst K, const double *__restrict__ tmp, const double *__restrict__ ls0,
                           const double *base, double *out, int mirror) {
    const int j = NB + blockIdx.x * TJ + threadIdx.x, i = NB + blockIdx.y * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    const int64_t c = IX(g, i, j);
    const double hd = heaviside_deriv(tmp[c], K.eps);
    const double val = base[c] + sussman_constraint(g, K, tmp, ls0, hd, i, j);
    out[c] = val;
    if (mirror) p_mirror_store(g, out, i, j, val);
}

// First-time mode normalisation (levelset2d.cpp:388-395): phi0 / |grad phi0|
// where positive, written to a separate buffer.
__global__ void k_reinit_normalize(Grid g, LsConst K, const double *__restrict__ ls0, double *__restrict__ out) {
    const int j = NB + blockIdx.x * TJ + threadIdx.x, i = NB + blockIdx.y * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    const int64_t c = IX(g, i, j);
    const double a = absgrad<false>(g, K, ls0, ls0, i, j);
    const double v = a > 0.0 ? ls0[c] / a : ls0[c];
    out[c] = v;
    if (g.p_mirror) p_mirror_store(g, out, i, j, v);
}

// ------------------------------------------------------------------------
// Building blocks with fresh-vector semantics (interior written; the caller
// zeroes the array first).
template <bool SUB>
__global__ void k_absgrad(Grid g, LsConst K, const double *__restrict__ ls, const double *__restrict__ ls0,
                          double *__restrict__ out) {
    const int j = NB + blockIdx.x * TJ + threadIdx.x, i = NB + blockIdx.y * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    out[IX(g, i, j)] = absgrad<SUB>(g, K, ls, ls0, i, j);
}

__global__ void k_sussman_only(Grid g, LsConst K, const double *__restrict__ ls, const double *__restrict__ ls0,
                               const double *__restrict__ hd, double *__restrict__ out) {
    const int j = NB + blockIdx.x * TJ + threadIdx.x, i = NB + blockIdx.y * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    out[IX(g, i, j)] = sussman_constraint(g, K, ls, ls0, hd[IX(g, i, j)], i, j);
}

// Whole-array maps: 0 = heaviside derivative, 1 = smoothed sign.
__global__ void k_pointwise_ls(int64_t n, int which, double eps, const double *__restrict__ a, double *__restrict__ out) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        out[k] = which == 0 ? heaviside_deriv(a[k], eps) : smoothed_sign(a[k], eps);
}

// ------------------------------------------------------------------------
// UnitHJWENO5 on one line F[0 .. n+5] (levelset2d.cpp:159-262): FP, FM at
// points 3 .. n+2.
__global__ void k_weno_line(const double *__restrict__ F, double *__restrict__ FP, double *__restrict__ FM, DivH dv,
                            int n) {
    const int i = NB + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n + NB) return;
    double D[6], fp, fm;
#pragma unroll
    for (int k = 0; k < 6; k++) D[k] = F[i - 2 + k] - F[i - 3 + k];
    weno5_point(D, dv, fp, fm);
    FP[i] = fp;
    FM[i] = fm;
}

// HJWENO5_DerivAbsLS_2D (levelset2d.cpp:488-558): WENO5 one-sided derivatives
// of phi itself along each line, Godunov |grad phi| with the sign of phi0.
__global__ void k_weno_absgrad(Grid g, DivH ddx, DivH ddy, const double *__restrict__ ls,
                               const double *__restrict__ ls0, double *__restrict__ out) {
    const int j = NB + blockIdx.x * TJ + threadIdx.x, i = NB + blockIdx.y * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    double D[6], pX, mX, pY, mY;
#pragma unroll
    for (int k = 0; k < 6; k++) D[k] = ls[IX(g, i - 2 + k, j)] - ls[IX(g, i - 3 + k, j)];
    weno5_point(D, ddx, pX, mX);
#pragma unroll
    for (int k = 0; k < 6; k++) D[k] = ls[IX(g, i, j - 2 + k)] - ls[IX(g, i, j - 3 + k)];
    weno5_point(D, ddy, pY, mY);
    out[IX(g, i, j)] = godunov(ls0[IX(g, i, j)], pX, mX, pY, mY);
}

// ------------------------------------------------------------------------
// Host launchers
LsConst make_lsconst(const Grid &g) {
    LsConst K;
    K.ddx = make_divh(g.dx);
    K.ddy = make_divh(g.dy);
    K.ddx2 = make_divh(g.dx * g.dx);
    K.ddy2 = make_divh(g.dy * g.dy);
    K.dx = g.dx;
    K.dy = g.dy;
    K.eps = g.dx < g.dy ? g.dx : g.dy;  // kEps = min(dx, dy), levelset2d.cpp:4
    K.thick = 1.5 * K.eps;
    K.adt = K.eps * 0.5;
    return K;
}

void launch_center_vel(const Grid &g, const double *u, const double *v, double *tu, double *tv, cudaStream_t st) {
    k_center_vel<<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, u, v, tu, tv);
    if (!g.p_mirror) {
        launch_fill_p(g, tu, st);
        launch_fill_p(g, tv, st);
    }
}

void launch_ls_stage(int stage, const Grid &g, const double *phi_in, const double *tu, const double *tv,
                     const double *phi_n, double *out, const double *dt, cudaStream_t st) {
    const DivH ddx = make_divh(g.dx), ddy = make_divh(g.dy);
    const dim3 grd = cell_grid(g), blk(TJ, TI);
    switch (stage) {
    case 0: k_ls_stage<0><<<grd, blk, 0, st>>>(g, ddx, ddy, phi_in, tu, tv, phi_n, out, dt); break;
    case 1: k_ls_stage<1><<<grd, blk, 0, st>>>(g, ddx, ddy, phi_in, tu, tv, phi_n, out, dt); break;
    case 2: k_ls_stage<2><<<grd, blk, 0, st>>>(g, ddx, ddy, phi_in, tu, tv, phi_n, out, dt); break;
    default: k_ls_stage<3><<<grd, blk, 0, st>>>(g, ddx, ddy, phi_in, tu, tv, phi_n, out, dt); break;
    }
    if (stage != 0 && !g.p_mirror) launch_fill_p(g, out, st);
}

template <int MODE>
static void reinit_a(const Grid &g, const LsConst &K, const double *src, const double *ls0, double *out, bool bc,
                     cudaStream_t st) {
    k_reinit_a<MODE><<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, K, src, ls0, out, bc && g.p_mirror);
    if (bc && !g.p_mirror) launch_fill_p(g, out, st);
}
template <int MODE>
static void reinit_b(const Grid &g, const LsConst &K, const double *ls1, const double *ls0, const double *base,
                     double *out, bool bc, cudaStream_t st) {
    k_reinit_b<MODE><<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, K, ls1, ls0, base, out, bc && g.p_mirror);
    if (bc && !g.p_mirror) launch_fill_p(g, out, st);
}
static void reinit_c(const Grid &g, const LsConst &K, const double *tmp, const double *ls0, const double *base,
                     double *out, cudaStream_t st) {
    k_reinit_c<<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, K, tmp, ls0, base, out, g.p_mirror);
    if (!g.p_mirror) launch_fill_p(g, out, st);
}

// Number of pseudo steps of `while (m_atime < max) m_atime += kAdt;`.
int reinit_steps(double adt, double max_atime) {
    double t = 0.0;
    int n = 0;
    while (t < max_atime) {
        t += adt;
        n++;
    }
    return n;
}

// Full reinitialisation of ls in place.  w1, w2, w3 are padded work arrays
// whose ghost cells must be zero on entry for the Sussman mode (the
// reference's LS1/LS2/tmpLS are fresh zero vectors, and Sussman mode never
// fills LS1's ghosts).  ls0 receives lsInit.
void launch_reinit(const Grid &g, int mode, double max_atime, double *ls, double *ls0, double *w1, double *w2,
                   double *w3, cudaStream_t st) {
    const LsConst K = make_lsconst(g);
    const size_t bytes = sizeof(double) * (size_t)g.sx * g.sy;
    if (mode == RM_FIRST) {
        // levelset2d.cpp:377-431
        cudaMemcpyAsync(ls0, ls, bytes, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(w3, ls, bytes, cudaMemcpyDeviceToDevice, st);
        k_reinit_normalize<<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, K, ls0, w3);
        if (!g.p_mirror) launch_fill_p(g, w3, st);
        cudaMemcpyAsync(ls0, w3, bytes, cudaMemcpyDeviceToDevice, st);
        const double lx = g.dx * g.nx, ly = g.dy * g.ny;
        const int steps = reinit_steps(K.adt, lx > ly ? lx : ly);
        launch_fill_p(g, ls, st);
        for (int s = 0; s < steps; s++) {
            reinit_a<RM_FIRST>(g, K, ls, ls0, w1, true, st);
            reinit_b<RM_FIRST>(g, K, w1, ls0, ls, ls, true, st);
        }
        launch_fill_p(g, ls, st);
        return;
    }
    const double mt = max_atime > 0.0 ? max_atime : 1.5 * K.thick;  // kMaxATime, levelset2d.cpp:10
    const int steps = reinit_steps(K.adt, mt);
    if (mode == RM_MINRK2 || mode == RM_MINRK2_SUSS) {
        launch_fill_p(g, ls, st);  // ApplyBC_P_2D(ls) before lsInit = ls (:435-438)
        cudaMemcpyAsync(ls0, ls, bytes, cudaMemcpyDeviceToDevice, st);
    } else {
        // Original and Sussman copy lsInit first (:267-268, :325-326), then
        // fill ls at the top of the loop.
        cudaMemcpyAsync(ls0, ls, bytes, cudaMemcpyDeviceToDevice, st);
        launch_fill_p(g, ls, st);
    }
    if (mode == RM_SUSS) {
        cudaMemsetAsync(w1, 0, bytes, st);
        cudaMemsetAsync(w3, 0, bytes, st);
    } else if (mode == RM_MINRK2_SUSS) {
        cudaMemsetAsync(w3, 0, bytes, st);
    }
    for (int s = 0; s < steps; s++) {
        switch (mode) {
        case RM_ORIG:
            reinit_a<RM_ORIG>(g, K, ls, ls0, w1, true, st);
            reinit_b<RM_ORIG>(g, K, w1, ls0, ls, ls, true, st);
            break;
        case RM_SUSS:
            // LS1 without ghost fill; tmpLS with fill; ls += constraint.
            reinit_a<RM_SUSS>(g, K, ls, ls0, w1, false, st);
            reinit_b<RM_SUSS>(g, K, w1, ls0, ls, w3, true, st);
            reinit_c(g, K, w3, ls0, ls, ls, st);
            break;
        case RM_MINRK2:
            reinit_a<RM_MINRK2>(g, K, ls, ls0, w1, true, st);
            reinit_b<RM_MINRK2>(g, K, w1, ls0, ls, ls, true, st);
            break;
        default:  // RM_MINRK2_SUSS
            reinit_a<RM_MINRK2_SUSS>(g, K, ls, ls0, w1, true, st);
            reinit_b<RM_MINRK2_SUSS>(g, K, w1, ls0, ls, w3, true, st);
            reinit_c(g, K, w3, ls0, w3, ls, st);
            break;
        }
    }
    if (!g.p_mirror) launch_fill_p(g, ls, st);
    (void)w2;
}

void launch_absgrad(const Grid &g, bool sub, const double *ls, const double *ls0, double *out, cudaStream_t st) {
    const LsConst K = make_lsconst(g);
    cudaMemsetAsync(out, 0, sizeof(double) * (size_t)g.sx * g.sy, st);
    if (sub) k_absgrad<true><<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, K, ls, ls0, out);
    else k_absgrad<false><<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, K, ls, ls0, out);
}

void launch_sussman_only(const Grid &g, const double *ls, const double *ls0, const double *hd, double *out,
                         cudaStream_t st) {
    const LsConst K = make_lsconst(g);
    cudaMemsetAsync(out, 0, sizeof(double) * (size_t)g.sx * g.sy, st);
    k_sussman_only<<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, K, ls, ls0, hd, out);
}

void launch_weno_line(const double *F, double *FP, double *FM, double d, int n, cudaStream_t st) {
    k_weno_line<<<(n + 127) / 128, 128, 0, st>>>(F, FP, FM, make_divh(d), n);
}

void launch_weno_absgrad(const Grid &g, const double *ls, const double *ls0, double *out, cudaStream_t st) {
    cudaMemsetAsync(out, 0, sizeof(double) * (size_t)g.sx * g.sy, st);
    k_weno_absgrad<<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, make_divh(g.dx), make_divh(g.dy), ls, ls0, out);
}

void launch_pointwise_ls(const Grid &g, int which, const double *a, double *out, cudaStream_t st) {
    const int64_t n = (int64_t)g.sx * g.sy;
    const double eps = g.dx < g.dy ? g.dx : g.dy;
    k_pointwise_ls<<<(int)((n + 255) / 256), 256, 0, st>>>(n, which, eps, a, out);
}

}  // namespace asd2g
