// Level-set stencil kernels templated on the element type T: HJ-WENO5 +
// TVD-RK3 advection (Solve_LevelSet_2D, levelset2d.cpp:43-157) and the
// reinitialisation passes (:264-486, :560-893).  levelset.cu instantiates
// them for double (the bit-exact path, built with -fmad=false), levelset32.cu
// for float (the mixed-precision path).
//
// Each kernel computes final interior values and, when the pressure-grid
// boundary is Neumann/Dirichlet on all sides, also writes the ghost mirrors
// of the cells it owns (p_mirror_store), which is what the reference's
// ApplyBC_P_2D after the loop would produce.  Otherwise the host runs the
// P fill after the kernel.
#pragma once
#include "lsmath.cuh"

namespace asd2g {

// ------------------------------------------------------------------------
// Velocity centring (levelset2d.cpp:50-54).
// The face velocities are FP64 in every precision; the centred values are T.
// Every cell kernel below is a tile function of the TJ x TI tile (bx, by)
// of interior cells (one thread per cell, threadIdx = position in the tile),
// wrapped by a one-grid kernel (tile = blockIdx) and, in batch.cu, by a
// batched kernel over a work list of (instance, tile).
template <typename T>
__device__ __forceinline__ void center_vel_tile(const Grid &g, const double *__restrict__ u,
                                                const double *__restrict__ v, T *__restrict__ tu,
                                                T *__restrict__ tv, int bx, int by) {
    const int j = NB + bx * TJ + threadIdx.x, i = NB + by * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    const T a = T((u[IX(g, i, j)] + u[IX(g, i + 1, j)]) * 0.5);
    const T b = T((v[IX(g, i, j)] + v[IX(g, i, j + 1)]) * 0.5);
    tu[IX(g, i, j)] = a;
    tv[IX(g, i, j)] = b;
    if (g.p_mirror) {
        p_mirror_store(g, tu, i, j, a);
        p_mirror_store(g, tv, i, j, b);
    }
}
template <typename T>
__global__ void k_center_vel(Grid g, const double *__restrict__ u, const double *__restrict__ v, T *__restrict__ tu,
                             T *__restrict__ tv) {
    center_vel_tile<T>(g, u, v, tu, tv, blockIdx.x, blockIdx.y);
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
// dtp is the FP64 dt of the step (rounded to T for T = float).
template <int STAGE, typename T>
__device__ __forceinline__ void ls_stage_tile(const Grid &g, const DivHT<T> &ddx, const DivHT<T> &ddy,
                                              const T *__restrict__ phi_in, const T *__restrict__ tu,
                                              const T *__restrict__ tv, const T *phi_n, T *out,
                                              const double *__restrict__ dtp, int bx, int by) {
    __shared__ T sFx[TI + 2 * NB][TJ];      // rows i0-3 .. i0+TI+2, cols j0 .. j0+TJ-1
    __shared__ T sFy[TI][TJ + 2 * NB + 1];  // rows i0 .. i0+TI-1, cols j0-3 .. j0+TJ+2
    const int j0 = NB + bx * TJ, i0 = NB + by * TI;
    const int tid = threadIdx.y * TJ + threadIdx.x;
    for (int t = tid; t < (TI + 2 * NB) * TJ; t += TJ * TI) {
        const int r = t / TJ, c = t % TJ;
        const int i = i0 - NB + r, j = j0 + c;
        T f = T(0.0);
        if (i < g.sx && j < g.ny + NB) f = phi_in[IX(g, i, j)] * tu[IX(g, i, j)];
        sFx[r][c] = f;
    }
    for (int t = tid; t < TI * (TJ + 2 * NB); t += TJ * TI) {
        const int r = t / (TJ + 2 * NB), c = t % (TJ + 2 * NB);
        const int i = i0 + r, j = j0 - NB + c;
        T f = T(0.0);
        if (i < g.nx + NB && j < g.sy) f = phi_in[IX(g, i, j)] * tv[IX(g, i, j)];
        sFy[r][c] = f;
    }
    __syncthreads();
    const int ti = threadIdx.y, tj = threadIdx.x;
    const int i = i0 + ti, j = j0 + tj;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    T D[6], xp, xm, yp, ym;
#pragma unroll
    for (int k = 0; k < 6; k++) D[k] = sFx[ti + k + 1][tj] - sFx[ti + k][tj];
    weno5_point(D, ddx, xp, xm);
#pragma unroll
    for (int k = 0; k < 6; k++) D[k] = sFy[ti][tj + k + 1] - sFy[ti][tj + k];
    weno5_point(D, ddy, yp, ym);
    const int64_t c = IX(g, i, j);
    const T L = weno_blend(xp, xm, yp, ym, tu[c], tv[c]);
    const T dt = STAGE == 0 ? T(0.0) : T(*dtp);
    T val;
    if (STAGE == 0) val = L;
    else if (STAGE == 1) val = phi_n[c] - dt * L;
    else if (STAGE == 2) val = T(0.75) * phi_n[c] + T(0.25) * phi_in[c] - T(0.25) * dt * L;
    else val = T(1.0 / 3.0) * phi_n[c] + T(2.0 / 3.0) * phi_in[c] - T(2.0 / 3.0) * dt * L;
    out[c] = val;
    if (STAGE != 0 && g.p_mirror) p_mirror_store(g, out, i, j, val);
}
template <int STAGE, typename T>
__global__ void __launch_bounds__(TJ *TI) k_ls_stage(Grid g, DivHT<T> ddx, DivHT<T> ddy, const T *__restrict__ phi_in,
                                                       const T *__restrict__ tu, const T *__restrict__ tv,
                                                       const T *phi_n, T *out, const double *__restrict__ dtp) {
    ls_stage_tile<STAGE, T>(g, ddx, ddy, phi_in, tu, tv, phi_n, out, dtp, blockIdx.x, blockIdx.y);
}

// ------------------------------------------------------------------------
// Reinitialisation passes.  Every pass reads its stencil input from buffers
// other than the one it writes, except for the cell-local reads of `base`,
// so in-place use of `out == base` is safe.
enum { RM_ORIG = 0, RM_SUSS = 1, RM_MINRK2 = 2, RM_FIRST = 3, RM_MINRK2_SUSS = 4 };

template <typename T> __device__ __forceinline__ T reinit_sign(int mode, T l0, T eps) {
    // MinRK2 uses the smoothed sign of phi0 (levelset2d.cpp:445,456); the
    // other modes use sign(phi0) (:284).
    return (mode == RM_MINRK2 || mode == RM_MINRK2_SUSS) ? smoothed_sign(l0, eps) : (T)isgn(l0);
}

// Pass A: out = src - adt * S * (|grad src| - 1)   (LS1 of every mode)
template <int MODE, typename T>
__device__ __forceinline__ void reinit_a_tile(const Grid &g, const LsConstT<T> &K, const T *__restrict__ src,
                                              const T *__restrict__ ls0, T *__restrict__ out, int mirror, int bx,
                                              int by) {
    const int j = NB + bx * TJ + threadIdx.x, i = NB + by * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    constexpr bool SUB = (MODE == RM_MINRK2 || MODE == RM_MINRK2_SUSS);
    const int64_t c = IX(g, i, j);
    const T a = absgrad<SUB>(g, K, src, ls0, i, j);
    const T S = reinit_sign(MODE, ls0[c], K.eps);
    T val;
    if (SUB) val = src[c] - K.adt * S * (a - T(1.0));
    else val = src[c] - K.adt * (T)isgn(ls0[c]) * (a - T(1.0));
    out[c] = val;
    if (mirror) p_mirror_store(g, out, i, j, val);
}
template <int MODE, typename T>
__global__ void k_reinit_a(Grid g, LsConstT<T> K, const T *__restrict__ src, const T *__restrict__ ls0,
                           T *__restrict__ out, int mirror) {
    reinit_a_tile<MODE, T>(g, K, src, ls0, out, mirror, blockIdx.x, blockIdx.y);
}

// Pass B: LS2 = step_base - adt * S * (|grad ls1| - 1); out = 0.5 * (base + LS2)
// step_base is ls1 itself except for the first-time mode, which steps from
// phi again (levelset2d.cpp:413-416).
template <int MODE, typename T>
__device__ __forceinline__ void reinit_b_tile(const Grid &g, const LsConstT<T> &K, const T *__restrict__ ls1,
                                              const T *__restrict__ ls0, const T *base, T *out, int mirror, int bx,
                                              int by) {
    const int j = NB + bx * TJ + threadIdx.x, i = NB + by * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    constexpr bool SUB = (MODE == RM_MINRK2 || MODE == RM_MINRK2_SUSS);
    const int64_t c = IX(g, i, j);
    const T a = absgrad<SUB>(g, K, ls1, ls0, i, j);
    const T b = base[c];
    T ls2;
    if (SUB) ls2 = ls1[c] - K.adt * reinit_sign(MODE, ls0[c], K.eps) * (a - T(1.0));
    else if (MODE == RM_FIRST) ls2 = b - K.adt * (T)isgn(ls0[c]) * (a - T(1.0));
    else ls2 = ls1[c] - K.adt * (T)isgn(ls0[c]) * (a - T(1.0));
    const T val = T(0.5) * (b + ls2);
    out[c] = val;
    if (mirror) p_mirror_store(g, out, i, j, val);
}
template <int MODE, typename T>
__global__ void k_reinit_b(Grid g, LsConstT<T> K, const T *__restrict__ ls1, const T *__restrict__ ls0, const T *base,
                           T *out, int mirror) {
    reinit_b_tile<MODE, T>(g, K, ls1, ls0, base, out, mirror, blockIdx.x, blockIdx.y);
}

// Pass C (Sussman constraint, :787-893): out = base + constraint(tmp, ls0)
// with hd = UpdateHeavisideFuncDeriv(tmp).  Sussman mode: base = phi
// (levelset2d.cpp:368-372); MinRK2+Sussman: base = tmp.
template <typename T>
__device__ __forceinline__ void reinit_c_tile(const Grid &g, const LsConstT<T> &K, const T *__restrict__ tmp,
                                              const T *__restrict__ ls0, const T *base, T *out, int mirror, int bx,
                                              int by) {
    const int j = NB + bx * TJ + threadIdx.x, i = NB + by * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    const int64_t c = IX(g, i, j);
    const T hd = heaviside_deriv(tmp[c], K.eps);
    const T val = base[c] + sussman_constraint(g, K, tmp, ls0, hd, i, j);
    out[c] = val;
    if (mirror) p_mirror_store(g, out, i, j, val);
}
template <typename T>
__global__ void k_reinit_c(Grid g, LsConstT<T> K, const T *__restrict__ tmp, const T *__restrict__ ls0, const T *base,
                           T *out, int mirror) {
    reinit_c_tile<T>(g, K, tmp, ls0, base, out, mirror, blockIdx.x, blockIdx.y);
}


// Step and grid constants of the reinitialisation in precision T.
template <typename T> LsConstT<T> make_lsconst_t(const Grid &g);

}  // namespace asd2g
