// Reinitialisation pseudo-steps of the mixed-precision level-set step, FP32
// (Reinit_Original_2D / Reinit_MinRK2_2D with ENO_DerivAbsLS_2D /
// SubcellENO_Min_DerivAbsLS_2D, the smoothed sign and the Sussman constraint:
// levelset2d.cpp:264-316, :433-486, :560-711, :787-923).
//
// One pseudo-step is the reference's: LS1 = phi - adt S (|grad phi| - 1),
// LS2 = LS1 - adt S (|grad LS1| - 1), tmp = (phi + LS2) / 2, and in the
// MinRK2 + Sussman mode phi = tmp + the constraint.  Like the FP32 advection
// stage (weno32.cu) the passes are organised for instruction count:
//
//  * Pass A/B kernel: a lane owns the 2 x 2 cells (i, i+1) x (j, j+32).
//    Along x (a column pair, packed FP32x2) it slides down its rows with the
//    values, second differences and their minmods in registers: minmod(dd_k,
//    dd_{k+1}) serves dP at k and dM at k+1.  Along y (a row pair, packed)
//    the pair's phi and phi0 rows pass through a per-warp shared-memory row.
//    The Min-Gibou subcell fix runs only where phi0 changes sign between
//    neighbours, out of line.  Sign: phi0 * rsqrt(phi0^2 + eps^2).
//  * Sussman constraint only where it is nonzero.  It is nonzero only where
//    |tmp| <= eps (the Heaviside derivative of tmp vanishes elsewhere), a band
//    of a few cells around the interface.  Pass B writes tmp over phi and
//    appends the band cells to a list; one kernel evaluates the constraint at
//    the listed cells from tmp (read only), a second writes tmp + constraint
//    back.  Corner ghost cells of tmp read as 0, as the reference's tmpLS
//    corners are never written.
#include "levelset_impl.cuh"
#include "ls32.cuh"

namespace asd2g {
namespace {

constexpr int R32_WARPS = 4;
constexpr int R32_COLS = 64;

__device__ __forceinline__ float2 p2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 mm2(float2 a, float2 b) { return make_float2(minmod(a.x, b.x), minmod(a.y, b.y)); }
// (l_{k-1} - 2 l_k + l_{k+1}) / h^2
__device__ __forceinline__ float2 dd2(float2 lm, float2 l0, float2 lp, float2 inv2) {
    return mul2(fma2(p2(-2.f), l0, add2(lm, lp)), inv2);
}

struct Pass32Const {
    LsConstT<float> K;
    float2 invx, invy, invx2, invy2, hhx, hhy;  // 1/h, 1/h^2, h/2 (both lanes)
    float eps2;
};

// The subcell branches run at a few cells per row near the interface; out of
// line they keep the unrolled pass small enough for the instruction cache.
__device__ __noinline__ float subcell_plus32(float h, DivHT<float> dh, DivHT<float> dh2, float c, float a, float b,
                                             float cc, float d) {
    return subcell_plus(h, dh, dh2, c, a, b, cc, d);
}
__device__ __noinline__ float subcell_minus32(float h, DivHT<float> dh, DivHT<float> dh2, float c, float a, float b,
                                              float cc, float d) {
    return subcell_minus(h, dh, dh2, c, a, b, cc, d);
}

template <int MODE>
__device__ __forceinline__ float sign32(float l0, float eps2) {
    if (MODE == RM_MINRK2 || MODE == RM_MINRK2_SUSS) return l0 * rsqrtf(fmaf(l0, l0, eps2));
    return (float)isgn(l0);
}

// Pass A (PB = false): out = src - adt S (|grad src| - 1).
// Pass B (PB = true):  out = (base + src - adt S (|grad src| - 1)) / 2; in the
// Sussman mode the cells with |out| <= eps are appended to band / band_n.
// Pass A also clears band_n for the pass B that follows.
template <int MODE, bool PB, int R>
__global__ void __launch_bounds__(32 * R32_WARPS, 4)
    k_reinit32(Grid g, Pass32Const C, const float *__restrict__ src, const float *__restrict__ ls0, const float *base,
               float *out, int *__restrict__ band, unsigned *__restrict__ band_n) {
    constexpr bool SUB = (MODE == RM_MINRK2 || MODE == RM_MINRK2_SUSS);
    constexpr bool BAND = PB && MODE == RM_MINRK2_SUSS;
    __shared__ float2 sS[R32_WARPS][R32_COLS + 4];  // src of rows (i, i+1) at column j0-2+k
    __shared__ float2 sZ[R32_WARPS][R32_COLS + 4];  // phi0 of rows (i, i+1)
    if (!PB && MODE == RM_MINRK2_SUSS && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *band_n = 0u;
    const LsConstT<float> &K = C.K;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int sx = g.sx, sy = g.sy;
    const int ib = NB + (blockIdx.y * R32_WARPS + w) * R;
    if (ib >= g.nx + NB) return;  // whole warp
    const int ie = min(ib + R, g.nx + NB);
    const int j0 = NB + blockIdx.x * R32_COLS;
    const int cA = j0 + lane, cB = cA + 32;
    const bool inA = cA < sy, inB = cB < sy;
    float2 *ss = sS[w], *sz = sZ[w];
    const bool edge = blockIdx.x == 0 || j0 + R32_COLS > g.ny || ib < 2 * NB || ie > g.nx;

    auto ld = [&](const float *a, int i, int c, bool in) -> float {
        return (in && i < sx) ? __ldg(a + (int64_t)i * sy + c) : 0.f;
    };
    auto pr = [&](const float *a, int i) -> float2 { return make_float2(ld(a, i, cA, inA), ld(a, i, cB, inB)); };

    // x window: src rows i, i+1; dd_i; minmod_{i-1}; D_{i-1}; phi0 rows i-1, i
    float2 l0, l1, ddc, mmp, Dp, z0, z1;
    {
        const float2 a = pr(src, ib - 2), b = pr(src, ib - 1);
        l0 = pr(src, ib);
        l1 = pr(src, ib + 1);
        const float2 ddm = dd2(a, b, l0, C.invx2);
        ddc = dd2(b, l0, l1, C.invx2);
        mmp = mm2(ddm, ddc);
        Dp = sub2(l0, b);
        z0 = pr(ls0, ib - 1);
        z1 = pr(ls0, ib);
    }

#pragma unroll 1
    for (int k = 0; k < R / 2; k++) {
        const int i = ib + 2 * k;
        if (i >= ie) break;
        // rows i+2, i+3 enter the window; (z0, z1, z2, z3) = phi0 rows i-1 .. i+2
        const float2 l2 = pr(src, i + 2), l3 = pr(src, i + 3);
        const float2 z2 = pr(ls0, i + 1), z3 = pr(ls0, i + 2);
        const float2 dd1 = dd2(l0, l1, l2, C.invx2), dd2v = dd2(l1, l2, l3, C.invx2);
        const float2 mm0 = mm2(ddc, dd1), mm1 = mm2(dd1, dd2v);
        const float2 D0 = sub2(l1, l0), D1 = sub2(l2, l1);
        // x derivatives of rows i (r = 0) and i+1 (r = 1), columns (cA, cB)
        float2 dPX[2], dMX[2];
        dPX[0] = fma2(p2(-1.f), mul2(C.hhx, mm0), mul2(D0, C.invx));
        dMX[0] = fma2(C.hhx, mmp, mul2(Dp, C.invx));
        dPX[1] = fma2(p2(-1.f), mul2(C.hhx, mm1), mul2(D1, C.invx));
        dMX[1] = fma2(C.hhx, mm0, mul2(D0, C.invx));

        // y: the row pair's src and phi0 through shared memory
        ss[lane + 2] = make_float2(l0.x, l1.x);
        ss[lane + 34] = make_float2(l0.y, l1.y);
        sz[lane + 2] = make_float2(z1.x, z2.x);
        sz[lane + 34] = make_float2(z1.y, z2.y);
        if (lane < 4) {  // halo columns j0-2, j0-1, j0+64, j0+65
            const int hc = lane < 2 ? j0 - 2 + lane : j0 + 62 + lane;
            const bool hin = hc < sy;
            const int hk = lane < 2 ? lane : lane + 64;
            ss[hk] = make_float2(ld(src, i, hc, hin), ld(src, i + 1, hc, hin));
            sz[hk] = make_float2(ld(ls0, i, hc, hin), ld(ls0, i + 1, hc, hin));
        }
        __syncwarp();
        float2 dPY[2], dMY[2], zm[2], zp[2];
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int b = lane + 32 * c + 2;
            const float2 a0 = ss[b - 2], a1 = ss[b - 1], a2 = ss[b], a3 = ss[b + 1], a4 = ss[b + 2];
            const float2 e0 = dd2(a0, a1, a2, C.invy2), e1 = dd2(a1, a2, a3, C.invy2), e2 = dd2(a2, a3, a4, C.invy2);
            const float2 n0 = mm2(e0, e1), n1 = mm2(e1, e2);
            dPY[c] = fma2(p2(-1.f), mul2(C.hhy, n1), mul2(sub2(a3, a2), C.invy));
            dMY[c] = fma2(C.hhy, n0, mul2(sub2(a2, a1), C.invy));
            zm[c] = sz[b - 1];
            zp[c] = sz[b + 1];
        }

        float val[2][2];
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const float2 zc = r ? z2 : z1, zu = r ? z1 : z0, zd = r ? z3 : z2;  // phi0 at rows i+r, i+r-1, i+r+1
            const float2 lc = r ? l1 : l0;
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const int row = i + r, col = c ? cB : cA;
                const bool cin = c ? inB : inA;
                const float x0 = c ? zc.y : zc.x;
                const float cval = c ? lc.y : lc.x;
                float dpx = c ? dPX[r].y : dPX[r].x, dmx = c ? dMX[r].y : dMX[r].x;
                float dpy = r ? dPY[c].y : dPY[c].x, dmy = r ? dMY[c].y : dMY[c].x;
                if (SUB) {
                    const float xm1 = c ? zu.y : zu.x, xp1 = c ? zd.y : zd.x;
                    const float ym1 = r ? zm[c].y : zm[c].x, yp1 = r ? zp[c].y : zp[c].x;
                    if (x0 * xp1 < 0.f)
                        dpx = subcell_plus32(K.dx, K.ddx, K.ddx2, cval, xm1, x0, xp1, ld(ls0, row + 2, col, cin));
                    if (x0 * xm1 < 0.f)
                        dmx = subcell_minus32(K.dx, K.ddx, K.ddx2, cval, ld(ls0, row - 2, col, cin), xm1, x0, xp1);
                    if (x0 * yp1 < 0.f) {
                        const float2 q = sz[lane + 32 * c + 4];
                        dpy = subcell_plus32(K.dy, K.ddy, K.ddy2, cval, ym1, x0, yp1, r ? q.y : q.x);
                    }
                    if (x0 * ym1 < 0.f) {
                        const float2 q = sz[lane + 32 * c];
                        dmy = subcell_minus32(K.dy, K.ddy, K.ddy2, cval, r ? q.y : q.x, ym1, x0, yp1);
                    }
                }
                const float a = godunov(x0, dpx, dmx, dpy, dmy);
                const float upd = cval - K.adt * sign32<MODE>(x0, C.eps2) * (a - 1.f);
                if (PB) {
                    const bool ok = row < ie && col < g.ny + NB;
                    const float bv = ok ? base[(int64_t)row * sy + col] : 0.f;
                    val[r][c] = 0.5f * (bv + upd);
                } else {
                    val[r][c] = upd;
                }
            }
        }
        __syncwarp();  // shared rows are rewritten by the next iteration
#pragma unroll
        for (int r = 0; r < 2; r++) {
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const int row = i + r, col = c ? cB : cA;
                const bool ok = row < ie && col < g.ny + NB;
                if (ok) {
                    out[(int64_t)row * sy + col] = val[r][c];
                    if (edge) p_mirror_store(g, out, row, col, val[r][c]);
                }
                if (BAND) {
                    const bool in_band = ok && !(fabsf(val[r][c]) > K.eps);
                    const unsigned m = __ballot_sync(0xffffffffu, in_band);
                    if (m) {
                        unsigned b0 = 0;
                        if (lane == 0) b0 = atomicAdd(band_n, (unsigned)__popc(m));
                        b0 = __shfl_sync(0xffffffffu, b0, 0);
                        if (in_band) band[b0 + __popc(m & ((1u << lane) - 1u))] = (int)((int64_t)row * sy + col);
                    }
                }
            }
        }

        // slide the x window by two rows
        l0 = l2;
        l1 = l3;
        ddc = dd2v;
        mmp = mm1;
        Dp = D1;
        z0 = z2;
        z1 = z3;
    }
}

// Constraint at the listed band cells: vals[e] = tmp + constraint(tmp, phi0).
__global__ void __launch_bounds__(256) k_band_constraint(Grid g, LsConstT<float> K, const float *__restrict__ tmp,
                                                         const float *__restrict__ ls0, const int *__restrict__ band,
                                                         const unsigned *__restrict__ band_n, float *__restrict__ vals) {
    const unsigned n = *band_n;
    for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int idx = band[e];
        const int i = idx / g.sy, j = idx % g.sy;
        float Lr[3][3], Ir[3][3];
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const int ii = i + a - 1, jj = j + b - 1;
                const bool corner = (ii < NB || ii >= g.nx + NB) && (jj < NB || jj >= g.ny + NB);
                Lr[a][b] = corner ? 0.f : tmp[IX(g, ii, jj)];
                Ir[a][b] = ls0[IX(g, ii, jj)];
            }
        const float hd = heaviside_deriv(Lr[1][1], K.eps);
        vals[e] = Lr[1][1] + (hd == 0.f ? 0.f : sussman_constraint_nb(K, Lr, Ir));
    }
}

__global__ void __launch_bounds__(256) k_band_apply(Grid g, const int *__restrict__ band,
                                                    const unsigned *__restrict__ band_n,
                                                    const float *__restrict__ vals, float *__restrict__ phi) {
    const unsigned n = *band_n;
    for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int idx = band[e];
        const float v = vals[e];
        phi[idx] = v;
        p_mirror_store(g, phi, idx / g.sy, idx % g.sy, v);
    }
}

template <int MODE, bool PB, int R>
void launch_r(const Grid &g, const Pass32Const &C, const float *src, const float *ls0, const float *base, float *out,
              int *band, unsigned *band_n, cudaStream_t st) {
    const dim3 grd((g.ny + R32_COLS - 1) / R32_COLS, (g.nx + R32_WARPS * R - 1) / (R32_WARPS * R));
    k_reinit32<MODE, PB, R><<<grd, 32 * R32_WARPS, 0, st>>>(g, C, src, ls0, base, out, band, band_n);
}

template <int MODE, bool PB>
void launch_p(const Grid &g, const Pass32Const &C, const float *src, const float *ls0, const float *base, float *out,
              int *band, unsigned *band_n, cudaStream_t st) {
    switch (ls32_rows_per_warp(g)) {
    case 16: launch_r<MODE, PB, 16>(g, C, src, ls0, base, out, band, band_n, st); break;
    case 8: launch_r<MODE, PB, 8>(g, C, src, ls0, base, out, band, band_n, st); break;
    default: launch_r<MODE, PB, 4>(g, C, src, ls0, base, out, band, band_n, st); break;
    }
}

template <int MODE>
void pseudo_step(const Grid &g, const Pass32Const &C, const Ls32Work &w, cudaStream_t st) {
    // LS1 -> w.a; tmp -> w.phi (in place: each cell reads phi only at itself)
    launch_p<MODE, false>(g, C, w.phi, w.ls0, nullptr, w.a, w.band, w.band_n, st);
    launch_p<MODE, true>(g, C, w.a, w.ls0, w.phi, w.phi, w.band, w.band_n, st);
    if (MODE == RM_MINRK2_SUSS) {
        // band cells: at most nx * ny; a grid-stride loop over the device count
        const int blocks = 2 * 148;
        k_band_constraint<<<blocks, 256, 0, st>>>(g, C.K, w.phi, w.ls0, w.band, w.band_n, w.band_val);
        k_band_apply<<<blocks, 256, 0, st>>>(g, w.band, w.band_n, w.band_val, w.phi);
    }
}

float2 both(float v) { return make_float2(v, v); }

}  // namespace

void launch_reinit32(const Grid &g, const LsConstT<float> &K, int reinit_mode, int steps, const Ls32Work &w,
                     cudaStream_t st) {
    Pass32Const C;
    C.K = K;
    C.invx = both((float)(1.0 / g.dx));
    C.invy = both((float)(1.0 / g.dy));
    C.invx2 = both((float)(1.0 / (g.dx * g.dx)));
    C.invy2 = both((float)(1.0 / (g.dy * g.dy)));
    C.hhx = both(K.dx * 0.5f);
    C.hhy = both(K.dy * 0.5f);
    C.eps2 = K.eps * K.eps;
    for (int s = 0; s < steps; s++) {
        if (reinit_mode == RM_ORIG) pseudo_step<RM_ORIG>(g, C, w, st);
        else if (reinit_mode == RM_MINRK2) pseudo_step<RM_MINRK2>(g, C, w, st);
        else pseudo_step<RM_MINRK2_SUSS>(g, C, w, st);
    }
}

int reinit32_launches(int reinit_mode, int steps) { return steps * (reinit_mode == RM_MINRK2_SUSS ? 4 : 2); }

}  // namespace asd2g
