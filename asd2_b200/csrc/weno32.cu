// HJ-WENO5 + TVD-RK3 stage of the mixed-precision level-set step, FP32,
// organised for instruction count (Solve_LevelSet_2D / HJWENO5_LS_2D /
// UnitHJWENO5, levelset2d.cpp:43-262).
//
// The scheme is the reference's: fluxes F = phi*u along x and phi*v along y,
// first differences D, the three Jiang-Peng smoothness indicators and weights
// (0.1, 0.6, 0.3) / (1e-6 + IS)^2 of phi^- and phi^+, the signed-velocity
// blend and the TVD-RK3 stage.  These stencils are bound by instruction issue
// (a per-cell evaluation as written takes ~800 thread instructions against 20
// bytes of traffic), so this kernel cuts instructions:
//
//  * Triples shared between reconstructions.  With T_k = (D_{k-1}, D_k,
//    D_{k+1}), phi^- at i uses T_{i-2} in the form (a-4b+3c), T_{i-1} in
//    (a-c) and T_i in (3a-4b+c); phi^+ at i uses T_{i+1} (3a-4b+c), T_i (a-c)
//    and T_{i-1} (a-4b+3c).  Each triple's three indicators and their
//    reciprocal squares are computed once and serve phi^- at one cell and
//    phi^+ at the neighbour.
//  * Scaling folded out.  The reference divides every difference by the
//    spacing d; here IS is formed from the raw differences with the epsilon
//    scaled to 1e-6 d^2 (the same weights), and 1/d multiplies the blend.
//  * The weights d_k enter the candidate coefficients, so a reconstruction
//    is (sum r_k q'_k) / (sum d_k r_k): one reciprocal each.
//  * Packed FP32x2 arithmetic (sm_100 fma/add/mul .f32x2).  A lane owns the
//    2 x 2 cells (i, i+1) x (j, j+32).  Along x it works on the column pair
//    (same rows, same stencil), sliding down its rows with the x window in
//    registers; along y on the row pair, with the pair's fluxes and triple
//    reciprocals exchanged through a per-warp shared-memory row.
//  * Reciprocals by rcp.approx (one MUFU op); the indicators are a
//    smoothness heuristic and the weights are normalised.
//
// A warp owns a strip of 64 columns and R rows; a block is 4 independent
// warps (no block barrier).  Loads outside the padded array read 0; they only
// feed cells that are not written.  Warps with cells within three of a
// boundary also write the ghost mirrors (the FP32 path requires
// producer-side P fills).
#include <cstdlib>

#include "batch.cuh"
#include "internal.cuh"
#include "ls32.cuh"

namespace asd2g {
namespace {

constexpr int W32_WARPS = 4;
constexpr int W32_COLS = 64;

__device__ __forceinline__ float2 p2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b, rounded like a subtraction
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }

__device__ __forceinline__ float rcpa(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float2 rcp2(float2 x) { return make_float2(rcpa(x.x), rcpa(x.y)); }

// 1 / (eps + IS)^2 of the triple (x, y, z) = (D_{k-1}, D_k, D_{k+1}) in the
// three forms: a = (x-4y+3z), b = (3x-4y+z), c = (x-z), each with
// IS = 13/12 (x-2y+z)^2 + 1/4 form^2.
struct Tri {
    float2 a, b, c;
};
__device__ __forceinline__ Tri tri(float2 x, float2 y, float2 z, float2 eps) {
    const float2 s = fma2(p2(-2.f), y, add2(x, z));
    const float2 h = fma2(mul2(s, p2(13.f / 12.f)), s, eps);
    const float2 u = sub2(x, z);
    const float2 v = fma2(p2(3.f), z, fma2(p2(-4.f), y, x));
    const float2 w = fma2(p2(3.f), x, fma2(p2(-4.f), y, z));
    const float2 ia = fma2(mul2(v, p2(0.25f)), v, h);
    const float2 ib = fma2(mul2(w, p2(0.25f)), w, h);
    const float2 ic = fma2(mul2(u, p2(0.25f)), u, h);
    Tri t;
    t.a = rcp2(mul2(ia, ia));
    t.b = rcp2(mul2(ib, ib));
    t.c = rcp2(mul2(ic, ic));
    return t;
}

// One reconstruction on the window v0..v4 (phi^- order: D_{i-3..i+1}; phi^+
// passes D_{i+2..i-2}) with the reciprocals r0, r1, r2 of its IS0, IS1, IS2:
// (0.1 r0 q0 + 0.6 r1 q1 + 0.3 r2 q2) / (0.1 r0 + 0.6 r1 + 0.3 r2), not yet
// divided by the spacing.
__device__ __forceinline__ float2 weno2(float2 v0, float2 v1, float2 v2, float2 v3, float2 v4, float2 r0, float2 r1,
                                        float2 r2) {
    const float2 q0 = fma2(p2(1.1f / 6.f), v2, fma2(p2(-0.7f / 6.f), v1, mul2(p2(0.1f / 3.f), v0)));
    const float2 q1 = fma2(p2(0.2f), v3, fma2(p2(0.5f), v2, mul2(p2(-0.1f), v1)));
    const float2 q2 = fma2(p2(-0.05f), v4, fma2(p2(0.25f), v3, mul2(p2(0.1f), v2)));
    const float2 den = fma2(p2(0.3f), r2, fma2(p2(0.6f), r1, mul2(p2(0.1f), r0)));
    const float2 num = fma2(r2, q2, fma2(r1, q1, mul2(r0, q0)));
    return mul2(num, rcp2(den));
}

// One strip (64 columns, bx) x row block (by) of the stage; the single-grid
// kernel takes them from its block index, the batched one from its work list.
template <int STAGE, int R>
__device__ __forceinline__ void ls_stage32_strip(const Grid &g, const Weno32Const &K, const float *__restrict__ phi_in,
                                                 const float *__restrict__ tu, const float *__restrict__ tv,
                                                 const float *phi_n, float *out, const double *__restrict__ dtp,
                                                 int bx, int by) {
    __shared__ float2 sF[W32_WARPS][W32_COLS + 6];     // F_y of rows (i, i+1) at column j0-3+k
    __shared__ float2 sT[W32_WARPS][3][W32_COLS + 4];  // reciprocals a, b, c of rows (i, i+1) at column j0-2+k
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int sx = g.sx, sy = g.sy;
    const int ib = NB + (by * W32_WARPS + w) * R;
    if (ib >= g.nx + NB) return;  // whole warp
    const int ie = min(ib + R, g.nx + NB);
    const int j0 = NB + bx * W32_COLS;
    const int cA = j0 + lane, cB = cA + 32;
    const bool inA = cA < sy, inB = cB < sy;
    float2 *sf = sF[w];
    float2(*st)[W32_COLS + 4] = sT[w];
    const float2 epsx = p2(K.epsx), epsy = p2(K.epsy);
    const float dt = (float)*dtp;
    // warps whose cells include ones within three of a boundary write ghost mirrors
    const bool edge = bx == 0 || j0 + W32_COLS > g.ny || ib < 2 * NB || ie > g.nx;

    auto ld = [&](const float *a, int i, int c, bool in) -> float {
        return (in && i < sx) ? __ldg(a + (int64_t)i * sy + c) : 0.f;
    };
    // phi_n may be the output array (stage 3 writes phi in place): read with a
    // coherent load, own cells only, before they are written
    auto ldn = [&](int i, int c, bool in) -> float { return in ? phi_n[(int64_t)i * sy + c] : 0.f; };
    auto fx = [&](int i) -> float2 {  // F_x at (i, cA), (i, cB)
        return mul2(make_float2(ld(phi_in, i, cA, inA), ld(phi_in, i, cB, inB)),
                    make_float2(ld(tu, i, cA, inA), ld(tu, i, cB, inB)));
    };

    // x window: D_{i-3..i+1} and the triples at i-2 (a), i-1 (a, c), i (all)
    float2 Fp = fx(ib - 3), d0, d1, d2, d3, d4;
    {
        float2 f = fx(ib - 2);
        d0 = sub2(f, Fp);
        Fp = fx(ib - 1);
        d1 = sub2(Fp, f);
        f = fx(ib);
        d2 = sub2(f, Fp);
        Fp = fx(ib + 1);
        d3 = sub2(Fp, f);
        f = fx(ib + 2);
        d4 = sub2(f, Fp);
        Fp = f;
    }
    float2 rAm2 = tri(d0, d1, d2, epsx).a, rAm1, rCm1;
    {
        const Tri t = tri(d1, d2, d3, epsx);
        rAm1 = t.a;
        rCm1 = t.c;
    }
    Tri T0 = tri(d2, d3, d4, epsx);

#pragma unroll
    for (int k = 0; k < R / 2; k++) {
        const int i = ib + 2 * k;
        if (i >= ie) break;
        // rows i+3, i+4 enter the x window (loads issued first, used last)
        const float2 fa = fx(i + 3), fb = fx(i + 4);
        // own cells (rows i, i+1; columns cA, cB) and the y fluxes of the row pair
        float ph[2][2], ux[2][2], vy[2][2], pn[2][2];
#pragma unroll
        for (int r = 0; r < 2; r++) {
            ph[r][0] = ld(phi_in, i + r, cA, inA);
            ph[r][1] = ld(phi_in, i + r, cB, inB);
            ux[r][0] = ld(tu, i + r, cA, inA);
            ux[r][1] = ld(tu, i + r, cB, inB);
            vy[r][0] = ld(tv, i + r, cA, inA);
            vy[r][1] = ld(tv, i + r, cB, inB);
            if (STAGE == 1) {
                pn[r][0] = ph[r][0];
                pn[r][1] = ph[r][1];
            } else {
                pn[r][0] = ldn(i + r, cA, inA);
                pn[r][1] = ldn(i + r, cB, inB);
            }
        }
        sf[lane + 3] = make_float2(ph[0][0] * vy[0][0], ph[1][0] * vy[1][0]);
        sf[lane + 35] = make_float2(ph[0][1] * vy[0][1], ph[1][1] * vy[1][1]);
        if (lane < 6) {  // halo columns j0-3..j0-1 and j0+64..j0+66
            const int hc = lane < 3 ? j0 - 3 + lane : j0 + 61 + lane;
            const bool hin = hc < sy;
            sf[lane < 3 ? lane : lane + 64] = make_float2(ld(phi_in, i, hc, hin) * ld(tv, i, hc, hin),
                                                          ld(phi_in, i + 1, hc, hin) * ld(tv, i + 1, hc, hin));
        }

        // y direction: differences and own triples of both columns
        __syncwarp();
        float2 dy[2][6];
        Tri ty[2];
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int b = lane + 32 * c;
            float2 e[7];
#pragma unroll
            for (int q = 0; q < 7; q++) e[q] = sf[b + q];
#pragma unroll
            for (int q = 0; q < 6; q++) dy[c][q] = sub2(e[q + 1], e[q]);
            ty[c] = tri(dy[c][2], dy[c][3], dy[c][4], epsy);
            st[0][b + 2] = ty[c].a;
            st[1][b + 2] = ty[c].b;
            st[2][b + 2] = ty[c].c;
        }
        if (lane < 3) {  // triples at columns j0-2, j0-1 and j0+64
            const int hp = lane < 2 ? lane : W32_COLS + 2;
            const float2 a0 = sf[hp], a1 = sf[hp + 1], a2 = sf[hp + 2], a3 = sf[hp + 3];
            const Tri h = tri(sub2(a1, a0), sub2(a2, a1), sub2(a3, a2), epsy);
            st[0][hp] = h.a;
            st[1][hp] = h.b;
            st[2][hp] = h.c;
        }
        __syncwarp();
        float2 ym[2], yp[2];
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const int b = lane + 32 * c;
            const float2 *v = dy[c];
            ym[c] = weno2(v[0], v[1], v[2], v[3], v[4], st[0][b], st[2][b + 1], ty[c].b);
            yp[c] = weno2(v[5], v[4], v[3], v[2], v[1], st[1][b + 3], ty[c].c, st[0][b + 1]);
        }

        // blend (x: column pairs per row; y: row pairs per column) and the RK stage
        const float2 hx = p2(K.hx), hy = p2(K.hy), nhx = p2(-K.hx), nhy = p2(-K.hy);
        float2 Y[2];
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const float2 a = make_float2(vy[0][c], vy[1][c]);
            Y[c] = fma2(yp[c], fma2(a, nhy, hy), mul2(ym[c], fma2(a, hy, hy)));
        }

        // x direction
        const float2 d5 = sub2(fa, Fp), d6 = sub2(fb, fa);
        Fp = fb;
        const Tri T1 = tri(d3, d4, d5, epsx), T2 = tri(d4, d5, d6, epsx);
        const float2 xm0 = weno2(d0, d1, d2, d3, d4, rAm2, rCm1, T0.b);
        const float2 xp0 = weno2(d5, d4, d3, d2, d1, T1.b, T0.c, rAm1);
        const float2 xm1 = weno2(d1, d2, d3, d4, d5, rAm1, T0.c, T1.b);
        const float2 xp1 = weno2(d6, d5, d4, d3, d2, T2.b, T1.c, T0.a);

        float2 X[2];
        {
            const float2 a0 = make_float2(ux[0][0], ux[0][1]), a1 = make_float2(ux[1][0], ux[1][1]);
            X[0] = fma2(xp0, fma2(a0, nhx, hx), mul2(xm0, fma2(a0, hx, hx)));
            X[1] = fma2(xp1, fma2(a1, nhx, hx), mul2(xm1, fma2(a1, hx, hx)));
        }
#pragma unroll
        for (int r = 0; r < 2; r++) {
            const int row = i + r;
            if (row >= ie) break;
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const int col = c ? cB : cA;
                if (col >= g.ny + NB) continue;
                const float Lc = (r ? (c ? X[1].y : X[1].x) : (c ? X[0].y : X[0].x)) + (r ? Y[c].y : Y[c].x);
                float val;
                if (STAGE == 1) val = pn[r][c] - dt * Lc;
                else if (STAGE == 2) val = 0.75f * pn[r][c] + 0.25f * ph[r][c] - 0.25f * dt * Lc;
                else val = (1.f / 3.f) * pn[r][c] + (2.f / 3.f) * ph[r][c] - (2.f / 3.f) * dt * Lc;
                out[(int64_t)row * sy + col] = val;
                if (edge) p_mirror_store(g, out, row, col, val);
            }
        }

        // slide the x window by two rows
        d0 = d2;
        d1 = d3;
        d2 = d4;
        d3 = d5;
        d4 = d6;
        rAm2 = T0.a;
        rAm1 = T1.a;
        rCm1 = T1.c;
        T0 = T2;
    }
}

template <int STAGE, int R>
__global__ void __launch_bounds__(32 * W32_WARPS, 4)
    k_ls_stage32(Grid g, Weno32Const K, const float *__restrict__ phi_in, const float *__restrict__ tu,
                 const float *__restrict__ tv, const float *phi_n, float *out, const double *__restrict__ dtp) {
    ls_stage32_strip<STAGE, R>(g, K, phi_in, tu, tv, phi_n, out, dtp, blockIdx.x, blockIdx.y);
}

// Batched: work-list entry = (instance, strip, row block) of the mixed
// instances; arrays by index into the instance's FP32 work (0 phi, 2 a, 3 b).
template <int STAGE, int R>
__global__ void __launch_bounds__(32 * W32_WARPS, 4)
    k_bls_stage32(const BInst *__restrict__ insts, const BTile *__restrict__ tiles, int in, int n, int out) {
    const BTile t = tiles[blockIdx.x];
    const BInst &I = insts[t.inst];
    const Grid g = I.g;
    const Weno32Const K = I.wk32;
    float *const a[4] = {I.w32.phi, I.w32.ls0, I.w32.a, I.w32.b};
    ls_stage32_strip<STAGE, R>(g, K, a[in], I.w32.tu, I.w32.tv, a[n], a[out], I.sc, t.bx, t.by);
}

template <int STAGE, int R>
void launch_r(const Grid &g, const Weno32Const &K, const float *phi_in, const float *tu, const float *tv,
              const float *phi_n, float *out, const double *dtp, cudaStream_t st) {
    const dim3 grd((g.ny + W32_COLS - 1) / W32_COLS, (g.nx + W32_WARPS * R - 1) / (W32_WARPS * R));
    k_ls_stage32<STAGE, R><<<grd, 32 * W32_WARPS, 0, st>>>(g, K, phi_in, tu, tv, phi_n, out, dtp);
}

template <int STAGE>
void launch_s(const Grid &g, const Weno32Const &K, const float *phi_in, const float *tu, const float *tv,
              const float *phi_n, float *out, const double *dtp, cudaStream_t st) {
    switch (ls32_rows_per_warp(g)) {
    case 16: launch_r<STAGE, 16>(g, K, phi_in, tu, tv, phi_n, out, dtp, st); break;
    case 8: launch_r<STAGE, 8>(g, K, phi_in, tu, tv, phi_n, out, dtp, st); break;
    default: launch_r<STAGE, 4>(g, K, phi_in, tu, tv, phi_n, out, dtp, st); break;
    }
}

}  // namespace

// Rows per warp of the FP32 stage kernel: 4 (at
// 2048^2 the advection took 0.19 / 0.22 / 0.30 ms with 4 / 8 / 16 rows: with
// 16 warps per SM the serial row walk of a warp is latency-bound, and more,
// shorter walks hide it better than the fewer window loads of long ones).
// ASD2G_LS32_ROWS = 8 or 16 selects the longer walks.
int ls32_rows_per_warp(const Grid &) {
    static int rows = -1;
    if (rows < 0) {
        const char *e = getenv("ASD2G_LS32_ROWS");
        const int v = e ? atoi(e) : 0;
        rows = (v == 8 || v == 16) ? v : 4;
    }
    return rows;
}

Weno32Const make_weno32_const(const Grid &g) {
    Weno32Const K;
    K.hx = (float)(0.5 / g.dx);
    K.hy = (float)(0.5 / g.dy);
    K.epsx = (float)(1e-6 * g.dx * g.dx);
    K.epsy = (float)(1e-6 * g.dy * g.dy);
    return K;
}

void launch_bstep_ls_stage32(const BStepPlan &P, int stage, int in, int n, int out, cudaStream_t st) {
    if (P.ns32 == 0) return;
    constexpr int R = 4;  // the tile lists are built for 4 rows per warp
#define BS32(S) k_bls_stage32<S, R><<<P.ns32, 32 * W32_WARPS, 0, st>>>(P.insts, P.s32_tiles, in, n, out)
    if (stage == 1) BS32(1);
    else if (stage == 2) BS32(2);
    else BS32(3);
#undef BS32
}

void launch_ls_stage32(const Grid &g, int stage, const float *phi_in, const float *tu, const float *tv,
                       const float *phi_n, float *out, const double *dtp, cudaStream_t st) {
    const Weno32Const K = make_weno32_const(g);
    if (stage == 1) launch_s<1>(g, K, phi_in, tu, tv, phi_n, out, dtp, st);
    else if (stage == 2) launch_s<2>(g, K, phi_in, tu, tv, phi_n, out, dtp, st);
    else launch_s<3>(g, K, phi_in, tu, tv, phi_n, out, dtp, st);
}

}  // namespace asd2g
