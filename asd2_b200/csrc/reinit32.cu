// Reinitialisation pseudo-steps of the mixed-precision level-set step, FP32,
// organised for instruction count (Reinit_MinRK2_2D / Reinit_Original_2D /
// Reinit_Sussman_2D with ENO_DerivAbsLS_2D, SubcellENO_Min_DerivAbsLS_2D and
// GetSussmanReinitConstraint, levelset2d.cpp:264-486, :560-893).
//
// The scheme is the reference's: second-order ENO one-sided differences
// (minmod of the neighbouring second differences), the Min-Gibou subcell fix
// where phi0 changes sign towards a neighbour, Godunov |grad phi|, the sign
// of phi0 (smoothed for MinRK2), the two RK2 passes, and for MinRK2 +
// Sussman the volume constraint on the interface band.  Evaluated per cell as
// written these passes take ~330 thread instructions per cell against 12-16
// bytes of traffic, so they were issue-bound at a fifth of HBM bandwidth.
// This form cuts instructions:
//
//  * Differences and minmods shared between cells.  First differences live
//    on faces, second differences on cells and the minmod of two neighbouring
//    second differences on faces again: each is formed once and serves the
//    one-sided derivatives of both cells beside it.  minmod(a, b) is the
//    median of (a, b, 0): min(max(a, b), max(a, 0), max(b, 0)), with the
//    sm_100 three-input minimum.
//  * Spacings folded out.  The one-sided derivatives are formed from raw
//    differences, (D1 -/+ minmod(D2, D2') / 2); Godunov's max/min commute with
//    the positive factor, and 1/dx, 1/dy scale the two squares at the end.
//    Godunov's upwind choice (levelset2d.cpp:596-610) is a three-input
//    maximum of sign-scaled differences: max(-sg D+, sg D-, 0), sg = 1 where
//    phi0 >= 0 and -1 elsewhere (the scaling runs packed on the FMA pipe, the
//    maxima on the ALU pipe, which minmods and maxima saturate first).
//  * Packed FP32x2 arithmetic (sm_100 fma/add/mul .f32x2).  A lane owns the
//    two neighbouring columns (c, c+1) of a 64-column strip and walks R rows:
//    along x the five-row window and its differences slide in registers,
//    along y the neighbour columns come from the adjacent lanes by shuffles.
//    Lanes 1..30 write (60 columns per strip); lanes 0 and 31 only supply
//    neighbours.
//  * The subcell fix runs only in warps where some written cell has a sign
//    change of phi0 towards a neighbour (a few rows per strip around the
//    interface), on the flagged lanes, with the per-cell routine.
//  * The Sussman pass: the second RK2 pass also stores its result into phi,
//    so the constraint kernel only touches the band |tmp| <= eps where the
//    Heaviside derivative is nonzero (elsewhere the constraint is zero and
//    phi = tmp already).
//
// Square roots are sqrt.approx (one MUFU op).  Loads outside the padded
// array read 0; they only feed cells that are not written.  Warps with cells
// within three of a boundary also write the ghost mirrors (the FP32 path
// requires producer-side P fills).
#include <cstdint>
#include <cstdlib>

#include "batch.cuh"
#include "levelset_impl.cuh"
#include "ls32.cuh"

namespace asd2g {
namespace {

constexpr int RI_WARPS = 4;  // warps per block, stacked along x (rows)
constexpr int RI_OUT = 60;   // columns written per strip (lanes 1..30, two each)
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ float2 p2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
// a - b, rounded like a subtraction
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }

__device__ __forceinline__ float max3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float min3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
// LevelSetSolver2D::MinMod (levelset2d.cpp:1036-1046) as the median of
// (a, b, 0): a when a, b have one sign and |a| <= |b|, b when |b| < |a|, 0
// when the signs differ or either is zero.
__device__ __forceinline__ float mmod(float a, float b) { return min3(fmaxf(a, b), fmaxf(a, 0.f), fmaxf(b, 0.f)); }
__device__ __forceinline__ float2 mmod2(float2 a, float2 b) { return make_float2(mmod(a.x, b.x), mmod(a.y, b.y)); }

__device__ __forceinline__ float sqrta(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Spacings for the subcell routine, passed by value.
struct SubK {
    float dx, dy, idx, idy, idx2, idy2;  // dx, dy, 1/dx, 1/dy, 1/dx^2, 1/dy^2
};

// The subcell one-sided derivatives at the interior cell at offset c (row
// pitch sy) where phi0 changes sign towards a neighbour
// (SubcellENO_Min_DerivAbsLS_2D, levelset2d.cpp:620-711), as raw differences
// (times the spacing).  d = (D+x, D-x, D+y, D-y) from ENO; the entries
// without a sign change are returned unchanged.
__device__ __noinline__ float4 subcell_fix(const float *__restrict__ src, const float *__restrict__ ls0, int64_t c,
                                           int sy, SubK s, float4 d) {
    const DivHT<float> ddx{s.dx, s.idx, 0}, ddy{s.dy, s.idy, 0};
    const DivHT<float> ddx2{s.dx * s.dx, s.idx2, 0}, ddy2{s.dy * s.dy, s.idy2, 0};
    const float v = __ldg(src + c);
    const float x0 = __ldg(ls0 + c);
    const float xm1 = __ldg(ls0 + c - sy), xp1 = __ldg(ls0 + c + sy);
    const float ym1 = __ldg(ls0 + c - 1), yp1 = __ldg(ls0 + c + 1);
    if (x0 * xp1 < 0.f) d.x = subcell_plus(s.dx, ddx, ddx2, v, xm1, x0, xp1, __ldg(ls0 + c + 2 * sy)) * s.dx;
    if (x0 * xm1 < 0.f) d.y = subcell_minus(s.dx, ddx, ddx2, v, __ldg(ls0 + c - 2 * sy), xm1, x0, xp1) * s.dx;
    if (x0 * yp1 < 0.f) d.z = subcell_plus(s.dy, ddy, ddy2, v, ym1, x0, yp1, __ldg(ls0 + c + 2)) * s.dy;
    if (x0 * ym1 < 0.f) d.w = subcell_minus(s.dy, ddy, ddy2, v, __ldg(ls0 + c - 2), ym1, x0, yp1) * s.dy;
    return d;
}

// One RK2 pass of the reinitialisation over a strip of 60 columns x R rows
// per warp.
//   PASS 0: out = src - adt S (|grad src| - 1)                 (LS1)
//   PASS 1: out = (base + src - adt S (|grad src| - 1)) / 2    (LS2, averaged)
// S = sign(phi0) (Original) or the smoothed sign (MinRK2 modes); the MinRK2
// modes use the subcell derivatives next to the interface.  out2, when not
// null, receives the same values (the Sussman mode's phi).  base may alias
// out2: it is read only at the lane's own cells, before they are written.
// The strip bx x row block by; the single-grid kernel takes them from its
// block index, the batched one from its work list.
template <int PASS, int MODE, bool VEC, int R>
__device__ __forceinline__ void reinit32_strip(const Grid &g, const LsConstT<float> &K, const float *__restrict__ src,
                                               const float *__restrict__ ls0, const float *base, float *out,
                                               float *out2, int *band, unsigned *band_n, int bx, int by) {
    constexpr bool SUB = (MODE == RM_MINRK2 || MODE == RM_MINRK2_SUSS);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    // the first pass of a pseudo-step empties the band list the second fills
    if (PASS == 0 && band_n && bx == 0 && by == 0 && threadIdx.x == 0) *band_n = 0u;
    const int ib = NB + (by * RI_WARPS + w) * R;
    if (ib >= g.nx + NB) return;  // whole warp
    const int ie = min(ib + R, g.nx + NB);
    const int J0 = bx * RI_OUT;
    const int c0 = J0 + 2 * lane;
    const int sx = g.sx, sy = g.sy;
    const bool own = lane >= 1 && lane <= 30;
    const bool wA = own && c0 >= NB && c0 < g.ny + NB;  // column c0 is interior and written
    const bool wB = own && c0 + 1 < g.ny + NB;          // column c0 + 1
    const bool edge = J0 <= 2 * NB || J0 + RI_OUT + 1 >= g.ny || ib <= 2 * NB - 1 || ie - 1 >= g.nx;

    auto ld2 = [&](const float *a, int r) -> float2 {
        if (r >= sx) return p2(0.f);
        const float *p = a + (int64_t)r * sy + c0;
        if constexpr (VEC) {
            return c0 < sy ? __ldg(reinterpret_cast<const float2 *>(p)) : p2(0.f);
        } else {
            return make_float2(c0 < sy ? __ldg(p) : 0.f, c0 + 1 < sy ? __ldg(p + 1) : 0.f);
        }
    };
    // the whole window first: R + 4 rows of src, R + 2 rows of phi0
    float2 P[R + 4], Q[R + 2];
    if (VEC && ib + R + 1 < sx && J0 + 63 < sy) {  // the whole window inside the array: no guards
        const float *ps = src + (int64_t)(ib - 2) * sy + c0, *pq = ls0 + (int64_t)(ib - 1) * sy + c0;
#pragma unroll
        for (int m = 0; m < R + 4; m++) P[m] = __ldg(reinterpret_cast<const float2 *>(ps + (int64_t)m * sy));
#pragma unroll
        for (int m = 0; m < R + 2; m++) Q[m] = __ldg(reinterpret_cast<const float2 *>(pq + (int64_t)m * sy));
    } else {
#pragma unroll
        for (int m = 0; m < R + 4; m++) P[m] = ld2(src, ib - 2 + m);
#pragma unroll
        for (int m = 0; m < R + 2; m++) Q[m] = ld2(ls0, ib - 1 + m);
    }
    // the second pass's base values at the lane's own cells (base may alias
    // out2, so plain loads, issued with the window)
    float2 Bv[PASS == 1 ? R : 1];
    if constexpr (PASS == 1) {
#pragma unroll
        for (int m = 0; m < R; m++) {
            const int64_t o = (int64_t)(ib + m) * sy + c0;
            if (ib + m >= ie) {
                Bv[m] = p2(0.f);
            } else if (VEC && wA && wB) {
                Bv[m] = *reinterpret_cast<const float2 *>(base + o);
            } else {
                Bv[m] = make_float2(wA ? base[o] : 0.f, wB ? base[o + 1] : 0.f);
            }
        }
    }

    const float2 ihx = p2(K.ddx.inv), ihy = p2(K.ddy.inv);
    const float2 half = p2(0.5f), nhalf = p2(-0.5f), nadt = p2(-K.adt);
    const float eps2 = K.eps * K.eps;

    // x window for row ib: faces (ib-1|ib), (ib|ib+1); second differences at
    // ib; the minmod on face (ib-1|ib)
    float2 dx0 = sub2(P[2], P[1]), dxp = sub2(P[3], P[2]);
    float2 d20 = sub2(dxp, dx0);
    float2 mm_m = mmod2(sub2(dx0, sub2(P[1], P[0])), d20);

#pragma unroll
    for (int k = 0; k < R; k++) {
        const int i = ib + k;
        if (i >= ie) break;  // whole warp
        const float2 p = P[k + 2], q = Q[k + 1];
        // x: forward face (i|i+1), backward face (i-1|i)
        const float2 dxpp = sub2(P[k + 4], P[k + 3]);
        const float2 d2p = sub2(dxpp, dxp);
        const float2 mm_p = mmod2(d20, d2p);
        const float2 dPx = fma2(mm_p, nhalf, dxp), dMx = fma2(mm_m, half, dx0);
        // y: columns c0-1 and c0+2 from the neighbour lanes
        const float vL = __shfl_up_sync(FULL, p.y, 1), vR = __shfl_down_sync(FULL, p.x, 1);
        const float2 el = sub2(p, make_float2(vL, p.x));   // faces (c0-1|c0), (c0|c0+1)
        const float2 er = sub2(make_float2(p.y, vR), p);   // faces (c0|c0+1), (c0+1|c0+2)
        const float2 d2y = sub2(er, el);                    // second differences at c0, c0+1
        const float d2R = __shfl_down_sync(FULL, d2y.x, 1);
        const float mB = mmod(d2y.x, d2y.y), mC = mmod(d2y.y, d2R);
        const float mA = __shfl_up_sync(FULL, mC, 1);  // face (c0-1|c0): the left lane's (c0+1|c0+2)
        const float2 dPy = fma2(make_float2(mB, mC), nhalf, er);
        const float2 dMy = fma2(make_float2(mA, mB), half, el);
        float4 dA = make_float4(dPx.x, dMx.x, dPy.x, dMy.x), dB = make_float4(dPx.y, dMx.y, dPy.y, dMy.y);
        if constexpr (SUB) {
            // phi0 changes sign towards a neighbour: x0 * x_nb < 0 (levelset2d.cpp:629-642)
            const float qL = __shfl_up_sync(FULL, q.y, 1), qR = __shfl_down_sync(FULL, q.x, 1);
            const float2 px = mul2(q, Q[k + 2]), pm = mul2(q, Q[k]);
            const float2 py = mul2(q, make_float2(q.y, qR));  // (c0|c0+1), (c0+1|c0+2)
            const float pl = q.x * qL;                          // (c0-1|c0)
            const bool any = own && min3(min3(px.x, px.y, pm.x), min3(pm.y, py.x, py.y), pl) < 0.f;
            if (__any_sync(FULL, any)) {
                const bool fA = wA && fminf(fminf(px.x, pm.x), fminf(py.x, pl)) < 0.f;
                const bool fB = wB && fminf(fminf(px.y, pm.y), fminf(py.y, py.x)) < 0.f;
                const SubK sk{K.dx, K.dy, K.ddx.inv, K.ddy.inv, K.ddx2.inv, K.ddy2.inv};
                const int64_t o = (int64_t)i * sy + c0;
                if (fA) dA = subcell_fix(src, ls0, o, sy, sk, dA);
                if (fB) dB = subcell_fix(src, ls0, o + 1, sy, sk, dB);
            }
        }
        // Godunov |grad|, the sign of phi0 and the RK2 update
        // sg = +1 where phi0 >= 0, else -1: max(-sg D+, sg D-, 0) per axis
        const float2 sg = make_float2(q.x >= 0.f ? 1.f : -1.f, q.y >= 0.f ? 1.f : -1.f);
        const float2 ux_p = mul2(sg, make_float2(dA.x, dB.x)), ux_m = mul2(sg, make_float2(dA.y, dB.y));
        const float2 uy_p = mul2(sg, make_float2(dA.z, dB.z)), uy_m = mul2(sg, make_float2(dA.w, dB.w));
        const float2 gx = mul2(make_float2(max3(-ux_p.x, ux_m.x, 0.f), max3(-ux_p.y, ux_m.y, 0.f)), ihx);
        const float2 gy = mul2(make_float2(max3(-uy_p.x, uy_m.x, 0.f), max3(-uy_p.y, uy_m.y, 0.f)), ihy);
        const float2 G = fma2(gx, gx, mul2(gy, gy));
        const float2 a = make_float2(sqrta(G.x), sqrta(G.y));
        float2 S;
        if constexpr (SUB) {
            S = mul2(q, make_float2(rsqrtf(fmaf(q.x, q.x, eps2)), rsqrtf(fmaf(q.y, q.y, eps2))));
        } else {
            S = make_float2((float)isgn(q.x), (float)isgn(q.y));
        }
        float2 val = fma2(mul2(S, nadt), sub2(a, p2(1.f)), p);
        const int64_t o = (int64_t)i * sy + c0;
        if constexpr (PASS == 1) val = mul2(half, __fadd2_rn(Bv[k], val));
        if (VEC && wA && wB) {
            *reinterpret_cast<float2 *>(out + o) = val;
            if (out2) *reinterpret_cast<float2 *>(out2 + o) = val;
        } else {
            if (wA) out[o] = val.x;
            if (wB) out[o + 1] = val.y;
            if (out2) {
                if (wA) out2[o] = val.x;
                if (wB) out2[o + 1] = val.y;
            }
        }
        if (PASS == 1 && band) {
            // cells where the Heaviside derivative of tmp is nonzero (not |tmp| > eps)
            const bool bA = wA && !(fabsf(val.x) > K.eps), bB = wB && !(fabsf(val.y) > K.eps);
            const unsigned mA = __ballot_sync(FULL, bA), mB = __ballot_sync(FULL, bB);
            if (mA | mB) {
                unsigned at = 0;
                if (lane == 0) at = atomicAdd(band_n, (unsigned)(__popc(mA) + __popc(mB)));
                at = __shfl_sync(FULL, at, 0);
                const unsigned below = (1u << lane) - 1u;
                const unsigned pos = at + __popc(mA & below) + __popc(mB & below);
                if (bA) band[pos] = (int)o;
                if (bB) band[pos + (bA ? 1u : 0u)] = (int)(o + 1);
            }
        }
        if (edge) {
            if (wA) p_mirror_store(g, out, i, c0, val.x);
            if (wB) p_mirror_store(g, out, i, c0 + 1, val.y);
            if (out2) {
                if (wA) p_mirror_store(g, out2, i, c0, val.x);
                if (wB) p_mirror_store(g, out2, i, c0 + 1, val.y);
            }
        }
        // slide the x window by one row
        dx0 = dxp;
        dxp = dxpp;
        d20 = d2p;
        mm_m = mm_p;
    }
}

// The Sussman constraint on the interface band (GetSussmanReinitConstraint,
// levelset2d.cpp:787-893; MinRK2 + Sussman adds it to tmp, :368-372):
// out = tmp + constraint(tmp, phi0) at the cells the second RK2 pass listed
// (|tmp| <= eps).  Elsewhere the Heaviside derivative of tmp is zero, the
// constraint with it, and out already holds tmp.  The list is a few cells
// wide along the interface; one thread per listed cell.
__global__ void __launch_bounds__(128)
    k_sussman32_band(Grid g, LsConstT<float> K, const float *__restrict__ tmp, const float *__restrict__ ls0,
                     float *out, const int *__restrict__ band, const unsigned *__restrict__ band_n) {
    const unsigned n = *band_n;
    for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int o = band[k];
        const int i = o / g.sy, j = o - i * g.sy;
        const float t = __ldg(tmp + o);
        const float val = t + sussman_constraint(g, K, tmp, ls0, heaviside_deriv(t, K.eps), i, j);
        out[o] = val;
        p_mirror_store(g, out, i, j, val);
    }
}

template <int PASS, int MODE, bool VEC, int R>
__global__ void __launch_bounds__(32 * RI_WARPS, R == 1 ? 8 : (R == 2 ? 7 : (R == 4 ? 6 : 4)))
    k_reinit32(Grid g, LsConstT<float> K, const float *__restrict__ src, const float *__restrict__ ls0,
               const float *base, float *out, float *out2, int *band, unsigned *band_n) {
    reinit32_strip<PASS, MODE, VEC, R>(g, K, src, ls0, base, out, out2, band, band_n, blockIdx.x, blockIdx.y);
}

// Batched (modes Original and MinRK2, 2 rows per warp): work-list entry =
// (instance, strip, row block) of the mixed instances; pseudo-step k of
// every instance that has it.  Pass a: phi -> a; pass b: (phi, a) -> phi.
template <int PASS, int MODE>
__global__ void __launch_bounds__(32 * RI_WARPS, 7)
    k_breinit32(const BInst *__restrict__ insts, const BTile *__restrict__ tiles, int k) {
    const BTile t = tiles[blockIdx.x];
    const BInst &I = insts[t.inst];
    if (k >= I.nreinit) return;
    const Grid g = I.g;
    const LsConstT<float> K = I.K32;
    const Ls32Work w = I.w32;
    const float *src = PASS == 0 ? w.phi : w.a;
    float *out = PASS == 0 ? w.a : w.phi;
    const float *base = PASS == 0 ? nullptr : w.phi;
    if (g.sy % 2 == 0) reinit32_strip<PASS, MODE, true, 2>(g, K, src, w.ls0, base, out, nullptr, nullptr, nullptr, t.bx, t.by);
    else reinit32_strip<PASS, MODE, false, 2>(g, K, src, w.ls0, base, out, nullptr, nullptr, nullptr, t.bx, t.by);
}

template <int PASS, int MODE, bool VEC>
void launch_v(const Grid &g, const LsConstT<float> &K, int rows, const float *src, const float *ls0,
              const float *base, float *out, float *out2, int *band, unsigned *band_n, cudaStream_t st) {
    const int nbx = (g.ny + 1 + RI_OUT - 1) / RI_OUT;  // strips cover padded columns 2 .. ny + 2
    auto grid = [&](int R) { return dim3(nbx, (g.nx + RI_WARPS * R - 1) / (RI_WARPS * R)); };
    const int nt = 32 * RI_WARPS;
#define RI32_LAUNCH(R) \
    k_reinit32<PASS, MODE, VEC, R><<<grid(R), nt, 0, st>>>(g, K, src, ls0, base, out, out2, band, band_n)
    switch (rows) {
    case 1: RI32_LAUNCH(1); break;
    case 4: RI32_LAUNCH(4); break;
    case 8: RI32_LAUNCH(8); break;
    default: RI32_LAUNCH(2); break;
    }
#undef RI32_LAUNCH
}

template <int PASS, int MODE>
void launch_p(const Grid &g, const LsConstT<float> &K, int rows, bool vec, const float *src, const float *ls0,
              const float *base, float *out, float *out2, int *band, unsigned *band_n, cudaStream_t st) {
    if (vec) launch_v<PASS, MODE, true>(g, K, rows, src, ls0, base, out, out2, band, band_n, st);
    else launch_v<PASS, MODE, false>(g, K, rows, src, ls0, base, out, out2, band, band_n, st);
}

bool aligned8(const void *p) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) & 7u) == 0; }

}  // namespace

void launch_bstep_reinit32(const BStepPlan &P, int mode, bool pass_b, int k, cudaStream_t st) {
    if (P.nr32 == 0) return;
    const int nt = 32 * RI_WARPS;
    if (mode == RM_ORIG) {
        if (pass_b) k_breinit32<1, RM_ORIG><<<P.nr32, nt, 0, st>>>(P.insts, P.r32_tiles, k);
        else k_breinit32<0, RM_ORIG><<<P.nr32, nt, 0, st>>>(P.insts, P.r32_tiles, k);
    } else {
        if (pass_b) k_breinit32<1, RM_MINRK2><<<P.nr32, nt, 0, st>>>(P.insts, P.r32_tiles, k);
        else k_breinit32<0, RM_MINRK2><<<P.nr32, nt, 0, st>>>(P.insts, P.r32_tiles, k);
    }
}

// Rows per warp of the FP32 reinitialisation passes: 2 (one pseudo-step at
// 2048^2 took 50.7 / 48.6 / 55.8 / 74.7 us with 1 / 2 / 4 / 8 rows: the
// longer walks load fewer window rows per cell but hold more registers, and
// the passes are bound by instruction issue with few resident warps).
// ASD2G_RI32_ROWS = 1, 4 or 8 selects the others.
int ri32_rows_per_warp() {
    static int rows = -1;
    if (rows < 0) {
        const char *e = getenv("ASD2G_RI32_ROWS");
        const int v = e ? atoi(e) : 0;
        rows = (v == 1 || v == 4 || v == 8) ? v : 2;
    }
    return rows;
}

void launch_reinit32_step(const Grid &g, int reinit_mode, const Ls32Work &w, cudaStream_t st) {
    const LsConstT<float> K = make_lsconst_t<float>(g);
    const int rows = ri32_rows_per_warp();
    // paired float2 accesses need an even row pitch and 8-byte aligned arrays
    const bool vec = (g.sy % 2 == 0) && aligned8(w.phi) && aligned8(w.ls0) && aligned8(w.a) && aligned8(w.b);
    if (reinit_mode == RM_ORIG) {
        launch_p<0, RM_ORIG>(g, K, rows, vec, w.phi, w.ls0, nullptr, w.a, nullptr, nullptr, nullptr, st);
        launch_p<1, RM_ORIG>(g, K, rows, vec, w.a, w.ls0, w.phi, w.phi, nullptr, nullptr, nullptr, st);
    } else if (reinit_mode == RM_MINRK2) {
        launch_p<0, RM_MINRK2>(g, K, rows, vec, w.phi, w.ls0, nullptr, w.a, nullptr, nullptr, nullptr, st);
        launch_p<1, RM_MINRK2>(g, K, rows, vec, w.a, w.ls0, w.phi, w.phi, nullptr, nullptr, nullptr, st);
    } else {
        launch_p<0, RM_MINRK2_SUSS>(g, K, rows, vec, w.phi, w.ls0, nullptr, w.a, nullptr, nullptr, w.band_n, st);
        launch_p<1, RM_MINRK2_SUSS>(g, K, rows, vec, w.a, w.ls0, w.phi, w.b, w.phi, w.band, w.band_n, st);
        k_sussman32_band<<<2 * 148, 128, 0, st>>>(g, K, w.b, w.ls0, w.phi, w.band, w.band_n);
    }
}

}  // namespace asd2g
