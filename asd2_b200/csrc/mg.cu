// Mixed-precision multigrid-preconditioned flexible CG for the GFM system.
//
// Outer solver: flexible CG (Polak-Ribiere beta) in FP64 on the assembled
// system (x, r, p, q FP64; the residual that decides convergence is the FP64
// recurrence residual, checked against the true FP64 residual by the host).
// Preconditioner: one symmetric V(1,1)-cycle in FP32 of cell-centred
// geometric multigrid:
//   * coarse operators by Galerkin aggregation of 2x2 cells (piecewise-
//     constant prolongation P, restriction R = P^T): coarse face couplings are
//     the sums of the fine couplings across the coarse face, the coarse
//     diagonal the aggregate's row sums; 5-point, SPD, and exact across the
//     density jumps (no coefficient averaging);
//   * red-black Gauss-Seidel smoothing, red then black before restriction and
//     black then red after prolongation (the adjoint), so the cycle is
//     symmetric; the prolonged correction is over-relaxed by omega = 1.9,
//     which compensates the piecewise-constant coarse space;
//   * the coarsest level (<= 64 cells) is solved exactly with its dense
//     inverse, formed once per assembly.
// Each level costs two kernels: "pre" = red sweep + black sweep + residual +
// restriction, "post" = prolongation + black sweep + red sweep.  A 16 x 32
// tile loads a two-cell halo into shared memory and recomputes the halo's
// red/black values itself, so one kernel produces exactly the result of the
// separate sweeps (no grid-wide barrier between them).  The level-0 "post"
// kernel also converts z to FP64 and forms the two FCG dot products.
#include "lsmath.cuh"
#include <cstdlib>

#include "mg.cuh"
#include "asd2g.h"
#include "batch.cuh"

namespace asd2g {

namespace {

constexpr int MT_I = 16, MT_J = 32;  // tile (rows i, columns j), must be even
constexpr int KMODE_LEARNED = 5;      // KState mode of ASD2G_SOLVER_UNET (V-cycle + learned correction)

// Programmatic dependent launch: the single-system FCG / V-cycle kernels are
// launched with programmatic stream serialisation, so the next kernel's CTAs
// are scheduled while this one runs; each waits for its predecessor's
// completion (and memory) before touching data, then lets its own successor
// launch.  Both are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
constexpr int MG_COARSE_MAX = 64;   // cells on the coarsest level

// block sum and grid reduction (same fixed-order scheme as pressure.cu)
template <int NV>
__device__ __forceinline__ void mg_block_sum(double (&v)[NV], double (&sh)[NV][32]) {
#pragma unroll
    for (int q = 0; q < NV; q++)
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int lane = tid & 31, wid = tid >> 5, nw = (blockDim.x * blockDim.y) >> 5;
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NV; q++) sh[q][wid] = v[q];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double s = lane < nw ? sh[q][lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            v[q] = s;
        }
    }
}

// Sum NV values over the nb blocks (ids bid) that share partial and counter:
// every block writes its block sum, the last one to arrive adds them in
// block order (deterministic) and returns true with the totals in thread 0.
template <int NV>
__device__ __forceinline__ bool mg_reduce(double (&v)[NV], double *partial, unsigned *counter, unsigned bid,
                                          unsigned nb, double (&tot)[NV]) {
    __shared__ double sh[NV][32];
    __shared__ bool last;
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    mg_block_sum<NV>(v, sh);
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) partial[NV * bid + q] = v[q];
        __threadfence();
        last = atomicAdd(counter, 1u) == nb - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double a[NV];
#pragma unroll
    for (int q = 0; q < NV; q++) a[q] = 0.0;
    for (unsigned b = tid; b < nb; b += blockDim.x * blockDim.y)
#pragma unroll
        for (int q = 0; q < NV; q++) a[q] += __ldcg(partial + NV * b + q);
    mg_block_sum<NV>(a, sh);
    if (tid != 0) return false;
#pragma unroll
    for (int q = 0; q < NV; q++) tot[q] = a[q];
    *counter = 0u;
    return true;
}

template <int NV>
__device__ __forceinline__ bool mg_grid_reduce(double (&v)[NV], double *partial, unsigned *counter,
                                               double (&tot)[NV]) {
    return mg_reduce<NV>(v, partial, counter, blockIdx.x + gridDim.x * blockIdx.y, gridDim.x * gridDim.y, tot);
}

__device__ __forceinline__ int64_t LK(const MgLevel &L, int i, int j) { return (int64_t)j + (int64_t)L.ny * i; }

// ------------------------------------------------------------- set-up --
// Level 0 in FP32 from the assembled FP64 system; the pinned cell keeps its
// diagonal and loses its couplings (its rhs is always 0, so it stays 0).
__device__ __forceinline__ void mg_l0_cell(int nx, int ny, const Sys &S, const MgLevel &L, int64_t k) {
    const int i = (int)(k / ny), j = (int)(k % ny);
    const bool pin0 = S.pinned && k == 0;
    L.diag[k] = (float)S.diag[k];
    L.ce[k] = (i < nx - 1 && !pin0) ? (float)S.ce[k] : 0.0f;
    L.cn[k] = (j < ny - 1 && !pin0) ? (float)S.cn[k] : 0.0f;
}

__global__ void k_mg_l0(int nx, int ny, Sys S, MgLevel L) {
    const int64_t n = (int64_t)nx * ny;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        mg_l0_cell(nx, ny, S, L, k);
}

// Galerkin aggregation R A P with piecewise-constant P (2x2 aggregates; the
// last aggregate of an odd dimension has one cell in that direction).
__device__ __forceinline__ void mg_coarsen_cell(const MgLevel &F, const MgLevel &C, int64_t k) {
    const int I = (int)(k / C.ny), J = (int)(k % C.ny);
    const int i0 = 2 * I, j0 = 2 * J;
    const bool hi = i0 + 1 < F.nx, hj = j0 + 1 < F.ny;
    float d = F.diag[LK(F, i0, j0)];
    if (hi) d += F.diag[LK(F, i0 + 1, j0)];
    if (hj) d += F.diag[LK(F, i0, j0 + 1)];
    if (hi && hj) d += F.diag[LK(F, i0 + 1, j0 + 1)];
    float inner = 0.0f;
    if (hi) inner += F.ce[LK(F, i0, j0)];
    if (hi && hj) inner += F.ce[LK(F, i0, j0 + 1)];
    if (hj) inner += F.cn[LK(F, i0, j0)];
    if (hi && hj) inner += F.cn[LK(F, i0 + 1, j0)];
    C.diag[k] = d - 2.0f * inner;
    const int ie = hi ? i0 + 1 : i0, je = hj ? j0 + 1 : j0;
    float ce = F.ce[LK(F, ie, j0)];
    if (hj) ce += F.ce[LK(F, ie, j0 + 1)];
    float cn = F.cn[LK(F, i0, je)];
    if (hi) cn += F.cn[LK(F, i0 + 1, je)];
    C.ce[k] = ce;
    C.cn[k] = cn;
}

__global__ void k_mg_coarsen(MgLevel F, MgLevel C) {
    const int64_t n = (int64_t)C.nx * C.ny;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        mg_coarsen_cell(F, C, k);
}

// ---------------------------------------------------------- tile loads --
// A tile of TI_ x TJ_ cells plus its 2-cell halo (the batched solve picks TI_
// x TJ_ from MG_SHAPES by timing them on its own hierarchy).
template <int TI_, int TJ_> struct TileT {
    static constexpr int HI = TI_ + 4, HJ = TJ_ + 4;
    float e[HI][HJ], f[HI][HJ], d[HI][HJ], ce[HI][HJ], cn[HI][HJ];
};

// Load f, d, ce, cn on the tile + 2-cell halo (out of domain: f 0, d 1,
// couplings 0).  Level 0 reads f from the FP64 residual.
template <bool L0, class TT>
__device__ __forceinline__ void load_tile(TT &T, const MgLevel &L, const double *__restrict__ r64, int i0, int j0) {
    constexpr int HI = TT::HI, HJ = TT::HJ;
    const int tid = threadIdx.x + blockDim.x * threadIdx.y, nt = blockDim.x * blockDim.y;
    for (int t = tid; t < HI * HJ; t += nt) {
        const int a = t / HJ, b = t % HJ;
        const int i = i0 - 2 + a, j = j0 - 2 + b;
        float f = 0.0f, d = 1.0f, ce = 0.0f, cn = 0.0f;
        if (i >= 0 && i < L.nx && j >= 0 && j < L.ny) {
            const int64_t k = LK(L, i, j);
            f = L0 ? (float)r64[k] : L.f[k];
            d = L.diag[k];
            ce = L.ce[k];
            cn = L.cn[k];
        }
        T.f[a][b] = f;
        T.d[a][b] = d;
        T.ce[a][b] = ce;
        T.cn[a][b] = cn;
    }
}

// Gauss-Seidel update of local cell (a, b) from its four neighbours.
template <class TT> __device__ __forceinline__ float gs_cell(const TT &T, int a, int b) {
    const float s = T.f[a][b] + T.ce[a - 1][b] * T.e[a - 1][b] + T.ce[a][b] * T.e[a + 1][b] +
                    T.cn[a][b - 1] * T.e[a][b - 1] + T.cn[a][b] * T.e[a][b + 1];
    return s / T.d[a][b];
}

// ------------------------------------------------------------ pre pass --
// From e = 0: red sweep on tile+2, black on tile+1, residual on the tile,
// restriction (2x2 sums) into the next level's f.  Stores e (tile).
template <bool L0, int TI_ = MT_I, int TJ_ = MT_J>
__device__ __forceinline__ void mg_pre_tile(const MgLevel &L, const MgLevel &C, const double *__restrict__ r64,
                                            int i0, int j0) {
    using TT = TileT<TI_, TJ_>;
    constexpr int HI = TT::HI, HJ = TT::HJ;
    __shared__ TT T;
    __shared__ float res[TI_][TJ_];
    load_tile<L0>(T, L, r64, i0, j0);
    __syncthreads();
    const int tid = threadIdx.x + blockDim.x * threadIdx.y, nt = blockDim.x * blockDim.y;
    // red (i+j even) on tile+2 from zero: e = f / d; black cells start at 0
    for (int t = tid; t < HI * HJ; t += nt) {
        const int a = t / HJ, b = t % HJ;
        const int i = i0 - 2 + a, j = j0 - 2 + b;
        T.e[a][b] = (((i + j) & 1) == 0) ? T.f[a][b] / T.d[a][b] : 0.0f;
    }
    __syncthreads();
    // black on tile+1
    for (int t = tid; t < (HI - 2) * (HJ - 2); t += nt) {
        const int a = 1 + t / (HJ - 2), b = 1 + t % (HJ - 2);
        const int i = i0 - 2 + a, j = j0 - 2 + b;
        if (((i + j) & 1) == 1) T.e[a][b] = gs_cell(T, a, b);
    }
    __syncthreads();
    // residual on the tile; store e
    for (int t = tid; t < TI_ * TJ_; t += nt) {
        const int a = 2 + t / TJ_, b = 2 + t % TJ_;
        const int i = i0 + t / TJ_, j = j0 + t % TJ_;
        float rr = 0.0f;
        if (i < L.nx && j < L.ny) {
            const float Ae = T.d[a][b] * T.e[a][b] - T.ce[a - 1][b] * T.e[a - 1][b] - T.ce[a][b] * T.e[a + 1][b] -
                             T.cn[a][b - 1] * T.e[a][b - 1] - T.cn[a][b] * T.e[a][b + 1];
            rr = T.f[a][b] - Ae;
            L.e[LK(L, i, j)] = T.e[a][b];
        }
        res[t / TJ_][t % TJ_] = rr;
    }
    __syncthreads();
    // restriction: coarse cells of this tile
    for (int t = tid; t < (TI_ / 2) * (TJ_ / 2); t += nt) {
        const int ci = t / (TJ_ / 2), cj = t % (TJ_ / 2);
        const int I = i0 / 2 + ci, J = j0 / 2 + cj;
        if (I < C.nx && J < C.ny)
            C.f[LK(C, I, J)] = res[2 * ci][2 * cj] + res[2 * ci + 1][2 * cj] + res[2 * ci][2 * cj + 1] +
                               res[2 * ci + 1][2 * cj + 1];
    }
}

template <bool L0, int TI_ = MT_I, int TJ_ = MT_J>
__global__ void __launch_bounds__(256) k_mg_pre(MgLevel L, MgLevel C, const double *__restrict__ r64,
                                                const KState *ks) {
    pdl_enter();
    if (ks->done || ks->skip_vc) return;
    mg_pre_tile<L0, TI_, TJ_>(L, C, r64, blockIdx.y * TI_, blockIdx.x * TJ_);
}

// ----------------------------------------------------------- post pass --
// e += omega * P ep_coarse on tile+2, black sweep on tile+1, red sweep on the
// tile; stores the result in ep.  The halo reads the pre-smoothed e of the
// neighbouring tiles, so the result goes to a separate array: an in-place
// store would race with neighbours still reading their halo.  Level 0
// instead writes z = (double) e (0 at the pinned cell) and reduces z.r and
// z.q into the FCG beta.
template <bool L0, int TI_ = MT_I, int TJ_ = MT_J>
__device__ __forceinline__ void mg_post_tile(const MgLevel &L, const MgLevel &C, float omega,
                                             const double *__restrict__ r64, const double *__restrict__ q64,
                                             double *__restrict__ z64, int pinned, int i0, int j0,
                                             double (&acc)[2]) {
    using TT = TileT<TI_, TJ_>;
    constexpr int HI = TT::HI, HJ = TT::HJ;
    __shared__ TT T;
    __shared__ float ec[TI_ / 2 + 2][TJ_ / 2 + 2];
    // the tile's global reads are issued before the first barrier: its
    // coefficients and rhs, the pre-smoothed e, the coarse correction
    const int tid = threadIdx.x + blockDim.x * threadIdx.y, nt = blockDim.x * blockDim.y;
    load_tile<L0>(T, L, r64, i0, j0);
    const int I0 = i0 / 2 - 1, J0 = j0 / 2 - 1;
    for (int t = tid; t < HI * HJ; t += nt) {
        const int a = t / HJ, b = t % HJ;
        const int i = i0 - 2 + a, j = j0 - 2 + b;
        T.e[a][b] = (i >= 0 && i < L.nx && j >= 0 && j < L.ny) ? L.e[LK(L, i, j)] : 0.0f;
    }
    for (int t = tid; t < (TI_ / 2 + 2) * (TJ_ / 2 + 2); t += nt) {
        const int a = t / (TJ_ / 2 + 2), b = t % (TJ_ / 2 + 2);
        const int I = I0 + a, J = J0 + b;
        ec[a][b] = (I >= 0 && I < C.nx && J >= 0 && J < C.ny) ? C.ep[LK(C, I, J)] : 0.0f;
    }
    __syncthreads();
    for (int t = tid; t < HI * HJ; t += nt) {
        const int a = t / HJ, b = t % HJ;
        const int i = i0 - 2 + a, j = j0 - 2 + b;
        if (i >= 0 && i < L.nx && j >= 0 && j < L.ny) T.e[a][b] += omega * ec[(i >> 1) - I0][(j >> 1) - J0];
    }
    __syncthreads();
    for (int t = tid; t < (HI - 2) * (HJ - 2); t += nt) {
        const int a = 1 + t / (HJ - 2), b = 1 + t % (HJ - 2);
        const int i = i0 - 2 + a, j = j0 - 2 + b;
        if (((i + j) & 1) == 1 && i >= 0 && i < L.nx && j >= 0 && j < L.ny) T.e[a][b] = gs_cell(T, a, b);
    }
    __syncthreads();
    acc[0] = acc[1] = 0.0;
    for (int t = tid; t < TI_ * TJ_; t += nt) {
        const int a = 2 + t / TJ_, b = 2 + t % TJ_;
        const int i = i0 + t / TJ_, j = j0 + t % TJ_;
        if (i < L.nx && j < L.ny) {
            float e = T.e[a][b];
            if (((i + j) & 1) == 0) e = gs_cell(T, a, b);
            const int64_t k = LK(L, i, j);
            if (L0) {
                const double z = (pinned && k == 0) ? 0.0 : (double)e;
                z64[k] = z;
                acc[0] += z * r64[k];
                acc[1] += z * q64[k];
            } else {
                L.ep[k] = e;
            }
        }
    }
}

// flexible CG: beta = z_{k+1}.(r_{k+1} - r_k) / (z_k.r_k), r_{k+1} - r_k = -alpha q_k
// (tot = {z.r, z.q} of the new z; thread 0 of the last block).
__device__ __forceinline__ void fcg_beta(KState *ks, const double (&tot)[2]) {
    if (ks->it == 0 || ks->restart) ks->beta = 0.0;
    else ks->beta = -ks->alpha * tot[1] / ks->rho;
    ks->restart = 0;
    ks->rho = tot[0];
    if (!(tot[0] > 0.0) && ks->it == 0 && ks->res > ks->tol) {
        ks->status = -6;
        ks->done = 1;
    }
}

template <bool L0, int TI_ = MT_I, int TJ_ = MT_J>
__global__ void __launch_bounds__(256) k_mg_post(MgLevel L, MgLevel C, float omega, const double *__restrict__ r64,
                                                 const double *__restrict__ q64, double *__restrict__ z64, int pinned,
                                                 KState *ks, double *partial) {
    pdl_enter();
    if (ks->done || ks->skip_vc) return;
    double acc[2];
    mg_post_tile<L0, TI_, TJ_>(L, C, omega, r64, q64, z64, pinned, blockIdx.y * TI_, blockIdx.x * TJ_, acc);
    if (L0) {
        double tot[2];
        // in the learned mode the V-cycle's z is only part of the preconditioner: beta comes later
        if (mg_grid_reduce<2>(acc, partial, &ks->counter, tot) && ks->mode != KMODE_LEARNED) fcg_beta(ks, tot);
    }
}

// ----------------------------------------------------------- coarsest --
// The coarsest level (<= MG_COARSE_MAX cells) is solved exactly: its dense
// inverse is formed once per assembly (Gauss-Jordan in FP64 in one CTA; the
// aggregated operator is SPD, so no pivoting is needed) and each V-cycle
// applies it as one small matrix-vector product.
// Augmented [A | I] of n x 2n doubles, row stride 2 * MG_COARSE_MAX; 32 x 32
// threads (ty: rows, tx: columns) eliminate each pivot step in parallel.
constexpr int MG_INV_THREADS = 1024;
__device__ __forceinline__ void mg_invert_body(const MgLevel &L, double *inv) {
    extern __shared__ double sm[];
    constexpr int W = 2 * MG_COARSE_MAX;
    double *M = sm, *col = sm + MG_COARSE_MAX * W;
    const int n = L.nx * L.ny, ny = L.ny, tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
    for (int r = ty; r < n; r += 32)
        for (int c = tx; c < 2 * n; c += 32) M[r * W + c] = (c == n + r) ? 1.0 : 0.0;
    __syncthreads();
    if (tid < n) {
        const int t = tid, i = t / ny, j = t % ny;
        M[t * W + t] = L.diag[t];
        if (i < L.nx - 1) M[t * W + t + ny] = M[(t + ny) * W + t] = -(double)L.ce[t];
        if (j < ny - 1) M[t * W + t + 1] = M[(t + 1) * W + t] = -(double)L.cn[t];
    }
    __syncthreads();
    for (int c = 0; c < n; c++) {
        const double rpiv = 1.0 / M[c * W + c];
        if (tid < n) col[tid] = M[tid * W + c];
        __syncthreads();
        if (tid < 2 * n) M[c * W + tid] *= rpiv;
        __syncthreads();
        for (int r = ty; r < n; r += 32) {
            if (r == c) continue;
            const double f = col[r];
            for (int t = tx; t < 2 * n; t += 32) M[r * W + t] -= f * M[c * W + t];
        }
        __syncthreads();
    }
    for (int r = ty; r < n; r += 32)
        for (int c = tx; c < n; c += 32) inv[r * MG_COARSE_MAX + c] = M[r * W + n + c];
}

__global__ void __launch_bounds__(MG_INV_THREADS) k_mg_coarse_invert(MgLevel L, double *inv) { mg_invert_body(L, inv); }

// ------------------------------------------------------ coarse V-cycle --
// Levels s .. nlev-1 (level s has at most MG_CTA_CELLS cells) in ONE CTA:
// every level's operator, restricted residual and correction live in shared
// memory, the sweeps are separated by __syncthreads instead of kernel
// boundaries, and the coarsest level is solved with its dense inverse.  Same
// sweeps as the tile kernels (red from zero, black; residual, 2x2
// restriction; descend; coarsest; prolongation with omega, black, red), so
// the preconditioner is the same.  Reads lv[s].f, writes lv[s].ep.
constexpr int MG_CTA_CELLS = 4096;
constexpr int MG_CTA_THREADS = 1024;

struct MgHier {
    MgLevel l[MG_MAX_LEVELS];
};

__host__ __device__ inline size_t mg_cta_smem(const MgHier &H, int s, int nlev) {
    size_t n = 0;
    for (int l = s; l < nlev; l++) n += 5 * (size_t)H.l[l].nx * H.l[l].ny;
    return n * sizeof(float);
}

__device__ __forceinline__ void mg_cta_body(const MgLevel *__restrict__ lv, int s, int nlev,
                                            const double *__restrict__ inv, float omega) {
    extern __shared__ float smf[];
    // 32 x 32 threads: ty walks rows i, tx columns j (no integer division)
    const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
    size_t off[MG_MAX_LEVELS];
    {
        size_t o = 0;
        for (int l = s; l < nlev; l++) {
            off[l] = o;
            o += 5 * (size_t)lv[l].nx * lv[l].ny;
        }
    }
    for (int l = s; l < nlev; l++) {
        const MgLevel &L = lv[l];
        const int n = L.nx * L.ny;
        float *D = smf + off[l], *CE = D + n, *CN = CE + n, *F = CN + n;
        for (int k = tid; k < n; k += MG_CTA_THREADS) {
            D[k] = L.diag[k];
            CE[k] = L.ce[k];
            CN[k] = L.cn[k];
            if (l == s) F[k] = L.f[k];
        }
    }
    __syncthreads();
    for (int l = s; l < nlev - 1; l++) {
        const int nx = lv[l].nx, ny = lv[l].ny, n = nx * ny;
        const float *D = smf + off[l], *CE = D + n, *CN = CE + n, *F = CN + n;
        float *E = smf + off[l] + 4 * (size_t)n;
        // red from zero (e = f / d) and black from those red values, in one
        // pass: a black cell evaluates its red neighbours' f / d itself
        for (int i = ty; i < nx; i += 32)
            for (int j = tx; j < ny; j += 32) {
                const int k = j + ny * i;
                if (((i + j) & 1) == 0) {
                    E[k] = F[k] / D[k];
                } else {
                    float acc = F[k];
                    if (i > 0) acc += CE[k - ny] * (F[k - ny] / D[k - ny]);
                    if (i < nx - 1) acc += CE[k] * (F[k + ny] / D[k + ny]);
                    if (j > 0) acc += CN[k - 1] * (F[k - 1] / D[k - 1]);
                    if (j < ny - 1) acc += CN[k] * (F[k + 1] / D[k + 1]);
                    E[k] = acc / D[k];
                }
            }
        __syncthreads();
        const int cnx = lv[l + 1].nx, cny = lv[l + 1].ny;
        float *Fc = smf + off[l + 1] + 3 * (size_t)cnx * cny;
        for (int I = ty; I < cnx; I += 32)
            for (int J = tx; J < cny; J += 32) {
                float sum = 0.0f;
#pragma unroll
                for (int a = 0; a < 2; a++)
#pragma unroll
                    for (int b = 0; b < 2; b++) {
                        const int i = 2 * I + a, j = 2 * J + b;
                        if (i >= nx || j >= ny) continue;
                        const int k = j + ny * i;
                        float Ae = D[k] * E[k];
                        if (i > 0) Ae -= CE[k - ny] * E[k - ny];
                        if (i < nx - 1) Ae -= CE[k] * E[k + ny];
                        if (j > 0) Ae -= CN[k - 1] * E[k - 1];
                        if (j < ny - 1) Ae -= CN[k] * E[k + 1];
                        sum += F[k] - Ae;
                    }
                Fc[J + cny * I] = sum;
            }
        __syncthreads();
    }
    {
        // e = inv f on the coarsest level (<= 64 cells): 16 lanes per row
        const int l = nlev - 1, n = lv[l].nx * lv[l].ny;
        const float *F = smf + off[l] + 3 * (size_t)n;
        float *E = smf + off[l] + 4 * (size_t)n;
        const int row = tid >> 4, c = tid & 15;
        double acc = 0.0;
        if (row < n)
#pragma unroll
            for (int q = 0; q < MG_COARSE_MAX / 16; q++)
                if (c + 16 * q < n) acc += inv[row * MG_COARSE_MAX + c + 16 * q] * (double)F[c + 16 * q];
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, 16);
        if (row < n && c == 0) E[row] = (float)acc;
        __syncthreads();
    }
    for (int l = nlev - 2; l >= s; l--) {
        const int nx = lv[l].nx, ny = lv[l].ny, n = nx * ny;
        const int cny = lv[l + 1].ny, cn = lv[l + 1].nx * cny;
        const float *D = smf + off[l], *CE = D + n, *CN = CE + n, *F = CN + n;
        float *E = smf + off[l] + 4 * (size_t)n;
        const float *Ec = smf + off[l + 1] + 4 * (size_t)cn;
        // prolongation fused into the black sweep: a black cell reads its red
        // neighbours as e + omega * e_coarse (its own old value is not used)
        auto pe = [&](int k, int i, int j) { return E[k] + omega * Ec[(j >> 1) + cny * (i >> 1)]; };
        for (int i = ty; i < nx; i += 32)
            for (int j = 2 * tx + ((i + 1) & 1); j < ny; j += 64) {
                // black cells: lane tx takes j = 2 tx + ((i + 1) & 1) + 64 m
                const int k = j + ny * i;
                float acc = F[k];
                if (i > 0) acc += CE[k - ny] * pe(k - ny, i - 1, j);
                if (i < nx - 1) acc += CE[k] * pe(k + ny, i + 1, j);
                if (j > 0) acc += CN[k - 1] * pe(k - 1, i, j - 1);
                if (j < ny - 1) acc += CN[k] * pe(k + 1, i, j + 1);
                E[k] = acc / D[k];
            }
        __syncthreads();
        for (int i = ty; i < nx; i += 32)
            for (int j = 2 * tx + (i & 1); j < ny; j += 64) {
                // red cells from the new black values
                const int k = j + ny * i;
                float acc = F[k];
                if (i > 0) acc += CE[k - ny] * E[k - ny];
                if (i < nx - 1) acc += CE[k] * E[k + ny];
                if (j > 0) acc += CN[k - 1] * E[k - 1];
                if (j < ny - 1) acc += CN[k] * E[k + 1];
                E[k] = acc / D[k];
            }
        __syncthreads();
    }
    const int n = lv[s].nx * lv[s].ny;
    const float *E = smf + off[s] + 4 * (size_t)n;
    for (int k = tid; k < n; k += MG_CTA_THREADS) lv[s].ep[k] = E[k];
}

__global__ void __launch_bounds__(MG_CTA_THREADS) k_mg_cta_cycle(MgHier H, int s, int nlev,
                                                                const double *__restrict__ inv, float omega,
                                                                const KState *ks) {
    pdl_enter();
    if (ks->done || ks->skip_vc) return;
    mg_cta_body(H.l, s, nlev, inv, omega);
}

// ------------------------------------------------------------ FCG FP64 --
// p = z + beta p_old (cell and neighbours), q = A p, partial p.q -> alpha
__global__ void __launch_bounds__(256) k_fcg_a(int nx, int ny, Sys S, const double *__restrict__ z,
                                               const double *__restrict__ p_old, double *__restrict__ p_new,
                                               double *__restrict__ q, KState *ks, double *partial) {
    pdl_enter();
    if (ks->done) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) ks->skip_vc = 0;
    const double beta = ks->beta;
    const int64_t n = (int64_t)nx * ny;
    double v[1] = {0.0};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int ii = (int)(k / ny), jj = (int)(k % ny);
        auto pv = [&](int64_t m) { return z[m] + beta * p_old[m]; };
        const double pc = pv(k);
        double y = 0.0;
        if (!(S.pinned && k == 0)) {
            if (jj > 0) y += -S.cn[k - 1] * pv(k - 1);
            if (ii > 0) y += -S.ce[k - ny] * pv(k - ny);
            y += S.diag[k] * pc;
            if (ii < nx - 1) y += -S.ce[k] * pv(k + ny);
            if (jj < ny - 1) y += -S.cn[k] * pv(k + 1);
        }
        p_new[k] = pc;
        q[k] = y;
        v[0] += pc * y;
    }
    double tot[1];
    if (mg_grid_reduce<1>(v, partial, &ks->counter, tot)) {
        if (!(tot[0] != 0.0) || !isfinite(tot[0])) {
            ks->status = -6;
            ks->done = 1;
        } else {
            ks->alpha = ks->rho / tot[0];
        }
    }
}

// x += alpha p, r -= alpha q, ||r|| -> convergence
__global__ void __launch_bounds__(256) k_fcg_b(int64_t n, double *__restrict__ x, double *__restrict__ r,
                                               const double *__restrict__ p, const double *__restrict__ q, KState *ks,
                                               double *partial) {
    pdl_enter();
    if (ks->done) return;
    const double alpha = ks->alpha;
    double v[1] = {0.0};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        x[k] += alpha * p[k];
        const double rk = r[k] - alpha * q[k];
        r[k] = rk;
        v[0] += rk * rk;
    }
    double tot[1];
    if (mg_grid_reduce<1>(v, partial, &ks->counter, tot)) {
        const int it = ks->it + 1;
        ks->it = it;
        ks->res = sqrt(tot[0]) / ks->bn;
        if (!isfinite(ks->res)) {
            ks->status = -5;
            ks->done = 1;
        } else if (!(ks->res > ks->tol) || it >= ks->maxit) {
            ks->done = 1;
        }
    }
}

// FP64 residual replacement.  Once the recurrence residual has met tol, r is
// recomputed as b - A x in FP64 (the recurrence drifts from it by rounding,
// by up to a few 1e-9 relative at density ratio 1000 on 1024^2 grids).  The
// solve ends when that residual meets tol, when maxit is reached, or when it
// has stagnated at FP64 rounding level (a replacement that did not halve the
// previous one: tol is below what FP64 can verify for this system);
// otherwise it resumes from x with the fresh r and a new direction (beta = 0).
__global__ void __launch_bounds__(256) k_fcg_replace(int nx, int ny, Sys S, const double *__restrict__ x,
                                                     double *__restrict__ r, KState *ks, double *partial) {
    pdl_enter();
    if (!ks->done) {  // mid-solve: nothing to replace, and the V-cycle after the check must not run
        if (blockIdx.x == 0 && threadIdx.x == 0) ks->skip_vc = 1;
        return;
    }
    if (ks->verified || ks->status != 0) return;
    const int64_t n = (int64_t)nx * ny;
    double v[1] = {0.0};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int ii = (int)(k / ny), jj = (int)(k % ny);
        double rk = 0.0;
        if (!(S.pinned && k == 0)) {
            double y = 0.0;
            if (jj > 0) y += -S.cn[k - 1] * x[k - 1];
            if (ii > 0) y += -S.ce[k - ny] * x[k - ny];
            y += S.diag[k] * x[k];
            if (ii < nx - 1) y += -S.ce[k] * x[k + ny];
            if (jj < ny - 1) y += -S.cn[k] * x[k + 1];
            rk = S.b[k] - y;
        }
        r[k] = rk;
        v[0] += rk * rk;
    }
    double tot[1];
    if (mg_grid_reduce<1>(v, partial, &ks->counter, tot)) {
        const double res = sqrt(tot[0]) / ks->bn;
        const double prev = ks->res_true_prev;
        ks->res = res;
        ks->res_true_prev = res;
        if (!isfinite(res)) {
            ks->status = -5;
            ks->verified = 1;
        } else if (!(res > ks->tol) || ks->it >= ks->maxit) {
            ks->verified = 1;
        } else if (prev >= 0.0 && res > 0.5 * prev) {
            ks->status = 2;  // stagnated at rounding level
            ks->verified = 1;
        } else {
            ks->done = 0;
            ks->restart = 1;
        }
    }
}

// r = b, x = 0, p = 0, ||b||; the first V-cycle follows.
__global__ void k_fcg_init(int64_t n, Sys S, double *__restrict__ x, double *__restrict__ r, double *__restrict__ p,
                           KState *ks, double *partial) {
    pdl_enter();
    double v[1] = {0.0};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const double bk = S.b[k];
        x[k] = 0.0;
        r[k] = bk;
        p[k] = 0.0;
        v[0] += bk * bk;
    }
    double tot[1];
    if (mg_grid_reduce<1>(v, partial, &ks->counter, tot)) {
        double bn = sqrt(tot[0]);
        if (bn == 0.0) bn = 1.0;
        ks->bn = bn;
        ks->res = sqrt(tot[0]) / bn;
        ks->it = 0;
        ks->status = 0;
        ks->alpha = 0.0;
        ks->verified = 0;
        ks->restart = 0;
        ks->res_true_prev = -1.0;
        ks->skip_vc = 0;
        ks->done = (!(ks->res > ks->tol) || ks->maxit <= 0) ? 1 : 0;
    }
}

// ------------------------------------------------------------ batched --
// The kernels below serve every instance of a batch in one launch: block b
// takes work-list entry b, reads that instance's descriptor and returns at
// entry once the instance has converged (every block of an instance sees the
// same flag: it only changes in the last block of a reduction, after all of
// them have arrived).  Per-instance sums use the instance's own partial slots
// and KState ticket, with block ids local to the instance.

__global__ void k_bmg_l0(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    const int64_t k0 = (int64_t)w.c * FCG_CHUNK;
    for (int t = threadIdx.x; t < FCG_CHUNK; t += blockDim.x)
        if (k0 + t < I.n) mg_l0_cell(I.g.nx, I.g.ny, I.S, I.lv[0], k0 + t);
}

__global__ void k_bmg_coarsen(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks, int l) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    const MgLevel &C = I.lv[l];
    const int64_t k0 = (int64_t)w.c * FCG_CHUNK, n = (int64_t)C.nx * C.ny;
    for (int t = threadIdx.x; t < FCG_CHUNK; t += blockDim.x)
        if (k0 + t < n) mg_coarsen_cell(I.lv[l - 1], C, k0 + t);
}

__global__ void __launch_bounds__(MG_INV_THREADS) k_bmg_invert(const BInst *__restrict__ insts) {
    const BInst &I = insts[blockIdx.x];
    mg_invert_body(I.lv[I.nlev - 1], I.coarse_inv);
}

__global__ void k_bset_kstate(const BInst *__restrict__ insts, int count, double tol, int maxit, int mode) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= count) return;
    KState *ks = insts[b].ks;
    ks->tol = tol;
    ks->maxit = maxit;
    ks->mode = mode;
    ks->fm_mask = 0;
    ks->reg = 0.0;
    ks->done = 0;
    ks->status = 0;
    ks->it = 0;
    ks->counter = 0u;
    ks->verified = 0;
    ks->restart = 0;
    ks->res_true_prev = -1.0;
    ks->skip_vc = 0;
}

__global__ void __launch_bounds__(256) k_bfcg_init(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    const int64_t n = I.n, k0 = (int64_t)w.c * FCG_CHUNK;
    const double *__restrict__ b = I.S.b;
    double *__restrict__ x = I.x;
    double *__restrict__ r = I.r;
    double *__restrict__ pa = I.pa;
    double *__restrict__ q = I.q;
    double v[1] = {0.0};
#pragma unroll
    for (int u = 0; u < FCG_CHUNK / 256; u++) {
        const int64_t k = k0 + threadIdx.x + 256 * u;
        if (k < n) {
            const double bk = b[k];
            x[k] = 0.0;
            r[k] = bk;
            pa[k] = 0.0;
            q[k] = 0.0;
            v[0] += bk * bk;
        }
    }
    double tot[1];
    KState *ks = I.ks;
    if (mg_reduce<1>(v, I.partial, &ks->counter, w.c, I.chunks, tot)) {
        double bn = sqrt(tot[0]);
        if (bn == 0.0) bn = 1.0;
        ks->bn = bn;
        ks->res = sqrt(tot[0]) / bn;
        ks->it = 0;
        ks->status = 0;
        ks->alpha = 0.0;
        ks->verified = 0;
        ks->restart = 0;
        ks->res_true_prev = -1.0;
        ks->done = (!(ks->res > ks->tol) || ks->maxit <= 0) ? 1 : 0;
    }
}

// (A x)_k of one instance's compact system (pinned row: 0)
__device__ __forceinline__ double sys_apply(const Sys &S, int nx, int ny, const double *__restrict__ x, int64_t k) {
    if (S.pinned && k == 0) return 0.0;
    const int ii = (int)(k / ny), jj = (int)(k % ny);
    double y = 0.0;
    if (jj > 0) y += -S.cn[k - 1] * x[k - 1];
    if (ii > 0) y += -S.ce[k - ny] * x[k - ny];
    y += S.diag[k] * x[k];
    if (ii < nx - 1) y += -S.ce[k] * x[k + ny];
    if (jj < ny - 1) y += -S.cn[k] * x[k + 1];
    return y;
}

// The batched kernels copy what they use of the instance descriptor into
// registers first: through a reference into global memory every store to a
// field would force the compiler to reload the descriptor's pointers.
__global__ void __launch_bounds__(256) k_bfcg_a(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks,
                                                int parity) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    KState *ks = I.ks;
    if (ks->done) return;
    if (w.c == 0 && threadIdx.x == 0) ks->skip_vc = 0;
    const double beta = ks->beta;
    const double *__restrict__ p_old = parity ? I.pb : I.pa;
    double *__restrict__ p_new = parity ? I.pa : I.pb;
    const double *__restrict__ z = I.z;
    const double *__restrict__ diag = I.S.diag;
    const double *__restrict__ ce = I.S.ce;
    const double *__restrict__ cn = I.S.cn;
    double *__restrict__ q = I.q;
    const int nx = I.g.nx, ny = I.g.ny, pinned = I.S.pinned;
    const int64_t n = I.n, k0 = (int64_t)w.c * FCG_CHUNK;
    double v[1] = {0.0};
#pragma unroll
    for (int u = 0; u < FCG_CHUNK / 256; u++) {
        const int64_t k = k0 + threadIdx.x + 256 * u;
        if (k < n) {
            const int ii = (int)(k / ny), jj = (int)(k % ny);
            auto pv = [&](int64_t m) { return z[m] + beta * p_old[m]; };
            const double pc = pv(k);
            double y = 0.0;
            if (!(pinned && k == 0)) {
                if (jj > 0) y += -cn[k - 1] * pv(k - 1);
                if (ii > 0) y += -ce[k - ny] * pv(k - ny);
                y += diag[k] * pc;
                if (ii < nx - 1) y += -ce[k] * pv(k + ny);
                if (jj < ny - 1) y += -cn[k] * pv(k + 1);
            }
            p_new[k] = pc;
            q[k] = y;
            v[0] += pc * y;
        }
    }
    double tot[1];
    if (mg_reduce<1>(v, I.partial, &ks->counter, w.c, I.chunks, tot)) {
        if (!(tot[0] != 0.0) || !isfinite(tot[0])) {
            ks->status = -6;
            ks->done = 1;
        } else {
            ks->alpha = ks->rho / tot[0];
        }
    }
}

__global__ void __launch_bounds__(256) k_bfcg_b(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks,
                                                int parity) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    KState *ks = I.ks;
    if (ks->done) return;
    const double alpha = ks->alpha;
    const double *__restrict__ p = parity ? I.pa : I.pb;
    const double *__restrict__ q = I.q;
    double *__restrict__ x = I.x;
    double *__restrict__ r = I.r;
    const int64_t n = I.n, k0 = (int64_t)w.c * FCG_CHUNK;
    double v[1] = {0.0};
#pragma unroll
    for (int u = 0; u < FCG_CHUNK / 256; u++) {
        const int64_t k = k0 + threadIdx.x + 256 * u;
        if (k < n) {
            x[k] += alpha * p[k];
            const double rk = r[k] - alpha * q[k];
            r[k] = rk;
            v[0] += rk * rk;
        }
    }
    double tot[1];
    if (mg_reduce<1>(v, I.partial, &ks->counter, w.c, I.chunks, tot)) {
        const int it = ks->it + 1;
        ks->it = it;
        ks->res = sqrt(tot[0]) / ks->bn;
        if (!isfinite(ks->res)) {
            ks->status = -5;
            ks->done = 1;
        } else if (!(ks->res > ks->tol) || it >= ks->maxit) {
            ks->done = 1;
        }
    }
}

// FP64 residual replacement with the single-system rules (k_fcg_replace).
__global__ void __launch_bounds__(256) k_bfcg_replace(const BInst *__restrict__ insts,
                                                      const BChunk *__restrict__ chunks) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    KState *ks = I.ks;
    if (!ks->done) {  // mid-solve: the V-cycle after the check must not run
        if (w.c == 0 && threadIdx.x == 0) ks->skip_vc = 1;
        return;
    }
    if (ks->verified || ks->status != 0) return;
    const Sys S = I.S;
    const int nx = I.g.nx, ny = I.g.ny;
    const double *__restrict__ x = I.x;
    double *__restrict__ r = I.r;
    const int64_t n = I.n, k0 = (int64_t)w.c * FCG_CHUNK;
    double v[1] = {0.0};
#pragma unroll
    for (int u = 0; u < FCG_CHUNK / 256; u++) {
        const int64_t k = k0 + threadIdx.x + 256 * u;
        if (k < n) {
            const double rk = (S.pinned && k == 0) ? 0.0 : S.b[k] - sys_apply(S, nx, ny, x, k);
            r[k] = rk;
            v[0] += rk * rk;
        }
    }
    double tot[1];
    if (mg_reduce<1>(v, I.partial, &ks->counter, w.c, I.chunks, tot)) {
        const double res = sqrt(tot[0]) / ks->bn;
        const double prev = ks->res_true_prev;
        ks->res = res;
        ks->res_true_prev = res;
        if (!isfinite(res)) {
            ks->status = -5;
            ks->verified = 1;
        } else if (!(res > ks->tol) || ks->it >= ks->maxit) {
            ks->verified = 1;
        } else if (prev >= 0.0 && res > 0.5 * prev) {
            ks->status = 2;
            ks->verified = 1;
        } else {
            ks->done = 0;
            ks->restart = 1;
        }
    }
}

// ------------------------------------- batched learned preconditioner --
// The two-level preconditioner of ASD2G_SOLVER_UNET (the single-system
// kernels k_pc_* / k_pcm_a below) for every instance of a batch: one launch
// per phase over the FCG chunks, per-instance sums with the instance's
// partial slots and ticket.  The network itself runs between these phases
// on the instances' feature planes, grouped by grid size.

// scal[0] = max |diag| of each instance (1 if zero): one CTA per instance
__global__ void __launch_bounds__(1024) k_bpc_diag_max(const BInst *__restrict__ insts) {
    const BInst &I = insts[blockIdx.x];
    const double *__restrict__ diag = I.S.diag;
    double v = 0.0;
    for (int64_t k = threadIdx.x; k < I.n; k += blockDim.x) v = fmax(v, fabs(diag[k]));
    __shared__ double sm[32];
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double mx = 0.0;
        for (int wi = 0; wi < (int)(blockDim.x >> 5); wi++) mx = fmax(mx, sm[wi]);
        I.pc_scal[0] = (float)(mx > 0.0 ? mx : 1.0);
    }
}

// feature channels 1..3: diag, ce, cn over the instance's scale
__global__ void __launch_bounds__(256) k_bpc_consts(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    const Sys S = I.S;
    float *__restrict__ f = I.pc_feats;
    const float is = 1.0f / I.pc_scal[0];
    const int64_t n = I.n, k0 = (int64_t)w.c * FCG_CHUNK;
#pragma unroll
    for (int u = 0; u < FCG_CHUNK / 256; u++) {
        const int64_t k = k0 + threadIdx.x + 256 * u;
        if (k < n) {
            f[4 * k + 1] = (float)S.diag[k] * is;
            f[4 * k + 2] = (float)S.ce[k] * is;
            f[4 * k + 3] = (float)S.cn[k] * is;
        }
    }
}

// r1 = r - A z (0 at the pinned row); |r1| -> ks->snorm
__global__ void __launch_bounds__(256) k_bpc_resid(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    KState *ks = I.ks;
    if (ks->done) return;
    const Sys S = I.S;
    const int nx = I.g.nx, ny = I.g.ny;
    const double *__restrict__ r = I.r;
    const double *__restrict__ z = I.z;
    double *__restrict__ r1 = I.pc_r1;
    const int64_t n = I.n, k0 = (int64_t)w.c * FCG_CHUNK;
    double v[1] = {0.0};
#pragma unroll
    for (int u = 0; u < FCG_CHUNK / 256; u++) {
        const int64_t k = k0 + threadIdx.x + 256 * u;
        if (k < n) {
            const double rk = (S.pinned && k == 0) ? 0.0 : r[k] - sys_apply(S, nx, ny, z, k);
            r1[k] = rk;
            v[0] += rk * rk;
        }
    }
    double tot[1];
    if (mg_reduce<1>(v, I.partial, &ks->counter, w.c, I.chunks, tot)) ks->snorm = sqrt(tot[0]);
}

// feature channel 0: r1 / rms(r1)
__global__ void __launch_bounds__(256) k_bpc_feat0(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    const KState *ks = I.ks;
    if (ks->done) return;
    const int64_t n = I.n, k0 = (int64_t)w.c * FCG_CHUNK;
    const double rms = ks->snorm / sqrt((double)n);
    const double inv = (rms > 0.0 && isfinite(rms)) ? 1.0 / rms : 0.0;
    const double *__restrict__ r1 = I.pc_r1;
    float *__restrict__ f = I.pc_feats;
#pragma unroll
    for (int u = 0; u < FCG_CHUNK / 256; u++) {
        const int64_t k = k0 + threadIdx.x + 256 * u;
        if (k < n) f[4 * k] = (float)(r1[k] * inv);
    }
}

// omega = (u . r1) / (u . A u) -> ks->omega (u: the network output, 0 at the pinned cell)
__global__ void __launch_bounds__(256) k_bpc_omega(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    KState *ks = I.ks;
    if (ks->done) return;
    const Sys S = I.S;
    const int nx = I.g.nx, ny = I.g.ny;
    const float *__restrict__ uo = I.pc_out;
    const double *__restrict__ r1 = I.pc_r1;
    auto U = [&](int64_t m) { return (S.pinned && m == 0) ? 0.0 : (double)uo[m]; };
    const int64_t n = I.n, k0 = (int64_t)w.c * FCG_CHUNK;
    double acc[2] = {0.0, 0.0};
#pragma unroll
    for (int u = 0; u < FCG_CHUNK / 256; u++) {
        const int64_t k = k0 + threadIdx.x + 256 * u;
        if (k < n) {
            double y = 0.0;
            if (!(S.pinned && k == 0)) {
                const int ii = (int)(k / ny), jj = (int)(k % ny);
                if (jj > 0) y += -S.cn[k - 1] * U(k - 1);
                if (ii > 0) y += -S.ce[k - ny] * U(k - ny);
                y += S.diag[k] * U(k);
                if (ii < nx - 1) y += -S.ce[k] * U(k + ny);
                if (jj < ny - 1) y += -S.cn[k] * U(k + 1);
            }
            const double uk = U(k);
            acc[0] += uk * r1[k];
            acc[1] += uk * y;
        }
    }
    double tot[2];
    if (mg_reduce<2>(acc, I.partial, &ks->counter, w.c, I.chunks, tot))
        ks->omega = (tot[1] > 0.0 && isfinite(tot[0] / tot[1])) ? tot[0] / tot[1] : 0.0;
}

// z += omega u (with_u) and the orthogonalisation coefficients of the valid
// direction slots from z . q_j (none at the first iteration or after a
// residual replacement)
__global__ void __launch_bounds__(256) k_bpc_final(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks,
                                                   int with_u) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    KState *ks = I.ks;
    if (ks->done || ks->skip_vc) return;
    const double om = with_u ? ks->omega : 0.0;
    const float *__restrict__ uo = I.pc_out;
    double *__restrict__ z = I.z;
    const FmDirs D = I.fm;
    const int pinned = I.S.pinned;
    const int64_t n = I.n, k0 = (int64_t)w.c * FCG_CHUNK;
    double acc[FM_SLOTS] = {};
#pragma unroll
    for (int u = 0; u < FCG_CHUNK / 256; u++) {
        const int64_t k = k0 + threadIdx.x + 256 * u;
        if (k < n) {
            const double zk = (pinned && k == 0) ? 0.0 : z[k] + (with_u ? om * (double)uo[k] : 0.0);
            z[k] = zk;
#pragma unroll
            for (int j = 0; j < FM_SLOTS; j++) acc[j] += zk * D.q[j][k];
        }
    }
    double tot[FM_SLOTS];
    if (mg_reduce<FM_SLOTS>(acc, I.partial, &ks->counter, w.c, I.chunks, tot)) {
        if (ks->it == 0 || ks->restart) {
            ks->fm_mask = 0;
            ks->restart = 0;
        }
        for (int j = 0; j < FM_SLOTS; j++)
            ks->fm_beta[j] = ((ks->fm_mask >> j) & 1) ? -tot[j] / ks->fm_pq[j] : 0.0;
    }
}

// p_w = z + sum over the other valid slots of beta_j p_j, q_w = A p_w;
// alpha = (p_w . r) / (p_w . q_w)
__global__ void __launch_bounds__(256) k_bpcm_a(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks,
                                                int wslot) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    KState *ks = I.ks;
    if (ks->done) return;
    if (w.c == 0 && threadIdx.x == 0) ks->skip_vc = 0;
    double b[FM_SLOTS];
#pragma unroll
    for (int j = 0; j < FM_SLOTS; j++) b[j] = j == wslot ? 0.0 : ks->fm_beta[j];
    const Sys S = I.S;
    const int nx = I.g.nx, ny = I.g.ny;
    const FmDirs D = I.fm;
    const double *__restrict__ z = I.z;
    const double *__restrict__ r = I.r;
    double *__restrict__ pw = D.p[wslot];
    double *__restrict__ qw = D.q[wslot];
    const int64_t n = I.n, k0 = (int64_t)w.c * FCG_CHUNK;
    auto pv = [&](int64_t m) {
        double v = z[m];
#pragma unroll
        for (int j = 0; j < FM_SLOTS; j++)
            if (j != wslot) v += b[j] * D.p[j][m];
        return v;
    };
    double acc[2] = {0.0, 0.0};
#pragma unroll
    for (int u = 0; u < FCG_CHUNK / 256; u++) {
        const int64_t k = k0 + threadIdx.x + 256 * u;
        if (k < n) {
            const int ii = (int)(k / ny), jj = (int)(k % ny);
            const double pc = pv(k);
            double y = 0.0;
            if (!(S.pinned && k == 0)) {
                if (jj > 0) y += -S.cn[k - 1] * pv(k - 1);
                if (ii > 0) y += -S.ce[k - ny] * pv(k - ny);
                y += S.diag[k] * pc;
                if (ii < nx - 1) y += -S.ce[k] * pv(k + ny);
                if (jj < ny - 1) y += -S.cn[k] * pv(k + 1);
            }
            pw[k] = pc;
            qw[k] = y;
            acc[0] += pc * y;
            acc[1] += pc * r[k];
        }
    }
    double tot[2];
    if (mg_reduce<2>(acc, I.partial, &ks->counter, w.c, I.chunks, tot)) {
        if (!(tot[0] > 0.0) || !isfinite(tot[0]) || !isfinite(tot[1])) {
            ks->status = -6;
            ks->done = 1;
        } else {
            ks->alpha = tot[1] / tot[0];
            ks->fm_pq[wslot] = tot[0];
            ks->fm_mask |= 1 << wslot;
        }
    }
}

// x += alpha p_w, r -= alpha q_w; |r| and the stopping test (k_bfcg_b on the slot's vectors)
__global__ void __launch_bounds__(256) k_bpcm_b(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks,
                                                int wslot) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    KState *ks = I.ks;
    if (ks->done) return;
    const double alpha = ks->alpha;
    const double *__restrict__ p = I.fm.p[wslot];
    const double *__restrict__ q = I.fm.q[wslot];
    double *__restrict__ x = I.x;
    double *__restrict__ r = I.r;
    const int64_t n = I.n, k0 = (int64_t)w.c * FCG_CHUNK;
    double v[1] = {0.0};
#pragma unroll
    for (int u = 0; u < FCG_CHUNK / 256; u++) {
        const int64_t k = k0 + threadIdx.x + 256 * u;
        if (k < n) {
            x[k] += alpha * p[k];
            const double rk = r[k] - alpha * q[k];
            r[k] = rk;
            v[0] += rk * rk;
        }
    }
    double tot[1];
    if (mg_reduce<1>(v, I.partial, &ks->counter, w.c, I.chunks, tot)) {
        const int it = ks->it + 1;
        ks->it = it;
        ks->res = sqrt(tot[0]) / ks->bn;
        if (!isfinite(ks->res)) {
            ks->status = -5;
            ks->done = 1;
        } else if (!(ks->res > ks->tol) || it >= ks->maxit) {
            ks->done = 1;
        }
    }
}

template <bool L0, int TI_, int TJ_>
__global__ void __launch_bounds__(256) k_bmg_pre(const BInst *__restrict__ insts, const BTile *__restrict__ tiles,
                                                 int l) {
    const BTile w = tiles[blockIdx.x];
    const BInst &I = insts[w.inst];
    if (I.ks->done || I.ks->skip_vc) return;
    mg_pre_tile<L0, TI_, TJ_>(I.lv[l], I.lv[l + 1], L0 ? I.r : nullptr, w.by * TI_, w.bx * TJ_);
}

__global__ void __launch_bounds__(MG_CTA_THREADS) k_bmg_cta(const BInst *__restrict__ insts, float omega) {
    const BInst &I = insts[blockIdx.x];
    if (I.ks->done || I.ks->skip_vc) return;
    mg_cta_body(I.lv, I.s_cta, I.nlev, I.coarse_inv, omega);
}

template <bool L0, int TI_, int TJ_>
__global__ void __launch_bounds__(256) k_bmg_post(const BInst *__restrict__ insts, const BTile *__restrict__ tiles,
                                                  int l, float omega) {
    const BTile w = tiles[blockIdx.x];
    const BInst &I = insts[w.inst];
    KState *ks = I.ks;
    if (ks->done || ks->skip_vc) return;
    double acc[2];
    mg_post_tile<L0, TI_, TJ_>(I.lv[l], I.lv[l + 1], omega, L0 ? I.r : nullptr, L0 ? I.q : nullptr,
                               L0 ? I.z : nullptr, I.S.pinned, w.by * TI_, w.bx * TJ_, acc);
    if (L0) {
        const int gx = (I.lv[0].ny + TJ_ - 1) / TJ_;
        double tot[2];
        if (mg_reduce<2>(acc, I.partial, &ks->counter, w.bx + gx * w.by, I.tiles0, tot) &&
            ks->mode != KMODE_LEARNED)
            fcg_beta(ks, tot);
    }
}

// ------------------------------------------------- learned preconditioner --
// Two-level preconditioner of ASD2G_SOLVER_UNET: the FP32 V-cycle gives z_mg
// (the coarse, global part); the network sees what it leaves, r1 = r - A
// z_mg, and returns u ~ A^-1 r1 up to scale; z = z_mg + omega u with omega
// minimising the A-norm of the error left along u (FP64).  scal[0] = s = max diag (coefficient
// scale of the features); |r1| in ks->snorm; omega in ks->omega.

__global__ void __launch_bounds__(256) k_pc_diag_max(int64_t n, const double *__restrict__ diag, double *partial,
                                                     unsigned *counter, float *scal) {
    double v = 0.0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        v = fmax(v, fabs(diag[k]));
    __shared__ double sm[256];
    sm[threadIdx.x] = v;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
        __syncthreads();
    }
    __shared__ bool last;
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = sm[0];
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double mx = 0.0;
    for (unsigned b = 0; b < gridDim.x; b++) mx = fmax(mx, __ldcg(partial + b));
    scal[0] = (float)(mx > 0.0 ? mx : 1.0);
    *counter = 0u;
}

// r1 = r - A z (0 at the pinned row); |r1| -> ks->snorm
__global__ void __launch_bounds__(256) k_pc_resid(int nx, int ny, Sys S, const double *__restrict__ r,
                                                  const double *__restrict__ z, double *__restrict__ r1, KState *ks,
                                                  double *partial) {
    if (ks->done) return;
    const int64_t n = (int64_t)nx * ny;
    double v[1] = {0.0};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const double rk = (S.pinned && k == 0) ? 0.0 : r[k] - sys_apply(S, nx, ny, z, k);
        r1[k] = rk;
        v[0] += rk * rk;
    }
    double tot[1];
    if (mg_grid_reduce<1>(v, partial, &ks->counter, tot)) ks->snorm = sqrt(tot[0]);
}

// feats [nx][ny][4]: channel 0 = r1 / rms(r1), channels 1..3 = diag, ce, cn
// over s (written when consts != 0).
__global__ void k_pc_features(int nx, int ny, Sys S, const double *__restrict__ r1, const KState *ks,
                              const float *__restrict__ scal, float *__restrict__ feats, int consts) {
    if (ks->done && !consts) return;
    const int64_t n = (int64_t)nx * ny;
    const double rms = ks->snorm / sqrt((double)n);
    const double inv = (rms > 0.0 && isfinite(rms)) ? 1.0 / rms : 0.0;
    const float is = 1.0f / scal[0];
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        if (!consts) feats[4 * k] = (float)(r1[k] * inv);
        else {
            feats[4 * k + 1] = (float)S.diag[k] * is;
            feats[4 * k + 2] = (float)S.ce[k] * is;
            feats[4 * k + 3] = (float)S.cn[k] * is;
        }
    }
}

// u: the network's FP32 output (0 at the pinned cell); omega =
// (u . r1) / (u . A u) -> ks->omega, the step that minimises the A-norm of
// the error left along u (A e1 = r1)
__global__ void __launch_bounds__(256) k_pc_omega(int nx, int ny, Sys S, const float *__restrict__ u,
                                                  const double *__restrict__ r1, KState *ks,
                                                  double *partial) {
    if (ks->done) return;
    const int64_t n = (int64_t)nx * ny;
    auto U = [&](int64_t m) { return (S.pinned && m == 0) ? 0.0 : (double)u[m]; };
    double acc[2] = {0.0, 0.0};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double y = 0.0;
        if (!(S.pinned && k == 0)) {
            const int ii = (int)(k / ny), jj = (int)(k % ny);
            if (jj > 0) y += -S.cn[k - 1] * U(k - 1);
            if (ii > 0) y += -S.ce[k - ny] * U(k - ny);
            y += S.diag[k] * U(k);
            if (ii < nx - 1) y += -S.ce[k] * U(k + ny);
            if (jj < ny - 1) y += -S.cn[k] * U(k + 1);
        }
        const double uk = U(k);
        acc[0] += uk * r1[k];
        acc[1] += uk * y;
    }
    double tot[2];
    if (mg_grid_reduce<2>(acc, partial, &ks->counter, tot))
        ks->omega = (tot[1] > 0.0 && isfinite(tot[0] / tot[1])) ? tot[0] / tot[1] : 0.0;
}

// z += omega u; z . q_j for every slot -> the orthogonalisation
// coefficients of the valid slots (none at the first iteration or after a
// residual replacement)
__global__ void __launch_bounds__(256) k_pc_final(int64_t n, const float *__restrict__ u, double *__restrict__ z,
                                                  FmDirs D, int pinned, KState *ks, double *partial) {
    if (ks->done || ks->skip_vc) return;
    const double om = u ? ks->omega : 0.0;  // u == nullptr: the V-cycle alone this iteration
    double acc[FM_SLOTS] = {};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const double zk = (pinned && k == 0) ? 0.0 : z[k] + (u ? om * (double)u[k] : 0.0);
        z[k] = zk;
#pragma unroll
        for (int j = 0; j < FM_SLOTS; j++) acc[j] += zk * D.q[j][k];
    }
    double tot[FM_SLOTS];
    if (mg_grid_reduce<FM_SLOTS>(acc, partial, &ks->counter, tot)) {
        if (ks->it == 0 || ks->restart) {
            ks->fm_mask = 0;
            ks->restart = 0;
        }
        for (int j = 0; j < FM_SLOTS; j++)
            ks->fm_beta[j] = ((ks->fm_mask >> j) & 1) ? -tot[j] / ks->fm_pq[j] : 0.0;
    }
}

// p_w = z + sum over the other valid slots of beta_j p_j, q_w = A p_w;
// alpha = (p_w . r) / (p_w . q_w)
__global__ void __launch_bounds__(256) k_pcm_a(int nx, int ny, Sys S, const double *__restrict__ z, FmDirs D, int w,
                                               const double *__restrict__ r, KState *ks, double *partial) {
    if (ks->done) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) ks->skip_vc = 0;
    double b[FM_SLOTS];
#pragma unroll
    for (int j = 0; j < FM_SLOTS; j++) b[j] = j == w ? 0.0 : ks->fm_beta[j];
    const int64_t n = (int64_t)nx * ny;
    double *__restrict__ pw = D.p[w];
    double *__restrict__ qw = D.q[w];
    double acc[2] = {0.0, 0.0};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int ii = (int)(k / ny), jj = (int)(k % ny);
        auto pv = [&](int64_t m) {
            double v = z[m];
#pragma unroll
            for (int j = 0; j < FM_SLOTS; j++)
                if (j != w) v += b[j] * D.p[j][m];
            return v;
        };
        const double pc = pv(k);
        double y = 0.0;
        if (!(S.pinned && k == 0)) {
            if (jj > 0) y += -S.cn[k - 1] * pv(k - 1);
            if (ii > 0) y += -S.ce[k - ny] * pv(k - ny);
            y += S.diag[k] * pc;
            if (ii < nx - 1) y += -S.ce[k] * pv(k + ny);
            if (jj < ny - 1) y += -S.cn[k] * pv(k + 1);
        }
        pw[k] = pc;
        qw[k] = y;
        acc[0] += pc * y;
        acc[1] += pc * r[k];
    }
    double tot[2];
    if (mg_grid_reduce<2>(acc, partial, &ks->counter, tot)) {
        if (!(tot[0] > 0.0) || !isfinite(tot[0]) || !isfinite(tot[1])) {
            ks->status = -6;
            ks->done = 1;
        } else {
            ks->alpha = tot[1] / tot[0];
            ks->fm_pq[w] = tot[0];
            ks->fm_mask |= 1 << w;
        }
    }
}

// Training pair: feats = (r1 / rms(r1), diag / s, ce / s, cn / s) with r1 =
// r - A V(r) for a residual r = b - A x0; target = e / rms(e) with e = x - x0
// - V(r), the error the network must supply (omega makes the output scale
// irrelevant).
__global__ void __launch_bounds__(256) k_pc_err(int64_t n, const double *__restrict__ x,
                                                const double *__restrict__ x0, const double *__restrict__ z,
                                                double *__restrict__ e, double *partial, unsigned *counter,
                                                float *scal) {
    double v[1] = {0.0};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const double d = x[k] - x0[k] - z[k];
        e[k] = d;
        v[0] += d * d;
    }
    double tot[1];
    if (mg_grid_reduce<1>(v, partial, counter, tot)) scal[2] = (float)tot[0];
}

__global__ void k_pc_pair(int nx, int ny, Sys S, const double *__restrict__ r1, const double *__restrict__ e,
                          const KState *ks, const float *__restrict__ scal, float *__restrict__ feats,
                          float *__restrict__ target) {
    const int64_t n = (int64_t)nx * ny;
    const double rr = ks->snorm / sqrt((double)n), inv = rr > 0.0 ? 1.0 / rr : 0.0;
    const double er = sqrt((double)scal[2] / (double)n), einv = er > 0.0 ? 1.0 / er : 0.0;
    const float is = 1.0f / scal[0];
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        feats[4 * k] = (float)(r1[k] * inv);
        feats[4 * k + 1] = (float)S.diag[k] * is;
        feats[4 * k + 2] = (float)S.ce[k] * is;
        feats[4 * k + 3] = (float)S.cn[k] * is;
        target[k] = (float)(e[k] * einv);
    }
}

}  // namespace

// ------------------------------------------------------------------ host --
int mg_levels_for(int nx, int ny, int *dims, int max_levels) {
    int n = 0, a = nx, b = ny;
    for (;;) {
        dims[2 * n] = a;
        dims[2 * n + 1] = b;
        n++;
        if ((int64_t)a * b <= MG_COARSE_MAX || n == max_levels) break;
        a = (a + 1) / 2;
        b = (b + 1) / 2;
    }
    return ((int64_t)a * b <= MG_COARSE_MAX) ? n : 0;
}

void launch_mg_setup(const Sys &S, MgLevel *lv, int nlev, double *coarse_inv, cudaStream_t st) {
    const int64_t n0 = (int64_t)lv[0].nx * lv[0].ny;
    k_mg_l0<<<red_blocks(n0), 256, 0, st>>>(lv[0].nx, lv[0].ny, S, lv[0]);
    for (int l = 1; l < nlev; l++) {
        const int64_t n = (int64_t)lv[l].nx * lv[l].ny;
        k_mg_coarsen<<<red_blocks(n), 256, 0, st>>>(lv[l - 1], lv[l]);
    }
    const size_t smem = sizeof(double) * (MG_COARSE_MAX * 2 * MG_COARSE_MAX + MG_COARSE_MAX);
    k_mg_coarse_invert<<<1, MG_INV_THREADS, smem, st>>>(lv[nlev - 1], coarse_inv);
}

template <int TI_ = MT_I, int TJ_ = MT_J> static dim3 tile_grid(const MgLevel &L) {
    return dim3((L.ny + TJ_ - 1) / TJ_, (L.nx + TI_ - 1) / TI_);
}

int64_t mg_partial_len(int nx, int ny) {
    const int64_t tiles = (int64_t)((ny + MT_J - 1) / MT_J) * ((nx + MT_I - 1) / MT_I);
    const int64_t a = 2 * tiles, b = (int64_t)FM_SLOTS * RED_BLOCKS_MAX;  // the widest grid-stride reduction
    return a > b ? a : b;
}

// First level handled by the single-CTA coarse cycle: the first level
// after level 0 with at most MG_CTA_CELLS cells.
static int mg_cta_level(const MgLevel *lv, int nlev) {
    int s = 1;
    while (s < nlev - 1 && (int64_t)lv[s].nx * lv[s].ny > MG_CTA_CELLS) s++;
    return s;
}

int mg_cta_first_level(const MgLevel *lv, int nlev) { return mg_cta_level(lv, nlev); }

// Shared memory of the coarse cycle: level s has at most 4096 cells and each
// coarser level at most half of the previous one plus one (a one-cell-wide
// level halves in one direction only), so 5 floats x 8192 cells = 160 KiB
// bounds every hierarchy; the kernel attribute is set to that bound (it is
// process-wide, so it must cover every session's hierarchy).
constexpr size_t MG_CTA_SMEM_BOUND = 5 * sizeof(float) * 2 * (size_t)MG_CTA_CELLS;
bool mg_cta_prepare(const MgLevel *lv, int nlev) {
    // process-wide attributes, set when a hierarchy is allocated (before any stream capture uses them)
    const size_t inv = sizeof(double) * (MG_COARSE_MAX * 2 * MG_COARSE_MAX + MG_COARSE_MAX);
    if (cudaFuncSetAttribute(k_mg_coarse_invert, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)inv) !=
        cudaSuccess)
        return false;
    MgHier H{};
    for (int l = 0; l < nlev; l++) H.l[l] = lv[l];
    if (mg_cta_smem(H, mg_cta_level(lv, nlev), nlev) > MG_CTA_SMEM_BOUND) return false;
    return cudaFuncSetAttribute(k_mg_cta_cycle, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)MG_CTA_SMEM_BOUND) == cudaSuccess;
}

// Over-correction of the coarse-grid correction (e += omega P e_c): 1.9
// unless ASD2G_MG_OMEGA in the environment gives another value in (0, 2.5].
static float mg_omega() {
    static const float w = [] {
        const char *e = std::getenv("ASD2G_MG_OMEGA");
        const float v = e ? (float)std::atof(e) : 1.9f;
        return v > 0.0f && v <= 2.5f ? v : 1.9f;
    }();
    return w;
}

float mg_omega_value() { return mg_omega(); }

// Launch with programmatic stream serialisation (see pdl_enter); ASD2G_PDL=0
// in the environment launches plainly (for comparisons).
static bool pdl_enabled() {
    static const bool on = [] {
        const char *e = std::getenv("ASD2G_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}
template <typename... P, typename... A>
static void pdl_launch(void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A... args) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    cudaLaunchKernelEx(&cfg, k, static_cast<P>(args)...);
}

template <int TI_, int TJ_>
static void enqueue_vcycle_t(MgLevel *lv, int nlev, const double *coarse_inv, const double *r, const double *q,
                             double *z, int pinned, KState *ks, double *partial, cudaStream_t st) {
    const dim3 blk(32, 8);
    const int s = mg_cta_level(lv, nlev);
    for (int l = 0; l < s; l++) {
        if (l == 0) pdl_launch(k_mg_pre<true, TI_, TJ_>, tile_grid<TI_, TJ_>(lv[0]), blk, 0, st, lv[0], lv[1], r, ks);
        else
            pdl_launch(k_mg_pre<false, TI_, TJ_>, tile_grid<TI_, TJ_>(lv[l]), blk, 0, st, lv[l], lv[l + 1],
                       (const double *)nullptr, ks);
    }
    MgHier H{};
    for (int l = 0; l < nlev; l++) H.l[l] = lv[l];
    const float omega = mg_omega();
    pdl_launch(k_mg_cta_cycle, dim3(1), dim3(MG_CTA_THREADS), mg_cta_smem(H, s, nlev), st, H, s, nlev, coarse_inv, omega,
               ks);
    for (int l = s - 1; l >= 0; l--) {
        if (l == 0)
            pdl_launch(k_mg_post<true, TI_, TJ_>, tile_grid<TI_, TJ_>(lv[0]), blk, 0, st, lv[0], lv[1], omega, r, q, z,
                       pinned, ks, partial);
        else
            pdl_launch(k_mg_post<false, TI_, TJ_>, tile_grid<TI_, TJ_>(lv[l]), blk, 0, st, lv[l], lv[l + 1], omega,
                       (const double *)nullptr, (const double *)nullptr, (double *)nullptr, 0, ks, partial);
    }
}

// One V-cycle: input r (FP64 level-0 rhs), output z (FP64), with the FCG
// beta update folded into the level-0 post pass.  Levels 0 .. s-1 run as
// tile kernels over the whole GPU (tiles of MG_SHAPES[lv[0].tile]), levels
// s .. nlev-1 in one CTA.
static void enqueue_vcycle(MgLevel *lv, int nlev, const double *coarse_inv, const double *r, const double *q,
                           double *z, int pinned, KState *ks, double *partial, cudaStream_t st) {
    switch (lv[0].tile) {
    case 1:
        enqueue_vcycle_t<MG_SHAPES[1][0], MG_SHAPES[1][1]>(lv, nlev, coarse_inv, r, q, z, pinned, ks, partial, st);
        break;
    case 2:
        enqueue_vcycle_t<MG_SHAPES[2][0], MG_SHAPES[2][1]>(lv, nlev, coarse_inv, r, q, z, pinned, ks, partial, st);
        break;
    default: enqueue_vcycle_t<MT_I, MT_J>(lv, nlev, coarse_inv, r, q, z, pinned, ks, partial, st); break;
    }
}

bool launch_fcg_init(const Sys &S, int nx, int ny, MgLevel *lv, int nlev, const double *coarse_inv, double *x,
                     double *r, double *p, double *q, double *z, KState *ks, double *partial, int64_t partial_len,
                     cudaStream_t st) {
    if (partial_len < mg_partial_len(nx, ny)) return false;
    const int64_t n = (int64_t)nx * ny;
    pdl_launch(k_fcg_init, dim3(red_blocks(n)), dim3(256), 0, st, n, S, x, r, p, ks, partial);
    cudaMemsetAsync(q, 0, sizeof(double) * n, st);
    enqueue_vcycle(lv, nlev, coarse_inv, r, q, z, S.pinned, ks, partial, st);
    return true;
}

bool launch_fcg_iter(const Sys &S, int nx, int ny, MgLevel *lv, int nlev, const double *coarse_inv, double *x,
                     double *r, const double *p_old, double *p_new, double *q, double *z, KState *ks,
                     double *partial, int64_t partial_len, cudaStream_t st) {
    if (partial_len < mg_partial_len(nx, ny)) return false;
    const int64_t n = (int64_t)nx * ny;
    const int nb = red_blocks(n);
    pdl_launch(k_fcg_a, dim3(nb), dim3(256), 0, st, nx, ny, S, (const double *)z, p_old, p_new, q, ks, partial);
    pdl_launch(k_fcg_b, dim3(nb), dim3(256), 0, st, n, x, r, (const double *)p_new, (const double *)q, ks, partial);
    enqueue_vcycle(lv, nlev, coarse_inv, r, q, z, S.pinned, ks, partial, st);
    return true;
}

bool launch_fcg_check(const Sys &S, int nx, int ny, MgLevel *lv, int nlev, const double *coarse_inv, const double *x,
                      double *r, const double *q, double *z, KState *ks, double *partial, int64_t partial_len,
                      cudaStream_t st) {
    if (partial_len < mg_partial_len(nx, ny)) return false;
    const int64_t n = (int64_t)nx * ny;
    pdl_launch(k_fcg_replace, dim3(red_blocks(n)), dim3(256), 0, st, nx, ny, S, x, r, ks, partial);
    enqueue_vcycle(lv, nlev, coarse_inv, r, q, z, S.pinned, ks, partial, st);
    return true;
}

// ---------------------------------------------------------- batched host --
int batch_tiles0(int nx, int ny) { return ((ny + MT_J - 1) / MT_J) * ((nx + MT_I - 1) / MT_I); }
static_assert(MG_SHAPES[0][0] == MT_I && MG_SHAPES[0][1] == MT_J, "shape 0 is the single-system tile");

int64_t batch_partial_len(int nx, int ny) {
    const int64_t chunks = ((int64_t)nx * ny + FCG_CHUNK - 1) / FCG_CHUNK;
    const int64_t a = 2 * (int64_t)batch_tiles0(nx, ny), b = (int64_t)FM_SLOTS * chunks;  // learned: 4 sums
    return a > b ? a : b;
}

bool batch_cta_prepare() {
    const size_t inv = sizeof(double) * (MG_COARSE_MAX * 2 * MG_COARSE_MAX + MG_COARSE_MAX);
    return cudaFuncSetAttribute(k_bmg_cta, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MG_CTA_SMEM_BOUND) ==
               cudaSuccess &&
           cudaFuncSetAttribute(k_bmg_invert, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)inv) == cudaSuccess;
}

void launch_batch_set_kstate(const BatchPlan &P, double tol, int maxit, cudaStream_t st, int mode) {
    k_bset_kstate<<<(P.count + 127) / 128, 128, 0, st>>>(P.insts, P.count, tol, maxit, mode);
}

void launch_batch_mg_setup(const BatchPlan &P, cudaStream_t st) {
    k_bmg_l0<<<P.nchunks, 256, 0, st>>>(P.insts, P.chunks);
    for (int l = 1; l < P.max_nlev; l++)
        if (P.nlvl_chunks[l] > 0) k_bmg_coarsen<<<P.nlvl_chunks[l], 256, 0, st>>>(P.insts, P.lvl_chunks[l], l);
    const size_t inv = sizeof(double) * (MG_COARSE_MAX * 2 * MG_COARSE_MAX + MG_COARSE_MAX);
    k_bmg_invert<<<P.count, MG_INV_THREADS, inv, st>>>(P.insts);
}

template <int TI_, int TJ_> static void batch_vcycle_t(const BatchPlan &P, cudaStream_t st) {
    const dim3 blk(32, 8);
    const float omega = mg_omega();
    for (int l = 0; l < P.max_s; l++) {
        if (P.nmg_tiles[l] == 0) continue;
        if (l == 0) k_bmg_pre<true, TI_, TJ_><<<P.nmg_tiles[0], blk, 0, st>>>(P.insts, P.mg_tiles[0], 0);
        else k_bmg_pre<false, TI_, TJ_><<<P.nmg_tiles[l], blk, 0, st>>>(P.insts, P.mg_tiles[l], l);
    }
    k_bmg_cta<<<P.count, MG_CTA_THREADS, MG_CTA_SMEM_BOUND, st>>>(P.insts, omega);
    for (int l = P.max_s - 1; l >= 0; l--) {
        if (P.nmg_tiles[l] == 0) continue;
        if (l == 0) k_bmg_post<true, TI_, TJ_><<<P.nmg_tiles[0], blk, 0, st>>>(P.insts, P.mg_tiles[0], 0, omega);
        else k_bmg_post<false, TI_, TJ_><<<P.nmg_tiles[l], blk, 0, st>>>(P.insts, P.mg_tiles[l], l, omega);
    }
}

static void batch_vcycle(const BatchPlan &P, cudaStream_t st) {
    switch (P.shape) {
    case 1: batch_vcycle_t<MG_SHAPES[1][0], MG_SHAPES[1][1]>(P, st); break;
    case 2: batch_vcycle_t<MG_SHAPES[2][0], MG_SHAPES[2][1]>(P, st); break;
    default: batch_vcycle_t<MG_SHAPES[0][0], MG_SHAPES[0][1]>(P, st); break;
    }
}

bool launch_batch_fcg_init(const BatchPlan &P, cudaStream_t st) {
    k_bfcg_init<<<P.nchunks, 256, 0, st>>>(P.insts, P.chunks);
    batch_vcycle(P, st);
    return true;
}

bool launch_batch_fcg_iter(const BatchPlan &P, int parity, cudaStream_t st) {
    k_bfcg_a<<<P.nchunks, 256, 0, st>>>(P.insts, P.chunks, parity);
    k_bfcg_b<<<P.nchunks, 256, 0, st>>>(P.insts, P.chunks, parity);
    batch_vcycle(P, st);
    return true;
}

bool launch_batch_fcg_check(const BatchPlan &P, cudaStream_t st) {
    k_bfcg_replace<<<P.nchunks, 256, 0, st>>>(P.insts, P.chunks);
    batch_vcycle(P, st);
    return true;
}

void launch_batch_pc_setup(const BatchPlan &P, cudaStream_t st) {
    k_bpc_diag_max<<<P.count, 1024, 0, st>>>(P.insts);
    k_bpc_consts<<<P.nchunks, 256, 0, st>>>(P.insts, P.chunks);
}

void launch_batch_pc_input(const BatchPlan &P, cudaStream_t st) {
    k_bpc_resid<<<P.nchunks, 256, 0, st>>>(P.insts, P.chunks);
    k_bpc_feat0<<<P.nchunks, 256, 0, st>>>(P.insts, P.chunks);
}

void launch_batch_pc_output(const BatchPlan &P, bool with_u, cudaStream_t st) {
    if (with_u) k_bpc_omega<<<P.nchunks, 256, 0, st>>>(P.insts, P.chunks);
    k_bpc_final<<<P.nchunks, 256, 0, st>>>(P.insts, P.chunks, with_u ? 1 : 0);
}

void launch_batch_pcm_iter(const BatchPlan &P, int wslot, cudaStream_t st) {
    k_bpcm_a<<<P.nchunks, 256, 0, st>>>(P.insts, P.chunks, wslot);
    k_bpcm_b<<<P.nchunks, 256, 0, st>>>(P.insts, P.chunks, wslot);
    batch_vcycle(P, st);
}

// ------------------------------------------------- learned preconditioner --
void launch_pc_setup(const Sys &S, int nx, int ny, float *feats, float *scal, double *partial, unsigned *counter,
                     const KState *ks, cudaStream_t st) {
    const int64_t n = (int64_t)nx * ny;
    const int nb = red_blocks(n);
    k_pc_diag_max<<<nb, 256, 0, st>>>(n, S.diag, partial, counter, scal);
    k_pc_features<<<nb, 256, 0, st>>>(nx, ny, S, nullptr, ks, scal, feats, 1);
}

void launch_pc_input(const Sys &S, int nx, int ny, const double *r, const double *z, double *r1, KState *ks,
                     const float *scal, float *feats, double *partial, cudaStream_t st) {
    const int nb = red_blocks((int64_t)nx * ny);
    k_pc_resid<<<nb, 256, 0, st>>>(nx, ny, S, r, z, r1, ks, partial);
    k_pc_features<<<nb, 256, 0, st>>>(nx, ny, S, r1, ks, scal, feats, 0);
}

void launch_pc_output(const Sys &S, int nx, int ny, const float *u, const double *r1, double *z, const FmDirs &D,
                      KState *ks, double *partial, cudaStream_t st) {
    const int64_t n = (int64_t)nx * ny;
    const int nb = red_blocks(n);
    if (u) k_pc_omega<<<nb, 256, 0, st>>>(nx, ny, S, u, r1, ks, partial);
    k_pc_final<<<nb, 256, 0, st>>>(n, u, z, D, S.pinned, ks, partial);
}

bool launch_pcm_iter(const Sys &S, int nx, int ny, MgLevel *lv, int nlev, const double *coarse_inv, double *x,
                     double *r, double *z, const FmDirs &D, int w, KState *ks, double *partial, int64_t partial_len,
                     cudaStream_t st) {
    if (partial_len < mg_partial_len(nx, ny) || w < 0 || w >= FM_SLOTS) return false;
    const int64_t n = (int64_t)nx * ny;
    const int nb = red_blocks(n);
    k_pcm_a<<<nb, 256, 0, st>>>(nx, ny, S, z, D, w, r, ks, partial);
    k_fcg_b<<<nb, 256, 0, st>>>(n, x, r, D.p[w], D.q[w], ks, partial);
    enqueue_vcycle(lv, nlev, coarse_inv, r, D.q[w], z, S.pinned, ks, partial, st);
    return true;
}

bool launch_pcm_check(const Sys &S, int nx, int ny, MgLevel *lv, int nlev, const double *coarse_inv, const double *x,
                      double *r, double *z, const FmDirs &D, KState *ks, double *partial, int64_t partial_len,
                      cudaStream_t st) {
    if (partial_len < mg_partial_len(nx, ny)) return false;
    const int64_t n = (int64_t)nx * ny;
    k_fcg_replace<<<red_blocks(n), 256, 0, st>>>(nx, ny, S, x, r, ks, partial);
    enqueue_vcycle(lv, nlev, coarse_inv, r, D.q[0], z, S.pinned, ks, partial, st);
    return true;
}

void launch_pc_pair(const Sys &S, int nx, int ny, const double *x, const double *x0, const double *z, const double *r1, double *e,
                    const KState *ks, float *scal, double *partial, unsigned *counter, float *feats, float *target,
                    cudaStream_t st) {
    const int64_t n = (int64_t)nx * ny;
    const int nb = red_blocks(n);
    k_pc_diag_max<<<nb, 256, 0, st>>>(n, S.diag, partial, counter, scal);
    k_pc_err<<<nb, 256, 0, st>>>(n, x, x0, z, e, partial, counter, scal);
    k_pc_pair<<<nb, 256, 0, st>>>(nx, ny, S, r1, e, ks, scal, feats, target);
}

}  // namespace asd2g
