// The whole multigrid-preconditioned flexible CG solve in ONE launch.
//
// Same method as the multi-kernel MG-FCG in mg.cu (FP64 flexible CG with
// Polak-Ribiere beta and FP64 residual replacement; preconditioner one FP32
// V(1,1)-cycle of Galerkin 2x2 aggregation with red-black Gauss-Seidel,
// over-relaxed prolongation and an exact coarsest solve), run by a
// cooperative grid of one CTA per 16 x 32 tile of the system with grid
// barriers between the phases that exchange data.
//
// Why: at 256^2 every multi-kernel phase is latency-bound (7 dependent
// launches of 7-11 us per iteration: launch gap, dependent L2 loads of the
// tile, grid reduction, the one-SM coarse cycle).  The smoothers multiply by
// stored reciprocal diagonals (the per-phase kernels divide), so the two
// paths agree to FP32 rounding of the V-cycle, not bit for bit.  Here each CTA keeps its
// tile's state resident (level-0 FP32 operator on the tile + 2 halo, the
// level-1 operator on its level-1 cells + 5, the level-2 operator on its
// level-2 cells + 6, every level from 3 down in full) and an iteration has
// five grid barriers:
//
//   A   p = z + beta p_old and q = A p on the tile + halo (FP64) -> p.q
//   --- barrier 1: alpha
//   B   r = r_old - alpha q on the tile + 2 (recomputed from the neighbours'
//       q, which each CTA computed itself), x += alpha p, r.r; level-0
//       pre-smoothing (red on the tile + 2, black on the tile + 1), residual,
//       restriction into level 1
//   --- barrier 2: convergence (FP64 residual replacement when met)
//   D   level-1 pre-smoothing on the CTA's level-1 cells + 5 (red on +5,
//       black on +4, so the pre-smoothed level-1 correction is right on +4
//       without a barrier), residual, restriction into level 2
//   --- barrier 3: level-2 right-hand side complete
//   D2  the same for level 2 on its level-2 cells + 6, restriction into
//       level 3
//   --- barrier 4: level-3 right-hand side complete
//   E   every CTA gathers the level-3 right-hand side and runs levels 3..
//       itself (redundantly: no barrier needed to share the result), then
//       the level-2 post-smoothing on its cells + 2, the level-1 one on its
//       cells + 1 and the level-0 one on its tile (the neighbours'
//       pre-smoothed level-0 correction read from global memory) -> z, z.r,
//       z.q
//   --- barrier 5: beta
//
// A value a CTA computes for a neighbour's cell (halo recomputation) uses the
// same inputs and the same code as the owner's, so it is the owner's value.
// Reductions: every CTA writes its block sum to a slot; after the barrier
// every CTA adds the slots in the same fixed order, so all CTAs hold the same
// scalars and take the same branches.  Data written by other CTAs during the
// launch is read with L2-only loads (ld.global.cg); the system itself is
// read-only for the launch.
//
// The grid barrier is a monotonic arrival counter (zeroed before the launch)
// with a bounded wait: after GRID_SPIN_LIMIT polls a CTA sets the error word and
// returns, every other CTA stops at its next barrier, the solve reports
// status -8 and the host solves the system with the multi-kernel path.
// The launch is cooperative (all CTAs co-resident) or is not made at all.
#include <cstdint>
#include <cstdlib>

#include "asd2g.h"
#include "gridsync.cuh"
#include "mg.cuh"

namespace asd2g {
namespace {

constexpr int PTI = 16, PTJ = 32;                      // level-0 tile (rows i x columns j)
constexpr int NT = PTI * PTJ;                          // threads: one per tile cell
constexpr int H3I = PTI + 6, H3J = PTJ + 6;            // tile + 3
constexpr int H2I = PTI + 4, H2J = PTJ + 4;            // tile + 2
constexpr int CMAX = 1800;                             // cells of levels 3.. (32^2 + 16^2 + 8^2 and odd sizes)
constexpr int NINV = MG_COARSE_CELLS;                  // coarsest level <= 64 cells
static_assert(NINV == 64, "the coarsest inverse works on 8 x 8 blocks of a 64 x 64 matrix");
constexpr int STATUS_BARRIER = -8;                     // KState.status when a barrier wait gave up

// A level distributed over the CTAs: the CTA's CI x CJ cells of it (the
// cells under its level-0 tile) plus a halo of H cells, recomputed rather
// than exchanged.  Pre-smoothing (red on +H, black on +(H-1)) makes the
// pre-smoothed correction right on +(H-1); the post-smoothing of a target
// region +T (prolongation on +(T+2), black on +(T+1), red on +T) needs it on
// +(T+2), so T + 2 <= H - 1.
template <int CI_, int CJ_, int H_> struct DLev {
    static constexpr int CI = CI_, CJ = CJ_, H = H_, RI = CI_ + 2 * H_, RJ = CJ_ + 2 * H_;
    float d[RI][RJ], di[RI][RJ], ce[RI][RJ], cn[RI][RJ], f[RI][RJ], e[RI][RJ];
    float res[CI_][CJ_];
};
using Lev1 = DLev<PTI / 2, PTJ / 2, 5>;  // post target +1 (what level-0 post-smoothing reads)
using Lev2 = DLev<PTI / 4, PTJ / 4, 6>;  // post target +2 (what level-1 post-smoothing reads)

struct Smem {
    double p[H3I][H3J];        // direction on the tile + 3
    double q[H2I][H2J];        // A p on the tile + 2
    double r[H2I][H2J];        // residual on the tile + 2
    double inv[NINV * NINV];   // coarsest inverse (row-major, stride NINV)
    double gj_row[8][NINV], gj_col[NINV][8], gj_q[8][NINV], gj_p[8][8];  // block Gauss-Jordan panels
    double red[4][NT / 32];    // per-warp partial sums
    double tot[4];             // reduced sums (the same in every CTA)
    float d0[H2I][H2J], di0[H2I][H2J], ce0[H2I][H2J], cn0[H2I][H2J], f0[H2I][H2J], e0[H2I][H2J];  // level 0
    float res0[PTI][PTJ];
    Lev1 l1;
    Lev2 l2;
    float co[6 * CMAX];        // levels 3..: d, ce, cn, f, e, 1/d of each level
    int flag;
};

struct PArgs {
    int nx, ny, ntj, ncta, nlev;
    int dims[2 * MG_MAX_LEVELS];
    int off[MG_MAX_LEVELS];  // offset (floats) of level l >= 3 in Smem::co
    Sys S;
    double *x, *rbuf0, *rbuf1, *pbuf0, *pbuf1, *z;
    float *e0g;                          // level-0 pre-smoothed correction
    float *lg[4][4];                     // levels 1..3: [l][0..3] = diag, ce, cn, f (global)
    double *partial;                     // 4 slots per CTA
    unsigned *bar;                       // [0] arrivals, [1] error word
    KState *ks;
    double tol;
    int maxit;
    float omega;
};

__device__ __forceinline__ bool gsync(const PArgs &A, Smem &sm, unsigned &epoch) {
    return grid_sync(A.bar, A.ncta, epoch, sm.flag);
}
template <int NV> __device__ __forceinline__ void put_partial(const PArgs &A, Smem &sm, double (&v)[NV]) {
    grid_put_partial<NV, NT>(A.partial, &sm.red[0][0], v);
}
template <int NV> __device__ __forceinline__ void get_total(const PArgs &A, Smem &sm) {
    grid_get_total<NV>(A.partial, A.ncta, sm.tot);
}

// Gauss-Seidel update of local cell (a, b) from its four neighbours (times
// the stored reciprocal of the diagonal).
template <int W> __device__ __forceinline__ float gs(const float (*f)[W], const float (*di)[W], const float (*ce)[W],
                                                     const float (*cn)[W], const float (*e)[W], int a, int b) {
    const float s = f[a][b] + ce[a - 1][b] * e[a - 1][b] + ce[a][b] * e[a + 1][b] + cn[a][b - 1] * e[a][b - 1] +
                    cn[a][b] * e[a][b + 1];
    return s * di[a][b];
}

// Galerkin 2x2 aggregation of one coarse cell (as mg_coarsen_cell in mg.cu)
// from a fine operator given by accessors.
template <class FD, class FE, class FN>
__device__ __forceinline__ void coarsen_cell(int fnx, int fny, int I, int J, FD fd, FE fe, FN fn, float &cd,
                                             float &cce, float &ccn) {
    const int i0 = 2 * I, j0 = 2 * J;
    const bool hi = i0 + 1 < fnx, hj = j0 + 1 < fny;
    float d = fd(i0, j0);
    if (hi) d += fd(i0 + 1, j0);
    if (hj) d += fd(i0, j0 + 1);
    if (hi && hj) d += fd(i0 + 1, j0 + 1);
    float inner = 0.0f;
    if (hi) inner += fe(i0, j0);
    if (hi && hj) inner += fe(i0, j0 + 1);
    if (hj) inner += fn(i0, j0);
    if (hi && hj) inner += fn(i0 + 1, j0);
    cd = d - 2.0f * inner;
    const int ie = hi ? i0 + 1 : i0, je = hj ? j0 + 1 : j0;
    float ce = fe(ie, j0);
    if (hj) ce += fe(ie, j0 + 1);
    float cn = fn(i0, je);
    if (hi) cn += fn(i0 + 1, je);
    cce = ce;
    ccn = cn;
}

// ---------------------------------------------------------------- level 0 --
// Pre-smoothing of level 0 from the FP64 residual on the tile + 2 (sm.r):
// red on +2 from zero, black on +1, residual on the tile; stores e0 (tile)
// and the restricted residual of the tile's level-1 cells.
__device__ void l0_pre(const PArgs &A, Smem &sm, int i0, int j0) {
    const int tid = threadIdx.x, nx = A.nx, ny = A.ny;
    for (int t = tid; t < H2I * H2J; t += NT) {
        const int a = t / H2J, b = t % H2J, i = i0 - 2 + a, j = j0 - 2 + b;
        const float f = (float)sm.r[a][b];
        sm.f0[a][b] = f;
        sm.e0[a][b] = (((i + j) & 1) == 0) ? f * sm.di0[a][b] : 0.0f;
    }
    __syncthreads();
    for (int t = tid; t < (H2I - 2) * (H2J - 2); t += NT) {
        const int a = 1 + t / (H2J - 2), b = 1 + t % (H2J - 2), i = i0 - 2 + a, j = j0 - 2 + b;
        if (((i + j) & 1) == 1) sm.e0[a][b] = gs<H2J>(sm.f0, sm.di0, sm.ce0, sm.cn0, sm.e0, a, b);
    }
    __syncthreads();
    {
        const int ta = tid / PTJ, tb = tid % PTJ, a = 2 + ta, b = 2 + tb, i = i0 + ta, j = j0 + tb;
        float rr = 0.0f;
        if (i < nx && j < ny) {
            const float Ae = sm.d0[a][b] * sm.e0[a][b] - sm.ce0[a - 1][b] * sm.e0[a - 1][b] -
                             sm.ce0[a][b] * sm.e0[a + 1][b] - sm.cn0[a][b - 1] * sm.e0[a][b - 1] -
                             sm.cn0[a][b] * sm.e0[a][b + 1];
            rr = sm.f0[a][b] - Ae;
            __stcg(A.e0g + (int64_t)j + (int64_t)ny * i, sm.e0[a][b]);
        }
        sm.res0[ta][tb] = rr;
    }
    __syncthreads();
    if (tid < (PTI / 2) * (PTJ / 2)) {
        const int ci = tid / (PTJ / 2), cj = tid % (PTJ / 2), I = i0 / 2 + ci, J = j0 / 2 + cj;
        const int n1x = A.dims[2], n1y = A.dims[3];
        if (I < n1x && J < n1y)
            __stcg(A.lg[1][3] + (int64_t)J + (int64_t)n1y * I, sm.res0[2 * ci][2 * cj] + sm.res0[2 * ci + 1][2 * cj] +
                                                                sm.res0[2 * ci][2 * cj + 1] +
                                                                sm.res0[2 * ci + 1][2 * cj + 1]);
    }
}

// ------------------------------------------------- distributed levels 1, 2 --
// Pre-smoothing of level l on the CTA's cells + H (tile origin I0, J0 in
// level-l cells): right-hand side from global memory, red on +H from zero,
// black on +(H-1), residual on the tile, restriction into the tile's level
// l+1 cells (global).
template <class L> __device__ void dist_pre(const PArgs &A, L &v, int l, int I0, int J0) {
    const int tid = threadIdx.x, nx = A.dims[2 * l], ny = A.dims[2 * l + 1];
    const float *fg = A.lg[l][3];
    for (int t = tid; t < L::RI * L::RJ; t += NT) {
        const int a = t / L::RJ, b = t % L::RJ, I = I0 - L::H + a, J = J0 - L::H + b;
        const bool in = I >= 0 && I < nx && J >= 0 && J < ny;
        const float f = in ? __ldcg(fg + (int64_t)J + (int64_t)ny * I) : 0.0f;
        v.f[a][b] = f;
        v.e[a][b] = (((I + J) & 1) == 0) ? f * v.di[a][b] : 0.0f;
    }
    __syncthreads();
    for (int t = tid; t < (L::RI - 2) * (L::RJ - 2); t += NT) {
        const int a = 1 + t / (L::RJ - 2), b = 1 + t % (L::RJ - 2), I = I0 - L::H + a, J = J0 - L::H + b;
        if (((I + J) & 1) == 1) v.e[a][b] = gs<L::RJ>(v.f, v.di, v.ce, v.cn, v.e, a, b);
    }
    __syncthreads();
    if (tid < L::CI * L::CJ) {
        const int ta = tid / L::CJ, tb = tid % L::CJ, a = L::H + ta, b = L::H + tb, I = I0 + ta, J = J0 + tb;
        float rr = 0.0f;
        if (I < nx && J < ny) {
            const float Ae = v.d[a][b] * v.e[a][b] - v.ce[a - 1][b] * v.e[a - 1][b] - v.ce[a][b] * v.e[a + 1][b] -
                             v.cn[a][b - 1] * v.e[a][b - 1] - v.cn[a][b] * v.e[a][b + 1];
            rr = v.f[a][b] - Ae;
        }
        v.res[ta][tb] = rr;
    }
    __syncthreads();
    if (tid < (L::CI / 2) * (L::CJ / 2)) {
        const int ci = tid / (L::CJ / 2), cj = tid % (L::CJ / 2), I = I0 / 2 + ci, J = J0 / 2 + cj;
        const int cnx = A.dims[2 * l + 2], cny = A.dims[2 * l + 3];
        if (I < cnx && J < cny)
            __stcg(A.lg[l + 1][3] + (int64_t)J + (int64_t)cny * I,
                   v.res[2 * ci][2 * cj] + v.res[2 * ci + 1][2 * cj] + v.res[2 * ci][2 * cj + 1] +
                       v.res[2 * ci + 1][2 * cj + 1]);
    }
}

// Post-smoothing of level l on the CTA's cells + T: prolongation of the
// coarse correction ec(I >> 1, J >> 1) with omega on +(T+2), black on +(T+1),
// red on +T, in v.e.
template <int T, class L, class EC> __device__ void dist_post(const PArgs &A, L &v, int l, int I0, int J0, EC ec) {
    static_assert(T + 2 <= L::H - 1, "the pre-smoothed correction must be right where it is prolonged");
    const int tid = threadIdx.x, nx = A.dims[2 * l], ny = A.dims[2 * l + 1];
    constexpr int P = L::H - T - 2;  // first local index of the +(T+2) region
    for (int t = tid; t < (L::RI - 2 * P) * (L::RJ - 2 * P); t += NT) {
        const int a = P + t / (L::RJ - 2 * P), b = P + t % (L::RJ - 2 * P), I = I0 - L::H + a, J = J0 - L::H + b;
        if (I >= 0 && I < nx && J >= 0 && J < ny) v.e[a][b] += A.omega * ec(I >> 1, J >> 1);
    }
    __syncthreads();
    for (int t = tid; t < (L::RI - 2 * P - 2) * (L::RJ - 2 * P - 2); t += NT) {
        const int a = P + 1 + t / (L::RJ - 2 * P - 2), b = P + 1 + t % (L::RJ - 2 * P - 2);
        const int I = I0 - L::H + a, J = J0 - L::H + b;
        if (((I + J) & 1) == 1 && I >= 0 && I < nx && J >= 0 && J < ny)
            v.e[a][b] = gs<L::RJ>(v.f, v.di, v.ce, v.cn, v.e, a, b);
    }
    __syncthreads();
    for (int t = tid; t < (L::RI - 2 * P - 4) * (L::RJ - 2 * P - 4); t += NT) {
        const int a = P + 2 + t / (L::RJ - 2 * P - 4), b = P + 2 + t % (L::RJ - 2 * P - 4);
        const int I = I0 - L::H + a, J = J0 - L::H + b;
        if (((I + J) & 1) == 0 && I >= 0 && I < nx && J >= 0 && J < ny)
            v.e[a][b] = gs<L::RJ>(v.f, v.di, v.ce, v.cn, v.e, a, b);
    }
    __syncthreads();
}

// ------------------------------------------------------ levels 3 .. nlev-1 --
// The coarse part of the V-cycle on the full levels held by this CTA (the
// same sweeps as k_mg_cta_cycle in mg.cu, red and black in separate passes):
// f of level 3 must be in place; leaves the corrected, post-smoothed level-3
// correction in its e.
__device__ void coarse_cycle(const PArgs &A, Smem &sm) {
    const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;  // 16 rows x 32 columns of threads
    constexpr int RS = NT / 32;
    const int nlev = A.nlev;
    const float omega = A.omega;
    for (int l = 3; l < nlev - 1; l++) {
        const int nx = A.dims[2 * l], ny = A.dims[2 * l + 1], n = nx * ny;
        const float *D = sm.co + A.off[l], *CE = D + n, *CN = CE + n, *F = CN + n, *DI = F + 2 * n;
        float *E = sm.co + A.off[l] + 4 * n;
        for (int i = ty; i < nx; i += RS)
            for (int j = tx; j < ny; j += 32) {
                const int k = j + ny * i;
                E[k] = (((i + j) & 1) == 0) ? F[k] * DI[k] : 0.0f;
            }
        __syncthreads();
        for (int i = ty; i < nx; i += RS)
            for (int j = 2 * tx + ((i + 1) & 1); j < ny; j += 64) {
                const int k = j + ny * i;
                float acc = F[k];
                if (i > 0) acc += CE[k - ny] * E[k - ny];
                if (i < nx - 1) acc += CE[k] * E[k + ny];
                if (j > 0) acc += CN[k - 1] * E[k - 1];
                if (j < ny - 1) acc += CN[k] * E[k + 1];
                E[k] = acc * DI[k];
            }
        __syncthreads();
        const int cnx = A.dims[2 * l + 2], cny = A.dims[2 * l + 3];
        float *Fc = sm.co + A.off[l + 1] + 3 * cnx * cny;
        for (int I = ty; I < cnx; I += RS)
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
        // coarsest: e = inv f, 8 lanes per row
        const int l = nlev - 1, n = A.dims[2 * l] * A.dims[2 * l + 1];
        const float *F = sm.co + A.off[l] + 3 * n;
        float *E = sm.co + A.off[l] + 4 * n;
        const int row = tid >> 3, c = tid & 7;
        double acc = 0.0;
        if (row < n)
#pragma unroll
            for (int qq = 0; qq < NINV / 8; qq++)
                if (c + 8 * qq < n) acc += sm.inv[row * NINV + c + 8 * qq] * (double)F[c + 8 * qq];
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, 8);
        if (row < n && c == 0) E[row] = (float)acc;
        __syncthreads();
    }
    for (int l = nlev - 2; l >= 3; l--) {
        const int nx = A.dims[2 * l], ny = A.dims[2 * l + 1], n = nx * ny;
        const int cny = A.dims[2 * l + 3], cn = A.dims[2 * l + 2] * cny;
        const float *D = sm.co + A.off[l], *CE = D + n, *CN = CE + n, *F = CN + n, *DI = F + 2 * n;
        float *E = sm.co + A.off[l] + 4 * n;
        const float *Ec = sm.co + A.off[l + 1] + 4 * cn;
        (void)D;
        for (int i = ty; i < nx; i += RS)
            for (int j = tx; j < ny; j += 32) {
                const int k = j + ny * i;
                E[k] += omega * Ec[(j >> 1) + cny * (i >> 1)];
            }
        __syncthreads();
        for (int pass = 1; pass >= 0; pass--) {  // black (i + j odd), then red
            for (int i = ty; i < nx; i += RS)
                for (int j = 2 * tx + ((i + pass) & 1); j < ny; j += 64) {
                    const int k = j + ny * i;
                    float acc = F[k];
                    if (i > 0) acc += CE[k - ny] * E[k - ny];
                    if (i < nx - 1) acc += CE[k] * E[k + ny];
                    if (j > 0) acc += CN[k - 1] * E[k - 1];
                    if (j < ny - 1) acc += CN[k] * E[k + 1];
                    E[k] = acc * DI[k];
                }
            __syncthreads();
        }
    }
}

// Post-smoothing of level 0 on the tile: the neighbours' pre-smoothed e0 on
// the tile + 2, prolongation of the level-1 correction (sm.l1.e on the
// level-1 tile + 1) with omega, black on +1, red on the tile -> z (FP64; 0 at
// the pinned cell) and the sums z.r, z.q of the tile.
__device__ void l0_post(const PArgs &A, Smem &sm, int i0, int j0, double (&acc)[2]) {
    const int tid = threadIdx.x, nx = A.nx, ny = A.ny, I0 = i0 / 2 - Lev1::H, J0 = j0 / 2 - Lev1::H;
    for (int t = tid; t < H2I * H2J; t += NT) {
        const int a = t / H2J, b = t % H2J, i = i0 - 2 + a, j = j0 - 2 + b;
        float e = 0.0f;
        if (i >= 0 && i < nx && j >= 0 && j < ny)
            e = __ldcg(A.e0g + (int64_t)j + (int64_t)ny * i) + A.omega * sm.l1.e[(i >> 1) - I0][(j >> 1) - J0];
        sm.e0[a][b] = e;
    }
    __syncthreads();
    for (int t = tid; t < (H2I - 2) * (H2J - 2); t += NT) {
        const int a = 1 + t / (H2J - 2), b = 1 + t % (H2J - 2), i = i0 - 2 + a, j = j0 - 2 + b;
        if (((i + j) & 1) == 1 && i >= 0 && i < nx && j >= 0 && j < ny)
            sm.e0[a][b] = gs<H2J>(sm.f0, sm.di0, sm.ce0, sm.cn0, sm.e0, a, b);
    }
    __syncthreads();
    acc[0] = acc[1] = 0.0;
    const int ta = tid / PTJ, tb = tid % PTJ, a = 2 + ta, b = 2 + tb, i = i0 + ta, j = j0 + tb;
    if (i < nx && j < ny) {
        float e = sm.e0[a][b];
        if (((i + j) & 1) == 0) e = gs<H2J>(sm.f0, sm.di0, sm.ce0, sm.cn0, sm.e0, a, b);
        const int64_t k = (int64_t)j + (int64_t)ny * i;
        const double z = (A.S.pinned && k == 0) ? 0.0 : (double)e;
        __stcg(A.z + k, z);
        acc[0] = z * sm.r[a][b];
        acc[1] = z * sm.q[a][b];
    }
}

// ------------------------------------------------------------------ set-up --
// Level-0 FP32 operator on the tile + 2 from the FP64 system; the tile's
// level-1 and level-2 operator cells (Galerkin) written to global memory.
__device__ void setup_local(const PArgs &A, Smem &sm, int i0, int j0) {
    const int tid = threadIdx.x, nx = A.nx, ny = A.ny;
    const Sys &S = A.S;
    for (int t = tid; t < H2I * H2J; t += NT) {
        const int a = t / H2J, b = t % H2J, i = i0 - 2 + a, j = j0 - 2 + b;
        float d = 1.0f, ce = 0.0f, cn = 0.0f;
        if (i >= 0 && i < nx && j >= 0 && j < ny) {
            const int64_t k = (int64_t)j + (int64_t)ny * i;
            const bool pin0 = S.pinned && k == 0;
            d = (float)S.diag[k];
            ce = (i < nx - 1 && !pin0) ? (float)S.ce[k] : 0.0f;
            cn = (j < ny - 1 && !pin0) ? (float)S.cn[k] : 0.0f;
        }
        sm.d0[a][b] = d;
        sm.di0[a][b] = 1.0f / d;
        sm.ce0[a][b] = ce;
        sm.cn0[a][b] = cn;
    }
    __syncthreads();
    // the tile's level-1 cells (into the middle of sm.l1), then its level-2 cells
    const int n1x = A.dims[2], n1y = A.dims[3];
    constexpr int H1 = Lev1::H;
    if (tid < Lev1::CI * Lev1::CJ) {
        const int ci = tid / Lev1::CJ, cj = tid % Lev1::CJ, I = i0 / 2 + ci, J = j0 / 2 + cj;
        float cd = 1.0f, cce = 0.0f, ccn = 0.0f;
        if (I < n1x && J < n1y) {
            auto fd = [&](int i, int j) { return sm.d0[i - i0 + 2][j - j0 + 2]; };
            auto fe = [&](int i, int j) { return sm.ce0[i - i0 + 2][j - j0 + 2]; };
            auto fn = [&](int i, int j) { return sm.cn0[i - i0 + 2][j - j0 + 2]; };
            coarsen_cell(nx, ny, I, J, fd, fe, fn, cd, cce, ccn);
            const int64_t k = (int64_t)J + (int64_t)n1y * I;
            __stcg(A.lg[1][0] + k, cd);
            __stcg(A.lg[1][1] + k, cce);
            __stcg(A.lg[1][2] + k, ccn);
        }
        sm.l1.d[H1 + ci][H1 + cj] = cd;
        sm.l1.ce[H1 + ci][H1 + cj] = cce;
        sm.l1.cn[H1 + ci][H1 + cj] = ccn;
    }
    __syncthreads();
    const int n2x = A.dims[4], n2y = A.dims[5];
    if (tid < Lev2::CI * Lev2::CJ) {
        const int ci = tid / Lev2::CJ, cj = tid % Lev2::CJ, I = i0 / 4 + ci, J = j0 / 4 + cj;
        if (I < n2x && J < n2y) {
            const int I0 = i0 / 2, J0 = j0 / 2;
            auto fd = [&](int i, int j) { return sm.l1.d[i - I0 + H1][j - J0 + H1]; };
            auto fe = [&](int i, int j) { return sm.l1.ce[i - I0 + H1][j - J0 + H1]; };
            auto fn = [&](int i, int j) { return sm.l1.cn[i - I0 + H1][j - J0 + H1]; };
            float cd, cce, ccn;
            coarsen_cell(n1x, n1y, I, J, fd, fe, fn, cd, cce, ccn);
            const int64_t k = (int64_t)J + (int64_t)n2y * I;
            __stcg(A.lg[2][0] + k, cd);
            __stcg(A.lg[2][1] + k, cce);
            __stcg(A.lg[2][2] + k, ccn);
        }
    }
}

// A distributed level's operator on the CTA's cells + H from global memory.
template <class L> __device__ void load_dist_op(const PArgs &A, L &v, int l, int I0, int J0) {
    const int nx = A.dims[2 * l], ny = A.dims[2 * l + 1];
    for (int t = threadIdx.x; t < L::RI * L::RJ; t += NT) {
        const int a = t / L::RJ, b = t % L::RJ, I = I0 - L::H + a, J = J0 - L::H + b;
        float d = 1.0f, ce = 0.0f, cn = 0.0f;
        if (I >= 0 && I < nx && J >= 0 && J < ny) {
            const int64_t k = (int64_t)J + (int64_t)ny * I;
            d = __ldcg(A.lg[l][0] + k);
            ce = __ldcg(A.lg[l][1] + k);
            cn = __ldcg(A.lg[l][2] + k);
        }
        v.d[a][b] = d;
        v.di[a][b] = 1.0f / d;
        v.ce[a][b] = ce;
        v.cn[a][b] = cn;
    }
}

// After the level-1/2 operators are complete: the CTA's parts of levels 1
// and 2, level 3 aggregated from the global level 2, and the coarser levels
// built here (all with reciprocal diagonals).
__device__ void setup_coarse(const PArgs &A, Smem &sm, int i0, int j0) {
    const int tid = threadIdx.x;
    load_dist_op(A, sm.l1, 1, i0 / 2, j0 / 2);
    load_dist_op(A, sm.l2, 2, i0 / 4, j0 / 4);
    for (int l = 3; l < A.nlev; l++) {
        const int fnx = A.dims[2 * l - 2], fny = A.dims[2 * l - 1], fn = fnx * fny;
        const int cny = A.dims[2 * l + 1], cn = A.dims[2 * l] * cny;
        float *D = sm.co + A.off[l], *CE = D + cn, *CN = CE + cn, *DI = CN + 3 * cn;
        for (int k = tid; k < cn; k += NT) {
            const int I = k / cny, J = k % cny;
            if (l == 3) {
                const float *FD = A.lg[2][0], *FE = A.lg[2][1], *FN = A.lg[2][2];
                auto fd = [&](int i, int j) { return __ldcg(FD + j + fny * i); };
                auto fe = [&](int i, int j) { return __ldcg(FE + j + fny * i); };
                auto fnn = [&](int i, int j) { return __ldcg(FN + j + fny * i); };
                coarsen_cell(fnx, fny, I, J, fd, fe, fnn, D[k], CE[k], CN[k]);
            } else {
                const float *FD = sm.co + A.off[l - 1], *FE = FD + fn, *FN = FE + fn;
                auto fd = [&](int i, int j) { return FD[j + fny * i]; };
                auto fe = [&](int i, int j) { return FE[j + fny * i]; };
                auto fnn = [&](int i, int j) { return FN[j + fny * i]; };
                coarsen_cell(fnx, fny, I, J, fd, fe, fnn, D[k], CE[k], CN[k]);
            }
            DI[k] = 1.0f / D[k];
        }
        __syncthreads();
    }
}

// 1/x in FP64: the hardware approximation refined by two Newton steps
// (each squares the relative error: 2^-20 -> 2^-40 -> below FP64 rounding).
__device__ __forceinline__ double recip64(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    r = fma(r, fma(-x, r, 1.0), r);
    return fma(r, fma(-x, r, 1.0), r);
}

// Dense inverse of the coarsest operator (SPD, <= 64 cells) in sm.inv,
// computed by every CTA: block Gauss-Jordan without pivoting in FP64 over
// 8 x 8 blocks of the matrix padded to 64 x 64 with the identity (the
// inverse of diag(A, I) is diag(A^-1, I)), so 8 sequential block steps
// instead of 64 scalar ones (each scalar step cost ~1600 cycles of
// dependent latency).  The matrix lives in registers: thread -> row
// tid >> 3, columns (tid & 7) + 8 m (one column in each block column m).
// Block step K with pivot block B = M_KK, P = B^-1:
//   M_KJ <- P M_KJ,  M_IJ <- M_IJ - M_IK P M_KJ,  M_IK <- -M_IK P,  M_KK <- P.
// P comes from an 8 x 8 Gauss-Jordan inside warp 0 (two entries per lane,
// shuffles), Q = P M_K* from all threads, then each thread's rank-8 update.
__device__ void coarsest_inverse(const PArgs &A, Smem &sm) {
    const int tid = threadIdx.x, l = A.nlev - 1, nx = A.dims[2 * l], ny = A.dims[2 * l + 1], n = nx * ny;
    const float *D = sm.co + A.off[l], *CE = D + n, *CN = CE + n;
    const int row = tid >> 3, c0 = tid & 7;
    double a[8];
#pragma unroll
    for (int m = 0; m < 8; m++) {
        const int c = c0 + 8 * m;
        double v = 0.0;
        if (row >= n || c >= n) {
            v = row == c ? 1.0 : 0.0;
        } else {
            const int lo = row < c ? row : c, hi = row < c ? c : row;
            if (c == row) v = D[row];
            else if (hi - lo == ny) v = -(double)CE[lo];
            else if (hi - lo == 1 && (hi % ny) != 0) v = -(double)CN[lo];
        }
        a[m] = v;
    }
    for (int K = 0; K < 8; K++) {
        // publish the pivot block row and this row's entries of block column K
        if ((row >> 3) == K)
#pragma unroll
            for (int m = 0; m < 8; m++) sm.gj_row[row & 7][8 * m + c0] = a[m];
#pragma unroll
        for (int m = 0; m < 8; m++)
            if (m == K) sm.gj_col[row][c0] = a[m];
        __syncthreads();
        if (tid < 32) {  // P = inverse of the pivot block, lane -> row r, columns cc, cc + 1
            const int lane = tid, r = lane >> 2, cc = 2 * (lane & 3);
            double p0 = sm.gj_row[r][8 * K + cc], p1 = sm.gj_row[r][8 * K + cc + 1];
            for (int t = 0; t < 8; t++) {
                const int src_piv = (t << 2) + (t >> 1), src_col = (r << 2) + (t >> 1), src_row = (t << 2) + (lane & 3);
                const double vt = (t & 1) ? p1 : p0;
                const double piv = __shfl_sync(0xffffffffu, vt, src_piv);
                const double f = __shfl_sync(0xffffffffu, vt, src_col);
                const double q0 = __shfl_sync(0xffffffffu, p0, src_row), q1 = __shfl_sync(0xffffffffu, p1, src_row);
                const double rp = recip64(piv);
                if (r == t) {
                    p0 = (cc == t) ? rp : q0 * rp;
                    p1 = (cc + 1 == t) ? rp : q1 * rp;
                } else {
                    p0 = (cc == t) ? -f * rp : p0 - f * (q0 * rp);
                    p1 = (cc + 1 == t) ? -f * rp : p1 - f * (q1 * rp);
                }
            }
            sm.gj_p[r][cc] = p0;
            sm.gj_p[r][cc + 1] = p1;
        }
        __syncthreads();
        {  // Q = P M_K* (the new pivot block row), thread -> (t, column)
            const int t = tid >> 6, col = tid & 63;
            double q = 0.0;
#pragma unroll
            for (int u = 0; u < 8; u++) q += sm.gj_p[t][u] * sm.gj_row[u][col];
            sm.gj_q[t][col] = q;
        }
        __syncthreads();
        if ((row >> 3) == K) {
#pragma unroll
            for (int m = 0; m < 8; m++) a[m] = (m == K) ? sm.gj_p[row & 7][c0] : sm.gj_q[row & 7][8 * m + c0];
        } else {
            double f[8];
#pragma unroll
            for (int t = 0; t < 8; t++) f[t] = sm.gj_col[row][t];
#pragma unroll
            for (int m = 0; m < 8; m++) {
                double acc = 0.0;
                if (m == K) {
#pragma unroll
                    for (int t = 0; t < 8; t++) acc -= f[t] * sm.gj_p[t][c0];
                    a[m] = acc;
                } else {
#pragma unroll
                    for (int t = 0; t < 8; t++) acc += f[t] * sm.gj_q[t][8 * m + c0];
                    a[m] -= acc;
                }
            }
        }
        __syncthreads();
    }
    if (row < n)
#pragma unroll
        for (int m = 0; m < 8; m++)
            if (c0 + 8 * m < n) sm.inv[row * NINV + c0 + 8 * m] = a[m];
    __syncthreads();
}

__global__ void __launch_bounds__(NT, 1) k_mgfcg_persist(PArgs A) {
    extern __shared__ __align__(16) unsigned char smraw[];
    Smem &sm = *reinterpret_cast<Smem *>(smraw);
    const int tid = threadIdx.x, nx = A.nx, ny = A.ny;
    const int ti = blockIdx.x / A.ntj, tj = blockIdx.x % A.ntj, i0 = ti * PTI, j0 = tj * PTJ;
    const int ta = tid / PTJ, tb = tid % PTJ, mi = i0 + ta, mj = j0 + tb;  // this thread's cell of the tile
    const bool mine = mi < nx && mj < ny;
    const int64_t mk = (int64_t)mj + (int64_t)ny * mi;
    const Sys &S = A.S;
    unsigned epoch = 0;
    double *rcur = A.rbuf0, *rnext = A.rbuf1, *pold = A.pbuf0, *pnew = A.pbuf1;

    // ---- set-up: x = 0, r = b, p = 0; operators of levels 0-2 ----
    double xk = 0.0;
    {
        double v[1] = {0.0};
        if (mine) {
            const double bk = S.b[mk];
            __stcg(rcur + mk, bk);
            __stcg(pold + mk, 0.0);
            v[0] = bk * bk;
        }
        setup_local(A, sm, i0, j0);
        put_partial<1>(A, sm, v);
    }
    bool ok = gsync(A, sm, epoch);
    double bn = 1.0, res = 0.0, rho = 0.0, alpha = 0.0, beta = 0.0, res_true_prev = -1.0;
    int it = 0, status = 0, restart = 0;
    bool done = true;
    if (ok) {
        get_total<1>(A, sm);
        const double bb = sm.tot[0];
        bn = sqrt(bb);
        if (bn == 0.0) bn = 1.0;
        res = sqrt(bb) / bn;
        done = !(res > A.tol) || A.maxit <= 0;
    }
    if (ok && !done) {
        setup_coarse(A, sm, i0, j0);
        coarsest_inverse(A, sm);
        {
            // the first V-cycle's right-hand side r = b on the tile + 2; q = 0
            for (int t = tid; t < H2I * H2J; t += NT) {
                const int a = t / H2J, b = t % H2J, i = i0 - 2 + a, j = j0 - 2 + b;
                sm.r[a][b] = (i >= 0 && i < nx && j >= 0 && j < ny) ? __ldcg(rcur + (int64_t)j + (int64_t)ny * i)
                                                                       : 0.0;
                sm.q[a][b] = 0.0;
            }
            __syncthreads();
            l0_pre(A, sm, i0, j0);
            ok = gsync(A, sm, epoch);  // level-1 rhs and level-0 e of the first V-cycle complete
        }
    }
    // ---- iterations: rest of the V-cycle (levels 1.., z, beta), then A, B ----
    while (ok && !done) {
        dist_pre(A, sm.l1, 1, i0 / 2, j0 / 2);
        ok = gsync(A, sm, epoch);  // level-2 rhs complete
        if (!ok) break;
        dist_pre(A, sm.l2, 2, i0 / 4, j0 / 4);
        ok = gsync(A, sm, epoch);  // level-3 rhs complete
        if (!ok) break;
        {
            const int n3 = A.dims[6] * A.dims[7];
            float *F3 = sm.co + A.off[3] + 3 * n3;
            for (int k = tid; k < n3; k += NT) F3[k] = __ldcg(A.lg[3][3] + k);
            __syncthreads();
        }
        coarse_cycle(A, sm);
        {
            const int n3x = A.dims[6], n3y = A.dims[7];
            const float *E3 = sm.co + A.off[3] + 4 * n3x * n3y;
            dist_post<2>(A, sm.l2, 2, i0 / 4, j0 / 4, [&](int I, int J) { return E3[J + n3y * I]; });
            const int I2 = i0 / 4 - Lev2::H, J2 = j0 / 4 - Lev2::H;
            dist_post<1>(A, sm.l1, 1, i0 / 2, j0 / 2, [&](int I, int J) { return sm.l2.e[I - I2][J - J2]; });
        }
        {
            double acc[2];
            l0_post(A, sm, i0, j0, acc);
            put_partial<2>(A, sm, acc);
        }
        ok = gsync(A, sm, epoch);  // z complete -> beta
        if (!ok) break;
        get_total<2>(A, sm);
        {
            const double zr = sm.tot[0], zq = sm.tot[1];
            beta = (it == 0 || restart) ? 0.0 : -alpha * zq / rho;
            restart = 0;
            rho = zr;
            if (!(zr > 0.0) && it == 0 && res > A.tol) {
                status = -6;
                break;
            }
        }
        // A: p = z + beta p_old and q = A p on the tile + halo, p.q
        for (int t = tid; t < H3I * H3J; t += NT) {
            const int a = t / H3J, b = t % H3J, i = i0 - 3 + a, j = j0 - 3 + b;
            double v = 0.0;
            if (i >= 0 && i < nx && j >= 0 && j < ny) {
                const int64_t k = (int64_t)j + (int64_t)ny * i;
                v = __ldcg(A.z + k) + beta * __ldcg(pold + k);
            }
            sm.p[a][b] = v;
        }
        __syncthreads();
        for (int t = tid; t < H2I * H2J; t += NT) {
            const int a = t / H2J, b = t % H2J, i = i0 - 2 + a, j = j0 - 2 + b, ha = a + 1, hb = b + 1;
            double y = 0.0;
            if (i >= 0 && i < nx && j >= 0 && j < ny) {
                const int64_t k = (int64_t)j + (int64_t)ny * i;
                if (!(S.pinned && k == 0)) {
                    if (j > 0) y += -__ldg(S.cn + k - 1) * sm.p[ha][hb - 1];
                    if (i > 0) y += -__ldg(S.ce + k - ny) * sm.p[ha - 1][hb];
                    y += __ldg(S.diag + k) * sm.p[ha][hb];
                    if (i < nx - 1) y += -__ldg(S.ce + k) * sm.p[ha + 1][hb];
                    if (j < ny - 1) y += -__ldg(S.cn + k) * sm.p[ha][hb + 1];
                }
            }
            sm.q[a][b] = y;
        }
        __syncthreads();
        {
            double pq[1] = {0.0};
            if (mine) {
                __stcg(pnew + mk, sm.p[3 + ta][3 + tb]);
                pq[0] = sm.p[3 + ta][3 + tb] * sm.q[2 + ta][2 + tb];
            }
            put_partial<1>(A, sm, pq);
        }
        ok = gsync(A, sm, epoch);  // p.q -> alpha
        if (!ok) break;
        get_total<1>(A, sm);
        {
            const double t = sm.tot[0];
            if (!(t != 0.0) || !isfinite(t)) {
                status = -6;
                break;
            }
            alpha = rho / t;
        }
        // B: r and x updates, r.r, level-0 pre-smoothing of the new r
        for (int t = tid; t < H2I * H2J; t += NT) {
            const int a = t / H2J, b = t % H2J, i = i0 - 2 + a, j = j0 - 2 + b;
            double v = 0.0;
            if (i >= 0 && i < nx && j >= 0 && j < ny)
                v = __ldcg(rcur + (int64_t)j + (int64_t)ny * i) - alpha * sm.q[a][b];
            sm.r[a][b] = v;
        }
        __syncthreads();
        {
            double rr[1] = {0.0};
            if (mine) {
                xk += alpha * sm.p[3 + ta][3 + tb];
                const double rk = sm.r[2 + ta][2 + tb];
                __stcg(rnext + mk, rk);
                rr[0] = rk * rk;
            }
            put_partial<1>(A, sm, rr);
        }
        l0_pre(A, sm, i0, j0);
        {
            double *tp = rcur;
            rcur = rnext;
            rnext = tp;
            tp = pold;
            pold = pnew;
            pnew = tp;
        }
        ok = gsync(A, sm, epoch);  // r.r; level-1 rhs and level-0 e complete
        if (!ok) break;
        get_total<1>(A, sm);
        it++;
        res = sqrt(sm.tot[0]) / bn;
        if (!isfinite(res)) {
            status = -5;
            break;
        }
        if (res > A.tol && it < A.maxit) continue;
        // FP64 residual replacement: r = b - A x, judged in FP64
        if (mine) __stcg(A.x + mk, xk);
        ok = gsync(A, sm, epoch);
        if (!ok) break;
        {
            double tr[1] = {0.0};
            if (mine) {
                double rk = 0.0;
                if (!(S.pinned && mk == 0)) {
                    double y = 0.0;
                    if (mj > 0) y += -S.cn[mk - 1] * __ldcg(A.x + mk - 1);
                    if (mi > 0) y += -S.ce[mk - ny] * __ldcg(A.x + mk - ny);
                    y += S.diag[mk] * xk;
                    if (mi < nx - 1) y += -S.ce[mk] * __ldcg(A.x + mk + ny);
                    if (mj < ny - 1) y += -S.cn[mk] * __ldcg(A.x + mk + 1);
                    rk = S.b[mk] - y;
                }
                __stcg(rcur + mk, rk);
                tr[0] = rk * rk;
            }
            put_partial<1>(A, sm, tr);
        }
        ok = gsync(A, sm, epoch);
        if (!ok) break;
        get_total<1>(A, sm);
        {
            const double rt = sqrt(sm.tot[0]) / bn, prev = res_true_prev;
            res = rt;
            res_true_prev = rt;
            if (!isfinite(rt)) {
                status = -5;
                break;
            }
            if (!(rt > A.tol) || it >= A.maxit) break;
            if (prev >= 0.0 && rt > 0.5 * prev) {
                status = 2;  // stagnated at rounding level
                break;
            }
        }
        // resume from x with the replaced r and a new direction
        restart = 1;
        for (int t = tid; t < H2I * H2J; t += NT) {
            const int a = t / H2J, b = t % H2J, i = i0 - 2 + a, j = j0 - 2 + b;
            sm.r[a][b] = (i >= 0 && i < nx && j >= 0 && j < ny) ? __ldcg(rcur + (int64_t)j + (int64_t)ny * i) : 0.0;
        }
        __syncthreads();
        l0_pre(A, sm, i0, j0);
        ok = gsync(A, sm, epoch);  // level-1 rhs and level-0 e complete
    }
    if (mine) __stcg(A.x + mk, xk);
    if (blockIdx.x == 0 && tid == 0) {
        KState *ks = A.ks;
        ks->it = it;
        ks->res = res;
        ks->status = ok ? status : STATUS_BARRIER;
        ks->done = 1;
        ks->verified = 1;
        ks->rho = rho;
        ks->bn = bn;
        ks->alpha = alpha;
        ks->beta = beta;
    }
}

}  // namespace

// ------------------------------------------------------------------ host --
static bool persist_shape(const MgLevel *lv, int nlev, int nx, int ny, PArgs &A) {
    if (nlev < 4 || nlev > MG_MAX_LEVELS) return false;
    const int nti = (nx + PTI - 1) / PTI, ntj = (ny + PTJ - 1) / PTJ;
    A.nx = nx;
    A.ny = ny;
    A.ntj = ntj;
    A.ncta = nti * ntj;
    A.nlev = nlev;
    int off = 0;
    for (int l = 0; l < nlev; l++) {
        A.dims[2 * l] = lv[l].nx;
        A.dims[2 * l + 1] = lv[l].ny;
        A.off[l] = 0;
        if (l >= 3) {
            A.off[l] = off;
            off += 6 * lv[l].nx * lv[l].ny;
        }
        if (l >= 1 && (lv[l].nx != (lv[l - 1].nx + 1) / 2 || lv[l].ny != (lv[l - 1].ny + 1) / 2)) return false;
    }
    const int last = lv[nlev - 1].nx * lv[nlev - 1].ny;
    return off <= 6 * CMAX && last <= NINV;
}

bool mg_persist_enabled() {
    static const bool on = [] {
        const char *e = std::getenv("ASD2G_MG_PERSIST");
        return !(e && e[0] == '0');
    }();
    return on;
}

bool mg_persist_prepare() {
    static int smem_set = -1;  // the attribute is process-wide: set once, outside any capture
    if (smem_set < 0) {
        smem_set = cudaFuncSetAttribute(k_mgfcg_persist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sizeof(Smem)) == cudaSuccess
                       ? 1
                       : 0;
        if (!smem_set) cudaGetLastError();
    }
    return smem_set == 1;
}

static bool persist_fits(const MgLevel *lv, int nlev, int nx, int ny, int64_t partial_len, PArgs &A) {
    if (!persist_shape(lv, nlev, nx, ny, A) || partial_len < 4 * (int64_t)A.ncta || !mg_persist_prepare())
        return false;
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mgfcg_persist, NT, sizeof(Smem)) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (int64_t)per_sm * sms >= A.ncta;
}

bool mg_persist_fits(const MgLevel *lv, int nlev, int nx, int ny, int64_t partial_len) {
    PArgs A{};
    return persist_fits(lv, nlev, nx, ny, partial_len, A);
}

bool launch_mg_persist(const Sys &S, int nx, int ny, const MgLevel *lv, int nlev, double *x, double *r0, double *r1,
                       double *p0, double *p1, double *z, double *partial, int64_t partial_len,
                       unsigned *bar, KState *ks, double tol, int maxit, float omega, cudaStream_t st) {
    PArgs A{};
    if (!persist_fits(lv, nlev, nx, ny, partial_len, A)) return false;
    const size_t smem = sizeof(Smem);
    A.S = S;
    A.x = x;
    A.rbuf0 = r0;
    A.rbuf1 = r1;
    A.pbuf0 = p0;
    A.pbuf1 = p1;
    A.z = z;
    A.e0g = lv[0].e;
    for (int l = 1; l <= 3; l++) {
        A.lg[l][0] = lv[l].diag;
        A.lg[l][1] = lv[l].ce;
        A.lg[l][2] = lv[l].cn;
        A.lg[l][3] = lv[l].f;
    }
    A.partial = partial;
    A.bar = bar;
    A.ks = ks;
    A.tol = tol;
    A.maxit = maxit;
    A.omega = omega;
    if (cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), st) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    void *args[] = {&A};
    if (cudaLaunchCooperativeKernel((const void *)k_mgfcg_persist, dim3(A.ncta), dim3(NT), args, smem, st) !=
        cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}

size_t mg_persist_smem() { return sizeof(Smem); }

}  // namespace asd2g
