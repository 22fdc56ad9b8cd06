// Level-set kernels in FP64 (the bit-exact path, built with -fmad=false):
// the templated stencils of levelset_impl.cuh instantiated for double, the
// reinitialisation driver and the building-block kernels of the ABI.
#include <type_traits>

#include "levelset_impl.cuh"
#include "batch.cuh"

namespace asd2g {

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
    k_center_vel<double><<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, u, v, tu, tv);
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
    case 0: k_ls_stage<0, double><<<grd, blk, 0, st>>>(g, ddx, ddy, phi_in, tu, tv, phi_n, out, dt); break;
    case 1: k_ls_stage<1, double><<<grd, blk, 0, st>>>(g, ddx, ddy, phi_in, tu, tv, phi_n, out, dt); break;
    case 2: k_ls_stage<2, double><<<grd, blk, 0, st>>>(g, ddx, ddy, phi_in, tu, tv, phi_n, out, dt); break;
    default: k_ls_stage<3, double><<<grd, blk, 0, st>>>(g, ddx, ddy, phi_in, tu, tv, phi_n, out, dt); break;
    }
    if (stage != 0 && !g.p_mirror) launch_fill_p(g, out, st);
}

template <int MODE>
static void reinit_a(const Grid &g, const LsConst &K, const double *src, const double *ls0, double *out, bool bc,
                     cudaStream_t st) {
    k_reinit_a<MODE, double><<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, K, src, ls0, out, bc && g.p_mirror);
    if (bc && !g.p_mirror) launch_fill_p(g, out, st);
}
template <int MODE>
static void reinit_b(const Grid &g, const LsConst &K, const double *ls1, const double *ls0, const double *base,
                     double *out, bool bc, cudaStream_t st) {
    k_reinit_b<MODE, double><<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, K, ls1, ls0, base, out, bc && g.p_mirror);
    if (bc && !g.p_mirror) launch_fill_p(g, out, st);
}
static void reinit_c(const Grid &g, const LsConst &K, const double *tmp, const double *ls0, const double *base,
                     double *out, cudaStream_t st) {
    k_reinit_c<double><<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, K, tmp, ls0, base, out, g.p_mirror);
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

// ------------------------------------------------------------------------
// Batched full step (asd2g_batch_step): the same tile functions over a work
// list of (instance, tile), one launch per phase for the whole batch.  Every
// batch grid mirrors its own P ghosts (Neumann/Dirichlet sides).
__global__ void __launch_bounds__(TJ *TI) k_bcenter_vel(const BInst *__restrict__ insts,
                                                          const BTile *__restrict__ tiles) {
    const BTile t = tiles[blockIdx.x];
    const BInst &I = insts[t.inst];
    if (I.mixed) return;  // the FP32 path
    center_vel_tile<double>(I.g, bslot(I, BS_U), bslot(I, BS_V), bslot(I, BS_TU), bslot(I, BS_TV), t.bx, t.by);
}

template <int STAGE>
__global__ void __launch_bounds__(TJ *TI) k_bls_stage(const BInst *__restrict__ insts, const BTile *__restrict__ tiles,
                                                        int in, int n, int out) {
    const BTile t = tiles[blockIdx.x];
    const BInst &I = insts[t.inst];
    if (I.mixed) return;
    ls_stage_tile<STAGE, double>(I.g, I.ddx, I.ddy, bslot(I, in), bslot(I, BS_TU), bslot(I, BS_TV), bslot(I, n),
                                 bslot(I, out), I.sc, t.bx, t.by);
}

// One pseudo-step of every instance, as launch_reinit does for a session:
// A: LS1 = LS - adt S (|grad LS| - 1) into W1 (the Sussman mode without its
// ghost mirrors, W1's ghosts stay 0: levelset2d.cpp:336-340);
// B: 0.5 (LS + LS2(W1)) into LS, or for the Sussman modes into W2 (the
// session's third work array);
// C (Sussman modes): LS = base + constraint(W2), base = LS (Sussman) or W2
// (MinRK2 + Sussman).
template <int MODE>
__global__ void __launch_bounds__(TJ *TI) k_breinit_a(const BInst *__restrict__ insts, const BTile *__restrict__ tiles,
                                                      int k) {
    const BTile t = tiles[blockIdx.x];
    const BInst &I = insts[t.inst];
    if (k >= I.nreinit || I.mixed) return;
    reinit_a_tile<MODE, double>(I.g, I.K, bslot(I, BS_LS), bslot(I, BS_LS0), bslot(I, BS_W1), MODE == RM_SUSS ? 0 : 1,
                                t.bx, t.by);
}
template <int MODE>
__global__ void __launch_bounds__(TJ *TI) k_breinit_b(const BInst *__restrict__ insts, const BTile *__restrict__ tiles,
                                                      int k) {
    const BTile t = tiles[blockIdx.x];
    const BInst &I = insts[t.inst];
    if (k >= I.nreinit || I.mixed) return;
    constexpr bool SUSS = MODE == RM_SUSS || MODE == RM_MINRK2_SUSS;
    reinit_b_tile<MODE, double>(I.g, I.K, bslot(I, BS_W1), bslot(I, BS_LS0), bslot(I, BS_LS),
                                bslot(I, SUSS ? BS_W2 : BS_LS), 1, t.bx, t.by);
}
template <int MODE>
__global__ void __launch_bounds__(TJ *TI) k_breinit_c(const BInst *__restrict__ insts, const BTile *__restrict__ tiles,
                                                      int k) {
    const BTile t = tiles[blockIdx.x];
    const BInst &I = insts[t.inst];
    if (k >= I.nreinit || I.mixed) return;
    reinit_c_tile<double>(I.g, I.K, bslot(I, BS_W2), bslot(I, BS_LS0), bslot(I, MODE == RM_SUSS ? BS_LS : BS_W2),
                          bslot(I, BS_LS), 1, t.bx, t.by);
}

void launch_bstep_center_vel(const BStepPlan &P, cudaStream_t st) {
    k_bcenter_vel<<<P.ntiles, dim3(TJ, TI), 0, st>>>(P.insts, P.tiles);
}

void launch_bstep_ls_stage(const BStepPlan &P, int stage, int in, int n, int out, cudaStream_t st) {
    const dim3 blk(TJ, TI);
    if (stage == 1) k_bls_stage<1><<<P.ntiles, blk, 0, st>>>(P.insts, P.tiles, in, n, out);
    else if (stage == 2) k_bls_stage<2><<<P.ntiles, blk, 0, st>>>(P.insts, P.tiles, in, n, out);
    else k_bls_stage<3><<<P.ntiles, blk, 0, st>>>(P.insts, P.tiles, in, n, out);
}

void launch_bstep_reinit_pass(const BStepPlan &P, int mode, int pass, int k, cudaStream_t st) {
    const dim3 blk(TJ, TI);
    auto run = [&](auto m) {
        constexpr int M = decltype(m)::value;
        if (pass == 0) k_breinit_a<M><<<P.ntiles, blk, 0, st>>>(P.insts, P.tiles, k);
        else if (pass == 1) k_breinit_b<M><<<P.ntiles, blk, 0, st>>>(P.insts, P.tiles, k);
        else k_breinit_c<M><<<P.ntiles, blk, 0, st>>>(P.insts, P.tiles, k);
    };
    if (mode == RM_ORIG) run(std::integral_constant<int, RM_ORIG>{});
    else if (mode == RM_SUSS) run(std::integral_constant<int, RM_SUSS>{});
    else if (mode == RM_MINRK2) run(std::integral_constant<int, RM_MINRK2>{});
    else run(std::integral_constant<int, RM_MINRK2_SUSS>{});
}

}  // namespace asd2g
