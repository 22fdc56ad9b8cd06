// Mixed-precision level-set step: the stencils of levelset_impl.cuh
// instantiated for float (this unit is built with fused multiply-adds), the
// FP64 <-> FP32 conversions of the level-set field around them, and the FP64
// volume check (sharp and smoothed Heaviside integrals, fixed-order
// reduction).
//
// The FP32 path keeps the reference's algorithm and pass structure (TVD-RK3
// over HJ-WENO5, then the reinitialisation pseudo-steps with the same count
// as the FP64 path); only the arithmetic type changes.  It needs the
// pressure-grid ghost fill to be producer-side (all P sides Neumann or
// Dirichlet): every FP32 kernel then writes its own ghost mirrors.
#include <cstdlib>
#include <cstring>

#include "batch.cuh"
#include "levelset_impl.cuh"
#include "ls32.cuh"

namespace asd2g {

template <> LsConstT<float> make_lsconst_t<float>(const Grid &g) {
    LsConstT<float> K;
    K.ddx = make_divh_f(g.dx);
    K.ddy = make_divh_f(g.dy);
    K.ddx2 = make_divh_f(g.dx * g.dx);
    K.ddy2 = make_divh_f(g.dy * g.dy);
    K.dx = (float)g.dx;
    K.dy = (float)g.dy;
    const double eps = g.dx < g.dy ? g.dx : g.dy;  // kEps = min(dx, dy), levelset2d.cpp:4
    K.eps = (float)eps;
    K.thick = (float)(1.5 * eps);
    K.adt = (float)(eps * 0.5);
    return K;
}

namespace {

__global__ void k_to_f32(int64_t n, const double *__restrict__ a, float *__restrict__ b) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        b[k] = (float)a[k];
}

__global__ void k_to_f64(int64_t n, const float *__restrict__ a, double *__restrict__ b) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        b[k] = (double)a[k];
}

// Interior sums of H and HS (FP64), block partials then the last block adds
// them in block order: the same result on every run.
__global__ void __launch_bounds__(256) k_volume(Grid g, const double *__restrict__ H, const double *__restrict__ HS,
                                                double *partial, unsigned *counter, double *out) {
    const int64_t n = (int64_t)g.nx * g.ny;
    double a = 0.0, b = 0.0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int i = NB + (int)(k / g.ny), j = NB + (int)(k % g.ny);
        a += H[IX(g, i, j)];
        b += HS[IX(g, i, j)];
    }
    __shared__ double sa[8], sb[8];
    __shared__ bool last;
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sa[wid] = a;
        sb[wid] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0.0, tb = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            ta += sa[w];
            tb += sb[w];
        }
        partial[2 * blockIdx.x] = ta;
        partial[2 * blockIdx.x + 1] = tb;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double ta = 0.0, tb = 0.0;
    for (unsigned blk = 0; blk < gridDim.x; blk++) {
        ta += __ldcg(partial + 2 * blk);
        tb += __ldcg(partial + 2 * blk + 1);
    }
    out[0] = ta * g.dx * g.dy;
    out[1] = tb * g.dx * g.dy;
    *counter = 0u;
}

// The FP32 advection stage in its packed form (weno32.cu: shared smoothness
// triples, FP32x2 arithmetic, a sliding row window) or in the per-cell tile
// form (the FP64 kernel's template instantiated for float); both compute the
// same scheme.  ASD2G_LS32_FORM=cell selects the per-cell form.  The
// reinitialisation pseudo-steps likewise run in their packed form
// (reinit32.cu) or as the per-cell templates (ASD2G_RI32_FORM=cell).
bool env_is_cell(const char *name) {
    const char *e = getenv(name);
    return e && std::strcmp(e, "cell") == 0;
}
bool packed_stage() {
    static const bool v = !env_is_cell("ASD2G_LS32_FORM");
    return v;
}
bool packed_reinit() {
    static const bool v = !env_is_cell("ASD2G_RI32_FORM");
    return v;
}

int64_t padded(const Grid &g) { return (int64_t)g.sx * g.sy; }
int conv_blocks(int64_t n) { return (int)((n + 255) / 256 < 4 * 148 ? (n + 255) / 256 : 4 * 148); }

// Batched (mixed instances): FP64 LS <-> FP32 phi over each instance's
// padded cells, and the FP32 centred velocities over its cell tiles.
__global__ void k_bls32_convert(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks, int to64) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    if (!I.mixed) return;
    const int64_t n = (int64_t)I.g.sx * I.g.sy, k = (int64_t)w.c * BSTEP_PAD_CHUNK + threadIdx.x;
    if (k >= n) return;
    double *ls = bslot(I, BS_LS);
    if (to64) ls[k] = (double)I.w32.phi[k];
    else I.w32.phi[k] = (float)ls[k];
}

__global__ void __launch_bounds__(TJ *TI) k_bcenter_vel32(const BInst *__restrict__ insts,
                                                            const BTile *__restrict__ tiles) {
    const BTile t = tiles[blockIdx.x];
    const BInst &I = insts[t.inst];
    if (!I.mixed) return;
    center_vel_tile<float>(I.g, bslot(I, BS_U), bslot(I, BS_V), I.w32.tu, I.w32.tv, t.bx, t.by);
}

}  // namespace

void launch_bstep_ls32_convert(const BStepPlan &P, bool to64, cudaStream_t st) {
    if (P.any_mixed) k_bls32_convert<<<P.npad, BSTEP_PAD_CHUNK, 0, st>>>(P.insts, P.pad_chunks, to64 ? 1 : 0);
}

void launch_bstep_center_vel32(const BStepPlan &P, cudaStream_t st) {
    if (P.any_mixed) k_bcenter_vel32<<<P.ntiles, dim3(TJ, TI), 0, st>>>(P.insts, P.tiles);
}

int reinit_steps(double adt, double max_atime);  // levelset.cu

bool ls32_supported(const Grid &g, int reinit_mode) {
    // the band list of the Sussman pass holds 32-bit cell offsets
    return g.p_mirror && (reinit_mode == 0 || reinit_mode == 2 || reinit_mode == 4) &&
           (int64_t)g.sx * g.sy < ((int64_t)1 << 31);
}

void launch_ls_step32(const Grid &g, int reinit_mode, double max_atime, const double *u, const double *v,
                      const double *dtp, double *ls64, const Ls32Work &w, cudaStream_t st) {
    const int64_t n = padded(g);
    const dim3 grd = cell_grid(g), blk(TJ, TI);
    k_to_f32<<<conv_blocks(n), 256, 0, st>>>(n, ls64, w.phi);
    k_center_vel<float><<<grd, blk, 0, st>>>(g, u, v, w.tu, w.tv);
    if (!packed_stage()) {
        const DivHT<float> ddx = make_divh_f(g.dx), ddy = make_divh_f(g.dy);
        k_ls_stage<1, float><<<grd, blk, 0, st>>>(g, ddx, ddy, w.phi, w.tu, w.tv, w.phi, w.a, dtp);
        k_ls_stage<2, float><<<grd, blk, 0, st>>>(g, ddx, ddy, w.a, w.tu, w.tv, w.phi, w.b, dtp);
        k_ls_stage<3, float><<<grd, blk, 0, st>>>(g, ddx, ddy, w.b, w.tu, w.tv, w.phi, w.phi, dtp);
    } else {
        launch_ls_stage32(g, 1, w.phi, w.tu, w.tv, w.phi, w.a, dtp, st);
        launch_ls_stage32(g, 2, w.a, w.tu, w.tv, w.phi, w.b, dtp, st);
        launch_ls_stage32(g, 3, w.b, w.tu, w.tv, w.phi, w.phi, dtp, st);
    }
    // reinitialisation: lsInit = phi, then the pseudo-steps (levelset2d.cpp:264-316, :433-486)
    const LsConstT<float> K = make_lsconst_t<float>(g);
    const double eps = g.dx < g.dy ? g.dx : g.dy;
    const double mt = max_atime > 0.0 ? max_atime : 1.5 * (1.5 * eps);  // kMaxATime, levelset2d.cpp:10
    const int steps = reinit_steps(eps * 0.5, mt);
    cudaMemcpyAsync(w.ls0, w.phi, sizeof(float) * (size_t)n, cudaMemcpyDeviceToDevice, st);
    for (int s = 0; s < steps; s++) {
        if (packed_reinit()) {
            launch_reinit32_step(g, reinit_mode, w, st);
        } else if (reinit_mode == 0) {
            k_reinit_a<0, float><<<grd, blk, 0, st>>>(g, K, w.phi, w.ls0, w.a, 1);
            k_reinit_b<0, float><<<grd, blk, 0, st>>>(g, K, w.a, w.ls0, w.phi, w.phi, 1);
        } else if (reinit_mode == 2) {
            k_reinit_a<2, float><<<grd, blk, 0, st>>>(g, K, w.phi, w.ls0, w.a, 1);
            k_reinit_b<2, float><<<grd, blk, 0, st>>>(g, K, w.a, w.ls0, w.phi, w.phi, 1);
        } else {
            k_reinit_a<4, float><<<grd, blk, 0, st>>>(g, K, w.phi, w.ls0, w.a, 1);
            k_reinit_b<4, float><<<grd, blk, 0, st>>>(g, K, w.a, w.ls0, w.phi, w.b, 1);
            k_reinit_c<float><<<grd, blk, 0, st>>>(g, K, w.b, w.ls0, w.b, w.phi, 1);
        }
    }
    k_to_f64<<<conv_blocks(n), 256, 0, st>>>(n, w.phi, ls64);
}

int ls32_launches(int reinit_mode, double max_atime, const Grid &g) {
    const double eps = g.dx < g.dy ? g.dx : g.dy;
    const double mt = max_atime > 0.0 ? max_atime : 1.5 * (1.5 * eps);
    const int steps = reinit_steps(eps * 0.5, mt);
    return 5 + steps * (reinit_mode == 4 ? 3 : 2) + 1;  // memcpy not counted
}

void launch_volume(const Grid &g, const double *H, const double *HS, double *partial, unsigned *counter, double *out2,
                   cudaStream_t st) {
    const int64_t n = (int64_t)g.nx * g.ny;
    int nb = (int)((n + 255) / 256);
    if (nb > VOLUME_BLOCKS) nb = VOLUME_BLOCKS;
    k_volume<<<nb, 256, 0, st>>>(g, H, HS, partial, counter, out2);
}

}  // namespace asd2g
