// Tensor-core building blocks of the learned preconditioner (U-Net): a 3x3
// "same" convolution as an implicit GEMM on tcgen05 (BF16 activations and
// weights, FP32 accumulation in tensor memory), and the weight packing it
// reads, and the weight gradient of a 3x3 convolution (k_wgrad_tc).  No
// reference counterpart (the reference has no learned solver).
//
// Implicit GEMM: D[p][co] = sum over taps t and input channels ci of
// X[p + off(t)][ci] * W[co][t][ci] for a tile of 128 consecutive output
// pixels p of one image row (M = 128) and all output channels (N = Cout).
// Activations are NHWC BF16 with Cin a multiple of 16.  For each chunk of 16
// input channels a pipeline stage in shared memory holds
//   * the input patch (3 rows x 130 pixels) as two 8-channel half-planes of
//     16-byte pixel rows -- the K-major canonical layout, so the A operand of
//     tap (dy, dx) is the same buffer started dy * 130 + dx rows later;
//   * the chunk's packed weights [tap][half][co][8] (the B operands).
// Stages are filled two chunks ahead: the patch by cp.async (zero-fill
// outside the image), the chunk's weights by one bulk copy completing on the
// stage's full barrier.  One thread waits for the weights, issues the nine
// tcgen05.mma of a chunk and commits them to the stage's MMA barrier, which
// frees the stage for the chunk that many stages later.  The epilogue reads the accumulator from tensor memory
// (warp w owns pixel rows 32w .. 32w+31), adds the bias, applies ReLU and
// stores BF16 NHWC (and optionally channel 0 in FP32).
#include <cstdlib>
#include <cstring>

#include <cuda_bf16.h>

#include "asd2g.h"
#include "internal.cuh"
#include "tc05.cuh"

namespace asd2g {
int api_exception(const char *fn);  // the entry points' exception handler (api.cu)
}  // namespace asd2g

namespace asd2g {

bool conv_cout_ok(int c) { return c == 16 || c == 32 || c == 48 || c == 64 || c == 96 || c == 128 || c == 192; }

namespace {

constexpr int CT_PIX = 128;             // output pixels per tile
constexpr int PATCH_W = CT_PIX + 2;     // patch row: one halo pixel each side
constexpr int PATCH_PIX = 3 * PATCH_W;  // pixels per half-plane
constexpr int PATCH_BYTES = 2 * PATCH_PIX * 16;
constexpr int CONV_THREADS = 128;
constexpr int CONV_SMEM_MAX = 227 * 1024;

__host__ __device__ constexpr int conv_stage_bytes(int cout) { return PATCH_BYTES + 288 * cout; }
// Four stages where they fit (loads two chunks ahead, and the MMAs of a chunk
// get one iteration to finish before their stage is refilled), else three
// (loads two chunks ahead, the stage of the previous chunk is refilled).
__host__ __device__ constexpr int conv_stages(int cout) {
    return 4 * conv_stage_bytes(cout) + 16 * 4 + 16 <= CONV_SMEM_MAX ? 4 : 3;
}
// stages, then two mbarriers per stage, the TMEM address and the abort flag
__host__ __device__ constexpr int conv_smem_bytes(int cout) {
    return conv_stages(cout) * conv_stage_bytes(cout) + 16 * conv_stages(cout) + 16;
}
static_assert(conv_smem_bytes(192) <= CONV_SMEM_MAX, "conv pipeline exceeds shared memory");

// Patch copies of one thread: slot i covers patch entry t = tid + 128 i of
// the two half-planes (2 x 3 x 130 pixel rows of 16 bytes).  The pixel
// offsets do not depend on the channel chunk, so they are formed once; a
// chunk adds its channel offset.  With low != nullptr the input is the
// channel concatenation of low (H/2 x W/2 x CL, nearest-upsampled: pixel
// (y, x) reads (y/2, x/2)) and in (H x W x (CIN - CL)); CL is a multiple of
// 16, so a chunk reads one of the two.
constexpr int PATCH_SLOTS = (2 * PATCH_PIX + CONV_THREADS - 1) / CONV_THREADS;
struct PatchPlan {
    int off_in[PATCH_SLOTS];   // element offset in `in` (pixel * channels + half * 8), -1: outside
    int off_low[PATCH_SLOTS];  // element offset in `low`
};

__device__ __forceinline__ void patch_plan(PatchPlan &P, int H, int W, int cs, int CL, int y, int x0, int tid) {
#pragma unroll
    for (int i = 0; i < PATCH_SLOTS; i++) {
        const int t = tid + CONV_THREADS * i;
        P.off_in[i] = -1;
        P.off_low[i] = -1;
        if (t < 2 * PATCH_PIX) {
            const int h = t / PATCH_PIX, q = t % PATCH_PIX, r = q / PATCH_W, c = q % PATCH_W;
            const int yy = y - 1 + r, xx = x0 - 1 + c;
            if (yy >= 0 && yy < H && xx >= 0 && xx < W) {
                P.off_in[i] = (yy * W + xx) * cs + h * 8;
                P.off_low[i] = ((yy >> 1) * (W >> 1) + (xx >> 1)) * CL + h * 8;
            }
        }
    }
}

// Chunk kc into one stage: the patch by cp.async (every thread), the
// chunk's packed weights (contiguous) by one bulk copy of thread 0 that
// completes on the stage's full barrier.
template <int COUT>
__device__ __forceinline__ void conv_load_chunk(uint8_t *stage, uint64_t *full, const PatchPlan &P,
                                                const __nv_bfloat16 *__restrict__ inb,
                                                const __nv_bfloat16 *__restrict__ lowb, int CL, int kc,
                                                const uint4 *__restrict__ wpack, int tid) {
    uint4 *patch = reinterpret_cast<uint4 *>(stage);
    const bool from_low = lowb != nullptr && kc * 16 < CL;
    const __nv_bfloat16 *base = from_low ? lowb + kc * 16 : inb + (lowb ? kc * 16 - CL : kc * 16);
#pragma unroll
    for (int i = 0; i < PATCH_SLOTS; i++) {
        const int t = tid + CONV_THREADS * i;
        if (t < 2 * PATCH_PIX) {
            const int off = from_low ? P.off_low[i] : P.off_in[i];
            cp_async16(patch + t, off >= 0 ? base + off : inb, off >= 0);
        }
    }
    if (tid == 0) {
        constexpr uint32_t WB = 288u * COUT;  // 9 taps x 16 channels x COUT x 2 bytes
        mbar_arrive_expect_tx(full, WB);
        bulk_g2s(stage + PATCH_BYTES, wpack + (size_t)kc * (WB / 16), WB, full);
    }
}

// S pipeline stages (conv_stages(COUT), or 1 / 2 for layers of one / two
// input-channel chunks: every chunk then has its own stage, all are loaded
// at once, and the smaller footprint lets more CTAs share an SM).
template <int COUT, int S>
__global__ void __launch_bounds__(CONV_THREADS) k_conv3x3_tc(const __nv_bfloat16 *__restrict__ in,
                                                             const __nv_bfloat16 *__restrict__ low, int CL, int H,
                                                             int W, int CIN, const uint4 *__restrict__ wpack,
                                                             const float *__restrict__ bias,
                                                             __nv_bfloat16 *__restrict__ out,
                                                             float *__restrict__ out32, int relu, int *err) {
    extern __shared__ __align__(128) uint8_t sm[];
    constexpr int SB = conv_stage_bytes(COUT);
    constexpr int SLACK = S >= 3 ? S - 3 : 0;            // iterations a chunk's MMAs get before their stage is refilled
    constexpr int AHEAD = S >= 3 ? S - 1 - SLACK : S;  // chunks in flight ahead of the one being multiplied
    uint64_t *mma_bar = reinterpret_cast<uint64_t *>(sm + S * SB);  // per stage: its MMAs completed
    uint64_t *full_bar = mma_bar + S;                               // per stage: its weights landed
    uint32_t *tslot = reinterpret_cast<uint32_t *>(full_bar + S);
    int *abort_flag = reinterpret_cast<int *>(tslot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int x0 = blockIdx.x * CT_PIX, y = blockIdx.y, img = blockIdx.z;
    const int cs = low ? CIN - CL : CIN;
    const __nv_bfloat16 *inb = in + (size_t)img * H * W * cs;
    const __nv_bfloat16 *lowb = low ? low + (size_t)img * (H >> 1) * (W >> 1) * CL : nullptr;
    constexpr uint32_t NCOL = COUT <= 32 ? 32 : COUT <= 64 ? 64 : COUT <= 128 ? 128 : 256;  // power of two
    constexpr uint32_t IDESC = umma_idesc_bf16(128, COUT);
    const int nkc = CIN / 16;
    if (S < 3 && nkc > S) {  // the launcher never does this: no stage may be refilled with S < 3
        if (tid == 0) atomicExch(err, 4);
        return;
    }
    if (tid == 0) {
        for (int k = 0; k < S; k++) {
            mbar_init(mma_bar + k, 1);
            mbar_init(full_bar + k, 1);
        }
        mbar_init_fence();
        *abort_flag = 0;
    }
    PatchPlan P;
    patch_plan(P, H, W, cs, CL, y, x0, tid);
    __syncthreads();  // barriers initialised before the first copy arrives on one
    // prologue: the first AHEAD chunks in flight (one cp.async group each, empty past the end)
    for (int k = 0; k < AHEAD; k++) {
        if (k < nkc) conv_load_chunk<COUT>(sm + k * SB, full_bar + k, P, inb, lowb, CL, k, wpack, tid);
        cp_async_commit();
    }
    if (warp == 0) {
        tmem_alloc(tslot, NCOL);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    bool ok = true;
    int issued = nkc < AHEAD ? nkc : AHEAD;  // chunks whose copies were started
    int consumed = 0;                        // chunks whose weights thread 0 has waited for
    for (int kc = 0; kc < nkc; kc++) {
        const int nk = kc + AHEAD;  // chunk to prefetch, into the stage chunk nk - S used
        if (nk < nkc) {             // block-uniform
            bool freed = true;
            const int pk = nk - S;
            if (pk >= 0) freed = mbar_wait_hw(mma_bar + pk % S, (uint32_t)(pk / S) & 1u, err, 1);
            if (!__syncthreads_and(freed && !*abort_flag)) {  // every thread leaves the loop together
                ok = false;
                break;
            }
            conv_load_chunk<COUT>(sm + (nk % S) * SB, full_bar + nk % S, P, inb, lowb, CL, nk, wpack, tid);
            issued = nk + 1;
        }
        cp_async_commit();
        cp_async_wait<AHEAD>();  // chunk kc's patch has landed (this thread's part)
        fence_async_smem();
        __syncthreads();  // ... and every thread's part
        if (tid == 0) {
            const bool wok = mbar_wait_hw(full_bar + kc % S, (uint32_t)(kc / S) & 1u, err, 2);
            consumed = kc + 1;
            tc_fence_after();
            if (wok) {
                const uint32_t base = smem_u32(sm + (kc % S) * SB);
                const uint32_t pa = base, pw = base + PATCH_BYTES;
                for (int tap = 0; tap < 9; tap++) {
                    const int dy = tap / 3, dx = tap % 3;
                    const uint64_t ad = umma_desc_k(pa + (uint32_t)(dy * PATCH_W + dx) * 16u, PATCH_PIX * 16u, 128u);
                    const uint64_t bd = umma_desc_k(pw + (uint32_t)tap * 2u * COUT * 16u, COUT * 16u, 128u);
                    umma_bf16(tmem, ad, bd, IDESC, (kc > 0 || tap > 0) ? 1u : 0u);
                }
            } else {
                *abort_flag = 1;
            }
            umma_commit(mma_bar + kc % S);  // always, so that waits on this stage end
        }
    }
    cp_async_wait<0>();  // no cp.async may still target shared memory when the CTA exits
    if (tid == 0)        // nor a bulk copy: wait (bounded) for the weights of chunks never multiplied
        for (int c = consumed; c < issued; c++) mbar_wait(full_bar + c % S, (uint32_t)(c / S) & 1u, err, 2);
    // the last commit arrives once every MMA of the tile has completed
    if (ok && nkc > 0) ok = mbar_wait_hw(mma_bar + (nkc - 1) % S, (uint32_t)((nkc - 1) / S) & 1u, err, 1);
    __syncthreads();
    ok = __syncthreads_and(ok && !*abort_flag);  // the TMEM loads below are warp-collective
    tc_fence_after();
    if (ok) {
        const int x = x0 + warp * 32 + lane;
        const size_t pix = (size_t)img * H * W + (size_t)y * W + x;
#pragma unroll
        for (int c0 = 0; c0 < COUT; c0 += 16) {
            uint32_t r[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
            tmem_wait_ld();
            if (x < W) {
                float v[16];
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    v[i] = __uint_as_float(r[i]) + bias[c0 + i];
                    if (relu) v[i] = fmaxf(v[i], 0.0f);
                }
                if (out) {
                    uint32_t w[8];
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
                        w[i] = *reinterpret_cast<const uint32_t *>(&b2);
                    }
                    uint4 *o = reinterpret_cast<uint4 *>(out + pix * COUT + c0);
                    o[0] = make_uint4(w[0], w[1], w[2], w[3]);
                    o[1] = make_uint4(w[4], w[5], w[6], w[7]);
                }
                if (out32 && c0 == 0) out32[pix] = v[0];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, NCOL);
}

// The patch of one tile and chunk into a patch stage (cp.async, every thread).
__device__ __forceinline__ void conv_load_patch(uint8_t *stage, const PatchPlan &P,
                                                const __nv_bfloat16 *__restrict__ inb,
                                                const __nv_bfloat16 *__restrict__ lowb, int CL, int kc, int tid) {
    uint4 *patch = reinterpret_cast<uint4 *>(stage);
    const bool from_low = lowb != nullptr && kc * 16 < CL;
    const __nv_bfloat16 *base = from_low ? lowb + kc * 16 : inb + (lowb ? kc * 16 - CL : kc * 16);
#pragma unroll
    for (int i = 0; i < PATCH_SLOTS; i++) {
        const int t = tid + CONV_THREADS * i;
        if (t < 2 * PATCH_PIX) {
            const int off = from_low ? P.off_low[i] : P.off_in[i];
            cp_async16(patch + t, off >= 0 ? base + off : inb, off >= 0);
        }
    }
}

// ---------------------------------------------------------------- workers --
// Layers of one or two 16-channel input chunks (the full-resolution and
// half-resolution convolutions, most of the network's time) as persistent
// CTAs of NW independent workers.  A worker is four warps (TMEM lanes
// 0..127 for the epilogue) that loops over its own row tiles: the layer's
// weights are copied into the worker's shared memory once, the patch of the
// next tile is copied while the current one is multiplied and written out
// (two patch buffers), one thread issues the tile's MMAs into the worker's
// accumulator and commits them to the worker's barrier.  The per-tile CTAs
// above are held by the rate at which CTAs can be launched (a few hundred
// nanoseconds of work each, ~2 of 12 possible resident per SM); here a CTA
// lives for the whole layer and NW tile chains run side by side per SM.
template <int COUT, int NKC> struct ConvW {
    static constexpr int NCOL = COUT <= 32 ? 32 : COUT <= 64 ? 64 : COUT <= 128 ? 128 : 256;
    static constexpr int WB = 288 * COUT;                       // one weight chunk
    static constexpr int PER = NKC * WB + 2 * NKC * PATCH_BYTES;  // weights + two patch buffers
    static constexpr int FIT = (220 * 1024) / PER;
    static constexpr int NW0 = FIT > 8 ? 8 : FIT;
    static constexpr int NW = NW0 * NCOL > 512 ? 512 / NCOL : NW0;  // workers per CTA
    static constexpr int COLS = NW * NCOL <= 32 ? 32 : NW * NCOL <= 64 ? 64 : NW * NCOL <= 128 ? 128
                                : NW * NCOL <= 256 ? 256 : 512;   // TMEM allocation (power of two)
    static constexpr int BAR_OFF = NW * PER;
    static constexpr int SMEM = BAR_OFF + NW * 16 + 16;           // per worker: weights and MMA barriers
};

__device__ __forceinline__ void bar_sync(int id, int count) {
    asm volatile("barrier.cta.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}
// named-barrier AND over the count threads of barrier id
__device__ __forceinline__ bool bar_and(int id, int count, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\tbarrier.cta.red.and.pred p, %2, %3, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id), "r"(count)
        : "memory");
    return r != 0;
}

template <int COUT, int NKC>
__global__ void __launch_bounds__(CONV_THREADS *ConvW<COUT, NKC>::NW, 1)
    k_conv3x3_tcw(const __nv_bfloat16 *__restrict__ in, const __nv_bfloat16 *__restrict__ low, int CL, int H,
                  int W, int CIN, const uint4 *__restrict__ wpack, const float *__restrict__ bias,
                  __nv_bfloat16 *__restrict__ out, float *__restrict__ out32, int relu, int *err, int tiles_x,
                  int ntiles) {
    using C = ConvW<COUT, NKC>;
    constexpr int NW = C::NW, WB = C::WB;
    constexpr uint32_t NCOL = C::NCOL;
    constexpr uint32_t IDESC = umma_idesc_bf16(128, COUT);
    extern __shared__ __align__(128) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wk = warp >> 2, wt = tid & (CONV_THREADS - 1);  // worker, thread within the worker
    uint8_t *wreg = sm + wk * C::PER;                          // the worker's weights, then its two patch buffers
    uint8_t *pbuf = wreg + NKC * WB;
    uint64_t *wfull = reinterpret_cast<uint64_t *>(sm + C::BAR_OFF) + 2 * wk;  // weights landed
    uint64_t *mbar = wfull + 1;                                                 // the tile's MMAs completed
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + C::BAR_OFF + NW * 16);
    const int bid = 1 + wk;  // the worker's named barrier
    const int cs = low ? CIN - CL : CIN;
    if (CIN != 16 * NKC) {  // the launcher never does this
        if (tid == 0) atomicExch(err, 4);
        return;
    }
    if (wt == 0) {
        mbar_init(wfull, 1);
        mbar_init(mbar, 1);
        mbar_init_fence();
    }
    if (warp == 0) {
        tmem_alloc(tslot, (uint32_t)C::COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tacc = *tslot + (uint32_t)wk * NCOL;
    const int workers = (int)gridDim.x * NW, gw = (int)blockIdx.x * NW + wk;
    const int my = gw < ntiles ? (ntiles - 1 - gw) / workers + 1 : 0;  // this worker's tiles
    auto coords = [&](int i, int &img, int &y, int &x0) {  // the worker's i-th tile
        const int t = gw + i * workers;
        const int r = t / tiles_x;
        x0 = (t - r * tiles_x) * CT_PIX;
        y = r % H;
        img = r / H;
    };
    PatchPlan P;
    auto load_tile = [&](int i) {  // every chunk's patch of tile i into buffer i & 1
        int img, y, x0;
        coords(i, img, y, x0);
        patch_plan(P, H, W, cs, CL, y, x0, wt);
        const __nv_bfloat16 *inb = in + (size_t)img * H * W * cs;
        const __nv_bfloat16 *lowb = low ? low + (size_t)img * (H >> 1) * (W >> 1) * CL : nullptr;
#pragma unroll
        for (int kc = 0; kc < NKC; kc++)
            conv_load_patch(pbuf + ((i & 1) * NKC + kc) * PATCH_BYTES, P, inb, lowb, CL, kc, wt);
    };
    bool ok = true, wwait = false;
    if (my > 0) {
        if (wt == 0) {  // the layer's weights, once
            mbar_arrive_expect_tx(wfull, (uint32_t)(NKC * WB));
            bulk_g2s(wreg, wpack, (uint32_t)(NKC * WB), wfull);
        }
        load_tile(0);
    }
    cp_async_commit();
    for (int i = 0; i < my; i++) {
        // the next tile's patches go into the other buffer (its MMAs, of tile
        // i - 1, completed before that tile's epilogue)
        if (i + 1 < my) load_tile(i + 1);
        cp_async_commit();
        cp_async_wait<1>();  // tile i's patches have landed (this thread's part)
        fence_async_smem();
        bar_sync(bid, CONV_THREADS);  // ... and the whole worker's
        tc_fence_after();
        bool good = true;
        if (wt == 0) {
            if (!wwait) {
                good = mbar_wait_hw(wfull, 0u, err, 2);
                wwait = true;
            }
            if (good) {
                const uint32_t pw0 = smem_u32(wreg);
#pragma unroll 1
                for (int kc = 0; kc < NKC; kc++) {
                    const uint32_t pa = smem_u32(pbuf + ((i & 1) * NKC + kc) * PATCH_BYTES);
                    const uint32_t pw = pw0 + (uint32_t)(kc * WB);
                    for (int tap = 0; tap < 9; tap++) {
                        const int dy = tap / 3, dx = tap % 3;
                        const uint64_t ad =
                            umma_desc_k(pa + (uint32_t)(dy * PATCH_W + dx) * 16u, PATCH_PIX * 16u, 128u);
                        const uint64_t bd = umma_desc_k(pw + (uint32_t)tap * 2u * COUT * 16u, COUT * 16u, 128u);
                        umma_bf16(tacc, ad, bd, IDESC, (kc > 0 || tap > 0) ? 1u : 0u);
                    }
                }
            }
            umma_commit(mbar);  // always, so that the wait below ends
            good = mbar_wait_hw(mbar, (uint32_t)(i & 1), err, 1) && good;
        }
        if (!bar_and(bid, CONV_THREADS, good)) {  // the TMEM loads below are warp-collective
            ok = false;
            break;
        }
        tc_fence_after();
        int img, y, x0;
        coords(i, img, y, x0);
        const int x = x0 + (warp & 3) * 32 + lane;
        const size_t pix = (size_t)img * H * W + (size_t)y * W + x;
        const uint32_t tb = tacc + ((uint32_t)((warp & 3) * 32) << 16);
#pragma unroll
        for (int c0 = 0; c0 < COUT; c0 += 16) {
            uint32_t r[16];
            tmem_ld16(tb + (uint32_t)c0, r);
            tmem_wait_ld();
            if (x < W) {
                float v[16];
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    v[k] = __uint_as_float(r[k]) + bias[c0 + k];
                    if (relu) v[k] = fmaxf(v[k], 0.0f);
                }
                if (out) {
                    uint32_t wv[8];
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
                        wv[k] = *reinterpret_cast<const uint32_t *>(&b2);
                    }
                    uint4 *o = reinterpret_cast<uint4 *>(out + pix * COUT + c0);
                    o[0] = make_uint4(wv[0], wv[1], wv[2], wv[3]);
                    o[1] = make_uint4(wv[4], wv[5], wv[6], wv[7]);
                }
                if (out32 && c0 == 0) out32[pix] = v[0];
            }
        }
        tc_fence_before();
        bar_sync(bid, CONV_THREADS);  // every TMEM read of this tile precedes the next tile's MMAs
    }
    (void)ok;
    cp_async_wait<0>();  // no cp.async may still target shared memory when the CTA exits
    if (wt == 0 && my > 0 && !wwait) mbar_wait(wfull, 0u, err, 2);  // nor the weights' bulk copy
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(*tslot, (uint32_t)C::COLS);
}

// ------------------------------------------------------------ weight grad --
// Weight gradient of a 3x3 convolution on the tensor cores:
//   dW[co][ci][t] = sum_p G[p][co] X[p + off(t)][ci],   db[co] = sum_p G[p][co]
// as D[r][co] = sum_p A[r][p] B[co][p] with rows r = t CI + ci (and one row of
// ones for the bias after the last), columns co (Cout padded, N = COS), K =
// output pixels.  A CTA owns one 128-row tile of r and a contiguous range of
// pixels (split-K); per chunk of 64 pixels its threads gather and transpose
// the X and G values into the K-major canonical layout (thread r of the tile
// builds row r; columns from consecutive channels, so each pixel's loads are
// coalesced across the warp), one thread issues four tcgen05.mma (K = 16
// each) into the TMEM accumulator, and two stages alternate.  The partial
// sums of every CTA go to a buffer that one more kernel adds in a fixed
// order (deterministic, no atomics).
constexpr int WG_KC = 64;                       // pixels per stage
constexpr int WG_ROWS = 128;                    // rows of r per CTA (M)
constexpr int WG_A_BYTES = WG_ROWS * WG_KC * 2; // 16 KB
__host__ __device__ constexpr int wg_b_bytes(int cos) { return cos * WG_KC * 2; }
__host__ __device__ constexpr int wg_smem(int cos) { return 2 * (WG_A_BYTES + wg_b_bytes(cos)) + 2 * 8 + 16; }

// 8 consecutive BF16 values -> one 16-byte core-matrix row
__device__ __forceinline__ uint4 pack8(const __nv_bfloat16 (&v)[8]) {
    uint4 u;
    u.x = (uint32_t)__bfloat16_as_ushort(v[0]) | ((uint32_t)__bfloat16_as_ushort(v[1]) << 16);
    u.y = (uint32_t)__bfloat16_as_ushort(v[2]) | ((uint32_t)__bfloat16_as_ushort(v[3]) << 16);
    u.z = (uint32_t)__bfloat16_as_ushort(v[4]) | ((uint32_t)__bfloat16_as_ushort(v[5]) << 16);
    u.w = (uint32_t)__bfloat16_as_ushort(v[6]) | ((uint32_t)__bfloat16_as_ushort(v[7]) << 16);
    return u;
}

template <int COS>
__global__ void __launch_bounds__(WG_ROWS) k_wgrad_tc(const __nv_bfloat16 *__restrict__ X,
                                                      const __nv_bfloat16 *__restrict__ G, int H, int W, int CIS,
                                                      int CI, int64_t P, int64_t KP, float *__restrict__ part,
                                                      int *err) {
    extern __shared__ __align__(128) uint8_t sm[];
    constexpr int BB = wg_b_bytes(COS);
    constexpr int SB = WG_A_BYTES + BB;  // one stage: A then B
    constexpr uint32_t NCOL = COS <= 32 ? 32 : COS <= 64 ? 64 : COS <= 128 ? 128 : 256;
    constexpr uint32_t IDESC = umma_idesc_bf16(128, COS);
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sm + 2 * SB);  // per stage: its MMAs completed
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int R = 9 * CI;                    // rows of dW; row R is the bias (ones)
    const int r = blockIdx.y * WG_ROWS + tid;  // this thread's A row
    const int t = r < R ? r / CI : 0, ci = r < R ? r - t * CI : 0;
    const int dy = t / 3 - 1, dx = t % 3 - 1;
    const int64_t p_begin = (int64_t)blockIdx.x * KP;
    const int64_t p_end = p_begin + KP < P ? p_begin + KP : P;
    const int nch = (int)((p_end - p_begin + WG_KC - 1) / WG_KC);
    if (tid == 0) {
        mbar_init(mbar, 1);
        mbar_init(mbar + 1, 1);
        mbar_init_fence();
    }
    if (warp == 0) {
        tmem_alloc(tslot, NCOL);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f), one = __float2bfloat16_rn(1.0f);
    bool ok = true;
    int issued = 0;  // chunks whose MMAs were committed
    for (int c = 0; c < nch; c++) {
        const int st = c & 1;
        uint8_t *A = sm + st * SB, *Bm = A + WG_A_BYTES;
        if (c >= 2) {  // the stage's previous MMAs (chunk c - 2) are done
            const bool w = tid != 0 || mbar_wait_hw(mbar + st, (uint32_t)((c - 2) >> 1) & 1u, err, 5);
            if (!__syncthreads_and(w)) {
                ok = false;
                break;
            }
        }
        // gather and transpose: 8 groups of 8 pixels, group g -> core-matrix plane g
        const int64_t p0 = p_begin + (int64_t)c * WG_KC;
        int64_t q = p0 / W;
        int x = (int)(p0 - q * W);
        int y = (int)(q % H);
        int64_t b = q / H;
#pragma unroll 1
        for (int g = 0; g < WG_KC / 8; g++) {
            __nv_bfloat16 va[8], vb0[8], vb1[8];
#pragma unroll
            for (int e = 0; e < 8; e++) {
                const int64_t p = p0 + g * 8 + e;
                const bool in = p < p_end;
                __nv_bfloat16 a = zero;
                if (in && r < R) {
                    const int yy = y + dy, xx = x + dx;
                    if (yy >= 0 && yy < H && xx >= 0 && xx < W) a = X[((b * H + yy) * W + xx) * CIS + ci];
                } else if (in && r == R) {
                    a = one;
                }
                va[e] = a;
                vb0[e] = (in && tid < COS) ? G[p * COS + tid] : zero;
                if (COS > WG_ROWS) vb1[e] = (in && tid + WG_ROWS < COS) ? G[p * COS + tid + WG_ROWS] : zero;
                if (++x == W) {  // next pixel
                    x = 0;
                    if (++y == H) {
                        y = 0;
                        b++;
                    }
                }
            }
            *reinterpret_cast<uint4 *>(A + g * (WG_ROWS * 16) + tid * 16) = pack8(va);
            if (tid < COS) *reinterpret_cast<uint4 *>(Bm + g * (COS * 16) + tid * 16) = pack8(vb0);
            if (COS > WG_ROWS && tid + WG_ROWS < COS)
                *reinterpret_cast<uint4 *>(Bm + g * (COS * 16) + (tid + WG_ROWS) * 16) = pack8(vb1);
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(A), b0 = smem_u32(Bm);
#pragma unroll
            for (int s = 0; s < WG_KC / 16; s++) {
                const uint64_t ad = umma_desc_k(a0 + (uint32_t)(2 * s) * (WG_ROWS * 16), WG_ROWS * 16, 128u);
                const uint64_t bd = umma_desc_k(b0 + (uint32_t)(2 * s) * (COS * 16), COS * 16, 128u);
                umma_bf16(tmem, ad, bd, IDESC, (c > 0 || s > 0) ? 1u : 0u);
            }
            umma_commit(mbar + st);
        }
        issued = c + 1;
    }
    // the last commit arrives once every MMA of the CTA completed (also
    // before TMEM is released on an early exit)
    const bool w = tid != 0 || issued == 0 ||
                   mbar_wait_hw(mbar + ((issued - 1) & 1), (uint32_t)((issued - 1) >> 1) & 1u, err, 5);
    ok = __syncthreads_and(ok && w && issued == nch && nch > 0);
    tc_fence_after();
    if (ok) {
        const int row = warp * 32 + lane;
        float *dst = part + ((size_t)blockIdx.x * gridDim.y + blockIdx.y) * (size_t)WG_ROWS * COS + (size_t)row * COS;
#pragma unroll
        for (int c0 = 0; c0 < COS; c0 += 16) {
            uint32_t v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 16; i++) dst[c0 + i] = __uint_as_float(v[i]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, NCOL);
}

// dW[co][ci][t] += sum over the split-K partials (fixed order), db[co] += the bias row's
__global__ void k_wgrad_reduce(const float *__restrict__ part, int Z, int MT, int COS, int CI, int CO,
                               float *__restrict__ dW, float *__restrict__ db) {
    const int R = 9 * CI;
    const int64_t n = (int64_t)(R + 1) * CO;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e / CO), co = (int)(e - (int64_t)r * CO);
        const size_t stride = (size_t)MT * WG_ROWS * COS;
        const size_t off = (size_t)(r / WG_ROWS) * WG_ROWS * COS + (size_t)(r % WG_ROWS) * COS + co;
        float s = 0.0f;
        for (int z = 0; z < Z; z++) s += part[(size_t)z * stride + off];
        if (r < R) {
            const int t = r / CI, ci = r - t * CI;
            dW[((size_t)co * CI + ci) * 9 + t] += s;
        } else {
            db[co] += s;
        }
    }
}

// w[co][ci][3][3] (FP32, cout x cin real channels) -> wpack[kc][tap][half][co][8]
// (BF16, padded to cout_pad x cin_pad with zeros).
__global__ void k_pack_conv(const float *__restrict__ w, int cout, int cin, int cout_pad, int cin_pad,
                            __nv_bfloat16 *__restrict__ wpack) {
    const int64_t n = (int64_t)cin_pad * 9 * cout_pad;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        // e enumerates (kc, tap, half, co, j) with ci = kc*16 + half*8 + j
        const int j = (int)(e % 8);
        int64_t r = e / 8;
        const int co = (int)(r % cout_pad);
        r /= cout_pad;
        const int half = (int)(r % 2);
        r /= 2;
        const int tap = (int)(r % 9);
        const int kc = (int)(r / 9);
        const int ci = kc * 16 + half * 8 + j;
        float v = 0.0f;
        if (co < cout && ci < cin) v = w[(((size_t)co * cin + ci) * 3 + tap / 3) * 3 + tap % 3];
        wpack[e] = __float2bfloat16_rn(v);
    }
}

__host__ __device__ constexpr int conv_smem_s(int cout, int S) { return S * conv_stage_bytes(cout) + 16 * S + 16; }

template <int COUT, int S> bool conv_prepare() {
    static bool done = false;
    if (!done)
        done = cudaFuncSetAttribute(k_conv3x3_tc<COUT, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    conv_smem_s(COUT, S)) == cudaSuccess;
    return done;
}

template <int COUT, int S>
int conv_launch_s(const void *in, const void *low, int cl, int n, int h, int w, int cin, const void *wpack,
                  const float *bias, void *out, float *out32, int relu, int *err, cudaStream_t st) {
    if (!conv_prepare<COUT, S>()) return ASD2G_E_CUDA;
    const dim3 grid((w + CT_PIX - 1) / CT_PIX, h, n);
    k_conv3x3_tc<COUT, S><<<grid, CONV_THREADS, conv_smem_s(COUT, S), st>>>(
        (const __nv_bfloat16 *)in, (const __nv_bfloat16 *)low, cl, h, w, cin, (const uint4 *)wpack, bias,
        (__nv_bfloat16 *)out, out32, relu, err);
    return cudaGetLastError() == cudaSuccess ? ASD2G_OK : ASD2G_E_CUDA;
}

// One or two input-channel chunks: as many stages as chunks (ASD2G_CONV_STAGES
// = full keeps the full pipeline for them, for measurements).
bool conv_small_stages() {
    static const bool v = [] {
        const char *e = std::getenv("ASD2G_CONV_STAGES");
        return !(e && std::strcmp(e, "full") == 0);
    }();
    return v;
}

int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 148;
    }
    return n;
}

// ASD2G_CONV_FORM=tile: the per-tile CTAs for every layer (no workers).
bool conv_workers() {
    static const bool v = [] {
        const char *e = std::getenv("ASD2G_CONV_FORM");
        return !(e && std::strcmp(e, "tile") == 0);
    }();
    return v;
}

// The worker form for NKC chunks, if it fits at least two workers per CTA;
// returns 1 when it does not apply.
template <int COUT, int NKC>
int conv_launch_w(const void *in, const void *low, int cl, int n, int h, int w, int cin, const void *wpack,
                  const float *bias, void *out, float *out32, int relu, int *err, cudaStream_t st) {
    using C = ConvW<COUT, NKC>;
    if constexpr (C::NW >= 2) {
        static bool attr = false;
        if (!attr)
            attr = cudaFuncSetAttribute(k_conv3x3_tcw<COUT, NKC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        C::SMEM) == cudaSuccess;
        if (!attr) return ASD2G_E_CUDA;
        const int tiles_x = (w + CT_PIX - 1) / CT_PIX;
        const int64_t nt = (int64_t)tiles_x * h * n;
        if (nt >= ((int64_t)1 << 31)) return ASD2G_E_ARG;
        const int64_t need = (nt + C::NW - 1) / C::NW, cap = sm_count();
        const int grid = (int)(need < cap ? need : cap);
        k_conv3x3_tcw<COUT, NKC><<<grid, CONV_THREADS * C::NW, C::SMEM, st>>>(
            (const __nv_bfloat16 *)in, (const __nv_bfloat16 *)low, cl, h, w, cin, (const uint4 *)wpack, bias,
            (__nv_bfloat16 *)out, out32, relu, err, tiles_x, (int)nt);
        return cudaGetLastError() == cudaSuccess ? ASD2G_OK : ASD2G_E_CUDA;
    } else {
        return 1;
    }
}

template <int COUT>
int conv_launch(const void *in, const void *low, int cl, int n, int h, int w, int cin, const void *wpack,
                const float *bias, void *out, float *out32, int relu, int *err, cudaStream_t st) {
    const int nkc = cin / 16;
    // one or two chunks: the worker form (three chunks fit two workers per CTA
    // at 16 output channels, measured slower than the per-tile CTAs)
    if (conv_workers() && nkc <= 2) {
        const int rc = nkc == 1
                           ? conv_launch_w<COUT, 1>(in, low, cl, n, h, w, cin, wpack, bias, out, out32, relu, err, st)
                           : conv_launch_w<COUT, 2>(in, low, cl, n, h, w, cin, wpack, bias, out, out32, relu, err, st);
        if (rc != 1) return rc;
    }
    if (conv_small_stages() && nkc == 1)
        return conv_launch_s<COUT, 1>(in, low, cl, n, h, w, cin, wpack, bias, out, out32, relu, err, st);
    if (conv_small_stages() && nkc == 2)
        return conv_launch_s<COUT, 2>(in, low, cl, n, h, w, cin, wpack, bias, out, out32, relu, err, st);
    return conv_launch_s<COUT, conv_stages(COUT)>(in, low, cl, n, h, w, cin, wpack, bias, out, out32, relu, err,
                                                   st);
}

}  // namespace


int conv3x3_tc(const void *in, int n, int h, int w, int cin, const void *wpack, const float *bias, int cout,
               void *out, float *out32, int relu, int *err, cudaStream_t st, const void *low, int cl) {
    if (low && (cl < 16 || cl % 16 || cl >= cin || h % 2 || w % 2)) return ASD2G_E_ARG;
    if ((int64_t)h * w * cin >= (int64_t)1 << 31) return ASD2G_E_ARG;  // per-image offsets are 32-bit
    if (((uintptr_t)wpack & 15u) != 0) return ASD2G_E_ARG;              // bulk copies start on 16 bytes
    switch (cout) {
    case 16: return conv_launch<16>(in, low, cl, n, h, w, cin, wpack, bias, out, out32, relu, err, st);
    case 32: return conv_launch<32>(in, low, cl, n, h, w, cin, wpack, bias, out, out32, relu, err, st);
    case 48: return conv_launch<48>(in, low, cl, n, h, w, cin, wpack, bias, out, out32, relu, err, st);
    case 64: return conv_launch<64>(in, low, cl, n, h, w, cin, wpack, bias, out, out32, relu, err, st);
    case 96: return conv_launch<96>(in, low, cl, n, h, w, cin, wpack, bias, out, out32, relu, err, st);
    case 128: return conv_launch<128>(in, low, cl, n, h, w, cin, wpack, bias, out, out32, relu, err, st);
    case 192: return conv_launch<192>(in, low, cl, n, h, w, cin, wpack, bias, out, out32, relu, err, st);
    default: return ASD2G_E_ARG;
    }
}

// Weight and bias gradients of one 3x3 convolution (k_wgrad_tc + the fixed-
// order reduction), added into dW [CO][CI][9] and db [CO]; part is a work
// buffer of part_len floats.  Returns 1 when COS has no tensor-core form.
int wgrad_tc(const void *X, const void *G, int B, int H, int W, int CIS, int CI, int COS, int CO, float *dW,
             float *db, float *part, size_t part_len, int *err, cudaStream_t st) {
    const int64_t P = (int64_t)B * H * W;
    const int MT = (9 * CI + 1 + WG_ROWS - 1) / WG_ROWS;
    int64_t Z = (2 * sm_count() + MT - 1) / MT;  // about two CTAs per SM
    int64_t KP = (P + Z - 1) / Z;
    KP = (KP + WG_KC - 1) / WG_KC * WG_KC;
    while ((size_t)((P + KP - 1) / KP) * MT * WG_ROWS * COS > part_len) KP *= 2;
    Z = (P + KP - 1) / KP;
    const dim3 grid((unsigned)Z, (unsigned)MT);
#define WGL(C)                                                                                                      \
    {                                                                                                                \
        static bool attr = false;                                                                                    \
        if (!attr)                                                                                                   \
            attr = cudaFuncSetAttribute(k_wgrad_tc<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, wg_smem(C)) == \
                   cudaSuccess;                                                                                      \
        if (!attr) return ASD2G_E_CUDA;                                                                              \
        k_wgrad_tc<C><<<grid, WG_ROWS, wg_smem(C), st>>>((const __nv_bfloat16 *)X, (const __nv_bfloat16 *)G, H, W,   \
                                                        CIS, CI, P, KP, part, err);                                  \
    }
    switch (COS) {
    case 16: WGL(16); break;
    case 32: WGL(32); break;
    case 64: WGL(64); break;
    case 128: WGL(128); break;
    default: return 1;
    }
#undef WGL
    const int64_t n = (int64_t)(9 * CI + 1) * CO;
    k_wgrad_reduce<<<(int)((n + 255) / 256), 256, 0, st>>>(part, (int)Z, MT, COS, CI, CO, dW, db);
    return cudaGetLastError() == cudaSuccess ? ASD2G_OK : ASD2G_E_CUDA;
}

}  // namespace asd2g

using namespace asd2g;

extern "C" {

size_t asd2g_conv_wpack_bytes(int cout_pad, int cin_pad) { return (size_t)cout_pad * cin_pad * 9 * 2; }

int asd2g_conv_pack_weights(const float *w, int cout, int cin, int cout_pad, int cin_pad, void *wpack, void *stream) try {
    if (!w || !wpack || cout < 1 || cin < 1 || cout > cout_pad || cin > cin_pad || cin_pad % 16 ||
        !conv_cout_ok(cout_pad))
        return ASD2G_E_ARG;
    const int64_t n = (int64_t)cin_pad * 9 * cout_pad;
    k_pack_conv<<<(int)((n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184), 256, 0, (cudaStream_t)stream>>>(
        w, cout, cin, cout_pad, cin_pad, (__nv_bfloat16 *)wpack);
    return cudaGetLastError() == cudaSuccess ? ASD2G_OK : ASD2G_E_CUDA;
} catch (...) {
    return asd2g::api_exception("asd2g_conv_pack_weights");
}

int asd2g_conv3x3_bf16(const void *in, int n, int h, int w, int cin, const void *wpack, const float *bias, int cout,
                       void *out, float *out32, int relu, int *err, void *stream) try {
    if (!in || !wpack || !bias || (!out && !out32) || n < 1 || h < 1 || w < 1 || cin < 16 || cin % 16)
        return ASD2G_E_ARG;
    return conv3x3_tc(in, n, h, w, cin, wpack, bias, cout, out, out32, relu, err, (cudaStream_t)stream, nullptr, 0);
} catch (...) {
    return asd2g::api_exception("asd2g_conv3x3_bf16");
}

}  // extern "C"
