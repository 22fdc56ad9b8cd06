// The learned preconditioner: a 4-level 2D U-Net (16/32/64/128 channels,
// 3x3 convolutions, ReLU, 2x2 average pooling, nearest upsampling with skip
// concatenation), BF16 weights and activations, FP32 accumulation.  Every
// forward convolution and every input-gradient convolution runs on the
// tcgen05 tensor cores (unet.cu); the weight gradients are FP32 split-K
// reductions on the CUDA cores; the optimiser is Adam on FP32 master weights.
// No reference counterpart.
//
// Input features (16 channels, 4 used) of one GFM system on its nx x ny
// grid (image rows = i, columns = j, the compact layout k = j + ny i):
//   0: the vector to precondition, divided by its RMS;
//   1: diag / s, 2: ce / s, 3: cn / s with s = max(diag) of the system.
// Output: channel 0 of the last convolution, in FP32; the preconditioned
// vector is that times RMS / s (the network sees a unit-scale problem, and
// the map is homogeneous of degree one in the input vector).
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include <cuda_bf16.h>

#include "asd2g.h"
#include "internal.cuh"

namespace asd2g {
int api_fail(int code, const char *msg);
int api_exception(const char *fn);  // the entry points' exception handler (api.cu)
bool conv_cout_ok(int c);
// low != nullptr: the input is concat(nearest-upsampled low with cl channels, in)
int wgrad_tc(const void *X, const void *G, int B, int H, int W, int CIS, int CI, int COS, int CO, float *dW,
             float *db, float *part, size_t part_len, int *err, cudaStream_t st);
int conv3x3_tc(const void *in, int n, int h, int w, int cin, const void *wpack, const float *bias, int cout,
               void *out, float *out32, int relu, int *err, cudaStream_t st, const void *low = nullptr, int cl = 0);
}  // namespace asd2g

using namespace asd2g;
typedef __nv_bfloat16 bf16;

namespace {

// ------------------------------------------------------------ elementwise --
__device__ __forceinline__ float bf(bf16 v) { return __bfloat162float(v); }
__device__ __forceinline__ bf16 tobf(float v) { return __float2bfloat16_rn(v); }

// 2x2 average pooling, NHWC, C channels (H, W even, C a multiple of 8):
// one thread per 8 channels of an output pixel (16-byte loads and stores).
__global__ void k_pool(const bf16 *__restrict__ in, int B, int H, int W, int C, bf16 *__restrict__ out) {
    const int h = H / 2, w = W / 2, c8 = C / 8;
    const int64_t n = (int64_t)B * h * w * c8;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % c8) * 8;
        int64_t q = e / c8;
        const int x = (int)(q % w);
        q /= w;
        const int y = (int)(q % h);
        const int b = (int)(q / h);
        const bf16 *s = in + (((int64_t)b * H + 2 * y) * W + 2 * x) * C + c;
        const uint4 v[4] = {*reinterpret_cast<const uint4 *>(s), *reinterpret_cast<const uint4 *>(s + C),
                            *reinterpret_cast<const uint4 *>(s + (int64_t)W * C),
                            *reinterpret_cast<const uint4 *>(s + (int64_t)W * C + C)};
        uint32_t o[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            float lo = 0.0f, hi = 0.0f;
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const uint32_t wv = (&v[t].x)[i];
                const __nv_bfloat162 b2 = *reinterpret_cast<const __nv_bfloat162 *>(&wv);
                lo += __low2float(b2);
                hi += __high2float(b2);
            }
            const __nv_bfloat162 r2 = __floats2bfloat162_rn(0.25f * lo, 0.25f * hi);
            o[i] = *reinterpret_cast<const uint32_t *>(&r2);
        }
        *reinterpret_cast<uint4 *>(out + (((int64_t)b * h + y) * w + x) * C + c) = make_uint4(o[0], o[1], o[2], o[3]);
    }
}

// out[B][2h][2w][CL + CS] = concat(nearest-upsampled low[B][h][w][CL], skip[B][2h][2w][CS])
__global__ void k_upcat(const bf16 *__restrict__ low, int CL, const bf16 *__restrict__ skip, int CS, int B, int H,
                        int W, bf16 *__restrict__ out) {
    const int C = CL + CS;
    const int64_t n = (int64_t)B * H * W * C;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        const int64_t pix = e / C;
        const int x = (int)(pix % W);
        const int64_t q = pix / W;
        const int y = (int)(q % H);
        const int b = (int)(q / H);
        out[e] = c < CL ? low[(((int64_t)b * (H / 2) + y / 2) * (W / 2) + x / 2) * CL + c] : skip[pix * CS + (c - CL)];
    }
}

// d(pre-activation) = dY * [Y > 0] (BF16 in, BF16 out)
__global__ void k_relu_mask(const bf16 *__restrict__ dy, const bf16 *__restrict__ y, int64_t n, bf16 *__restrict__ g) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        g[e] = bf(y[e]) > 0.0f ? dy[e] : tobf(0.0f);
}

// Gradient of k_upcat: dlow[b][y][x][c] = sum of the 4 children; dskip += its part
// (dskip is written, not accumulated: the caller adds the pooling gradient after).
__global__ void k_upcat_back(const bf16 *__restrict__ dout, int CL, int CS, int B, int H, int W, bf16 *__restrict__ dlow,
                             float *__restrict__ dskip) {
    const int C = CL + CS, h = H / 2, w = W / 2;
    const int64_t nl = (int64_t)B * h * w * CL, ns = (int64_t)B * H * W * CS;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nl + ns; e += (int64_t)gridDim.x * blockDim.x) {
        if (e < nl) {
            const int c = (int)(e % CL);
            int64_t q = e / CL;
            const int x = (int)(q % w);
            q /= w;
            const int y = (int)(q % h);
            const int b = (int)(q / h);
            const bf16 *s = dout + (((int64_t)b * H + 2 * y) * W + 2 * x) * C + c;
            dlow[e] = tobf(bf(s[0]) + bf(s[C]) + bf(s[(int64_t)W * C]) + bf(s[(int64_t)W * C + C]));
        } else {
            const int64_t f = e - nl;
            const int c = (int)(f % CS);
            const int64_t pix = f / CS;
            dskip[f] = bf(dout[pix * C + CL + c]);
        }
    }
}

// d(e) = dskip + pool gradient (dp / 4 spread to the 2x2 block), -> BF16
__global__ void k_pool_back_add(const float *__restrict__ dskip, const bf16 *__restrict__ dp, int B, int H, int W,
                                int C, bf16 *__restrict__ de) {
    const int64_t n = (int64_t)B * H * W * C;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        const int64_t pix = e / C;
        const int x = (int)(pix % W);
        const int64_t q = pix / W;
        const int y = (int)(q % H);
        const int b = (int)(q / H);
        const float g = bf(dp[(((int64_t)b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c]) * 0.25f;
        de[e] = tobf((dskip ? dskip[e] : 0.0f) + g);
    }
}

// Features of B systems: feats FP32 [B][H][W][4] -> BF16 [B][H][W][16] (zero
// padded), one thread per pixel (one 16-byte load, two 16-byte stores).
__global__ void k_feats_pack(const float *__restrict__ f, int64_t npix, bf16 *__restrict__ out) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npix; p += (int64_t)gridDim.x * blockDim.x) {
        const float4 v = *reinterpret_cast<const float4 *>(f + 4 * p);
        const __nv_bfloat162 a = __floats2bfloat162_rn(v.x, v.y), b = __floats2bfloat162_rn(v.z, v.w);
        uint4 *o = reinterpret_cast<uint4 *>(out + 16 * p);
        o[0] = make_uint4(*reinterpret_cast<const uint32_t *>(&a), *reinterpret_cast<const uint32_t *>(&b), 0u, 0u);
        o[1] = make_uint4(0u, 0u, 0u, 0u);
    }
}

// Loss of each sample: sum (o - t)^2 / sum t^2; gradient into channel 0 of
// a BF16 [B][H][W][16] tensor.  One block per sample (two passes).
__global__ void k_loss(const float *__restrict__ o, const float *__restrict__ t, int64_t npix, bf16 *__restrict__ g,
                       float *__restrict__ loss) {
    const int b = blockIdx.x;
    const float *ob = o + (int64_t)b * npix, *tb = t + (int64_t)b * npix;
    float se = 0.0f, st = 0.0f;
    for (int64_t k = threadIdx.x; k < npix; k += blockDim.x) {
        const float d = ob[k] - tb[k];
        se += d * d;
        st += tb[k] * tb[k];
    }
    __shared__ float sa[32], sb[32];
    for (int o2 = 16; o2 > 0; o2 >>= 1) {
        se += __shfl_down_sync(0xffffffffu, se, o2);
        st += __shfl_down_sync(0xffffffffu, st, o2);
    }
    if ((threadIdx.x & 31) == 0) {
        sa[threadIdx.x >> 5] = se;
        sb[threadIdx.x >> 5] = st;
    }
    __syncthreads();
    __shared__ float tot[2];
    if (threadIdx.x == 0) {
        float a = 0.0f, c = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            a += sa[w];
            c += sb[w];
        }
        tot[0] = a;
        tot[1] = c > 0.0f ? c : 1.0f;
        loss[b] = a / tot[1];
    }
    __syncthreads();
    const float sc = 2.0f / tot[1] / (float)gridDim.x;  // mean over the batch
    for (int64_t k = threadIdx.x; k < npix; k += blockDim.x) {
        bf16 *gp = g + ((int64_t)b * npix + k) * 16;
        gp[0] = tobf(sc * (ob[k] - tb[k]));
        for (int c = 1; c < 16; c++) gp[c] = tobf(0.0f);
    }
}

// 5-point operator of the features at pixel k = h W + w: channels 1..3 =
// diag, ce (coupling to h + 1), cn (coupling to w + 1), symmetric.
__device__ __forceinline__ float stencil_apply(const float *__restrict__ f, const float *__restrict__ v, int H, int W,
                                               int64_t k) {
    const int h = (int)(k / W), w = (int)(k % W);
    float y = f[4 * k + 1] * v[k];
    if (h + 1 < H) y -= f[4 * k + 2] * v[k + W];
    if (h > 0) y -= f[4 * (k - W) + 2] * v[k - W];
    if (w + 1 < W) y -= f[4 * k + 3] * v[k + 1];
    if (w > 0) y -= f[4 * (k - 1) + 3] * v[k - 1];
    return y;
}

__device__ __forceinline__ void block_sum3(float (&v)[3], float (*sm)[32]) {
    for (int o2 = 16; o2 > 0; o2 >>= 1)
        for (int i = 0; i < 3; i++) v[i] += __shfl_down_sync(0xffffffffu, v[i], o2);
    if ((threadIdx.x & 31) == 0)
        for (int i = 0; i < 3; i++) sm[i][threadIdx.x >> 5] = v[i];
    __syncthreads();
    for (int i = 0; i < 3; i++) {
        float t = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sm[i][w];
        v[i] = t;
    }
}

// Residual loss of each sample: with r = feats channel 0, A the operator of
// channels 1..3 and a = A o, loss = 1 - (a.r)^2 / (|a|^2 |r|^2) -- the
// squared relative residual |r - omega a|^2 / |r|^2 left by the best scalar
// omega (the one the solver applies).  d loss / d a = -2 c / (q rr) (r - (c /
// q) a) with c = a.r, q = a.a, rr = r.r; d loss / d o = A (d loss / d a).
// One block per sample; scr holds a, then the gradient in a.
__global__ void __launch_bounds__(1024) k_loss_stencil(const float *__restrict__ o, const float *__restrict__ feats,
                                                       int H, int W, float *__restrict__ scr, bf16 *__restrict__ g,
                                                       float *__restrict__ loss) {
    const int b = blockIdx.x;
    const int64_t npix = (int64_t)H * W;
    const float *ob = o + b * npix, *fb = feats + 4 * b * npix;
    float *sb = scr + b * npix;
    __shared__ float sm[3][32];
    float acc[3] = {0.0f, 0.0f, 0.0f};
    for (int64_t k = threadIdx.x; k < npix; k += blockDim.x) {
        const float a = stencil_apply(fb, ob, H, W, k), r = fb[4 * k];
        sb[k] = a;
        acc[0] += a * r;
        acc[1] += a * a;
        acc[2] += r * r;
    }
    block_sum3(acc, sm);
    const float c = acc[0], q = acc[1] > 0.0f ? acc[1] : 1.0f, rr = acc[2] > 0.0f ? acc[2] : 1.0f;
    if (threadIdx.x == 0) loss[b] = 1.0f - c * c / (q * rr);
    const float f1 = -2.0f * c / (q * rr) / (float)gridDim.x, f2 = c / q;  // mean over the batch
    __syncthreads();  // every a is stored before the gradient overwrites it
    for (int64_t k = threadIdx.x; k < npix; k += blockDim.x) sb[k] = f1 * (fb[4 * k] - f2 * sb[k]);
    __syncthreads();
    for (int64_t k = threadIdx.x; k < npix; k += blockDim.x) {
        bf16 *gp = g + (b * npix + k) * 16;
        gp[0] = tobf(stencil_apply(fb, sb, H, W, k));
        for (int ch = 1; ch < 16; ch++) gp[ch] = tobf(0.0f);
    }
}

// Energy loss of each sample: with e = target, A the operator of channels
// 1..3 and u = o, loss = 1 - (u' A e)^2 / ((u' A u)(e' A e)) -- the squared
// relative A-norm error |e - omega u|_A^2 / |e|_A^2 left by the best scalar
// omega (the one the solver applies).  d loss / d u = -2 p / (q E) (A e - (p
// / q) A u) with p = u' A e, q = u' A u, E = e' A e.  One block per sample;
// scr holds A u.
__global__ void __launch_bounds__(1024) k_loss_energy(const float *__restrict__ o, const float *__restrict__ feats,
                                                      const float *__restrict__ t, int H, int W,
                                                      float *__restrict__ scr, bf16 *__restrict__ g,
                                                      float *__restrict__ loss) {
    const int b = blockIdx.x;
    const int64_t npix = (int64_t)H * W;
    const float *ob = o + b * npix, *fb = feats + 4 * b * npix, *tb = t + b * npix;
    float *sb = scr + b * npix;
    __shared__ float sm[3][32];
    float acc[3] = {0.0f, 0.0f, 0.0f};
    for (int64_t k = threadIdx.x; k < npix; k += blockDim.x) {
        const float au = stencil_apply(fb, ob, H, W, k), ae = stencil_apply(fb, tb, H, W, k);
        sb[k] = au;
        acc[0] += ob[k] * ae;
        acc[1] += ob[k] * au;
        acc[2] += tb[k] * ae;
    }
    block_sum3(acc, sm);
    const float pp = acc[0], q = acc[1] > 0.0f ? acc[1] : 1.0f, E = acc[2] > 0.0f ? acc[2] : 1.0f;
    if (threadIdx.x == 0) loss[b] = 1.0f - pp * pp / (q * E);
    const float f1 = -2.0f * pp / (q * E) / (float)gridDim.x, f2 = pp / q;  // mean over the batch
    for (int64_t k = threadIdx.x; k < npix; k += blockDim.x) {
        bf16 *gp = g + (b * npix + k) * 16;
        gp[0] = tobf(f1 * (stencil_apply(fb, tb, H, W, k) - f2 * sb[k]));
        for (int ch = 1; ch < 16; ch++) gp[ch] = tobf(0.0f);
    }
}

// Weight gradient as a GEMM over pixels, dW[co][ci][t] += sum_p G[p][co] X[p + off(t)][ci]:
// M = co, N = (t, ci) with n = t * CI + ci (real channels), K = pixels.  A
// block owns a 32 x 32 output tile and a range of WG_PIX pixels (split K);
// 256 threads, 2 x 2 outputs each; the partial sums go to the FP32 gradient
// with atomics (blockIdx.y == 0 also sums the bias gradient).  X and G are
// NHWC with padded channel strides CIS, COS.
constexpr int WG_TM = 32, WG_TN = 32, WG_TK = 32, WG_PIX = 2048;
__global__ void __launch_bounds__(256) k_wgrad(const bf16 *__restrict__ X, const bf16 *__restrict__ G, int B, int H,
                                               int W, int CIS, int CI, int COS, int CO, float *__restrict__ dW,
                                               float *__restrict__ db) {
    __shared__ float sG[WG_TK][WG_TM + 1], sX[WG_TK][WG_TN + 1];
    const int m0 = blockIdx.x * WG_TM, n0 = blockIdx.y * WG_TN;
    const int64_t P = (int64_t)B * H * W, p_begin = (int64_t)blockIdx.z * WG_PIX;
    const int64_t p_end = p_begin + WG_PIX < P ? p_begin + WG_PIX : P;
    const int tid = threadIdx.x, tm = (tid % 16) * 2, tn = (tid / 16) * 2;
    float acc[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}}, accb[2] = {0.0f, 0.0f};
    const int N = 9 * CI;
    const bool bias_col = blockIdx.y == 0 && tn == 0;
    for (int64_t p0 = p_begin; p0 < p_end; p0 += WG_TK) {
        for (int e = tid; e < WG_TK * WG_TM; e += 256) {
            const int kk = e / WG_TM, mm = e % WG_TM;
            const int64_t p = p0 + kk;
            const int co = m0 + mm;
            sG[kk][mm] = (p < p_end && co < CO) ? bf(G[p * COS + co]) : 0.0f;
        }
        for (int e = tid; e < WG_TK * WG_TN; e += 256) {
            const int kk = e / WG_TN, nn = e % WG_TN;
            const int64_t p = p0 + kk;
            const int n = n0 + nn;
            float v = 0.0f;
            if (p < p_end && n < N) {
                const int t = n / CI, ci = n % CI;
                const int x = (int)(p % W);
                const int64_t q = p / W;
                const int y = (int)(q % H);
                const int64_t b = q / H;
                const int yy = y + t / 3 - 1, xx = x + t % 3 - 1;
                if (yy >= 0 && yy < H && xx >= 0 && xx < W) v = bf(X[((b * H + yy) * W + xx) * CIS + ci]);
            }
            sX[kk][nn] = v;
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < WG_TK; kk++) {
            const float g0 = sG[kk][tm], g1 = sG[kk][tm + 1], x0 = sX[kk][tn], x1 = sX[kk][tn + 1];
            acc[0][0] += g0 * x0;
            acc[0][1] += g0 * x1;
            acc[1][0] += g1 * x0;
            acc[1][1] += g1 * x1;
            if (bias_col) {
                accb[0] += g0;
                accb[1] += g1;
            }
        }
        __syncthreads();
    }
    for (int a = 0; a < 2; a++) {
        const int co = m0 + tm + a;
        if (co >= CO) continue;
        for (int c = 0; c < 2; c++) {
            const int n = n0 + tn + c;
            if (n >= N) continue;
            const int t = n / CI, ci = n % CI;
            atomicAdd(&dW[((size_t)co * CI + ci) * 9 + t], acc[a][c]);
        }
        if (bias_col) atomicAdd(&db[co], accb[a]);
    }
}

// dgrad weights: Wt[ci][co][ky][kx] = W[co][ci][2-ky][2-kx]
__global__ void k_flip_transpose(const float *__restrict__ w, int CO, int CI, float *__restrict__ wt) {
    const int64_t n = (int64_t)CO * CI * 9;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const int t = (int)(e % 9);
        const int64_t q = e / 9;
        const int co = (int)(q % CO), ci = (int)(q / CO);
        wt[e] = w[((size_t)co * CI + ci) * 9 + (8 - t)];
    }
}

__global__ void k_adam(float *__restrict__ w, float *__restrict__ m, float *__restrict__ v, const float *__restrict__ g,
                       int64_t n, float lr, float b1, float b2, float c1, float c2, float eps) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const float gg = g[e];
        const float mm = b1 * m[e] + (1.0f - b1) * gg, vv = b2 * v[e] + (1.0f - b2) * gg * gg;
        m[e] = mm;
        v[e] = vv;
        w[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    }
}

int blocks(int64_t n) { return (int)((n + 255) / 256 < 4 * 1184 ? (n + 255) / 256 : 4 * 1184); }

}  // namespace

// ----------------------------------------------------------------- network --
struct UnetLayer {
    int cin, cout;          // real channels
    int cin_p, cout_p;      // padded to multiples of 16
    int relu;
    size_t woff, boff;      // offsets in the parameter arrays: W [cout][cin][9], b [cout_p]
    void *wpack = nullptr;  // forward weights
    void *wpack_t = nullptr;  // input-gradient weights (taps flipped, in/out swapped)
};

struct asd2g_unet {
    cudaStream_t st = nullptr;       // the stream launches go to
    cudaStream_t own_st = nullptr;   // created here when none was given
    cudaStream_t home_st = nullptr;  // the creation-time stream (given or own)
    bool own_stream = false;
    int max_b = 0, max_h = 0, max_w = 0;
    std::vector<UnetLayer> L;
    size_t nparam = 0;
    float *w = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;
    float *wt_tmp = nullptr, *zero_bias = nullptr;
    int step = 0;
    float lr = 0.0f;
    int *err = nullptr;
    std::vector<void *> allocs;
    bf16 *x0 = nullptr, *a[4] = {}, *e[4] = {}, *p[3] = {}, *c[3] = {}, *da[3] = {}, *d[3] = {};
    float *out = nullptr;
    bf16 *gA = nullptr, *gB = nullptr, *gC = nullptr, *gL = nullptr;
    float *dskip[3] = {};
    float *loss = nullptr, *loss_host = nullptr;
    float *lscr = nullptr;  // residual loss: A out, then its gradient
    float *wpart = nullptr; // split-K partial sums of the tensor-core weight gradients
};

namespace {

// encoder e0a e0b e1a e1b e2a e2b e3a e3b | decoder d2a d2b d1a d1b d0a d0b | out
const int LAYERS[15][3] = {{4, 16, 1},   {16, 16, 1}, {16, 32, 1}, {32, 32, 1},  {32, 64, 1},
                           {64, 64, 1},  {64, 128, 1}, {128, 128, 1}, {192, 64, 1}, {64, 64, 1},
                           {96, 32, 1},  {32, 32, 1}, {48, 16, 1}, {16, 16, 1},  {16, 1, 0}};
const int CH[4] = {16, 32, 64, 128};

template <typename T> int ualloc(asd2g_unet *u, T **p, size_t n) {
    if (cudaMalloc(p, sizeof(T) * (n ? n : 1)) != cudaSuccess) {
        cudaGetLastError();
        return api_fail(ASD2G_E_NOMEM, "U-Net device allocation failed");
    }
    u->allocs.push_back(*p);
    return ASD2G_OK;
}

int pad16(int c) { return (c + 15) / 16 * 16; }

// split-K work buffer of the tensor-core weight gradient: about 2 x 148 CTAs
// of 128 rows x up to 128 columns (larger products take longer K ranges)
constexpr size_t UNET_WPART = (size_t)340 * 128 * 128;

bool wgrad_tensor_cores() {
    static const bool v = [] {
        const char *e = std::getenv("ASD2G_WGRAD");
        return !(e && std::strcmp(e, "cuda") == 0);
    }();
    return v;
}

int cuda_ok(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return ASD2G_OK;
    char msg[200];
    snprintf(msg, sizeof(msg), "U-Net %s: %s", what, cudaGetErrorString(e));
    return api_fail(ASD2G_E_CUDA, msg);
}

int repack(asd2g_unet *u) {
    for (auto &l : u->L) {
        int rc = asd2g_conv_pack_weights(u->w + l.woff, l.cout, l.cin, l.cout_p, l.cin_p, l.wpack, u->st);
        if (rc) return api_fail(rc, "weight packing");
        k_flip_transpose<<<blocks((int64_t)l.cout * l.cin * 9), 256, 0, u->st>>>(u->w + l.woff, l.cout, l.cin,
                                                                                  u->wt_tmp);
        rc = asd2g_conv_pack_weights(u->wt_tmp, l.cin, l.cout, pad16(l.cin), l.cout_p, l.wpack_t, u->st);
        if (rc) return api_fail(rc, "weight packing (input gradient)");
    }
    return cuda_ok("repack");
}

int conv(asd2g_unet *u, int li, const bf16 *in, int B, int H, int W, bf16 *out, float *out32) {
    const UnetLayer &l = u->L[li];
    const int rc = conv3x3_tc(in, B, H, W, l.cin_p, l.wpack, u->w + l.boff, l.cout_p, out, out32, l.relu, u->err, u->st);
    return rc ? api_fail(rc, "tensor-core convolution launch") : ASD2G_OK;
}

// keep_concat: materialise each decoder input (upsampled low + skip) in u->c
// for the weight gradients; otherwise the decoder convolutions read the two
// sources directly.
int forward(asd2g_unet *u, int B, int H, int W, bool keep_concat) {
    int rc = ASD2G_OK;
    const bf16 *in = u->x0;
    for (int lv = 0; lv < 4 && !rc; lv++) {
        const int h = H >> lv, w = W >> lv;
        rc = conv(u, 2 * lv, in, B, h, w, u->a[lv], nullptr);
        if (!rc) rc = conv(u, 2 * lv + 1, u->a[lv], B, h, w, u->e[lv], nullptr);
        if (!rc && lv < 3) {
            k_pool<<<blocks((int64_t)B * (h / 2) * (w / 2) * (CH[lv] / 8)), 256, 0, u->st>>>(u->e[lv], B, h, w,
                                                                                            CH[lv], u->p[lv]);
            in = u->p[lv];
        }
    }
    const bf16 *low = u->e[3];
    int cl = 128;
    for (int lv = 2; lv >= 0 && !rc; lv--) {
        const int h = H >> lv, w = W >> lv, cs = CH[lv];
        const int li = 8 + 2 * (2 - lv);
        if (keep_concat) {
            k_upcat<<<blocks((int64_t)B * h * w * (cl + cs)), 256, 0, u->st>>>(low, cl, u->e[lv], cs, B, h, w,
                                                                              u->c[lv]);
            rc = conv(u, li, u->c[lv], B, h, w, u->da[lv], nullptr);
        } else {
            const UnetLayer &l = u->L[li];
            const int rc2 = conv3x3_tc(u->e[lv], B, h, w, l.cin_p, l.wpack, u->w + l.boff, l.cout_p, u->da[lv],
                                       nullptr, l.relu, u->err, u->st, low, cl);
            rc = rc2 ? api_fail(rc2, "tensor-core convolution launch") : ASD2G_OK;
        }
        if (!rc) rc = conv(u, li + 1, u->da[lv], B, h, w, u->d[lv], nullptr);
        low = u->d[lv];
        cl = cs;
    }
    if (!rc) rc = conv(u, 14, u->d[0], B, H, W, nullptr, u->out);
    return rc ? rc : cuda_ok("forward");
}

// Backward of layer li: dY its output gradient, X its input, Y its output
// (nullptr for the linear last layer); accumulates dW, db; writes dX (BF16,
// padded input channels) unless dx is nullptr.
int layer_back(asd2g_unet *u, int li, const bf16 *X, const bf16 *Y, const bf16 *dY, int B, int H, int W, bf16 *dx) {
    const UnetLayer &l = u->L[li];
    const int64_t n = (int64_t)B * H * W * l.cout_p;
    const bf16 *G = dY;
    if (Y) {
        k_relu_mask<<<blocks(n), 256, 0, u->st>>>(dY, Y, n, u->gC);
        G = u->gC;
    }
    // weight and bias gradients on the tensor cores (FP32 CUDA-core form for
    // other padded widths, or with ASD2G_WGRAD=cuda)
    int wrc = 1;
    if (wgrad_tensor_cores())
        wrc = wgrad_tc(X, G, B, H, W, l.cin_p, l.cin, l.cout_p, l.cout, u->g + l.woff, u->g + l.boff, u->wpart,
                       UNET_WPART, u->err, u->st);
    if (wrc < 0) return api_fail(wrc, "tensor-core weight gradient launch");
    if (wrc == 1) {
        const int64_t P = (int64_t)B * H * W;
        const dim3 grid((l.cout + WG_TM - 1) / WG_TM, (9 * l.cin + WG_TN - 1) / WG_TN,
                        (int)((P + WG_PIX - 1) / WG_PIX));
        k_wgrad<<<grid, 256, 0, u->st>>>(X, G, B, H, W, l.cin_p, l.cin, l.cout_p, l.cout, u->g + l.woff,
                                         u->g + l.boff);
    }
    if (dx) {
        const int rc = conv3x3_tc(G, B, H, W, l.cout_p, l.wpack_t, u->zero_bias, pad16(l.cin), dx, nullptr, 0, u->err,
                                  u->st);
        if (rc) return api_fail(rc, "input-gradient convolution launch");
    }
    return cuda_ok("layer backward");
}

int backward(asd2g_unet *u, int B, int H, int W) {
    bf16 *gA = u->gA, *gB = u->gB;
    int rc = layer_back(u, 14, u->d[0], nullptr, u->gL, B, H, W, gA);
    // decoder levels 0, 1, 2 (reverse of the forward order 2, 1, 0)
    for (int lv = 0; lv < 3 && !rc; lv++) {
        const int h = H >> lv, w = W >> lv, li = 8 + 2 * (2 - lv);
        const int cs = CH[lv], cl = lv == 2 ? 128 : CH[lv + 1];
        // gA: gradient of d[lv]
        rc = layer_back(u, li + 1, u->da[lv], u->d[lv], gA, B, h, w, gB);
        if (!rc) rc = layer_back(u, li, u->c[lv], u->da[lv], gB, B, h, w, gA);  // gA: d c[lv] (cl + cs channels)
        if (rc) break;
        k_upcat_back<<<blocks((int64_t)B * h * w * (cl + cs)), 256, 0, u->st>>>(gA, cl, cs, B, h, w, gB, u->dskip[lv]);
        std::swap(gA, gB);  // gA: gradient of the level below's decoder output (or of e3)
    }
    // encoder: level 3, then 2, 1, 0 (gA holds the gradient of e[3])
    for (int lv = 3; lv >= 0 && !rc; lv--) {
        const int h = H >> lv, w = W >> lv;
        rc = layer_back(u, 2 * lv + 1, u->a[lv], u->e[lv], gA, B, h, w, gB);
        const bf16 *xin = lv == 0 ? u->x0 : u->p[lv - 1];
        if (!rc) rc = layer_back(u, 2 * lv, xin, u->a[lv], gB, B, h, w, lv == 0 ? nullptr : gA);
        if (rc || lv == 0) break;
        // gA: gradient of p[lv-1]; de[lv-1] = dskip[lv-1] + pool-back(gA)
        const int C = CH[lv - 1];
        k_pool_back_add<<<blocks((int64_t)B * (2 * h) * (2 * w) * C), 256, 0, u->st>>>(u->dskip[lv - 1], gA, B, 2 * h,
                                                                                      2 * w, C, gB);
        std::swap(gA, gB);
    }
    return rc ? rc : cuda_ok("backward");
}

void release(asd2g_unet *u) {
    for (void *p : u->allocs) cudaFree(p);
    if (u->loss_host) cudaFreeHost(u->loss_host);
    if (u->own_stream && u->own_st) cudaStreamDestroy(u->own_st);
    delete u;
}

}  // namespace

extern "C" {

int asd2g_unet_create(int max_batch, int max_h, int max_w, void *stream, asd2g_unet **out) try {
    if (!out || max_batch < 1 || max_h < 8 || max_w < 8 || max_h % 8 || max_w % 8)
        return api_fail(ASD2G_E_ARG, "unet_create: sizes must be positive multiples of 8");
    *out = nullptr;
    asd2g_unet *u = new (std::nothrow) asd2g_unet();
    if (!u) return api_fail(ASD2G_E_NOMEM, "host allocation failed");
    u->max_b = max_batch;
    u->max_h = max_h;
    u->max_w = max_w;
    if (stream) u->st = (cudaStream_t)stream;
    else {
        if (cudaStreamCreateWithFlags(&u->own_st, cudaStreamNonBlocking) != cudaSuccess) {
            delete u;
            return api_fail(ASD2G_E_CUDA, "cudaStreamCreate failed");
        }
        u->st = u->own_st;
        u->own_stream = true;
    }
    u->home_st = u->st;
    size_t off = 0;
    for (int i = 0; i < 15; i++) {
        UnetLayer l;
        l.cin = LAYERS[i][0];
        l.cout = LAYERS[i][1];
        l.relu = LAYERS[i][2];
        l.cin_p = pad16(l.cin);
        l.cout_p = pad16(l.cout);
        l.woff = off;
        off += (size_t)l.cout * l.cin * 9;
        l.boff = off;
        off += (size_t)l.cout_p;
        u->L.push_back(l);
    }
    u->nparam = off;
    int rc = ASD2G_OK;
    float **pa[] = {&u->w, &u->m, &u->v, &u->g};
    for (float **pp : pa)
        if (!rc) rc = ualloc(u, pp, u->nparam);
    if (!rc) rc = ualloc(u, &u->wt_tmp, (size_t)192 * 192 * 9);
    if (!rc) rc = ualloc(u, &u->zero_bias, 256);
    if (!rc) rc = ualloc(u, &u->err, 1);
    for (auto &l : u->L) {
        if (rc) break;
        rc = ualloc(u, reinterpret_cast<uint8_t **>(&l.wpack), asd2g_conv_wpack_bytes(l.cout_p, l.cin_p));
        if (!rc) rc = ualloc(u, reinterpret_cast<uint8_t **>(&l.wpack_t), asd2g_conv_wpack_bytes(pad16(l.cin), l.cout_p));
    }
    const size_t P = (size_t)max_batch * max_h * max_w;
    if (!rc) rc = ualloc(u, &u->x0, P * 16);
    for (int lv = 0; lv < 4 && !rc; lv++) {
        const size_t Pl = P >> (2 * lv);
        rc = ualloc(u, &u->a[lv], Pl * CH[lv]);
        if (!rc) rc = ualloc(u, &u->e[lv], Pl * CH[lv]);
        if (!rc && lv < 3) rc = ualloc(u, &u->p[lv], (Pl / 4) * CH[lv]);
        if (!rc && lv < 3) rc = ualloc(u, &u->c[lv], Pl * (CH[lv] + (lv == 2 ? 128 : CH[lv + 1])));
        if (!rc && lv < 3) rc = ualloc(u, &u->da[lv], Pl * CH[lv]);
        if (!rc && lv < 3) rc = ualloc(u, &u->d[lv], Pl * CH[lv]);
        if (!rc && lv < 3) rc = ualloc(u, &u->dskip[lv], Pl * CH[lv]);
    }
    if (!rc) rc = ualloc(u, &u->out, P);
    if (!rc) rc = ualloc(u, &u->gA, P * 48);
    if (!rc) rc = ualloc(u, &u->gB, P * 48);
    if (!rc) rc = ualloc(u, &u->gC, P * 16);
    if (!rc) rc = ualloc(u, &u->gL, P * 16);
    if (!rc) rc = ualloc(u, &u->loss, (size_t)max_batch);
    if (!rc) rc = ualloc(u, &u->lscr, P);
    if (!rc) rc = ualloc(u, &u->wpart, UNET_WPART);
    if (!rc && cudaMallocHost(&u->loss_host, sizeof(float) * max_batch) != cudaSuccess)
        rc = api_fail(ASD2G_E_NOMEM, "pinned allocation failed");
    if (rc) {
        release(u);
        return rc;
    }
    cudaMemsetAsync(u->zero_bias, 0, sizeof(float) * 256, u->st);
    cudaMemsetAsync(u->err, 0, sizeof(int), u->st);
    cudaMemsetAsync(u->w, 0, sizeof(float) * u->nparam, u->st);
    *out = u;
    return cuda_ok("create");
} catch (...) {
    return asd2g::api_exception("asd2g_unet_create");
}

int asd2g_unet_destroy(asd2g_unet *u) try {
    if (!u) return ASD2G_OK;
    cudaStreamSynchronize(u->st);
    release(u);
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_unet_destroy");
}

size_t asd2g_unet_nparams(asd2g_unet *u) { return u ? u->nparam : 0; }

// He-normal initialisation (std = sqrt(2 / (9 cin))), the last layer scaled by 0.1, zero biases.
int asd2g_unet_init(asd2g_unet *u, unsigned long long seed) try {
    if (!u) return api_fail(ASD2G_E_ARG, "null network");
    std::vector<float> h(u->nparam, 0.0f);
    std::mt19937_64 rng(seed);
    for (size_t li = 0; li < u->L.size(); li++) {
        const UnetLayer &l = u->L[li];
        std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (9.0f * (float)l.cin)) * (l.relu ? 1.0f : 0.1f));
        for (size_t k = 0; k < (size_t)l.cout * l.cin * 9; k++) h[l.woff + k] = nd(rng);
    }
    return asd2g_unet_set_params(u, h.data());
} catch (...) {
    return asd2g::api_exception("asd2g_unet_init");
}

int asd2g_unet_set_params(asd2g_unet *u, const float *host) try {
    if (!u || !host) return api_fail(ASD2G_E_ARG, "null argument");
    cudaMemcpyAsync(u->w, host, sizeof(float) * u->nparam, cudaMemcpyHostToDevice, u->st);
    cudaMemsetAsync(u->m, 0, sizeof(float) * u->nparam, u->st);
    cudaMemsetAsync(u->v, 0, sizeof(float) * u->nparam, u->st);
    u->step = 0;
    const int rc = repack(u);
    if (rc) return rc;
    return cudaStreamSynchronize(u->st) == cudaSuccess ? ASD2G_OK : cuda_ok("set_params");
} catch (...) {
    return asd2g::api_exception("asd2g_unet_set_params");
}

int asd2g_unet_get_params(asd2g_unet *u, float *host) try {
    if (!u || !host) return api_fail(ASD2G_E_ARG, "null argument");
    cudaMemcpyAsync(host, u->w, sizeof(float) * u->nparam, cudaMemcpyDeviceToHost, u->st);
    return cudaStreamSynchronize(u->st) == cudaSuccess ? ASD2G_OK : cuda_ok("get_params");
} catch (...) {
    return asd2g::api_exception("asd2g_unet_get_params");
}

// A forward pass fits when its B * H * W pixels fit the activation buffers
// (max_batch * max_h * max_w pixels, every level a quarter of the one
// above); a training step also needs B <= max_batch (per-image losses) and
// H * W <= max_h * max_w.
static int check_shape(asd2g_unet *u, int B, int H, int W, bool training = true) {
    const size_t cap = u ? (size_t)u->max_b * u->max_h * u->max_w : 0;
    if (!u || B < 1 || H < 8 || W < 8 || H % 8 || W % 8 || (size_t)B * H * W > cap ||
        (training && (B > u->max_b || (size_t)H * W > (size_t)u->max_h * u->max_w)))
        return api_fail(ASD2G_E_ARG, "U-Net batch or image size outside the created maximum (multiples of 8)");
    return ASD2G_OK;
}

// feats: device FP32 [B][H][W][4]; out: device FP32 [B][H][W].
int asd2g_unet_forward(asd2g_unet *u, int B, int H, int W, const float *feats, float *out) try {
    NvtxRange nv("U-Net forward");
    int rc = check_shape(u, B, H, W, false);
    if (rc) return rc;
    if (!feats || !out) return api_fail(ASD2G_E_ARG, "null argument");
    const int64_t npix = (int64_t)B * H * W;
    k_feats_pack<<<blocks(npix), 256, 0, u->st>>>(feats, npix, u->x0);
    rc = forward(u, B, H, W, false);
    if (rc) return rc;
    cudaMemcpyAsync(out, u->out, sizeof(float) * npix, cudaMemcpyDeviceToDevice, u->st);
    return cuda_ok("unet_forward");
} catch (...) {
    return asd2g::api_exception("asd2g_unet_forward");
}

static int train_finish(asd2g_unet *u, int B, int H, int W, float *loss_mean) {
    cudaMemsetAsync(u->g, 0, sizeof(float) * u->nparam, u->st);
    int rc = backward(u, B, H, W);
    if (rc) return rc;
    u->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)u->step), c2 = 1.0f - std::pow(b2, (float)u->step);
    k_adam<<<blocks((int64_t)u->nparam), 256, 0, u->st>>>(u->w, u->m, u->v, u->g, (int64_t)u->nparam, u->lr, b1, b2,
                                                         c1, c2, 1e-8f);
    rc = repack(u);
    if (rc) return rc;
    if (loss_mean) {
        cudaMemcpyAsync(u->loss_host, u->loss, sizeof(float) * B, cudaMemcpyDeviceToHost, u->st);
        if (cudaStreamSynchronize(u->st) != cudaSuccess) return cuda_ok("train_step");
        float s = 0.0f;
        for (int b = 0; b < B; b++) s += u->loss_host[b];
        *loss_mean = s / (float)B;
    }
    return cuda_ok("train_step");
}

// One Adam step on a batch: loss = mean over samples of |out - target|^2 / |target|^2.
int asd2g_unet_train_step(asd2g_unet *u, int B, int H, int W, const float *feats, const float *target, float lr,
                          float *loss_mean) try {
    NvtxRange nv("U-Net train step (MSE)");
    int rc = check_shape(u, B, H, W);
    if (rc) return rc;
    if (!feats || !target) return api_fail(ASD2G_E_ARG, "null argument");
    const int64_t npix = (int64_t)H * W;
    k_feats_pack<<<blocks((int64_t)B * npix), 256, 0, u->st>>>(feats, (int64_t)B * npix, u->x0);
    rc = forward(u, B, H, W, true);
    if (rc) return rc;
    k_loss<<<B, 256, 0, u->st>>>(u->out, target, npix, u->gL, u->loss);
    u->lr = lr;
    return train_finish(u, B, H, W, loss_mean);
} catch (...) {
    return asd2g::api_exception("asd2g_unet_train_step");
}

// One Adam step on the energy loss: mean over samples of the relative A-norm
// error 1 - (out' A t)^2 / ((out' A out)(t' A t)).
int asd2g_unet_train_step_energy(asd2g_unet *u, int B, int H, int W, const float *feats, const float *target,
                                 float lr, float *loss_mean) try {
    NvtxRange nv("U-Net train step (energy)");
    int rc = check_shape(u, B, H, W);
    if (rc) return rc;
    if (!feats || !target) return api_fail(ASD2G_E_ARG, "null argument");
    const int64_t npix = (int64_t)H * W;
    k_feats_pack<<<blocks((int64_t)B * npix), 256, 0, u->st>>>(feats, (int64_t)B * npix, u->x0);
    rc = forward(u, B, H, W, true);
    if (rc) return rc;
    k_loss_energy<<<B, 1024, 0, u->st>>>(u->out, feats, target, H, W, u->lscr, u->gL, u->loss);
    u->lr = lr;
    return train_finish(u, B, H, W, loss_mean);
} catch (...) {
    return asd2g::api_exception("asd2g_unet_train_step_energy");
}

// One Adam step on the residual loss: mean over samples of 1 - cos^2(A out, r).
int asd2g_unet_train_step_residual(asd2g_unet *u, int B, int H, int W, const float *feats, float lr,
                                   float *loss_mean) try {
    NvtxRange nv("U-Net train step (residual)");
    int rc = check_shape(u, B, H, W);
    if (rc) return rc;
    if (!feats) return api_fail(ASD2G_E_ARG, "null argument");
    const int64_t npix = (int64_t)H * W;
    k_feats_pack<<<blocks((int64_t)B * npix), 256, 0, u->st>>>(feats, (int64_t)B * npix, u->x0);
    rc = forward(u, B, H, W, true);
    if (rc) return rc;
    k_loss_stencil<<<B, 1024, 0, u->st>>>(u->out, feats, H, W, u->lscr, u->gL, u->loss);
    u->lr = lr;
    return train_finish(u, B, H, W, loss_mean);
} catch (...) {
    return asd2g::api_exception("asd2g_unet_train_step_residual");
}

// NULL returns the network to the stream it was created with.
int asd2g_unet_set_stream(asd2g_unet *u, void *stream) try {
    if (!u) return api_fail(ASD2G_E_ARG, "null network");
    u->st = stream ? (cudaStream_t)stream : u->home_st;
    return ASD2G_OK;
} catch (...) {
    return asd2g::api_exception("asd2g_unet_set_stream");
}

int asd2g_unet_get_grads(asd2g_unet *u, float *host) try {
    if (!u || !host) return api_fail(ASD2G_E_ARG, "null argument");
    cudaMemcpyAsync(host, u->g, sizeof(float) * u->nparam, cudaMemcpyDeviceToHost, u->st);
    return cudaStreamSynchronize(u->st) == cudaSuccess ? ASD2G_OK : cuda_ok("get_grads");
} catch (...) {
    return asd2g::api_exception("asd2g_unet_get_grads");
}

int asd2g_unet_error_flag(asd2g_unet *u, int *flag) try {
    if (!u || !flag) return api_fail(ASD2G_E_ARG, "null argument");
    cudaMemcpyAsync(flag, u->err, sizeof(int), cudaMemcpyDeviceToHost, u->st);
    return cudaStreamSynchronize(u->st) == cudaSuccess ? ASD2G_OK : cuda_ok("error flag");
} catch (...) {
    return asd2g::api_exception("asd2g_unet_error_flag");
}

}  // extern "C"
