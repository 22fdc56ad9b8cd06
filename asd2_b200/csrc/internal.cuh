// Declarations shared by the asd2g translation units (not part of the ABI).
#pragma once
#include <cstdio>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "common.cuh"

namespace asd2g {

// NVTX range for the host-side phases of the ABI calls (level set, momentum,
// assembly, solve, projection, batch phases): visible in an NVTX-aware
// profiler's timeline, free when none is attached.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// Division by a grid spacing.  When h is a power of two, x / h and
// x * (1/h) are the same IEEE result, so the multiply is used; otherwise the
// division is kept.  Either way the result equals the reference's x / h.
template <typename T>
struct DivHT {
    T h, inv;
    int pow2;
    __device__ __forceinline__ T operator()(T x) const { return pow2 ? x * inv : x / h; }
};
// FP32 (the mixed-precision path, not bit-exact by design): always the
// multiply by the rounded reciprocal, within 1.5 ulp of x / h and without
// the per-call branch.
template <>
struct DivHT<float> {
    float h, inv;
    int pow2;
    __device__ __forceinline__ float operator()(float x) const { return x * inv; }
};
using DivH = DivHT<double>;
DivH make_divh(double h);
DivHT<float> make_divh_f(double h);

// api.cu: set the thread's last-error text (read by asd2g_last_error)
void asd2g_set_error_text(const char *msg);

// bc.cu
void launch_fill_uv(const Grid &g, double *u, double *v, cudaStream_t st);
void launch_fill_p(const Grid &g, double *a, cudaStream_t st);
void launch_fill_side(const Grid &g, double *a, int grid_kind, int side, int kind, cudaStream_t st);

}  // namespace asd2g
