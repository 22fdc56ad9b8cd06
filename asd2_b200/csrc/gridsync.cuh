// Grid-wide barrier and reductions for one-launch (cooperative) solvers.
//
// The barrier is a monotonic arrival counter, zeroed before the launch:
// thread 0 of each CTA arrives with a release reduction (ordering the CTA's
// writes, made visible to it by the CTA barrier, before its arrival) and
// polls with acquire loads until every CTA of this barrier has arrived; the
// CTA barrier after it orders the other threads' reads.  The wait is
// bounded: after GRID_SPIN_LIMIT polls (L2 round trips, about 0.3 us each)
// the CTA sets the error word and returns false, and every other CTA sees
// the error word at its next poll and returns false too.  Data written by
// other CTAs during the launch must be read with L2-only loads (__ldcg).
//
// Reductions: every CTA writes its block sums to its own slots; after the
// barrier every CTA adds all slots in the same fixed order, so every CTA
// holds the same scalars and takes the same branches.
#pragma once
#include <cstdint>

namespace asd2g {

constexpr unsigned GRID_SPIN_LIMIT = 1u << 22;
constexpr int GRID_SLOTS = 4;  // reduction slots per CTA

__device__ __forceinline__ unsigned grid_ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// bar[0]: arrivals, bar[1]: error word; flag: a shared int of the CTA.
__device__ __forceinline__ bool grid_sync(unsigned *bar, int ncta, unsigned &epoch, int &flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        epoch++;
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
        const unsigned target = epoch * (unsigned)ncta;
        int good = 1;
        for (unsigned n = 0; grid_ld_acquire(bar) < target; n++) {
            if (n > GRID_SPIN_LIMIT || *(volatile unsigned *)(bar + 1)) {
                atomicExch(bar + 1, 1u);
                good = 0;
                break;
            }
        }
        flag = good;
    }
    __syncthreads();
    return flag != 0;
}

// Block sums of NV values (block of NT threads) into this CTA's slots; red
// holds NV x NT/32 doubles of shared memory.
template <int NV, int NT> __device__ __forceinline__ void grid_put_partial(double *partial, double *red, double (&v)[NV]) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++) {
        double s = v[q];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) red[q * (NT / 32) + wid] = s;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double s = lane < NT / 32 ? red[q * (NT / 32) + lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0) __stcg(partial + GRID_SLOTS * blockIdx.x + q, s);
        }
    }
}

// Sum of every CTA's slots, the same order in every CTA -> tot (shared).
template <int NV> __device__ __forceinline__ void grid_get_total(const double *partial, int ncta, double *tot) {
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double s = 0.0;
            for (int c = lane; c < ncta; c += 32) s += __ldcg(partial + GRID_SLOTS * c + q);
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0) tot[q] = s;
        }
    }
    __syncthreads();
}

}  // namespace asd2g
