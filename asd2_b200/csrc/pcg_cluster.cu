// Cluster-resident Jacobi-PCG: the whole solve in one launch of one
// thread-block cluster (up to 16 CTAs of 1024 threads on 16 SMs).
//
// The system's rows i are split into CS contiguous slabs, one per CTA.  Each
// CTA keeps its slab of the direction vector p and of the coefficients
// (diag, ce, cn, Minv) in shared memory; x, r and q stay in registers (at most
// four unknowns per thread).  The SpMV reads the rows just outside the slab
// from the neighbouring CTAs' shared memory (distributed shared memory), and
// the two dot products of an iteration are reduced by writing each CTA's
// partial into every CTA's slot array, so after the hardware cluster barrier
// each CTA sums the same CS values in the same order: every CTA holds
// identical, deterministic scalars and takes identical control decisions.
//
// Iteration (textbook PCG, as k_pcg_a/k_pcg_b):
//   p = Minv r + beta p                    (own slab, in place)
//   cluster barrier 1                      (p visible cluster-wide)
//   q = A p, partial p.q -> all slots A    (halo rows from the neighbours)
//   cluster barrier 2 -> alpha = rho / p.q
//   x += alpha p, r -= alpha q, partials r.Minv r, r.r -> all slots B
//   cluster barrier 3 -> beta, rho, convergence
// p is updated in place only after barrier 3, when every remote read of the
// previous p (between barriers 1 and 2) has completed; slot A is rewritten
// only after barrier 1 of the next iteration and slot B after barrier 2.
// All waits are hardware cluster barriers (no spin loops).
#include <cooperative_groups.h>

#include "pressure.cuh"

namespace cg = cooperative_groups;

namespace asd2g {

constexpr int PC_THREADS = 1024;
constexpr int PC_UPT = 4;  // unknowns per thread
constexpr int PC_MAX_CTA_UNKNOWNS = PC_THREADS * PC_UPT;
constexpr int PC_MAX_CLUSTER = 16;

// Sum of one value per thread over the block (fixed order); result in all
// threads.  sh must hold 32 doubles; the trailing barrier lets sh be reused.
__device__ __forceinline__ double cta_sum(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sh[w];
    __syncthreads();
    return s;
}

struct PcgClusterArgs {
    int nx, ny, cs, rows_max;
    Sys S;
    double *x;
    KState *ks;
    double tol;
    int maxit;
};

__global__ void __launch_bounds__(PC_THREADS, 1) k_pcg_cluster(PcgClusterArgs a) {
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int CS = a.cs, nx = a.nx, ny = a.ny;
    const int r0 = (int)((int64_t)rank * nx / CS), r1 = (int)((int64_t)(rank + 1) * nx / CS);
    const int rows = r1 - r0, nloc = rows * ny, cap = a.rows_max * ny;
    extern __shared__ double smem[];
    double *sp = smem, *sdiag = smem + cap, *sce = smem + 2 * cap, *scn = smem + 3 * cap, *sminv = smem + 4 * cap;
    double *slotA = smem + 5 * cap;            // [PC_MAX_CLUSTER]
    double *slotB = slotA + PC_MAX_CLUSTER;    // [3][PC_MAX_CLUSTER]
    double *red = slotB + 3 * PC_MAX_CLUSTER;  // [32]
    // neighbours' slabs (only rows r0-1 and r1 are read)
    const double *sp_lo = rank > 0 ? cluster.map_shared_rank(sp, rank - 1) : nullptr;
    const double *sce_lo = rank > 0 ? cluster.map_shared_rank(sce, rank - 1) : nullptr;
    const double *sp_hi = rank < CS - 1 ? cluster.map_shared_rank(sp, rank + 1) : nullptr;
    const int rows_lo = rank > 0 ? r0 - (int)((int64_t)(rank - 1) * nx / CS) : 0;
    const Sys &S = a.S;

    double x[PC_UPT], r[PC_UPT], q[PC_UPT];
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
#pragma unroll
    for (int u = 0; u < PC_UPT; u++) {
        const int t = threadIdx.x + u * PC_THREADS;
        x[u] = r[u] = q[u] = 0.0;
        if (t < nloc) {
            const int64_t k = (int64_t)r0 * ny + t;
            sdiag[t] = S.diag[k];
            sce[t] = S.ce[k];
            scn[t] = S.cn[k];
            const double mi = S.minv[k];
            sminv[t] = mi;
            sp[t] = 0.0;
            const double bk = S.b[k];
            r[u] = bk;
            acc0 += bk * bk;
            acc1 += bk * (mi * bk);
        }
    }
    // reduce (b.b, r.Minv r) -> slots B [0], [1]
    {
        const double s0 = cta_sum(acc0, red), s1 = cta_sum(acc1, red);
        if (threadIdx.x < CS) {
            double *dst = cluster.map_shared_rank(slotB, (int)threadIdx.x);
            dst[rank] = s0;
            dst[PC_MAX_CLUSTER + rank] = s1;
        }
    }
    cluster.sync();
    double bb = 0.0, rho = 0.0;
    for (int c = 0; c < CS; c++) {
        bb += slotB[c];
        rho += slotB[PC_MAX_CLUSTER + c];
    }
    double bn = sqrt(bb);
    if (bn == 0.0) bn = 1.0;
    double res = sqrt(bb) / bn, beta = 0.0;
    int it = 0, status = 0;
    bool done = !(res > a.tol) || a.maxit <= 0;
    const bool pin_here = S.pinned && rank == 0;

    while (!done) {
        // p = Minv r + beta p (own slab)
#pragma unroll
        for (int u = 0; u < PC_UPT; u++) {
            const int t = threadIdx.x + u * PC_THREADS;
            if (t < nloc) sp[t] = sminv[t] * r[u] + beta * sp[t];
        }
        cluster.sync();  // 1
        acc0 = 0.0;
#pragma unroll
        for (int u = 0; u < PC_UPT; u++) {
            const int t = threadIdx.x + u * PC_THREADS;
            if (t < nloc) {
                const int li = t / ny, j = t - li * ny, i = r0 + li;
                const double pc = sp[t];
                double y = 0.0;
                if (!(pin_here && t == 0)) {
                    if (j > 0) y += -scn[t - 1] * sp[t - 1];
                    if (i > 0) {
                        if (li > 0) y += -sce[t - ny] * sp[t - ny];
                        else y += -sce_lo[(rows_lo - 1) * ny + j] * sp_lo[(rows_lo - 1) * ny + j];
                    }
                    y += sdiag[t] * pc;
                    if (i < nx - 1) {
                        if (li < rows - 1) y += -sce[t] * sp[t + ny];
                        else y += -sce[t] * sp_hi[j];
                    }
                    if (j < ny - 1) y += -scn[t] * sp[t + 1];
                }
                q[u] = y;
                acc0 += pc * y;
            }
        }
        {
            const double s0 = cta_sum(acc0, red);
            if (threadIdx.x < CS) cluster.map_shared_rank(slotA, (int)threadIdx.x)[rank] = s0;
        }
        cluster.sync();  // 2
        double pq = 0.0;
        for (int c = 0; c < CS; c++) pq += slotA[c];
        if (!(pq != 0.0) || !isfinite(pq)) {
            status = -6;
            break;
        }
        const double alpha = rho / pq;
        acc1 = 0.0;
        acc2 = 0.0;
#pragma unroll
        for (int u = 0; u < PC_UPT; u++) {
            const int t = threadIdx.x + u * PC_THREADS;
            if (t < nloc) {
                x[u] += alpha * sp[t];
                const double rk = r[u] - alpha * q[u];
                r[u] = rk;
                acc1 += rk * (sminv[t] * rk);
                acc2 += rk * rk;
            }
        }
        {
            const double s1 = cta_sum(acc1, red), s2 = cta_sum(acc2, red);
            if (threadIdx.x < CS) {
                double *dst = cluster.map_shared_rank(slotB, (int)threadIdx.x);
                dst[rank] = s1;
                dst[PC_MAX_CLUSTER + rank] = s2;
            }
        }
        cluster.sync();  // 3
        double rz = 0.0, rr = 0.0;
        for (int c = 0; c < CS; c++) {
            rz += slotB[c];
            rr += slotB[PC_MAX_CLUSTER + c];
        }
        it++;
        res = sqrt(rr) / bn;
        beta = rz / rho;
        rho = rz;
        if (!isfinite(res)) {
            status = -5;
            break;
        }
        done = !(res > a.tol) || it >= a.maxit;
    }
#pragma unroll
    for (int u = 0; u < PC_UPT; u++) {
        const int t = threadIdx.x + u * PC_THREADS;
        if (t < nloc) a.x[(int64_t)r0 * ny + t] = x[u];
    }
    if (rank == 0 && threadIdx.x == 0) {
        a.ks->it = it;
        a.ks->res = res;
        a.ks->status = status;
        a.ks->done = 1;
        a.ks->rho = rho;
        a.ks->bn = bn;
    }
    cluster.sync();  // keep every CTA's shared memory alive until all remote reads are done
}

// Cluster size for an nx x ny system, or 0 when the system does not fit one
// cluster (more than PC_MAX_CTA_UNKNOWNS unknowns in some slab).
int pcg_cluster_size(int nx, int ny) {
    for (int cs = 1; cs <= PC_MAX_CLUSTER; cs *= 2) {
        if (cs > nx) break;
        const int rows_max = (nx + cs - 1) / cs;
        if ((int64_t)rows_max * ny <= PC_MAX_CTA_UNKNOWNS) return cs;
    }
    return 0;
}

static size_t pcg_cluster_smem(int rows_max, int ny) {
    return sizeof(double) * (5 * (size_t)rows_max * ny + 4 * PC_MAX_CLUSTER + 32);
}

// Returns true when the cluster launch was issued; false when the system
// does not fit or the device cannot schedule such a cluster (the caller then
// uses the multi-kernel path).
bool launch_pcg_cluster(int nx, int ny, const Sys &S, double *x, KState *ks, double tol, int maxit,
                        cudaStream_t st) {
    const int cs = pcg_cluster_size(nx, ny);
    if (!cs) return false;
    const int rows_max = (nx + cs - 1) / cs;
    const size_t smem = pcg_cluster_smem(rows_max, ny);
    if (cudaFuncSetAttribute(k_pcg_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(k_pcg_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs, 1, 1);
    cfg.blockDim = dim3(PC_THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, k_pcg_cluster, &cfg) != cudaSuccess || nclusters < 1) {
        cudaGetLastError();
        return false;
    }
    PcgClusterArgs a{nx, ny, cs, rows_max, S, x, ks, tol, maxit};
    if (cudaLaunchKernelEx(&cfg, k_pcg_cluster, a) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}

}  // namespace asd2g
