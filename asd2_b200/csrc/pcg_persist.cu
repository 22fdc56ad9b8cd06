// Textbook Jacobi-PCG (ASD2G_SOLVER_PCG, the reference's CG_2FUniformP_2D
// method, poisson2d.cpp:285-401) as ONE cooperative launch: one CTA of 512
// threads per 16 x 32 tile of the system, each thread one unknown, two grid
// barriers per iteration:
//
//   A   p = Minv r + beta p_old on the tile + 1 (the neighbours' r and p_old
//       read from global memory: each CTA recomputes the halo), q = A p on
//       the tile, p.q
//   --- barrier 1: alpha = rho / p.q
//   B   x += alpha p, r -= alpha q on the tile; r.Minv r, r.r
//   --- barrier 2: convergence, beta, rho
//
// Same arithmetic, in the same order and without fused multiply-adds, as
// k_pcg_a / k_pcg_b; only the reductions' summation order differs.  The
// grid barrier and reductions are those of gridsync.cuh (bounded waits;
// status -8 when a wait gave up, after which the host solves the system
// with the per-iteration kernels).
#include "asd2g.h"
#include "gridsync.cuh"
#include "pressure.cuh"

namespace asd2g {
namespace {

constexpr int QI = 16, QJ = 32, QT = QI * QJ;
constexpr int QHI = QI + 2, QHJ = QJ + 2;

struct QArgs {
    int nx, ny, ntj, ncta;
    Sys S;
    double *x, *r, *p0, *p1, *partial;
    unsigned *bar;
    KState *ks;
    double tol;
    int maxit;
};

struct QSmem {
    double p[QHI][QHJ];
    double red[GRID_SLOTS * QT / 32];
    double tot[GRID_SLOTS];
    int flag;
};

__global__ void __launch_bounds__(QT, 2) k_pcg_persist(QArgs A) {
    __shared__ QSmem sm;
    const int tid = threadIdx.x, nx = A.nx, ny = A.ny;
    const int ti = blockIdx.x / A.ntj, tj = blockIdx.x % A.ntj, i0 = ti * QI, j0 = tj * QJ;
    const int ta = tid / QJ, tb = tid % QJ, mi = i0 + ta, mj = j0 + tb;
    const bool mine = mi < nx && mj < ny;
    const int64_t mk = (int64_t)mj + (int64_t)ny * mi;
    const Sys &S = A.S;
    unsigned epoch = 0;
    double *pold = A.p0, *pnew = A.p1;
    double xk = 0.0, rk = 0.0, minv = 0.0;
    {
        double v[3] = {0.0, 0.0, 0.0};  // b.b, r.r, r.(Minv r)
        if (mine) {
            const double bk = S.b[mk];
            minv = S.minv[mk];
            rk = bk;
            __stcg(A.r + mk, bk);
            __stcg(pold + mk, 0.0);
            v[0] = bk * bk;
            v[1] = bk * bk;
            v[2] = bk * (minv * bk);
        }
        grid_put_partial<3, QT>(A.partial, sm.red, v);
    }
    bool ok = grid_sync(A.bar, A.ncta, epoch, sm.flag);
    double bn = 1.0, res = 0.0, rho = 0.0, beta = 0.0, alpha = 0.0;
    int it = 0, status = 0;
    bool done = true;
    if (ok) {
        grid_get_total<3>(A.partial, A.ncta, sm.tot);
        bn = sqrt(sm.tot[0]);
        if (bn == 0.0) bn = 1.0;
        res = sqrt(sm.tot[1]) / bn;
        rho = sm.tot[2];
        done = !(res > A.tol) || A.maxit <= 0;
    }
    while (ok && !done) {
        // A: p on the tile + 1, q = A p, p.q
        for (int t = tid; t < QHI * QHJ; t += QT) {
            const int a = t / QHJ, b = t % QHJ, i = i0 - 1 + a, j = j0 - 1 + b;
            double v = 0.0;
            if (i >= 0 && i < nx && j >= 0 && j < ny) {
                const int64_t k = (int64_t)j + (int64_t)ny * i;
                v = __ldg(S.minv + k) * __ldcg(A.r + k) + beta * __ldcg(pold + k);
            }
            sm.p[a][b] = v;
        }
        __syncthreads();
        double pc = 0.0, y = 0.0;
        {
            double v[1] = {0.0};
            if (mine) {
                const int a = ta + 1, b = tb + 1;
                pc = sm.p[a][b];
                if (!(S.pinned && mk == 0)) {
                    if (mj > 0) y += -__ldg(S.cn + mk - 1) * sm.p[a][b - 1];
                    if (mi > 0) y += -__ldg(S.ce + mk - ny) * sm.p[a - 1][b];
                    y += __ldg(S.diag + mk) * pc;
                    if (mi < nx - 1) y += -__ldg(S.ce + mk) * sm.p[a + 1][b];
                    if (mj < ny - 1) y += -__ldg(S.cn + mk) * sm.p[a][b + 1];
                }
                __stcg(pnew + mk, pc);
                v[0] = pc * y;
            }
            grid_put_partial<1, QT>(A.partial, sm.red, v);
        }
        ok = grid_sync(A.bar, A.ncta, epoch, sm.flag);
        if (!ok) break;
        grid_get_total<1>(A.partial, A.ncta, sm.tot);
        {
            const double den = sm.tot[0];
            if (!(den != 0.0) || !isfinite(den)) {
                status = -6;
                break;
            }
            alpha = rho / den;
        }
        // B: x, r; r.(Minv r), r.r
        {
            double v[2] = {0.0, 0.0};
            if (mine) {
                xk += alpha * pc;
                rk = rk - alpha * y;
                __stcg(A.r + mk, rk);
                v[0] = rk * (minv * rk);
                v[1] = rk * rk;
            }
            grid_put_partial<2, QT>(A.partial, sm.red, v);
        }
        {
            double *t = pold;
            pold = pnew;
            pnew = t;
        }
        ok = grid_sync(A.bar, A.ncta, epoch, sm.flag);
        if (!ok) break;
        grid_get_total<2>(A.partial, A.ncta, sm.tot);
        it++;
        res = sqrt(sm.tot[1]) / bn;
        beta = sm.tot[0] / rho;
        rho = sm.tot[0];
        if (!isfinite(res)) {
            status = -5;
            break;
        }
        done = !(res > A.tol) || it >= A.maxit;
    }
    if (mine) __stcg(A.x + mk, xk);
    if (blockIdx.x == 0 && tid == 0) {
        KState *ks = A.ks;
        ks->it = it;
        ks->res = res;
        ks->status = ok ? status : -8;
        ks->done = 1;
        ks->rho = rho;
        ks->bn = bn;
        ks->alpha = alpha;
        ks->beta = beta;
    }
}

}  // namespace

bool launch_pcg_persist(int nx, int ny, const Sys &S, double *x, double *r, double *p0, double *p1, double *partial,
                        int64_t partial_len, unsigned *bar, KState *ks, double tol, int maxit, cudaStream_t st) {
    QArgs A{};
    A.nx = nx;
    A.ny = ny;
    A.ntj = (ny + QJ - 1) / QJ;
    A.ncta = ((nx + QI - 1) / QI) * A.ntj;
    if (partial_len < (int64_t)GRID_SLOTS * A.ncta) return false;
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_persist, QT, 0) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if ((int64_t)per_sm * sms < A.ncta) return false;
    A.S = S;
    A.x = x;
    A.r = r;
    A.p0 = p0;
    A.p1 = p1;
    A.partial = partial;
    A.bar = bar;
    A.ks = ks;
    A.tol = tol;
    A.maxit = maxit;
    if (cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), st) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    void *args[] = {&A};
    if (cudaLaunchCooperativeKernel((const void *)k_pcg_persist, dim3(A.ncta), dim3(QT), args, 0, st) !=
        cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}

}  // namespace asd2g
