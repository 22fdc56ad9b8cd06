// GFM assembly of the variable-coefficient pressure Poisson operator
// (MACSolver2D::SolvePoisson, mac2d.cpp:1249-1656) into a matrix-free
// five-point form, and the Krylov solvers that replace PoissonSolver2D's MKL
// CSR + BLAS-1 loops (poisson2d.cpp:230-575).
//
// Reductions are deterministic: each block reduces with warp shuffles in a
// fixed order, writes one partial per block, and the last block to finish
// (atomic ticket) sums the partials in block order and updates the solver
// scalars in KState.  Every solver kernel returns at entry once KState.done is
// set, so a fixed-length chunk of iterations can be enqueued (or captured in
// a CUDA graph) and the host only polls between chunks.
#include "lsmath.cuh"
#include "pressure.cuh"
#include "batch.cuh"

namespace asd2g {

// ---------------------------------------------------------------- reduce --
// Block-wide sum of NV values per thread; thread 0 receives the totals.
// Fixed order (warp shuffles, then warps in index order): deterministic.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (&sh)[NV][32]) {
#pragma unroll
    for (int q = 0; q < NV; q++)
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();  // sh may still be read from a previous use
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

// Sum NV per-thread values over the grid.  Every block writes its partial;
// the last block to take a ticket sums the partials with all its threads
// (strided, then block_sum), so the result does not depend on which block
// finishes last.  Returns true on thread 0 of the last block, with the
// totals in tot.
template <int NV>
__device__ __forceinline__ bool grid_reduce(double (&v)[NV], double *partial, unsigned *counter, double (&tot)[NV]) {
    __shared__ double sh[NV][32];
    __shared__ bool last;
    block_sum<NV>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) partial[NV * blockIdx.x + q] = v[q];
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double a[NV];
#pragma unroll
    for (int q = 0; q < NV; q++) a[q] = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < NV; q++) a[q] += __ldcg(partial + NV * b + q);
    block_sum<NV>(a, sh);
    if (threadIdx.x != 0) return false;
#pragma unroll
    for (int q = 0; q < NV; q++) tot[q] = a[q];
    *counter = 0u;
    return true;
}

// ------------------------------------------------------------- assembly --
__device__ __forceinline__ void theta_first(double a, double b, double &thH, double &th) {
    // (W, M) / (S, M) pairs, mac2d.cpp:1341-1358, :1398-1415
    if (a >= 0.0 && b >= 0.0) { thH = 1.0; th = 0.0; }
    else if (a < 0.0 && b < 0.0) { thH = 0.0; th = 0.0; }
    else if (a >= 0.0 && b < 0.0) { thH = fabs(a) / (fabs(a) + fabs(b)); th = fabs(a) / (fabs(a) + fabs(b)); }
    else { thH = fabs(b) / (fabs(a) + fabs(b)); th = fabs(a) / (fabs(a) + fabs(b)); }
}
__device__ __forceinline__ void theta_second(double m, double e, double &thH, double &th) {
    // (M, E) / (M, N) pairs, mac2d.cpp:1372-1388, :1425-1441
    if (m >= 0.0 && e >= 0.0) { thH = 1.0; th = 0.0; }
    else if (m < 0.0 && e < 0.0) { thH = 0.0; th = 0.0; }
    else if (m >= 0.0 && e < 0.0) { thH = fabs(m) / (fabs(m) + fabs(e)); th = fabs(e) / (fabs(m) + fabs(e)); }
    else { thH = fabs(e) / (fabs(m) + fabs(e)); th = fabs(e) / (fabs(m) + fabs(e)); }
}
__device__ __forceinline__ bool p_dir_like(int b) {
    // Dirichlet branch of the assembly includes WALL (mac2d.cpp:1521-1523).
    return b == 2 /*DIRICHLET*/ || b == 5 /*INLET*/ || b == 6 /*OUTLET*/ || b == 7 /*PRESSURE*/ || b == 4 /*WALL*/;
}

// One interior cell (i, j) of the GFM system (mac2d.cpp:1330-1607).
__device__ __forceinline__ void assemble_cell(const Grid &g, const MomConst &M, const DivH &dxx, const DivH &dyy,
                                              const double *__restrict__ ls, const double *__restrict__ kappa,
                                              const double *__restrict__ H, const double *__restrict__ div,
                                              double dt, const Sys &S, int i, int j) {
    const double rH = M.rho_h, rL = M.rho_l, sig = M.sigma;
    const int64_t c = IX(g, i, j), cw = IX(g, i - 1, j), ce = IX(g, i + 1, j), cs = IX(g, i, j - 1),
                  cn = IX(g, i, j + 1);
    const double lsM = ls[c];
    double thH, th, kEff;
    theta_first(ls[cw], lsM, thH, th);
    double iW = 1.0 / (rH * thH + rL * (1.0 - thH));
    kEff = kappa[c] * th + kappa[cw] * (1.0 - th);
    double FW = -dt * (-sig * kEff) * (H[c] - H[cw]);
    FW *= dxx(iW);
    theta_second(lsM, ls[ce], thH, th);
    double iE = 1.0 / (rH * thH + rL * (1.0 - thH));
    kEff = kappa[c] * th + kappa[ce] * (1.0 - th);
    double FE = dt * (-sig * kEff) * (H[ce] - H[c]);
    FE *= dxx(iE);
    theta_first(ls[cs], lsM, thH, th);
    double iS = 1.0 / (rH * thH + rL * (1.0 - thH));
    kEff = kappa[c] * th + kappa[cs] * (1.0 - th);
    double FS = -dt * (-sig * kEff) * (H[c] - H[cs]);
    FS *= dyy(iS);
    theta_second(lsM, ls[cn], thH, th);
    double iN = 1.0 / (rH * thH + rL * (1.0 - thH));
    kEff = kappa[c] * th + kappa[cn] * (1.0 - th);
    double FN = dt * (-sig * kEff) * (H[cn] - H[c]);
    FN *= dyy(iN);
    double r = 0.0;
    r -= FW + FE + FS + FN;  // mac2d.cpp:1454
    r -= div[c];             // :1468-1470
    iS *= -1.0; iW *= -1.0; iE *= -1.0; iN *= -1.0;  // :1497-1500
    double aS = dyy(iS), aW = dxx(iW), aE = dxx(iE), aN = dyy(iN);
    double aC = -dxx(iW + iE) - dyy(iS + iN);
    const int nx = g.nx, ny = g.ny;
    // boundary edits :1515-1583 (periodic pressure is rejected at set-up)
    if (i == NB && g.bp[0] == 1) { aW = 0.0; aC += dxx(iW); }
    else if (i == NB && p_dir_like(g.bp[0])) { aW = 0.0; r -= dxx(iW) * g.cp[0]; }
    if (i == NB + nx - 1 && g.bp[1] == 1) { aE = 0.0; aC += dxx(iE); }
    else if (i == NB + nx - 1 && p_dir_like(g.bp[1])) { aE = 0.0; r -= dxx(iE) * g.cp[1]; }
    if (j == NB && g.bp[2] == 1) { aS = 0.0; aC += dyy(iS); }
    else if (j == NB && p_dir_like(g.bp[2])) { aS = 0.0; r -= dyy(iS) * g.cp[2]; }
    if (j == NB + ny - 1 && g.bp[3] == 1) { aN = 0.0; aC += dyy(iN); }
    else if (j == NB + ny - 1 && p_dir_like(g.bp[3])) { aN = 0.0; r -= dyy(iN) * g.cp[3]; }
    const int ii = i - NB, jj = j - NB;
    const int64_t k = (int64_t)jj + (int64_t)ny * ii;
    const bool pin0 = S.pinned && ii == 0 && jj == 0;
    S.diag[k] = aC;
    S.cw[k] = (S.pinned && ii == 1 && jj == 0) ? 0.0 : -aW;
    S.ce[k] = -aE;
    S.cs[k] = (S.pinned && ii == 0 && jj == 1) ? 0.0 : -aS;
    S.cn[k] = -aN;
    S.b[k] = pin0 ? 0.0 : r;
    S.minv[k] = pin0 ? 0.0 : 1.0 / aC;  // InvertMatrixDiagonal, poisson2d.cpp:577-585
}

__global__ void k_assemble(Grid g, MomConst M, DivH dxx, DivH dyy, const double *__restrict__ ls,
                           const double *__restrict__ kappa, const double *__restrict__ H,
                           const double *__restrict__ div, const double *__restrict__ dtp, Sys S) {
    const int j = NB + blockIdx.x * TJ + threadIdx.x, i = NB + blockIdx.y * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    assemble_cell(g, M, dxx, dyy, ls, kappa, H, div, *dtp, S, i, j);
}

// Batched: block b assembles cell tile b of its instance (32 x 8 cells).
__global__ void k_bassemble(const BInst *__restrict__ insts, const BTile *__restrict__ tiles) {
    const BTile w = tiles[blockIdx.x];
    const BInst &I = insts[w.inst];
    const int j = NB + w.bx * TJ + threadIdx.x, i = NB + w.by * TI + threadIdx.y;
    if (i >= I.g.nx + NB || j >= I.g.ny + NB) return;
    assemble_cell(I.g, I.M, I.dxx, I.dyy, I.ls, I.kappa, I.H, I.div, I.sc[0], I.S, i, j);
}

// Batched scatter: PS = x on the interior with its ghost mirrors (every
// batch instance has Neumann/Dirichlet pressure sides), P = PS / dt.
__global__ void k_bscatter(const BInst *__restrict__ insts, const BTile *__restrict__ tiles) {
    const BTile w = tiles[blockIdx.x];
    const BInst &I = insts[w.inst];
    const Grid &g = I.g;
    const int j = NB + w.bx * TJ + threadIdx.x, i = NB + w.by * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    const double v = I.x[(int64_t)(j - NB) + (int64_t)g.ny * (i - NB)];
    I.ps[IX(g, i, j)] = v;
    p_mirror_store(g, I.ps, i, j, v);
    I.p[IX(g, i, j)] = v / I.sc[0];  // mac2d.cpp:1722-1724
}

// ------------------------------------------------------------------ SpMV --
// y_k = (A x)_k in the reference's row order S, W, C, E, N; the pinned row is 0.
struct Nbr {
    int ii, jj;
    int64_t k;
};
__device__ __forceinline__ Nbr nbr_of(int64_t k, int ny) { return Nbr{(int)(k / ny), (int)(k % ny), k}; }

// --------------------------------------------------------------- PCG init --
__global__ void k_pcg_init(int64_t n, Sys S, double *__restrict__ x, double *__restrict__ r, double *__restrict__ p,
                           KState *ks, double *partial) {
    double v[3] = {0.0, 0.0, 0.0};  // b.b, r.r, r.(Minv r)
    const int ref = ks->mode == 1;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const double bk = S.b[k];
        x[k] = 0.0;
        r[k] = bk;
        p[k] = ref ? bk : 0.0;  // reference: p_0 = r_0 (poisson2d.cpp:331-332)
        v[0] += bk * bk;
        v[1] += bk * bk;
        v[2] += bk * (S.minv[k] * bk);
    }
    double tot[3];
    if (grid_reduce<3>(v, partial, &ks->counter, tot)) {
        double bn = sqrt(tot[0]);
        if (bn == 0.0) bn = 1.0;  // :336-337
        ks->bn = bn;
        ks->res = sqrt(tot[1]) / bn;
        ks->rho = tot[2];
        ks->beta = ref ? tot[2] / 1.0 : 0.0;  // reference iteration 0: beta = rho / rho1, rho1 = 1
        ks->it = 0;
        ks->status = 0;
        const bool conv = ref ? (ks->res <= ks->tol) : !(ks->res > ks->tol);
        ks->done = (conv || ks->maxit <= 0) ? 1 : 0;
        if (conv) ks->status = 0;
    }
}

// ------------------------------------------------------ PCG iteration A --
// p_new = Minv r + beta p_old (at the cell and, recomputed, at its four
// neighbours), q = A p_new, partial p_new . q.  Last block: alpha.
__global__ void __launch_bounds__(256) k_pcg_a(int nx, int ny, Sys S, const double *__restrict__ r,
                                               const double *__restrict__ p_old, double *__restrict__ p_new,
                                               double *__restrict__ q, KState *ks, double *partial) {
    if (ks->done) return;
    const double beta = ks->beta;
    const int64_t n = (int64_t)nx * ny;
    double v[1] = {0.0};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int ii = (int)(k / ny), jj = (int)(k % ny);
        auto pv = [&](int64_t m) { return S.minv[m] * r[m] + beta * p_old[m]; };
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
    if (grid_reduce<1>(v, partial, &ks->counter, tot)) {
        const double den = tot[0] + ks->reg;
        if (!(den != 0.0) || !isfinite(den)) {
            ks->status = -6;
            ks->done = 1;
        } else {
            ks->alpha = ks->rho / den;
        }
    }
}

// ------------------------------------------------------ PCG iteration B --
// x += alpha p; r -= alpha q; partials r.(Minv r), r.r.  Last block: the
// convergence test and the next beta.
__global__ void __launch_bounds__(256) k_pcg_b(int64_t n, Sys S, double *__restrict__ x, double *__restrict__ r,
                                               const double *__restrict__ p, const double *__restrict__ q, KState *ks,
                                               double *partial) {
    if (ks->done) return;
    const double alpha = ks->alpha;
    double v[2] = {0.0, 0.0};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        x[k] += alpha * p[k];
        const double rk = r[k] - alpha * q[k];
        r[k] = rk;
        v[0] += rk * (S.minv[k] * rk);
        v[1] += rk * rk;
    }
    double tot[2];
    if (grid_reduce<2>(v, partial, &ks->counter, tot)) {
        const int it = ks->it + 1;
        ks->it = it;
        ks->res = sqrt(tot[1]) / ks->bn;
        const bool ref = ks->mode == 1;
        if (ref) ks->beta = (it == 1) ? 0.0 : tot[0] / ks->rho;  // iteration 1 restarts p = z (:341-343)
        else ks->beta = tot[0] / ks->rho;
        ks->rho = tot[0];
        const bool conv = ref ? (ks->res <= ks->tol) : !(ks->res > ks->tol);
        if (!isfinite(ks->res)) { ks->status = -5; ks->done = 1; }
        else if (conv || it >= ks->maxit) ks->done = 1;
    }
}

// ---------------------------------------------------------------- BiCGStab --
// The reference's right-Jacobi BiCGStab (poisson2d.cpp:403-575); mode 3
// keeps rho_2 = 1 as the reference does, mode 2 carries rho_2 = rho_1.
__global__ void k_bicg_init(int64_t n, Sys S, double *__restrict__ x, double *__restrict__ r, double *__restrict__ rt,
                            double *__restrict__ p, double *__restrict__ v, KState *ks, double *partial) {
    double a[2] = {0.0, 0.0};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const double bk = S.b[k];
        x[k] = 0.0;
        r[k] = bk;
        rt[k] = bk;
        p[k] = 0.0;
        v[k] = 0.0;
        a[0] += bk * bk;
        a[1] += bk * bk;  // rt . r for the first rho_1
    }
    double tot[2];
    if (grid_reduce<2>(a, partial, &ks->counter, tot)) {
        double bn = sqrt(tot[0]);
        if (bn == 0.0) bn = 1.0;
        ks->bn = bn;
        ks->res = sqrt(tot[0]) / bn;
        ks->alpha = 1.0;
        ks->omega = 1.0;
        ks->rho2 = 1.0;
        ks->rho1 = tot[1];
        ks->it = 0;
        ks->status = 0;
        const bool conv = ks->res <= ks->tol;
        ks->done = (conv || ks->maxit <= 0 || ks->rho1 == 0.0) ? 1 : 0;
    }
}

// p = (it == 1) ? r : ((p - omega v) beta) + r ; phat = Minv p  (stored in t)
__global__ void k_bicg_p(int64_t n, Sys S, const double *__restrict__ r, double *__restrict__ p,
                         const double *__restrict__ v, double *__restrict__ phat, const KState *ks) {
    if (ks->done) return;
    const int it = ks->it;
    const double beta = (ks->rho1 / ks->rho2) * (ks->alpha / ks->omega), om = ks->omega;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double pk;
        if (it == 1) pk = r[k];
        else {
            pk = p[k] + -om * v[k];
            pk = pk * beta;
            pk = pk + 1.0 * r[k];
        }
        p[k] = pk;
        phat[k] = S.minv[k] * pk;
    }
}

// y = A xin; partial dots (NV = 1: rt . y; NV = 2: y . s, y . y)
template <int NV>
__global__ void __launch_bounds__(256) k_bicg_spmv(int nx, int ny, Sys S, const double *__restrict__ xin,
                                                   double *__restrict__ y, const double *__restrict__ w,
                                                   KState *ks, double *partial, int which) {
    if (ks->done) return;
    const int64_t n = (int64_t)nx * ny;
    double a[NV];
#pragma unroll
    for (int q = 0; q < NV; q++) a[q] = 0.0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int ii = (int)(k / ny), jj = (int)(k % ny);
        double s = 0.0;
        if (!(S.pinned && k == 0)) {
            if (jj > 0) s += -S.cn[k - 1] * xin[k - 1];
            if (ii > 0) s += -S.ce[k - ny] * xin[k - ny];
            s += S.diag[k] * xin[k];
            if (ii < nx - 1) s += -S.ce[k] * xin[k + ny];
            if (jj < ny - 1) s += -S.cn[k] * xin[k + 1];
        }
        y[k] = s;
        if (NV == 1) a[0] += w[k] * s;
        else { a[0] += s * w[k]; a[NV - 1] += s * s; }
    }
    double tot[NV];
    if (grid_reduce<NV>(a, partial, &ks->counter, tot)) {
        if (which == 0) {
            ks->alpha = ks->rho1 / tot[0];  // :482
        } else {
            ks->omega = tot[0] / tot[NV - 1];  // :499
        }
    }
}

// s = r - alpha v ; ||s|| ; early exit x += alpha phat when ||s||/||b|| < tol
__global__ void k_bicg_s(int64_t n, const double *__restrict__ r, const double *__restrict__ v, double *__restrict__ s,
                         KState *ks, double *partial) {
    if (ks->done) return;
    const double alpha = ks->alpha;
    double a[1] = {0.0};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const double sk = r[k] + -alpha * v[k];
        s[k] = sk;
        a[0] += sk * sk;
    }
    double tot[1];
    if (grid_reduce<1>(a, partial, &ks->counter, tot)) {
        ks->snorm = sqrt(tot[0]) / ks->bn;
        if (ks->snorm < ks->tol) ks->status = 2;  // converged on s (:488-492)
    }
}

// shat = Minv s (stored in phat's partner buffer)
__global__ void k_bicg_shat(int64_t n, Sys S, const double *__restrict__ s, double *__restrict__ shat, KState *ks,
                            double *__restrict__ x, const double *__restrict__ phat) {
    if (ks->done) return;
    if (ks->status == 2) {
        const double alpha = ks->alpha;
        for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
            x[k] += alpha * phat[k];
        return;
    }
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        shat[k] = S.minv[k] * s[k];
}

// x += alpha phat + omega shat ; r = s - omega t ; ||r|| ; rt . r
__global__ void k_bicg_x(int64_t n, double *__restrict__ x, double *__restrict__ r, const double *__restrict__ rt,
                         const double *__restrict__ phat, const double *__restrict__ shat, const double *__restrict__ s,
                         const double *__restrict__ t, KState *ks, double *partial) {
    if (ks->done) return;
    if (ks->status == 2) {  // converged on s in k_bicg_s (x updated in k_bicg_shat)
        __syncthreads();
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ks->res = ks->snorm;
            ks->status = 0;
            ks->done = 1;
        }
        return;
    }
    const double alpha = ks->alpha, om = ks->omega;
    double a[2] = {0.0, 0.0};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double xk = x[k] + alpha * phat[k];
        xk = xk + om * shat[k];
        x[k] = xk;
        const double rk = s[k] + -om * t[k];
        r[k] = rk;
        a[0] += rk * rk;
        a[1] += rt[k] * rk;
    }
    double tot[2];
    if (grid_reduce<2>(a, partial, &ks->counter, tot)) {
        ks->res = sqrt(tot[0]) / ks->bn;
        const int it = ks->it + 1;
        ks->it = it;
        if (ks->mode == 2) ks->rho2 = ks->rho1;  // IML++; the reference never updates rho_2
        ks->rho1 = tot[1];
        if (!isfinite(ks->res)) { ks->status = -5; ks->done = 1; }
        else if (ks->res <= ks->tol || it >= ks->maxit) ks->done = 1;
        else if (ks->rho1 == 0.0) { ks->status = -6; ks->done = 1; }  // :466-468
    }
}

// ------------------------------------------------------------------ CSR --
// PoissonSolver2D's CSR interface (poisson2d.cpp:230-575): a general CSR
// matrix from the caller, one thread per row.  Column indices outside
// [0, rows) are skipped (the reference's pinned all-Neumann matrix carries
// such entries, with value 0, which MKL would read out of bounds).
struct Csr {
    const int *ia, *ja;
    const double *a;
    int rows;
};
__device__ __forceinline__ double csr_row(const Csr &A, int r, const double *__restrict__ x) {
    double s = 0.0;
    for (int k = A.ia[r]; k < A.ia[r + 1]; k++) {
        const int c = A.ja[k];
        if (c < 0 || c >= A.rows) continue;
        s += A.a[k] * x[c];
    }
    return s;
}

// p = Minv r + beta p (PCG direction update)
__global__ void k_csr_pcg_p(int64_t n, Sys S, const double *__restrict__ r, double *__restrict__ p, const KState *ks) {
    if (ks->done) return;
    const double beta = ks->beta;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        p[k] = S.minv[k] * r[k] + beta * p[k];
}

// q = A p, p.q -> alpha
__global__ void __launch_bounds__(256) k_csr_pcg_q(Csr A, const double *__restrict__ p, double *__restrict__ q,
                                                   KState *ks, double *partial) {
    if (ks->done) return;
    double v[1] = {0.0};
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < A.rows; r += gridDim.x * blockDim.x) {
        const double y = csr_row(A, r, p);
        q[r] = y;
        v[0] += p[r] * y;
    }
    double tot[1];
    if (grid_reduce<1>(v, partial, &ks->counter, tot)) {
        const double den = tot[0] + ks->reg;
        if (!(den != 0.0) || !isfinite(den)) {
            ks->status = -6;
            ks->done = 1;
        } else {
            ks->alpha = ks->rho / den;
        }
    }
}

// y = A xin and dots (BiCGStab), as k_bicg_spmv with a CSR operator
template <int NV>
__global__ void __launch_bounds__(256) k_csr_bicg_spmv(Csr A, const double *__restrict__ xin, double *__restrict__ y,
                                                       const double *__restrict__ w, KState *ks, double *partial,
                                                       int which) {
    if (ks->done) return;
    double a[NV];
#pragma unroll
    for (int q = 0; q < NV; q++) a[q] = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < A.rows; r += gridDim.x * blockDim.x) {
        const double s = csr_row(A, r, xin);
        y[r] = s;
        if (NV == 1) a[0] += w[r] * s;
        else { a[0] += s * w[r]; a[NV - 1] += s * s; }
    }
    double tot[NV];
    if (grid_reduce<NV>(a, partial, &ks->counter, tot)) {
        if (which == 0) ks->alpha = ks->rho1 / tot[0];
        else ks->omega = tot[0] / tot[NV - 1];
    }
}

// ---------------------------------------------------------- scatter / res --
// PS = 0 everywhere, interior = x, then (host) P fill, then P = PS / dt.
__global__ void k_scatter_ps(Grid g, const double *__restrict__ x, double *__restrict__ ps) {
    const int j = NB + blockIdx.x * TJ + threadIdx.x, i = NB + blockIdx.y * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    ps[IX(g, i, j)] = x[(int64_t)(j - NB) + (int64_t)g.ny * (i - NB)];
}
__global__ void k_p_from_ps(Grid g, const double *__restrict__ ps, double *__restrict__ p, const double *__restrict__ dtp) {
    const int j = NB + blockIdx.x * TJ + threadIdx.x, i = NB + blockIdx.y * TI + threadIdx.y;
    if (i >= g.nx + NB || j >= g.ny + NB) return;
    p[IX(g, i, j)] = ps[IX(g, i, j)] / *dtp;  // mac2d.cpp:1722-1724
}

__global__ void k_true_residual(Grid g, Sys S, const double *__restrict__ ps, double *partial, unsigned *counter,
                                double *out2) {
    const int nx = g.nx, ny = g.ny;
    const int64_t n = (int64_t)nx * ny;
    double a[2] = {0.0, 0.0};
    auto X = [&](int64_t m) { return ps[IX(g, NB + (int)(m / ny), NB + (int)(m % ny))]; };
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        if (S.pinned && k == 0) continue;
        const int ii = (int)(k / ny), jj = (int)(k % ny);
        double s = 0.0;
        if (jj > 0) s += -S.cn[k - 1] * X(k - 1);
        if (ii > 0) s += -S.ce[k - ny] * X(k - ny);
        s += S.diag[k] * X(k);
        if (ii < nx - 1) s += -S.ce[k] * X(k + ny);
        if (jj < ny - 1) s += -S.cn[k] * X(k + 1);
        const double rk = S.b[k] - s;
        a[0] += rk * rk;
        a[1] += S.b[k] * S.b[k];
    }
    double tot[2];
    if (grid_reduce<2>(a, partial, counter, tot)) {
        out2[0] = tot[0];
        out2[1] = tot[1];
    }
}

__global__ void k_set_kstate(KState *ks, double tol, int maxit, int mode, double reg) {
    ks->tol = tol;
    ks->maxit = maxit;
    ks->mode = mode;
    ks->reg = reg;
    ks->done = 0;
    ks->status = 0;
    ks->it = 0;
    ks->counter = 0u;
    ks->verified = 0;
    ks->restart = 0;
    ks->res_true_prev = -1.0;
    ks->skip_vc = 0;
}

// ------------------------------------------------------------------ host --
void launch_assemble(const Grid &g, const MomConst &M, const double *ls, const double *kappa, const double *H,
                     const double *div, const double *dtp, const Sys &S, cudaStream_t st) {
    k_assemble<<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, M, make_divh(g.dx * g.dx), make_divh(g.dy * g.dy), ls,
                                                      kappa, H, div, dtp, S);
}

void launch_set_kstate(KState *ks, double tol, int maxit, int mode, double reg, cudaStream_t st) {
    k_set_kstate<<<1, 1, 0, st>>>(ks, tol, maxit, mode, reg);
}

void launch_pcg_init(const Grid &g, const Sys &S, double *x, double *r, double *p, KState *ks, double *partial,
                     cudaStream_t st) {
    const int64_t n = (int64_t)g.nx * g.ny;
    k_pcg_init<<<red_blocks(n), 256, 0, st>>>(n, S, x, r, p, ks, partial);
}

void launch_pcg_iter(const Grid &g, const Sys &S, double *x, double *r, const double *p_old, double *p_new,
                     double *q, KState *ks, double *partial, cudaStream_t st) {
    const int64_t n = (int64_t)g.nx * g.ny;
    const int nb = red_blocks(n);
    k_pcg_a<<<nb, 256, 0, st>>>(g.nx, g.ny, S, r, p_old, p_new, q, ks, partial);
    k_pcg_b<<<nb, 256, 0, st>>>(n, S, x, r, p_new, q, ks, partial);
}

void launch_bicg_init(const Grid &g, const Sys &S, double *x, double *r, double *rt, double *p, double *v,
                      KState *ks, double *partial, cudaStream_t st) {
    const int64_t n = (int64_t)g.nx * g.ny;
    k_bicg_init<<<red_blocks(n), 256, 0, st>>>(n, S, x, r, rt, p, v, ks, partial);
}

// buffers: p, v, s, t plus phat/shat carried in t's neighbours: the caller
// passes t pointing at a 3*n block [t | phat | shat].
void launch_bicg_iter(const Grid &g, const Sys &S, double *x, double *r, const double *rt, double *p, double *v,
                      double *s, double *t, KState *ks, double *partial, cudaStream_t st) {
    const int64_t n = (int64_t)g.nx * g.ny;
    const int nb = red_blocks(n);
    double *phat = t + n, *shat = t + 2 * n;
    k_bicg_p<<<nb, 256, 0, st>>>(n, S, r, p, v, phat, ks);
    k_bicg_spmv<1><<<nb, 256, 0, st>>>(g.nx, g.ny, S, phat, v, rt, ks, partial, 0);
    k_bicg_s<<<nb, 256, 0, st>>>(n, r, v, s, ks, partial);
    k_bicg_shat<<<nb, 256, 0, st>>>(n, S, s, shat, ks, x, phat);
    k_bicg_spmv<2><<<nb, 256, 0, st>>>(g.nx, g.ny, S, shat, t, s, ks, partial, 1);
    k_bicg_x<<<nb, 256, 0, st>>>(n, x, r, rt, phat, shat, s, t, ks, partial);
}

void launch_csr_pcg_iter(const int *ia, const int *ja, const double *a, int rows, const Sys &S, double *x,
                         double *r, double *p, double *q, KState *ks, double *partial, cudaStream_t st) {
    const Csr A{ia, ja, a, rows};
    const int nb = red_blocks(rows);
    k_csr_pcg_p<<<nb, 256, 0, st>>>(rows, S, r, p, ks);
    k_csr_pcg_q<<<nb, 256, 0, st>>>(A, p, q, ks, partial);
    k_pcg_b<<<nb, 256, 0, st>>>(rows, S, x, r, p, q, ks, partial);
}

void launch_csr_bicg_iter(const int *ia, const int *ja, const double *a, int rows, const Sys &S, double *x, double *r,
                          const double *rt, double *p, double *v, double *s, double *t, KState *ks, double *partial,
                          cudaStream_t st) {
    const Csr A{ia, ja, a, rows};
    const int64_t n = rows;
    const int nb = red_blocks(n);
    double *phat = t + n, *shat = t + 2 * n;
    k_bicg_p<<<nb, 256, 0, st>>>(n, S, r, p, v, phat, ks);
    k_csr_bicg_spmv<1><<<nb, 256, 0, st>>>(A, phat, v, rt, ks, partial, 0);
    k_bicg_s<<<nb, 256, 0, st>>>(n, r, v, s, ks, partial);
    k_bicg_shat<<<nb, 256, 0, st>>>(n, S, s, shat, ks, x, phat);
    k_csr_bicg_spmv<2><<<nb, 256, 0, st>>>(A, shat, t, s, ks, partial, 1);
    k_bicg_x<<<nb, 256, 0, st>>>(n, x, r, rt, phat, shat, s, t, ks, partial);
}

void launch_pcg_init_n(int64_t n, const Sys &S, double *x, double *r, double *p, KState *ks, double *partial,
                       cudaStream_t st) {
    k_pcg_init<<<red_blocks(n), 256, 0, st>>>(n, S, x, r, p, ks, partial);
}
void launch_bicg_init_n(int64_t n, const Sys &S, double *x, double *r, double *rt, double *p, double *v, KState *ks,
                        double *partial, cudaStream_t st) {
    k_bicg_init<<<red_blocks(n), 256, 0, st>>>(n, S, x, r, rt, p, v, ks, partial);
}

void launch_scatter_ps(const Grid &g, const double *x, double *ps, double *p, const double *dtp, cudaStream_t st) {
    cudaMemsetAsync(ps, 0, sizeof(double) * (size_t)g.sx * g.sy, st);  // mac2d.cpp:1324-1328
    k_scatter_ps<<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, x, ps);
    launch_fill_p(g, ps, st);
    k_p_from_ps<<<cell_grid(g), dim3(TJ, TI), 0, st>>>(g, ps, p, dtp);
}

void launch_true_residual(const Grid &g, const Sys &S, const double *ps, double *partial, double *out2,
                          cudaStream_t st) {
    const int64_t n = (int64_t)g.nx * g.ny;
    unsigned *counter = reinterpret_cast<unsigned *>(out2 + 2);
    k_true_residual<<<red_blocks(n), 256, 0, st>>>(g, S, ps, partial, counter, out2);
}

void launch_batch_assemble(const BInst *insts, const BTile *tiles, int ntiles, cudaStream_t st) {
    if (ntiles > 0) k_bassemble<<<ntiles, dim3(TJ, TI), 0, st>>>(insts, tiles);
}

void launch_batch_scatter(const BInst *insts, const BTile *tiles, int ntiles, cudaStream_t st) {
    if (ntiles > 0) k_bscatter<<<ntiles, dim3(TJ, TI), 0, st>>>(insts, tiles);
}

}  // namespace asd2g
