// GFM Poisson system and Krylov solvers (declarations shared with api.cu).
#pragma once
#include "momentum.cuh"

namespace asd2g {

// Matrix-free system over the nx*ny interior cells in the compact layout
// k = j' + ny*i' (j' = j-3, i' = i-3; y fastest like the padded fields):
//   (A x)_k = diag_k x_k - cw_k x_W - ce_k x_E - cs_k x_S - cn_k x_N
// cw_k equals ce of the west neighbour and cs_k cn of the south neighbour
// bit for bit (the face rule is symmetric), so the solvers read ce/cn only.
struct Sys {
    double *diag, *cw, *ce, *cs, *cn, *minv, *b;
    int pinned;
};

// Scalars of one Krylov solve, kept on the device so that iterations can be
// enqueued (and graph-captured) without host round trips.
struct KState {
    double rho, alpha, beta, bn, res, tol, reg;
    double omega, rho1, rho2, rtv, snorm;
    int it, maxit, done, status, mode;
    unsigned counter;
    int verified;  // MG-FCG: the converged residual was confirmed by b - A x in FP64
    int restart;   // MG-FCG: the next V-cycle starts a new direction (beta = 0)
    double res_true_prev;  // MG-FCG: true residual at the previous replacement (-1: none yet)
    // truncated flexible CG of the learned preconditioner: p_j . A p_j and the
    // orthogonalisation coefficients of the stored directions, valid-slot mask
    double fm_pq[4], fm_beta[4];
    int fm_mask;
    // MG-FCG: set by the residual check of a chunk when it changed nothing
    // (mid-solve), so the V-cycle enqueued after the check returns at entry
    // instead of redoing the last V-cycle and the direction update; cleared
    // by the next iteration's first kernel
    int skip_vc;
};

constexpr int RED_BLOCKS_MAX = 1184;  // 8 x 148 SMs
inline int red_blocks(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (int)(b < 1 ? 1 : (b > RED_BLOCKS_MAX ? RED_BLOCKS_MAX : b));
}

void launch_assemble(const Grid &g, const MomConst &M, const double *ls, const double *kappa, const double *H,
                     const double *div, const double *dtp, const Sys &S, cudaStream_t st);
void launch_pcg_init(const Grid &g, const Sys &S, double *x, double *r, double *p, KState *ks, double *partial,
                     cudaStream_t st);
void launch_pcg_iter(const Grid &g, const Sys &S, double *x, double *r, const double *p_old, double *p_new,
                     double *q, KState *ks, double *partial, cudaStream_t st);
void launch_bicg_init(const Grid &g, const Sys &S, double *x, double *r, double *rt, double *p, double *v,
                      KState *ks, double *partial, cudaStream_t st);
void launch_bicg_iter(const Grid &g, const Sys &S, double *x, double *r, const double *rt, double *p, double *v,
                      double *s, double *t, KState *ks, double *partial, cudaStream_t st);
void launch_scatter_ps(const Grid &g, const double *x, double *ps, double *p, const double *dtp, cudaStream_t st);
void launch_true_residual(const Grid &g, const Sys &S, const double *ps, double *partial, double *out2,
                          cudaStream_t st);
void launch_set_kstate(KState *ks, double tol, int maxit, int mode, double reg, cudaStream_t st);
// CSR-operator variants (PoissonSolver2D's CSR interface); Sys carries b and minv only.
void launch_pcg_init_n(int64_t n, const Sys &S, double *x, double *r, double *p, KState *ks, double *partial,
                       cudaStream_t st);
void launch_bicg_init_n(int64_t n, const Sys &S, double *x, double *r, double *rt, double *p, double *v, KState *ks,
                        double *partial, cudaStream_t st);
void launch_csr_pcg_iter(const int *ia, const int *ja, const double *a, int rows, const Sys &S, double *x,
                         double *r, double *p, double *q, KState *ks, double *partial, cudaStream_t st);
void launch_csr_bicg_iter(const int *ia, const int *ja, const double *a, int rows, const Sys &S, double *x, double *r,
                          const double *rt, double *p, double *v, double *s, double *t, KState *ks, double *partial,
                          cudaStream_t st);
// pcg_persist.cu: whole textbook PCG solve (mode 0) as one cooperative launch
// of one 512-thread CTA per 16 x 32 tile; false (nothing launched) when the
// tiles do not fit the GPU at once.  r, p0, p1: n-vectors of work space;
// partial: 4 doubles per tile; bar: two words, zeroed by the launch.  KState
// receives it, res, status (-8: a grid-barrier wait gave up) and done.
bool launch_pcg_persist(int nx, int ny, const Sys &S, double *x, double *r, double *p0, double *p1, double *partial,
                        int64_t partial_len, unsigned *bar, KState *ks, double tol, int maxit, cudaStream_t st);
// pcg_cluster.cu: whole textbook PCG solve in one thread-block cluster;
// false when the system does not fit one cluster or cannot be scheduled.
int pcg_cluster_size(int nx, int ny);
bool launch_pcg_cluster(int nx, int ny, const Sys &S, double *x, KState *ks, double tol, int maxit,
                        cudaStream_t st);
// axisym.cu: SolvePoisson's r-weighted assembly of the axisymmetric solver.
void launch_axi_assemble(const Grid &g, const MomConst &M, const double *ls, const double *kappa, const double *H,
                         const double *div, const double *dtp, const Sys &S, cudaStream_t st);

}  // namespace asd2g
