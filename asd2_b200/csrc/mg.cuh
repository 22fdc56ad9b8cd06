// Multigrid preconditioner and flexible CG (mg.cu).
#pragma once
#include "pressure.cuh"

namespace asd2g {

// One level of the FP32 hierarchy, compact layout k = j + ny*i: operator
// (diag, ce, cn), restricted residual f, pre-smoothed correction e and the
// corrected, post-smoothed result ep (the coarsest level's exact solve).
// Multigrid tile shapes (rows i x columns j) of the V-cycle's tile kernels,
// chosen per session or batch by timing (the first has the most tiles and
// sizes the partial-sum slots).
constexpr int MG_SHAPES[3][2] = {{16, 32}, {32, 32}, {16, 64}};
constexpr int MG_NSHAPES = 3;

struct MgLevel {
    int nx, ny;
    int tile;  // level 0 of a session's hierarchy: MG_SHAPES index of the V-cycle's tiles (host side)
    float *diag, *ce, *cn, *f, *e, *ep;
};

constexpr int MG_MAX_LEVELS = 16;
constexpr int MG_COARSE_CELLS = 64;

// Level sizes (halving, odd sizes rounded up) until the coarsest level has
// at most 64 cells; returns the number of levels (0 if max_levels is too small).
int mg_levels_for(int nx, int ny, int *dims, int max_levels);
// Doubles of per-block partial sums the flexible CG needs for this grid:
// two per level-0 tile of the fused post-smoothing pass (its dots), at
// least what the 1D reduction kernels use (three per block, RED_BLOCKS_MAX).
int64_t mg_partial_len(int nx, int ny);
// First level of the one-CTA coarse cycle for this hierarchy (at least 1).
int mg_cta_first_level(const MgLevel *lv, int nlev);
// Sets up the single-CTA coarse cycle for this hierarchy (its shared memory);
// false if it does not fit (not reachable with <= 4096-cell CTA levels).
bool mg_cta_prepare(const MgLevel *lv, int nlev);
// Level 0 from the FP64 system, Galerkin coarse levels, coarsest inverse.
void launch_mg_setup(const Sys &S, MgLevel *lv, int nlev, double *coarse_inv, cudaStream_t st);
// Flexible CG with one V-cycle per iteration: init (r = b, x = 0, first
// V-cycle) and one iteration (p, q, alpha; x, r, convergence; V-cycle, beta).
// partial holds partial_len doubles; both return false (launching nothing)
// when that is less than mg_partial_len(nx, ny).
bool launch_fcg_init(const Sys &S, int nx, int ny, MgLevel *lv, int nlev, const double *coarse_inv, double *x,
                     double *r, double *p, double *q, double *z, KState *ks, double *partial, int64_t partial_len,
                     cudaStream_t st);
bool launch_fcg_iter(const Sys &S, int nx, int ny, MgLevel *lv, int nlev, const double *coarse_inv, double *x,
                     double *r, const double *p_old, double *p_new, double *q, double *z, KState *ks,
                     double *partial, int64_t partial_len, cudaStream_t st);
// After a run of iterations: if the recurrence has converged, replace r by
// b - A x (FP64) and either confirm convergence or resume (V-cycle on the
// new r, beta = 0).  Every kernel returns at entry when there is nothing to do.
bool launch_fcg_check(const Sys &S, int nx, int ny, MgLevel *lv, int nlev, const double *coarse_inv, const double *x,
                      double *r, const double *q, double *z, KState *ks, double *partial, int64_t partial_len,
                      cudaStream_t st);

// Flexible CG with the two-level learned preconditioner (ASD2G_SOLVER_UNET),
// KState mode set to the solver id (the V-cycle then leaves the direction
// update to launch_pc_output).  Preconditioner: z_mg = V-cycle(r); r1 = r - A
// z_mg and the network's features; after the network (u), omega = (u . r1) /
// (u . A u) (the A-norm optimal step) and z = z_mg + omega u.  The network
// makes the preconditioner nonlinear, so each new direction is
// A-orthogonalised against the FM_SLOTS - 1 directions before it (truncated
// flexible CG), not only the last one: p = z - sum_j (z . q_j / p_j . q_j)
// p_j, alpha = (p . r) / (p . A p).  Directions live in FM_SLOTS ring slots;
// iteration k of a chunk writes slot k % FM_SLOTS (chunks are multiples of
// FM_SLOTS long, so the slot order is the same in every replay).
constexpr int FM_SLOTS = 4;
struct FmDirs {
    double *p[FM_SLOTS];
    double *q[FM_SLOTS];
};
void launch_pc_setup(const Sys &S, int nx, int ny, float *feats, float *scal, double *partial, unsigned *counter,
                     const KState *ks, cudaStream_t st);
void launch_pc_input(const Sys &S, int nx, int ny, const double *r, const double *z, double *r1, KState *ks,
                     const float *scal, float *feats, double *partial, cudaStream_t st);
void launch_pc_output(const Sys &S, int nx, int ny, const float *u, const double *r1, double *z, const FmDirs &D,
                      KState *ks, double *partial, cudaStream_t st);
// new direction in slot w (A-orthogonal to the other valid slots), x and r
// updates, then the V-cycle of the new r into z
bool launch_pcm_iter(const Sys &S, int nx, int ny, MgLevel *lv, int nlev, const double *coarse_inv, double *x,
                     double *r, double *z, const FmDirs &D, int w, KState *ks, double *partial, int64_t partial_len,
                     cudaStream_t st);
// FP64 residual replacement (as launch_fcg_check), then the V-cycle
bool launch_pcm_check(const Sys &S, int nx, int ny, MgLevel *lv, int nlev, const double *coarse_inv, const double *x,
                      double *r, double *z, const FmDirs &D, KState *ks, double *partial, int64_t partial_len,
                      cudaStream_t st);
// Training pair of a solved system x at the iterate x0: e = x - x0 - z (z =
// V(r), r1 = r - A z already computed, r = b - A x0), feats from r1, target
// e / rms(e).
void launch_pc_pair(const Sys &S, int nx, int ny, const double *x, const double *x0, const double *z, const double *r1, double *e,
                    const KState *ks, float *scal, double *partial, unsigned *counter, float *feats, float *target,
                    cudaStream_t st);

// mg_persist.cu: the whole MG-FCG solve (same method as launch_fcg_init /
// iter / check) as ONE cooperative launch of one CTA per 16 x 32 tile, for
// systems whose tiles fit the GPU at once and whose levels from 3 down fit
// one CTA's shared memory (up to about 256 x 256).  x receives the solution;
// r0/r1 and p0/p1 are two n-vectors each, z one; partial at least 4
// doubles per tile; bar two words (zeroed by the launch).  The levels'
// diag/ce/cn/f arrays of levels 1-3 and level 0's e serve as work space.  KState receives it, res, status (-8: a grid-barrier wait gave
// up, the solve did not finish) and done.  Returns false (nothing launched)
// when the system does not fit or the device cannot co-schedule the grid.
bool mg_persist_enabled();
// Sets the kernel's shared-memory attribute (once per process; call outside
// any stream capture); false if the device refuses it.
bool mg_persist_prepare();
// Whether launch_mg_persist would launch for this hierarchy (no launch).
bool mg_persist_fits(const MgLevel *lv, int nlev, int nx, int ny, int64_t partial_len);
bool launch_mg_persist(const Sys &S, int nx, int ny, const MgLevel *lv, int nlev, double *x, double *r0, double *r1,
                       double *p0, double *p1, double *z, double *partial, int64_t partial_len,
                       unsigned *bar, KState *ks, double tol, int maxit, float omega, cudaStream_t st);
size_t mg_persist_smem();
// The V-cycle's over-relaxation of the coarse-grid correction (mg.cu).
float mg_omega_value();

}  // namespace asd2g
