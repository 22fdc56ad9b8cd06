// Multigrid preconditioner and flexible CG (mg.cu).
#pragma once
#include "pressure.cuh"

namespace asd2g {

// One level of the FP32 hierarchy, compact layout k = j + ny*i.
struct MgLevel {
    int nx, ny;
    float *diag, *ce, *cn, *f, *e;
};

constexpr int MG_MAX_LEVELS = 16;
constexpr int MG_COARSE_CELLS = 64;

// Level sizes (halving, odd sizes rounded up) until the coarsest level has
// at most 64 cells; returns the number of levels (0 if max_levels is too small).
int mg_levels_for(int nx, int ny, int *dims, int max_levels);
// Level 0 from the FP64 system, Galerkin coarse levels, coarsest inverse.
void launch_mg_setup(const Sys &S, MgLevel *lv, int nlev, double *coarse_inv, cudaStream_t st);
// Flexible CG with one V-cycle per iteration: init (r = b, x = 0, first
// V-cycle) and one iteration (p, q, alpha; x, r, convergence; V-cycle, beta).
void launch_fcg_init(const Sys &S, int nx, int ny, MgLevel *lv, int nlev, const double *coarse_inv, double *x,
                     double *r, double *p, double *q, double *z, KState *ks, double *partial, cudaStream_t st);
void launch_fcg_iter(const Sys &S, int nx, int ny, MgLevel *lv, int nlev, const double *coarse_inv, double *x,
                     double *r, const double *p_old, double *p_new, double *q, double *z, KState *ks,
                     double *partial, cudaStream_t st);

}  // namespace asd2g
