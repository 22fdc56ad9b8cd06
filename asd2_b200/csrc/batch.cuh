// Batched GFM pressure systems: many independent droplets of uneven grid
// sizes assembled and solved together, one kernel launch per phase for the
// whole batch.  Device-side descriptors and work lists shared by pressure.cu
// (batched assembly), mg.cu (batched multigrid-preconditioned flexible CG)
// and batch.cu (host orchestration).
#pragma once
#include "mg.cuh"

namespace asd2g {

// One instance: its grid, physics and the pointers into the batch arenas.
struct BInst {
    Grid g;
    MomConst M;
    DivH dxx, dyy;                                 // / dx^2, / dy^2
    const double *ls, *kappa, *H, *div;            // padded FP64 inputs
    double *ps, *p;                                // padded FP64 outputs (P = PS / dt)
    double dt;                                     // this instance's step
    Sys S;                                         // compact system (diag, cw, ce, cs, cn, minv, b)
    double *x, *r, *pa, *pb, *q, *z;               // flexible CG vectors (compact, FP64)
    KState *ks;                                    // this instance's solver scalars
    double *partial;                               // its partial-sum slots (2 per block)
    int64_t n;                                     // unknowns nx * ny
    int chunks;                                    // vector chunks of FCG_CHUNK unknowns
    int tiles0;                                    // level-0 multigrid tiles
    int nlev, s_cta;                               // levels; first level of the one-CTA coarse cycle
    MgLevel lv[MG_MAX_LEVELS];
    double *coarse_inv;                            // MG_COARSE_CELLS^2
};

// Work-list entries.  A cell tile is 32 x 8 padded cells of one instance
// (assembly, scatter); an MG tile 16 x 32 cells of one level; a chunk
// FCG_CHUNK consecutive unknowns.
struct BTile {
    int inst, bx, by;
};
struct BChunk {
    int inst, c;
};
constexpr int FCG_CHUNK = 1024;  // 256 threads x 4

// pressure.cu
void launch_batch_assemble(const BInst *insts, const BTile *tiles, int ntiles, cudaStream_t st);
void launch_batch_scatter(const BInst *insts, const BTile *tiles, int ntiles, cudaStream_t st);

// mg.cu: set-up of every instance's hierarchy, then the solver phases.
// lvl_chunks[l] lists the chunks of level-l cells of the instances that have
// a level l (element-wise set-up kernels); mg_tiles[l] the 16 x 32 tiles of
// level l of the instances whose level l is a tile level (l < s_cta).
struct BatchPlan {
    const BInst *insts;
    int count;
    const BChunk *chunks;  // FCG chunks of all instances
    int nchunks;
    const BChunk *lvl_chunks[MG_MAX_LEVELS];
    int nlvl_chunks[MG_MAX_LEVELS];
    const BTile *mg_tiles[MG_MAX_LEVELS];
    int nmg_tiles[MG_MAX_LEVELS];
    int max_s;            // largest s_cta over the batch
    int max_nlev;
};
void launch_batch_mg_setup(const BatchPlan &P, cudaStream_t st);
bool launch_batch_fcg_init(const BatchPlan &P, cudaStream_t st);
bool launch_batch_fcg_iter(const BatchPlan &P, int parity, cudaStream_t st);
bool launch_batch_fcg_check(const BatchPlan &P, cudaStream_t st);
void launch_batch_set_kstate(const BatchPlan &P, double tol, int maxit, cudaStream_t st);
// Partial-sum doubles one instance needs (2 per level-0 tile or per chunk).
int64_t batch_partial_len(int nx, int ny);
int batch_tiles0(int nx, int ny);
bool batch_cta_prepare();

}  // namespace asd2g
