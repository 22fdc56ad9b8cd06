// Batched GFM pressure systems: many independent droplets of uneven grid
// sizes assembled and solved together, one kernel launch per phase for the
// whole batch.  Device-side descriptors and work lists shared by pressure.cu
// (batched assembly), mg.cu (batched multigrid-preconditioned flexible CG)
// and batch.cu (host orchestration).
#pragma once
#include "asd2g.h"
#include "ls32.cuh"
#include "lsmath.cuh"
#include "mg.cuh"

namespace asd2g {

// Padded-field slots of a batch arena: field slot f of instance i is
// pad + f * gtot + goff[i] (BInst::pad0 + f * gstride).  The first six
// hold the pressure problem; the rest serve the full droplet step.
enum BSlot {
    BS_LS = 0, BS_KAPPA, BS_H, BS_DIV, BS_PS, BS_P,
    BS_U, BS_V, BS_HS, BS_LSB, BS_LS0, BS_UHAT, BS_VHAT, BS_UA, BS_VA, BS_UB, BS_VB, BS_TU, BS_TV, BS_W1, BS_W2,
    BS_COUNT
};

// One instance: its grid, physics and the pointers into the batch arenas.
struct BInst {
    Grid g;
    MomConst M;
    DivH dxx, dyy;                                 // / dx^2, / dy^2
    const double *ls, *kappa, *H, *div;            // padded FP64 inputs
    double *ps, *p;                                // padded FP64 outputs (P = PS / dt)
    double *pad0;                                  // slot 0 of this instance (pad + goff)
    size_t gstride;                                // doubles between slots (gtot)
    double *sc;                                    // [0] dt of the step, [1] next dt, [2..3] volume (sharp, smooth)
    LsConst K;                                     // reinitialisation constants
    DivH ddx, ddy, d2x, d2y;                       // / dx, / dy, / (2 dx), / (2 dy)
    double kappa_lim, hs_eps;                      // 1 / min(dx, dy); 1.5 min(dx, dy)
    int kappa_fill;                                // the step fills kappa's ghosts (SolvePoisson's recompute)
    int nreinit;                                   // reinitialisation pseudo-steps of its step
    int order;                                     // time order of its intermediate velocity (0, 1, 2)
    // mixed precision: the level-set advection and reinitialisation in FP32
    int mixed;
    Ls32Work w32;                                  // FP32 work arrays (the batch's FP32 arena)
    Weno32Const wk32;                              // FP32 advection constants
    LsConstT<float> K32;                           // FP32 reinitialisation constants
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
    // learned preconditioner (allocated when a network is attached)
    FmDirs fm;                                     // truncated flexible CG direction slots
    double *pc_r1;                                 // r - A z_mg
    float *pc_feats;                               // network input [nx][ny][4] (inside its size group)
    float *pc_out;                                 // network output [nx][ny]
    float *pc_scal;                            // [0] coefficient scale (max |diag|)
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
// a level l (element-wise set-up kernels); mg_tiles[l] the tiles (shape
// MG_SHAPES[shape]) of level l of the instances whose level l is a tile level
// (l < s_cta).
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
    int shape;            // MG_SHAPES index of the tiles in mg_tiles
};
void launch_batch_mg_setup(const BatchPlan &P, cudaStream_t st);
bool launch_batch_fcg_init(const BatchPlan &P, cudaStream_t st);
bool launch_batch_fcg_iter(const BatchPlan &P, int parity, cudaStream_t st);
bool launch_batch_fcg_check(const BatchPlan &P, cudaStream_t st);
void launch_batch_set_kstate(const BatchPlan &P, double tol, int maxit, cudaStream_t st,
                             int mode = ASD2G_SOLVER_MGPCG);
// Batched learned preconditioner (ASD2G_SOLVER_UNET): set-up of the constant
// feature channels; r1 = r - A z and feature channel 0; omega and z += omega
// u (with_u) with the direction coefficients; one truncated-FCG iteration
// writing direction slot wslot, then the V-cycle of the new residual.
void launch_batch_pc_setup(const BatchPlan &P, cudaStream_t st);
void launch_batch_pc_input(const BatchPlan &P, cudaStream_t st);
void launch_batch_pc_output(const BatchPlan &P, bool with_u, cudaStream_t st);
void launch_batch_pcm_iter(const BatchPlan &P, int wslot, cudaStream_t st);
// Full droplet step of every instance (batch_step.cu): one launch per phase
// over the cell-tile list (tiles of TJ x TI interior cells), the padded-cell
// chunks (heaviside), the ghost-entry chunks (P-grid fill) or one CTA per
// instance (U/V fill); per-instance reductions (volume, dt) over the FCG
// chunks with the instance's partial slots and solver ticket.
struct BStepPlan {
    const BInst *insts;
    int count;
    const BTile *tiles;
    int ntiles;
    const BChunk *pad_chunks;    // 1024 padded cells each
    int npad;
    const BChunk *ghost_chunks;  // 256 P-grid ghost entries each
    int nghost;
    const BChunk *chunks;        // FCG chunks (1024 interior cells)
    int nchunks;
    const BTile *s32_tiles;      // mixed instances: FP32 advection strips (64 columns x 16 rows)
    int ns32;
    const BTile *r32_tiles;      // mixed instances: FP32 reinitialisation strips (60 columns x 8 rows)
    int nr32;
    int any_mixed;
};
__device__ __forceinline__ double *bslot(const BInst &I, int f) { return I.pad0 + (size_t)f * I.gstride; }
void launch_bstep_center_vel(const BStepPlan &P, cudaStream_t st);
void launch_bstep_fill_p(const BStepPlan &P, int slot, bool kappa_only_if_flagged, cudaStream_t st);
// U/V ghost fill of slots su, sv of the instances whose time order is at least min_order
void launch_bstep_fill_uv(const BStepPlan &P, int su, int sv, cudaStream_t st, int min_order = 0);
void launch_bstep_ls_stage(const BStepPlan &P, int stage, int in, int n, int out, cudaStream_t st);
// pass a or b of pseudo-step k (instances with fewer pseudo-steps skip it)
// pass 0: A (LS -> W1), 1: B (-> LS, or W2 for the Sussman modes), 2: C (the Sussman constraint -> LS)
void launch_bstep_reinit_pass(const BStepPlan &P, int mode, int pass, int k, cudaStream_t st);
// Mixed instances' FP32 level-set step (levelset32.cu, weno32.cu,
// reinit32.cu): FP64 LS <-> FP32 phi (interior and ghosts), the FP32
// centred velocities, one TVD-RK3 stage (arrays 0 phi, 2 a, 3 b), pass a or
// b of FP32 reinitialisation pseudo-step k.
void launch_bstep_ls32_convert(const BStepPlan &P, bool to64, cudaStream_t st);
void launch_bstep_center_vel32(const BStepPlan &P, cudaStream_t st);
void launch_bstep_ls_stage32(const BStepPlan &P, int stage, int in, int n, int out, cudaStream_t st);
void launch_bstep_reinit32(const BStepPlan &P, int mode, bool pass_b, int k, cudaStream_t st);
void launch_bstep_kappa(const BStepPlan &P, cudaStream_t st);
void launch_bstep_heaviside(const BStepPlan &P, cudaStream_t st);
void launch_bstep_volume(const BStepPlan &P, cudaStream_t st);
// RK stage `slot` (0, 1, 2) of every instance's intermediate velocity in its
// own time order: order 0: slot 0 = U -> UHAT; order 1: slot 0 = U -> UA,
// slot 1 = UA (base U) -> UHAT; order 2: slot 0 = U -> UA, slot 1 = UA -> UB,
// slot 2 = UB -> UHAT (GetIntermediateVel, mac2d.cpp); instances without the
// slot skip it
void launch_bstep_mom_slot(const BStepPlan &P, int slot, cudaStream_t st);
void launch_bstep_divergence(const BStepPlan &P, cudaStream_t st);
void launch_bstep_update_vel(const BStepPlan &P, cudaStream_t st);
void launch_bstep_update_dt(const BStepPlan &P, cudaStream_t st);
constexpr int BSTEP_GHOST_CHUNK = 256;
constexpr int BSTEP_PAD_CHUNK = 1024;

// Partial-sum doubles one instance needs (2 per level-0 tile or per chunk).
int64_t batch_partial_len(int nx, int ny);
int batch_tiles0(int nx, int ny);
bool batch_cta_prepare();

}  // namespace asd2g
