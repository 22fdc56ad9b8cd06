// Mixed-precision level-set step (levelset32.cu), declarations for api.cu.
#pragma once
#include "internal.cuh"

namespace asd2g {

// Constants of the FP32 advection stage.
struct Weno32Const {
    float hx, hy;      // 0.5 / dx, 0.5 / dy
    float epsx, epsy;  // 1e-6 dx^2, 1e-6 dy^2
};
Weno32Const make_weno32_const(const Grid &g);

// FP32 work arrays of the mixed level-set step, each (nx+6) x (ny+6).
struct Ls32Work {
    float *phi, *ls0, *a, *b, *tu, *tv;
    int *band;         // offsets of the Sussman band cells (capacity nx * ny)
    unsigned *band_n;  // their count
};
constexpr int LS32_ARRAYS = 6;
constexpr int VOLUME_BLOCKS = 592;  // partial sums: 2 per block

// The FP32 path needs producer-side ghost fills (all P sides Neumann or
// Dirichlet) and a reinitialisation mode it implements (0, 2 or 4).
bool ls32_supported(const Grid &g, int reinit_mode);
// ls64 (ghosts filled) -> FP32, TVD-RK3 advection with dt = *dtp, the
// reinitialisation pseudo-steps, -> ls64 (interior and ghosts).
void launch_ls_step32(const Grid &g, int reinit_mode, double max_atime, const double *u, const double *v,
                      const double *dtp, double *ls64, const Ls32Work &w, cudaStream_t st);
// One TVD-RK3 stage (1, 2 or 3) in FP32 (weno32.cu): out = stage(phi_n,
// phi_in, dt * HJWENO5(phi_in; tu, tv)), interior and ghost mirrors.
void launch_ls_stage32(const Grid &g, int stage, const float *phi_in, const float *tu, const float *tv,
                       const float *phi_n, float *out, const double *dtp, cudaStream_t st);
// Rows per warp of the FP32 stage kernel (64 columns x R rows per warp).
int ls32_rows_per_warp(const Grid &g);
// One reinitialisation pseudo-step (mode 0, 2 or 4) in FP32, packed form
// (reinit32.cu): phi <- pseudo-step(phi; phi0 = ls0), a and b as scratch.
void launch_reinit32_step(const Grid &g, int reinit_mode, const Ls32Work &w, cudaStream_t st);
// Kernel launches of one launch_ls_step32 call.
int ls32_launches(int reinit_mode, double max_atime, const Grid &g);
// out2[0] = sum over interior cells of H dx dy, out2[1] = of HS dx dy (FP64).
void launch_volume(const Grid &g, const double *H, const double *HS, double *partial, unsigned *counter, double *out2,
                   cudaStream_t st);

}  // namespace asd2g
