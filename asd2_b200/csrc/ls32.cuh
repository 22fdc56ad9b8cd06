// Mixed-precision level-set step (levelset32.cu), declarations for api.cu.
#pragma once
#include "internal.cuh"

namespace asd2g {

// FP32 work arrays of the mixed level-set step, each (nx+6) x (ny+6).
struct Ls32Work {
    float *phi, *ls0, *a, *b, *tu, *tv;
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
// Kernel launches of one launch_ls_step32 call.
int ls32_launches(int reinit_mode, double max_atime, const Grid &g);
// out2[0] = sum over interior cells of H dx dy, out2[1] = of HS dx dy (FP64).
void launch_volume(const Grid &g, const double *H, const double *HS, double *partial, unsigned *counter, double *out2,
                   cudaStream_t st);

}  // namespace asd2g
