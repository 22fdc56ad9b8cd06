// Ghost-cell fill for the staggered U, V and P grids.
// BoundaryCondition2D::ApplyBC_{U,V,P}_2D (bc2d.cpp:123-128, :239-244,
// :346-353) applies the W, E, S and N sides in that order, and later sides
// read cells earlier sides wrote (e.g. the U-grid W side writes the whole
// column i = 3, which a Dirichlet S side then overwrites in rows 0..2).  The
// U/V fill therefore runs in one CTA with a barrier between sides.  The P fill
// touches disjoint strips that only read interior cells for Neumann and
// Dirichlet sides, so those run fully parallel; periodic and extrapolating
// sides run side by side in order.
#include "batch.cuh"
#include "bc_fill.cuh"
#include "internal.cuh"

namespace asd2g {

// ---------------------------------------------------------------- U grid --
// side: 0 W, 1 E, 2 S, 3 N.  Work is split over [tid, n) with stride.
__device__ void fill_u_side(const Grid &g, double *a, int side, int tid, int nth) {
    const int nx = g.nx, ny = g.ny, k = g.ku[side];
    const double c = g.cu[side];
    if (k == K_NONE || k == K_LSF) return;
    if (side == 0) {
        if (k == K_PER) {  // bc2d.cpp:575-579 (i = 0..3)
            const int cnt = (NB + 1) * ny;
            for (int t = tid; t < cnt; t += nth) {
                const int i = t / ny, j = NB + t % ny;
                a[IX(g, i, j)] = a[IX(g, nx - 1 + i, j)];
            }
        } else if (k == K_NEU) {  // :599-606
            const int m = ny + 2 * NB, cnt2 = NB * (ny + 1);
            for (int t = tid; t < m + cnt2; t += nth) {
                if (t < m) a[IX(g, NB, t)] = a[IX(g, NB + 1, t)];
                else {
                    const int q = t - m, i = q / (ny + 1), j = NB + q % (ny + 1);
                    a[IX(g, i, j)] = a[IX(g, 2 * NB - i, j)];
                }
            }
        } else {  // K_DIR :631-640
            const int m = ny + 2 * NB, cnt2 = NB * ny;
            for (int t = tid; t < m + cnt2; t += nth) {
                if (t < m) a[IX(g, NB, t)] = c;
                else {
                    const int q = t - m, i = q / ny, j = NB + q % ny;
                    a[IX(g, i, j)] = -a[IX(g, 2 * NB - i, j)] + 2.0 * c;
                }
            }
        }
    } else if (side == 1) {
        if (k == K_PER) {  // :581-585
            for (int t = tid; t < NB * ny; t += nth) {
                const int i = t / ny, j = NB + t % ny;
                a[IX(g, nx + i + NB, j)] = a[IX(g, i + NB, j)];
            }
        } else if (k == K_NEU) {  // :608-615
            const int m = ny + 2 * NB, cnt2 = (NB - 1) * (ny + 1);
            for (int t = tid; t < m + cnt2; t += nth) {
                if (t < m) a[IX(g, nx + NB, t)] = a[IX(g, nx + NB - 1, t)];
                else {
                    const int q = t - m, i = 1 + q / (ny + 1), j = NB + q % (ny + 1);
                    a[IX(g, nx + 2 * NB - i, j)] = a[IX(g, nx + i, j)];
                }
            }
        } else {  // :642-650
            const int m = ny + 2 * NB, cnt2 = (NB - 1) * ny;
            for (int t = tid; t < m + cnt2; t += nth) {
                if (t < m) a[IX(g, nx + NB, t)] = c;
                else {
                    const int q = t - m, i = 1 + q / ny, j = NB + q % ny;
                    a[IX(g, nx + 2 * NB - i, j)] = -a[IX(g, nx + i, j)] + 2.0 * c;
                }
            }
        }
    } else {
        const bool north = side == 3;
        if (k == K_PER || k == K_NEU) {  // :587-597, :617-627 (i = 4..nx+2)
            const int ni = nx - 1;
            for (int t = tid; t < ni * NB; t += nth) {
                const int i = NB + 1 + t / NB, j = t % NB;
                if (!north) a[IX(g, i, j)] = k == K_PER ? a[IX(g, i, ny + j)] : a[IX(g, i, 2 * NB - j - 1)];
                else if (k == K_PER) a[IX(g, i, ny + j + NB)] = a[IX(g, i, j + NB)];
                else a[IX(g, i, ny + 2 * NB - j - 1)] = a[IX(g, i, ny + j)];
            }
        } else {  // K_DIR :652-664 (i = 3..nx+2)
            for (int t = tid; t < nx * NB; t += nth) {
                const int i = NB + t / NB, j = t % NB;
                if (!north) a[IX(g, i, j)] = -a[IX(g, i, 2 * NB - j - 1)] + 2.0 * c;
                else a[IX(g, i, ny + 2 * NB - j - 1)] = -a[IX(g, i, ny + j)] + 2.0 * c;
            }
        }
    }
}

// ---------------------------------------------------------------- V grid --
__device__ void fill_v_side(const Grid &g, double *a, int side, int tid, int nth) {
    const int nx = g.nx, ny = g.ny, k = g.kv[side];
    const double c = g.cv[side];
    if (k == K_NONE || k == K_LSF) return;
    if (side == 0 || side == 1) {  // :666-676, :690-700, :730-742 (j = 4..ny+2)
        const bool east = side == 1;
        const int nj = ny - 1;
        for (int t = tid; t < NB * nj; t += nth) {
            const int i = t / nj, j = NB + 1 + t % nj;
            if (!east) {
                if (k == K_PER) a[IX(g, i, j)] = a[IX(g, nx + i, j)];
                else if (k == K_NEU) a[IX(g, i, j)] = a[IX(g, 2 * NB - i - 1, j)];
                else a[IX(g, i, j)] = -a[IX(g, 2 * NB - i - 1, j)] + 2.0 * c;
            } else {
                if (k == K_PER) a[IX(g, nx + i + NB, j)] = a[IX(g, i + NB, j)];
                else if (k == K_NEU) a[IX(g, nx + 2 * NB - i - 1, j)] = a[IX(g, nx + i, j)];
                else a[IX(g, nx + 2 * NB - i - 1, j)] = -a[IX(g, nx + i, j)] + 2.0 * c;
            }
        }
    } else if (side == 2) {
        if (k == K_PER) {  // :678-682 (j = 0..3)
            for (int t = tid; t < nx * (NB + 1); t += nth) {
                const int i = NB + t / (NB + 1), j = t % (NB + 1);
                a[IX(g, i, j)] = a[IX(g, i, ny - 1 + j)];
            }
        } else {  // :702-709 Neumann, :744-752 Dirichlet
            const int m = nx + 2 * NB;
            for (int t = tid; t < m + nx * NB; t += nth) {
                if (t < m) a[IX(g, t, NB)] = k == K_NEU ? a[IX(g, t, NB + 1)] : c;
                else {
                    const int q = t - m, i = NB + q / NB, j = q % NB;
                    a[IX(g, i, j)] = k == K_NEU ? a[IX(g, i, 2 * NB - j)] : -a[IX(g, i, 2 * NB - j)] + 2.0 * c;
                }
            }
        }
    } else {
        if (k == K_PER) {  // :684-688
            for (int t = tid; t < nx * NB; t += nth) {
                const int i = NB + t / NB, j = t % NB;
                a[IX(g, i, ny + j + NB)] = a[IX(g, i, j + NB)];
            }
        } else {  // :711-718, :754-762
            const int m = nx + 2 * NB;
            for (int t = tid; t < m + nx * (NB - 1); t += nth) {
                if (t < m) a[IX(g, t, ny + NB)] = k == K_NEU ? a[IX(g, t, ny + NB - 1)] : c;
                else {
                    const int q = t - m, i = NB + q / (NB - 1), j = 1 + q % (NB - 1);
                    a[IX(g, i, ny + 2 * NB - j)] =
                        k == K_NEU ? a[IX(g, i, ny + j)] : -a[IX(g, i, ny + j)] + 2.0 * c;
                }
            }
        }
    }
}

// One CTA fills U and/or V (either pointer may be null), side by side.
__global__ void __launch_bounds__(1024) k_fill_uv(Grid g, double *u, double *v) {
    for (int side = 0; side < 4; side++) {
        if (u) fill_u_side(g, u, side, threadIdx.x, blockDim.x);
        if (v) fill_v_side(g, v, side, threadIdx.x, blockDim.x);
        __syncthreads();
    }
}

// ---------------------------------------------------------------- P grid --
// fill_p_cell / fill_p_lsfree / fill_p_entry: bc_fill.cuh

// side_mask selects the sides handled by this launch.
__global__ void k_fill_p(Grid g, double *a, int side_mask) {
    fill_p_entry(g, a, blockIdx.x * blockDim.x + threadIdx.x, side_mask);
}

// Batched fills (asd2g_batch_step): every instance's P grid in one launch
// over the ghost-entry chunks (Neumann/Dirichlet sides: all four at once),
// and the U/V fill with one CTA per instance.
__global__ void k_bfill_p(const BInst *__restrict__ insts, const BChunk *__restrict__ chunks, int slot,
                          int only_flagged) {
    const BChunk w = chunks[blockIdx.x];
    const BInst &I = insts[w.inst];
    if (only_flagged && !I.kappa_fill) return;
    fill_p_entry(I.g, bslot(I, slot), w.c * BSTEP_GHOST_CHUNK + threadIdx.x, 0xF);
}

__global__ void __launch_bounds__(1024) k_bfill_uv(const BInst *__restrict__ insts, int su, int sv, int min_order) {
    const BInst &I = insts[blockIdx.x];
    if (I.order < min_order) return;
    double *u = bslot(I, su), *v = bslot(I, sv);
    for (int side = 0; side < 4; side++) {
        fill_u_side(I.g, u, side, threadIdx.x, blockDim.x);
        fill_v_side(I.g, v, side, threadIdx.x, blockDim.x);
        __syncthreads();
    }
}

void launch_bstep_fill_p(const BStepPlan &P, int slot, bool kappa_only_if_flagged, cudaStream_t st) {
    k_bfill_p<<<P.nghost, BSTEP_GHOST_CHUNK, 0, st>>>(P.insts, P.ghost_chunks, slot, kappa_only_if_flagged ? 1 : 0);
}

void launch_bstep_fill_uv(const BStepPlan &P, int su, int sv, cudaStream_t st, int min_order) {
    k_bfill_uv<<<P.count, 1024, 0, st>>>(P.insts, su, sv, min_order);
}

// One side of one grid with an explicit fill kind (the per-side methods
// BC_UW, BC_NeumannUW, ... of bc2d.cpp).  grid_kind: 0 U, 1 V, 2 P.
void launch_fill_side(const Grid &g0, double *a, int grid_kind, int side, int kind, cudaStream_t st) {
    Grid g = g0;
    for (int s = 0; s < 4; s++) g.ku[s] = g.kv[s] = g.kp[s] = K_NONE;
    if (grid_kind == 0) g.ku[side] = kind;
    else if (grid_kind == 1) g.kv[side] = kind;
    else g.kp[side] = kind;
    if (grid_kind == 0) k_fill_uv<<<1, 1024, 0, st>>>(g, a, nullptr);
    else if (grid_kind == 1) k_fill_uv<<<1, 1024, 0, st>>>(g, nullptr, a);
    else {
        const int n = 2 * NB * g.ny + 2 * NB * g.nx;
        k_fill_p<<<(n + 255) / 256, 256, 0, st>>>(g, a, 1 << side);
    }
}

void launch_fill_uv(const Grid &g, double *u, double *v, cudaStream_t st) {
    k_fill_uv<<<1, 1024, 0, st>>>(g, u, v);
}

void launch_fill_p(const Grid &g, double *a, cudaStream_t st) {
    const int n = 2 * NB * g.ny + 2 * NB * g.nx;
    const int blocks = (n + 255) / 256;
    bool seq = false;
    for (int s = 0; s < 4; s++) seq |= (g.kp[s] == K_PER || g.kp[s] == K_LSF);
    if (!seq) {
        k_fill_p<<<blocks, 256, 0, st>>>(g, a, 0xF);
    } else {
        for (int s = 0; s < 4; s++) k_fill_p<<<blocks, 256, 0, st>>>(g, a, 1 << s);
    }
}

}  // namespace asd2g
