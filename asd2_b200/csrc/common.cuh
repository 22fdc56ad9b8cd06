// Shared device-side definitions for the asd2g kernels.
//
// Layout: padded (nx+6) x (ny+6) arrays, idx(i,j) = j + sy*i with sy = ny+6
// (the reference layout, levelset2d.cpp:1048-1050), j (y) fastest so that a
// warp's 32 lanes read 32 consecutive doubles along y.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace asd2g {

constexpr int NB = 3;  // ghost layers

// Resolved ghost-fill kinds (the dispatch of bc2d.cpp:355-573).
enum Kind : int32_t { K_NONE = 0, K_PER = 1, K_NEU = 2, K_DIR = 3, K_LSF = 4 };

struct Grid {
    int32_t nx, ny, sx, sy;    // interior sizes; padded sizes sx = nx+6, sy = ny+6
    double dx, dy;
    int32_t ku[4], kv[4], kp[4];  // resolved kinds W, E, S, N
    int32_t bp[4];                // raw BC2D values of P (assembly distinguishes NEUMANN / WALL)
    double cu[4], cv[4], cp[4];   // Dirichlet constants
    int32_t p_mirror;             // all four P sides are K_NEU/K_DIR: producers write ghost mirrors
    int32_t pinned;               // all four P sides Neumann/axisym/wall (mac2d.cpp:1496-1500)
    int32_t kappa_mode;           // ASD2G_CURVATURE_*
    int32_t bu[4], bv[4];         // raw BC2D values of U and V (the axisymmetric implicit step's end rows)
    double base_x;                // lower-left corner x (kBaseR of the axisymmetric solver)
};

__host__ __device__ __forceinline__ int64_t IX(const Grid &g, int i, int j) { return (int64_t)j + (int64_t)g.sy * i; }

// After a kernel computes the final interior value val of a cell-centred
// field at interior (i, j), write the ghost cells the P-grid fill
// (bc2d.cpp:788-810 Neumann, :835-861 Dirichlet) derives from this cell.
// Valid only when g.p_mirror is set; corners are never touched, as in the
// reference.
template <typename T>
__device__ __forceinline__ void p_mirror_store(const Grid &g, T *a, int i, int j, T val) {
    const int nx = g.nx, ny = g.ny;
    // W: a[t] = a[5-t]        (t = 0..2)  <- interior i = 3..5
    if (i <= 2 * NB - 1) {
        const int t = 2 * NB - 1 - i;
        a[IX(g, t, j)] = g.kp[0] == K_NEU ? val : -val + T(2.0) * T(g.cp[0]);
    }
    // E: a[nx+5-t] = a[nx+t]  (t = 0..2)  <- interior i = nx..nx+2
    if (i >= nx) {
        const int t = i - nx;
        a[IX(g, nx + 2 * NB - t - 1, j)] = g.kp[1] == K_NEU ? val : -val + T(2.0) * T(g.cp[1]);
    }
    // S: a[.,t] = a[.,5-t]
    if (j <= 2 * NB - 1) {
        const int t = 2 * NB - 1 - j;
        a[IX(g, i, t)] = g.kp[2] == K_NEU ? val : -val + T(2.0) * T(g.cp[2]);
    }
    // N: a[., ny+5-t] = a[., ny+t]
    if (j >= ny) {
        const int t = j - ny;
        a[IX(g, i, ny + 2 * NB - t - 1)] = g.kp[3] == K_NEU ? val : -val + T(2.0) * T(g.cp[3]);
    }
}

// Interior-cell launch shape: x over j (contiguous), y over i.
constexpr int TJ = 32, TI = 8;
__host__ inline dim3 cell_grid(const Grid &g, int i0 = NB, int i1 = -1, int j0 = NB, int j1 = -1) {
    const int ni = (i1 < 0 ? g.nx + NB : i1) - i0, nj = (j1 < 0 ? g.ny + NB : j1) - j0;
    return dim3((nj + TJ - 1) / TJ, (ni + TI - 1) / TI);
}

// Device status word bits (set by kernels, read by the host).
constexpr unsigned ST_NONFINITE = 1u, ST_BREAKDOWN = 2u;

}  // namespace asd2g
