// P-grid ghost fill of one entry (device functions shared by the fill
// kernels of bc.cu and the cluster-resident level-set step of levelset.cu):
// BoundaryCondition2D::ApplyBC_P_2D (bc2d.cpp:346-353, kernels :575-934).
#pragma once
#include "internal.cuh"

namespace asd2g {

__device__ __forceinline__ void fill_p_cell(const Grid &g, double *a, int side, int layer, int s) {
    // layer t = 0..2 is the ghost distance index the reference loops use;
    // s is the position along the side (interior j for W/E, interior i for S/N).
    const int nx = g.nx, ny = g.ny, k = g.kp[side];
    const double c = g.cp[side];
    if (side == 0) {
        const int j = s, i = layer;
        if (k == K_PER) a[IX(g, i, j)] = a[IX(g, nx + i, j)];
        else if (k == K_NEU) a[IX(g, i, j)] = a[IX(g, 2 * NB - i - 1, j)];
        else if (k == K_DIR) a[IX(g, i, j)] = -a[IX(g, 2 * NB - i - 1, j)] + 2.0 * c;
    } else if (side == 1) {
        const int j = s, i = layer;
        if (k == K_PER) a[IX(g, nx + i, j)] = a[IX(g, i + NB, j)];  // writes interior columns (bc2d.cpp:770-774)
        else if (k == K_NEU) a[IX(g, nx + 2 * NB - i - 1, j)] = a[IX(g, nx + i, j)];
        else if (k == K_DIR) a[IX(g, nx + 2 * NB - i - 1, j)] = -a[IX(g, nx + i, j)] + 2.0 * c;
    } else if (side == 2) {
        const int i = s, j = layer;
        if (k == K_PER) a[IX(g, i, j)] = a[IX(g, i, ny + j)];
        else if (k == K_NEU) a[IX(g, i, j)] = a[IX(g, i, 2 * NB - j - 1)];
        else if (k == K_DIR) a[IX(g, i, j)] = -a[IX(g, i, 2 * NB - j - 1)] + 2.0 * c;
    } else {
        const int i = s, j = layer;
        if (k == K_PER) a[IX(g, i, ny + j + NB)] = a[IX(g, i, j + NB)];
        else if (k == K_NEU) a[IX(g, i, ny + 2 * NB - j - 1)] = a[IX(g, i, ny + j)];
        else if (k == K_DIR) a[IX(g, i, ny + 2 * NB - j - 1)] = -a[IX(g, i, ny + j)] + 2.0 * c;
    }
}

// LS free boundary: linear extrapolation outward (bc2d.cpp:863-900), the
// three layers in the reference's order by one thread per line.
__device__ __forceinline__ void fill_p_lsfree(const Grid &g, double *a, int side, int s) {
    const int nx = g.nx, ny = g.ny;
    const double dx = g.dx, dy = g.dy;
    if (side == 0) {
        const int j = s;
        for (int i = NB - 1; i >= 0; i--)
            a[IX(g, i, j)] = a[IX(g, i + 1, j)] + dx * (a[IX(g, i + 1, j)] - a[IX(g, i + 2, j)]) / dx;
    } else if (side == 1) {
        const int j = s;
        for (int i = 0; i < NB; i++)
            a[IX(g, nx + NB + i, j)] =
                a[IX(g, nx + NB + i - 1, j)] + dx * (a[IX(g, nx + NB + i - 1, j)] - a[IX(g, nx + NB + i - 2, j)]) / dx;
    } else if (side == 2) {
        const int i = s;
        for (int j = NB - 1; j >= 0; j--)
            a[IX(g, i, j)] = a[IX(g, i, j + 1)] + dy * (a[IX(g, i, j + 1)] - a[IX(g, i, j + 2)]) / dy;
    } else {
        const int i = s;
        for (int j = 0; j < NB; j++)
            a[IX(g, i, ny + NB + j)] =
                a[IX(g, i, ny + NB + j - 1)] + dy * (a[IX(g, i, ny + NB + j - 1)] - a[IX(g, i, ny + NB + j - 2)]) / dy;
    }
}

// Ghost entry t of the P grid (W strip, E strip, S strip, N strip, each
// NB layers); side_mask selects the sides handled.
__device__ __forceinline__ void fill_p_entry(const Grid &g, double *a, int t, int side_mask) {
    const int nwe = NB * g.ny, nsn = NB * g.nx;
    int side, rem;
    if (t < nwe) { side = 0; rem = t; }
    else if (t < 2 * nwe) { side = 1; rem = t - nwe; }
    else if (t < 2 * nwe + nsn) { side = 2; rem = t - 2 * nwe; }
    else if (t < 2 * nwe + 2 * nsn) { side = 3; rem = t - 2 * nwe - nsn; }
    else return;
    if (!((side_mask >> side) & 1)) return;
    const int along = side < 2 ? g.ny : g.nx;
    const int layer = rem / along, s = NB + rem % along;
    if (g.kp[side] == K_LSF) {
        if (layer == 0) fill_p_lsfree(g, a, side, s);
    } else {
        fill_p_cell(g, a, side, layer, s);
    }
}

}  // namespace asd2g
