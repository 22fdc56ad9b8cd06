// Momentum/pressure constants shared by momentum.cu, pressure.cu and api.cu.
#pragma once
#include <cmath>

#include "internal.cuh"

namespace asd2g {

struct MomParams {
    double rho_h, rho_l, mu_h, mu_l, sigma, g, cfl;
    int g_axis, fix_gravity;
    int numbers_given;
    double re, we, fr;
};

struct MomConst {
    DivH ddx, ddy;
    double rho_h, rho_l, mu_h, mu_l, sigma, g, cfl;
    double gu, gv;     // gravity source on U and V faces
    int gv_from_u;     // V gets the AddGravityFU pattern (zero at i = 3)
    int visc;          // kRe > 0
    int dx_pow2, dy_pow2;
    double inv_dx, inv_dy;
};

constexpr int DT_BLOCKS = 148;

MomConst make_momconst(const Grid &g, const MomParams &p);
void launch_kappa(const Grid &g, const double *ls, double *kappa, cudaStream_t st);
void launch_heaviside(const Grid &g, const double *ls, double *H, double *HS, cudaStream_t st);
void launch_mom_stage(int kind, const Grid &g, const MomConst &M, const double *ls, const double *H, const double *uin,
                      const double *vin, const double *ub, const double *vb, double *uout, double *vout,
                      const double *dtp, cudaStream_t st);
void launch_divergence(const Grid &g, const double *u, const double *v, double *div, cudaStream_t st);
void launch_update_vel(const Grid &g, const MomConst &M, const double *us, const double *vs, const double *ps,
                       const double *ls, const double *H, const double *kappa, double *u, double *v,
                       const double *dtp, cudaStream_t st);
void launch_ntk(const Grid &g, const double *ls, const double *absg, double *nxo, double *nyo, cudaStream_t st);
// axisym.cu: the axisymmetric MAC step (MACSolver2DAxisym); x is r, y is z
void launch_axi_kappa(const Grid &g, const double *ls, double *kappa, cudaStream_t st);
void launch_axi_rhs_u(const Grid &g, const MomConst &M, const double *ls, const double *u, const double *v,
                      const double *H, const double *cU, const double *dtp, double *out, cudaStream_t st,
                      int visc_only = 0);
void launch_axi_rhs_v(const Grid &g, const MomConst &M, const double *ls, const double *u, const double *uhat,
                      const double *v, const double *H, const double *cV, const double *dtp, double *out,
                      cudaStream_t st, int visc_only = 0);
void launch_axi_hat(const Grid &g, const MomConst &M, int comp, const double *ls, const double *rhs,
                    const double *H, const double *dtp, double *out, double *const w[6], cudaStream_t st);
void launch_axi_div(const Grid &g, int for_poisson, const double *u, const double *v, double *div, cudaStream_t st);
void launch_axi_update_dt(const Grid &g, const MomConst &M, const double *u, const double *v, const double *kappa,
                          double *partial, unsigned *counter, double *dt_out, cudaStream_t st);
void launch_update_dt(const Grid &g, const MomConst &M, const double *u, const double *v, double *partial,
                      unsigned *counter, double *dt_out, cudaStream_t st);

}  // namespace asd2g
