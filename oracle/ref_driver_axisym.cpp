// C entry points over the reference's MACSolver2DAxisym (src/mac2dAxisym.cpp),
// compiled from the unmodified reference sources against the shims in
// ref_shim/.  Used only to pin the axisymmetric part of the C restatement in
// oracle/asd2_oracle.c and to generate golden vectors; nothing in the product
// links it.  Field arrays are padded (nr+6)*(nz+6) doubles in the reference
// layout idx(i,j) = j + (nz+6)*i, i along r.
#include <cstring>
#include <memory>
#include <algorithm>
#include <sstream>
#include <string>
#include <vector>

#include "mac2dAxisym.h"

extern "C" {
void ref_shim_capture_arm(void);
int ref_shim_capture_sizes(int *m, int *nnz, int *nb);
}

namespace {
struct AxiCtx {
    int64_t n;
    std::unique_ptr<MACSolver2DAxisym> mac;
};
std::vector<double> ain(const AxiCtx *c, const double *p) { return std::vector<double>(p, p + c->n); }
void aout(const AxiCtx *c, const std::vector<double> &v, double *p) { std::memcpy(p, v.data(), sizeof(double) * c->n); }
}  // namespace

extern "C" {

// MACSolver2DAxisym(rhoH, rhoL, muH, muL, g, GAxis, L = 1, U = 1, sigma, ...)
// with the Poisson solver set to CG, as the reference's axisymmetric drivers
// do (tests/LargeTests/test_mac2d_large.cpp:1145-1199).
void *ref_axi_create(int nr, int nz, double base_r, double base_z, double len_r, double len_z, double rho_h,
                     double rho_l, double mu_h, double mu_l, double g, int g_axis, double sigma, double cfl) {
    AxiCtx *c = new AxiCtx();
    c->n = (int64_t)(nr + 6) * (nz + 6);
    c->mac.reset(new MACSolver2DAxisym(rho_h, rho_l, mu_h, mu_l, g, static_cast<GAXISENUM2DAXISYM>(g_axis), 1.0,
                                       1.0, sigma, nr, nz, base_r, base_z, len_r, len_z, cfl, 1.0e30, 1 << 30, 1, 3,
                                       false));
    c->mac->AllocateVariables();
    c->mac->SetPoissonSolver(POISSONTYPE::CG);
    return c;
}
void ref_axi_destroy(void *h) { delete static_cast<AxiCtx *>(h); }

// MACSolver2DAxisym::SolveTDMA (mac2dAxisym.cpp:2255-2306) on one system of n
// rows: a, b, c the sub-, main and super-diagonal, d the right side; c and d
// come back as the solver leaves them (d the solution).
int ref_axi_tdma(void *h, double *a, double *b, double *c, double *d, int n) {
    AxiCtx *x = static_cast<AxiCtx *>(h);
    std::vector<double> A(a, a + n), B(b, b + n), Cv(c, c + n), D(d, d + n);
    const int rc = x->mac->SolveTDMA(A, B, Cv, D, n);
    std::copy(Cv.begin(), Cv.end(), c);
    std::copy(D.begin(), D.end(), d);
    return rc;
}

// kind 'U', 'V' or 'P'; spec: four lower-case names "W E S N"; k4: W E S N constants.
void ref_axi_set_bc(void *h, char kind, const char *spec, const double *k4) {
    AxiCtx *c = static_cast<AxiCtx *>(h);
    std::istringstream ss(spec);
    std::string s[4];
    for (int k = 0; k < 4; k++) ss >> s[k];
    MACSolver2DAxisym *m = c->mac.get();
    if (kind == 'U') {
        m->SetBC_U_2D(s[0], s[1], s[2], s[3]);
        m->SetBCConstantUW(k4[0]); m->SetBCConstantUE(k4[1]); m->SetBCConstantUS(k4[2]); m->SetBCConstantUN(k4[3]);
    } else if (kind == 'V') {
        m->SetBC_V_2D(s[0], s[1], s[2], s[3]);
        m->SetBCConstantVW(k4[0]); m->SetBCConstantVE(k4[1]); m->SetBCConstantVS(k4[2]); m->SetBCConstantVN(k4[3]);
    } else {
        m->SetBC_P_2D(s[0], s[1], s[2], s[3]);
        m->SetBCConstantPW(k4[0]); m->SetBCConstantPE(k4[1]); m->SetBCConstantPS(k4[2]); m->SetBCConstantPN(k4[3]);
    }
}
void ref_axi_apply_bc(void *h, char kind, double *arr) {
    AxiCtx *c = static_cast<AxiCtx *>(h);
    std::vector<double> a = ain(c, arr);
    if (kind == 'U') c->mac->ApplyBC_U_2D(a);
    else if (kind == 'V') c->mac->ApplyBC_V_2D(a);
    else c->mac->ApplyBC_P_2D(a);
    aout(c, a, arr);
}
void ref_axi_set_state(void *h, const double *u, const double *v, const double *kappa, double dt) {
    AxiCtx *c = static_cast<AxiCtx *>(h);
    c->mac->m_u = ain(c, u);
    c->mac->m_v = ain(c, v);
    c->mac->m_kappa = ain(c, kappa);
    c->mac->m_dt = dt;
}
void ref_axi_get_state(void *h, double *u, double *v, double *ps, double *p, double *kappa) {
    AxiCtx *c = static_cast<AxiCtx *>(h);
    if (u) aout(c, c->mac->m_u, u);
    if (v) aout(c, c->mac->m_v, v);
    if (ps) aout(c, c->mac->m_ps, ps);
    if (p) aout(c, c->mac->m_p, p);
    if (kappa) aout(c, c->mac->m_kappa, kappa);
}
void ref_axi_kappa(void *h, const double *ls, double *kappa) {
    AxiCtx *c = static_cast<AxiCtx *>(h);
    c->mac->UpdateKappa(ain(c, ls));
    aout(c, c->mac->m_kappa, kappa);
}
void ref_axi_visc(void *h, const double *u, const double *uhat, const double *v, const double *ls, const double *H,
                  double *dU, double *dV) {
    AxiCtx *c = static_cast<AxiCtx *>(h);
    aout(c, c->mac->AddExternalViscosityFU(ain(c, u), ain(c, v), ain(c, ls), ain(c, H)), dU);
    aout(c, c->mac->AddExternalViscosityFV(ain(c, u), ain(c, uhat), ain(c, v), ain(c, ls), ain(c, H)), dV);
}
void ref_axi_rhs_u(void *h, const double *ls, const double *u, const double *v, const double *H, double *out) {
    AxiCtx *c = static_cast<AxiCtx *>(h);
    aout(c, c->mac->GetRHSU(ain(c, ls), ain(c, u), ain(c, v), ain(c, H)), out);
}
void ref_axi_rhs_v(void *h, const double *ls, const double *u, const double *uhat, const double *v, const double *H,
                   double *out) {
    AxiCtx *c = static_cast<AxiCtx *>(h);
    aout(c, c->mac->GetRHSV(ain(c, ls), ain(c, u), ain(c, uhat), ain(c, v), ain(c, H)), out);
}
void ref_axi_uhat(void *h, const double *ls, const double *u, const double *rhs, const double *H, double *out) {
    AxiCtx *c = static_cast<AxiCtx *>(h);
    aout(c, c->mac->GetUHat(ain(c, ls), ain(c, u), ain(c, rhs), ain(c, H)), out);
}
void ref_axi_vhat(void *h, const double *ls, const double *v, const double *rhs, const double *H, double *out) {
    AxiCtx *c = static_cast<AxiCtx *>(h);
    aout(c, c->mac->GetVHat(ain(c, ls), ain(c, v), ain(c, rhs), ain(c, H)), out);
}
void ref_axi_div(void *h, const double *u, const double *v, double *div4p, double *div) {
    AxiCtx *c = static_cast<AxiCtx *>(h);
    aout(c, c->mac->GetDivergence4Poisson(ain(c, u), ain(c, v)), div4p);
    aout(c, c->mac->GetDivergence(ain(c, u), ain(c, v)), div);
}
// SolvePoisson with maxiter CG iterations and the capture hook armed (the
// system is then read with ref_capture_copy of ref_driver.cpp).
int ref_axi_poisson(void *h, double *ps, const double *div, const double *ls, const double *lsB, const double *H,
                    int maxiter, int *m, int *nnz, int *nb) {
    AxiCtx *c = static_cast<AxiCtx *>(h);
    std::vector<double> p = ain(c, ps);
    ref_shim_capture_arm();
    c->mac->SolvePoisson(p, ain(c, div), ain(c, ls), ain(c, lsB), c->mac->m_u, c->mac->m_v, ain(c, H), maxiter);
    aout(c, p, ps);
    return ref_shim_capture_sizes(m, nnz, nb);
}
void ref_axi_update_vel(void *h, const double *uhat, const double *vhat, const double *ps, const double *ls,
                        const double *lsB, const double *H) {
    AxiCtx *c = static_cast<AxiCtx *>(h);
    c->mac->UpdateVel(c->mac->m_u, c->mac->m_v, ain(c, uhat), ain(c, vhat), ain(c, ps), ain(c, ls), ain(c, lsB),
                      ain(c, H));
}
double ref_axi_update_dt(void *h, const double *u, const double *v) {
    AxiCtx *c = static_cast<AxiCtx *>(h);
    return c->mac->UpdateDt(ain(c, u), ain(c, v));
}
}
