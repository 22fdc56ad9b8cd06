// C entry points over the reference's own classes (LevelSetSolver2D,
// MACSolver2D, PoissonSolver2D), compiled from the unmodified reference
// sources against the shims in ref_shim/.  Used only to generate golden
// vectors and to pin the C restatement in oracle/asd2_oracle.c; nothing in
// the product links it.  All field arrays are padded (nx+6)*(ny+6) doubles in
// the reference layout idx(i,j) = j + (ny+6)*i.
#include <cstring>
#include <memory>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "levelset2d.h"
#include "mac2d.h"
#include "poisson2d.h"

extern "C" {
void ref_shim_capture_arm(void);
int ref_shim_capture_sizes(int *m, int *nnz, int *nb);
int ref_shim_capture_copy(double *a, int *ia, int *ja, double *b);
}

namespace {
struct RefCtx {
    int nx, ny;
    int64_t n;
    std::shared_ptr<LevelSetSolver2D> ls;
    std::unique_ptr<MACSolver2D> mac;
};

std::vector<double> vin(const RefCtx *c, const double *p) { return std::vector<double>(p, p + c->n); }
void vout(const RefCtx *c, const std::vector<double> &v, double *p) { std::memcpy(p, v.data(), sizeof(double) * c->n); }

void split4(const char *spec, std::string out[4]) {
    std::istringstream ss(spec);
    for (int k = 0; k < 4; k++) ss >> out[k];
}
}  // namespace

extern "C" {

void *ref_create(int nx, int ny, double base_x, double base_y, double len_x, double len_y, double rho_h,
                 double rho_l, double mu_h, double mu_l, double g, int g_axis, double sigma, int time_order,
                 double cfl, double ls_max_atime) {
    RefCtx *c = new RefCtx();
    c->nx = nx;
    c->ny = ny;
    c->n = (int64_t)(nx + 6) * (ny + 6);
    const double dx = len_x / nx, dy = len_y / ny;
    if (ls_max_atime > 0.0)
        c->ls = std::make_shared<LevelSetSolver2D>(nx, ny, 3, base_x, base_y, dx, dy, ls_max_atime);
    else
        c->ls = std::make_shared<LevelSetSolver2D>(nx, ny, 3, base_x, base_y, dx, dy);
    c->mac.reset(new MACSolver2D(rho_h, rho_l, mu_h, mu_l, g, static_cast<GAXISENUM2D>(g_axis), 1.0, 1.0, sigma,
                                 nx, ny, base_x, base_y, len_x, len_y, static_cast<TIMEORDERENUM>(time_order), cfl,
                                 1.0e30, 1 << 30, 1, 3, false));
    c->mac->AllocateVariables();
    c->mac->SetPoissonSolver(POISSONTYPE::CG);
    return c;
}

void ref_destroy(void *h) { delete static_cast<RefCtx *>(h); }

// which: 0 = level-set solver's BC object, 1 = MAC solver's BC object.
// kind: 'U', 'V' or 'P'.  spec: four lower-case names "W E S N".
void ref_set_bc(void *h, int which, char kind, const char *spec) {
    RefCtx *c = static_cast<RefCtx *>(h);
    std::string s[4];
    split4(spec, s);
    if (which == 0) {
        if (kind == 'U') c->ls->SetBC_U_2D(s[0], s[1], s[2], s[3]);
        if (kind == 'V') c->ls->SetBC_V_2D(s[0], s[1], s[2], s[3]);
        if (kind == 'P') c->ls->SetBC_P_2D(s[0], s[1], s[2], s[3]);
    } else {
        if (kind == 'U') c->mac->SetBC_U_2D(s[0], s[1], s[2], s[3]);
        if (kind == 'V') c->mac->SetBC_V_2D(s[0], s[1], s[2], s[3]);
        if (kind == 'P') c->mac->SetBC_P_2D(s[0], s[1], s[2], s[3]);
    }
}

void ref_set_bc_const(void *h, int which, char kind, const double *k4) {
    RefCtx *c = static_cast<RefCtx *>(h);
    std::shared_ptr<BoundaryCondition2D> bc = which == 0 ? c->ls->m_BC : c->mac->m_BC;
    if (kind == 'U') { bc->SetBCConstantUW(k4[0]); bc->SetBCConstantUE(k4[1]); bc->SetBCConstantUS(k4[2]); bc->SetBCConstantUN(k4[3]); }
    if (kind == 'V') { bc->SetBCConstantVW(k4[0]); bc->SetBCConstantVE(k4[1]); bc->SetBCConstantVS(k4[2]); bc->SetBCConstantVN(k4[3]); }
    if (kind == 'P') { bc->SetBCConstantPW(k4[0]); bc->SetBCConstantPE(k4[1]); bc->SetBCConstantPS(k4[2]); bc->SetBCConstantPN(k4[3]); }
}

void ref_apply_bc(void *h, int which, char kind, double *arr) {
    RefCtx *c = static_cast<RefCtx *>(h);
    std::vector<double> a = vin(c, arr);
    std::shared_ptr<BoundaryCondition2D> bc = which == 0 ? c->ls->m_BC : c->mac->m_BC;
    if (kind == 'U') bc->ApplyBC_U_2D(a);
    if (kind == 'V') bc->ApplyBC_V_2D(a);
    if (kind == 'P') bc->ApplyBC_P_2D(a);
    vout(c, a, arr);
}

// ---------------- level set ----------------
void ref_ls_advect(void *h, double *ls, const double *u, const double *v, double dt) {
    RefCtx *c = static_cast<RefCtx *>(h);
    std::vector<double> l = vin(c, ls);
    c->ls->Solve_LevelSet_2D(l, vin(c, u), vin(c, v), dt);
    vout(c, l, ls);
}

void ref_ls_weno_rhs(void *h, double *ls, const double *u, const double *v, double *out) {
    RefCtx *c = static_cast<RefCtx *>(h);
    std::vector<double> l = vin(c, ls);
    std::vector<double> r = c->ls->HJWENO5_LS_2D(l, vin(c, u), vin(c, v));
    vout(c, l, ls);
    vout(c, r, out);
}

void ref_unit_weno5(void *h, const double *F, double *FP, double *FM, double d, int n) {
    RefCtx *c = static_cast<RefCtx *>(h);
    std::vector<double> f(F, F + n + 6), fp(n + 6, 0.0), fm(n + 6, 0.0);
    c->ls->UnitHJWENO5(f, fp, fm, d, n);
    std::memcpy(FP, fp.data(), sizeof(double) * (n + 6));
    std::memcpy(FM, fm.data(), sizeof(double) * (n + 6));
}

// mode: 0 Reinit_Original_2D, 1 Reinit_Sussman_2D, 2 Reinit_MinRK2_2D,
//       3 FirstTimeOnlyReinit_Sussman_2D,
//       4 MinRK2 pseudo-steps with the Sussman area constraint applied after
//         each one, composed from the public pieces the reference exposes
//         (levelset2d.cpp:433-486 with the constraint call that is commented
//         out at :474 switched on).
void ref_reinit(void *h, int mode, double *ls) {
    RefCtx *c = static_cast<RefCtx *>(h);
    LevelSetSolver2D &L = *c->ls;
    std::vector<double> l = vin(c, ls);
    if (mode == 0) L.Reinit_Original_2D(l);
    if (mode == 1) L.Reinit_Sussman_2D(l);
    if (mode == 2) L.Reinit_MinRK2_2D(l);
    if (mode == 3) L.FirstTimeOnlyReinit_Sussman_2D(l);
    if (mode == 4) {
        const int nx = L.kNx, ny = L.kNy, nb = L.kNumBCGrid;
        auto I = [&](int i, int j) { return j + (ny + 2 * nb) * i; };
        L.m_atime = 0.0;
        L.ApplyBC_P_2D(l);
        std::vector<double> lsInit = l;
        std::vector<double> LS1(c->n, 0.0), LS2(c->n, 0.0), tmpLS(c->n, 0.0);
        std::vector<double> S = L.GetSmoothedSignFunc(lsInit);
        while (L.m_atime < L.kMaxATime) {
            L.m_atime += L.kAdt;
            L.ApplyBC_P_2D(l);
            std::vector<double> a1 = L.SubcellENO_Min_DerivAbsLS_2D(l, lsInit);
            for (int i = nb; i < nx + nb; i++)
                for (int j = nb; j < ny + nb; j++) LS1[I(i, j)] = l[I(i, j)] - L.kAdt * S[I(i, j)] * (a1[I(i, j)] - 1.0);
            L.ApplyBC_P_2D(LS1);
            std::vector<double> a2 = L.SubcellENO_Min_DerivAbsLS_2D(LS1, lsInit);
            for (int i = nb; i < nx + nb; i++)
                for (int j = nb; j < ny + nb; j++) LS2[I(i, j)] = LS1[I(i, j)] - L.kAdt * S[I(i, j)] * (a2[I(i, j)] - 1.0);
            L.ApplyBC_P_2D(LS2);
            for (int i = nb; i < nx + nb; i++)
                for (int j = nb; j < ny + nb; j++) tmpLS[I(i, j)] = 0.5 * (l[I(i, j)] + LS2[I(i, j)]);
            L.ApplyBC_P_2D(tmpLS);
            std::vector<double> hd = L.UpdateHeavisideFuncDeriv(tmpLS);
            std::vector<double> sc = L.GetSussmanReinitConstraint(tmpLS, lsInit, hd);
            for (int i = nb; i < nx + nb; i++)
                for (int j = nb; j < ny + nb; j++) l[I(i, j)] = tmpLS[I(i, j)] + sc[I(i, j)];
        }
        L.ApplyBC_P_2D(l);
    }
    vout(c, l, ls);
}

void ref_subcell_eno(void *h, const double *ls, const double *lsInit, double *out) {
    RefCtx *c = static_cast<RefCtx *>(h);
    vout(c, c->ls->SubcellENO_Min_DerivAbsLS_2D(vin(c, ls), vin(c, lsInit)), out);
}
void ref_eno(void *h, const double *ls, const double *lsInit, double *out) {
    RefCtx *c = static_cast<RefCtx *>(h);
    vout(c, c->ls->ENO_DerivAbsLS_2D(vin(c, ls), vin(c, lsInit)), out);
}
void ref_weno_absgrad(void *h, const double *ls, const double *lsInit, double *out) {
    RefCtx *c = static_cast<RefCtx *>(h);
    vout(c, c->ls->HJWENO5_DerivAbsLS_2D(vin(c, ls), vin(c, lsInit)), out);
}
void ref_sussman_constraint(void *h, const double *ls, const double *lsInit, const double *hd, double *out) {
    RefCtx *c = static_cast<RefCtx *>(h);
    vout(c, c->ls->GetSussmanReinitConstraint(vin(c, ls), vin(c, lsInit), vin(c, hd)), out);
}
void ref_heaviside_deriv(void *h, const double *ls, double *out) {
    RefCtx *c = static_cast<RefCtx *>(h);
    vout(c, c->ls->UpdateHeavisideFuncDeriv(vin(c, ls)), out);
}
void ref_smoothed_sign(void *h, const double *ls, double *out) {
    RefCtx *c = static_cast<RefCtx *>(h);
    vout(c, c->ls->GetSmoothedSignFunc(vin(c, ls)), out);
}

// ---------------- MAC solver ----------------
void ref_mac_set_state(void *h, const double *u, const double *v, const double *ps, double dt) {
    RefCtx *c = static_cast<RefCtx *>(h);
    c->mac->m_u = vin(c, u);
    c->mac->m_v = vin(c, v);
    c->mac->m_ps = vin(c, ps);
    c->mac->m_dt = dt;
}
double ref_mac_get_state(void *h, double *u, double *v, double *ps, double *p, double *kappa) {
    RefCtx *c = static_cast<RefCtx *>(h);
    if (u) vout(c, c->mac->m_u, u);
    if (v) vout(c, c->mac->m_v, v);
    if (ps) vout(c, c->mac->m_ps, ps);
    if (p) vout(c, c->mac->m_p, p);
    if (kappa) vout(c, c->mac->m_kappa, kappa);
    return c->mac->m_dt;
}
void ref_mac_set_kappa(void *h, const double *kappa) {
    RefCtx *c = static_cast<RefCtx *>(h);
    c->mac->m_kappa = vin(c, kappa);
}
void ref_mac_kappa(void *h, const double *ls, double *kappa) {
    RefCtx *c = static_cast<RefCtx *>(h);
    c->mac->UpdateKappa(vin(c, ls));
    vout(c, c->mac->m_kappa, kappa);
}
// UpdateNTK(LSolver, ls, (nx, ny), t1, t2, kappa): the normal components
// start from nxo / nyo (the reference leaves cells it does not reach as they
// were) and are copied back.
void ref_mac_ntk(void *h, const double *ls, double *nxo, double *nyo) {
    RefCtx *c = static_cast<RefCtx *>(h);
    std::vector<double> nx = vin(c, nxo), ny = vin(c, nyo);
    std::vector<double> t1x(c->n), t1y(c->n), t1z(c->n), t2x(c->n), t2y(c->n), t2z(c->n), kap(c->n);
    c->mac->UpdateNTK(c->ls, vin(c, ls), std::tie(nx, ny), std::tie(t1x, t1y, t1z), std::tie(t2x, t2y, t2z), kap);
    vout(c, nx, nxo);
    vout(c, ny, nyo);
}
void ref_mac_heaviside(void *h, const double *ls, double *H, double *HS) {
    RefCtx *c = static_cast<RefCtx *>(h);
    vout(c, c->mac->UpdateHeavisideFunc(vin(c, ls)), H);
    vout(c, c->mac->UpdateSmoothHeavisideFunc(vin(c, ls)), HS);
}
void ref_mac_conv(void *h, const double *u, const double *v, double *cU, double *cV) {
    RefCtx *c = static_cast<RefCtx *>(h);
    vout(c, c->mac->AddConvectionFU(vin(c, u), vin(c, v)), cU);
    vout(c, c->mac->AddConvectionFV(vin(c, u), vin(c, v)), cV);
}
void ref_mac_visc(void *h, const double *u, const double *v, const double *ls, const double *H, double *dU,
                  double *dV) {
    RefCtx *c = static_cast<RefCtx *>(h);
    vout(c, c->mac->AddViscosityFU(vin(c, u), vin(c, v), vin(c, ls), vin(c, H)), dU);
    vout(c, c->mac->AddViscosityFV(vin(c, u), vin(c, v), vin(c, ls), vin(c, H)), dV);
}
void ref_mac_rhs(void *h, const double *ls, const double *u, const double *v, const double *H, double *FU,
                 double *FV) {
    RefCtx *c = static_cast<RefCtx *>(h);
    vout(c, c->mac->UpdateFU(c->ls, vin(c, ls), vin(c, u), vin(c, v), vin(c, H)), FU);
    vout(c, c->mac->UpdateFV(c->ls, vin(c, ls), vin(c, u), vin(c, v), vin(c, H)), FV);
}
void ref_mac_intermediate(void *h, const double *ls, const double *u, const double *v, double *uhat, double *vhat,
                          const double *H) {
    RefCtx *c = static_cast<RefCtx *>(h);
    std::vector<double> uh = vin(c, uhat), vh = vin(c, vhat);
    c->mac->GetIntermediateVel(c->ls, vin(c, ls), vin(c, u), vin(c, v), uh, vh, vin(c, H));
    vout(c, uh, uhat);
    vout(c, vh, vhat);
}
void ref_mac_div(void *h, const double *u, const double *v, double *div) {
    RefCtx *c = static_cast<RefCtx *>(h);
    vout(c, c->mac->GetDivergence(vin(c, u), vin(c, v)), div);
}
// MACSolver2D::OutRes with PLTTYPE::ASCII; m_iter (0 writes the file headers) set first.
int ref_mac_outres(void *h, int m_iter, int iter, double t, const char *vel_base, const char *div_base,
                   const double *u, const double *v, const double *ps, const double *ls) {
    RefCtx *c = static_cast<RefCtx *>(h);
    c->mac->SetPLTType(PLTTYPE::ASCII);
    c->mac->m_iter = m_iter;
    return c->mac->OutRes(iter, t, vel_base, div_base, vin(c, u), vin(c, v), vin(c, ps), vin(c, ls));
}
// Runs MACSolver2D::SolvePoisson with maxiter iterations of the reference CG
// and the capture hook armed.  Writes the solver's ps (and m_p) back, and
// returns the captured system sizes in m/nnz/nb (-1 if nothing was captured).
int ref_mac_poisson(void *h, double *ps, const double *div, const double *ls, const double *lsB, const double *H,
                    int maxiter, int *m, int *nnz, int *nb) {
    RefCtx *c = static_cast<RefCtx *>(h);
    std::vector<double> p = vin(c, ps);
    ref_shim_capture_arm();
    c->mac->SolvePoisson(p, vin(c, div), vin(c, ls), vin(c, lsB), c->mac->m_u, c->mac->m_v, vin(c, H), maxiter);
    vout(c, p, ps);
    return ref_shim_capture_sizes(m, nnz, nb);
}
int ref_capture_copy(double *a, int *ia, int *ja, double *b) { return ref_shim_capture_copy(a, ia, ja, b); }

// PoissonSolver2D::CG_2FUniformP_2D on a caller-supplied CSR system (e.g. one
// captured above).  rhs and ps are padded arrays; mdiag holds the diagonal
// used for the Jacobi preconditioner (one value per row).
void ref_mac_cg(void *h, double *ps, const double *rhs, const double *a, const int *ia, const int *ja, int rows,
                const double *mdiag, int maxiter) {
    RefCtx *c = static_cast<RefCtx *>(h);
    std::vector<double> p = vin(c, ps);
    const int nnz = ia[rows];
    std::vector<double> A(a, a + nnz), M(mdiag, mdiag + rows);
    std::vector<MKL_INT> IA(ia, ia + rows + 1), JA(ja, ja + nnz), MR(rows + 1), MC(rows);
    for (int r = 0; r <= rows; r++) MR[r] = r;
    for (int r = 0; r < rows; r++) MC[r] = r;
    c->mac->m_Poisson->CG_2FUniformP_2D(p, vin(c, rhs), A, JA, IA, M, MC, MR, c->mac->m_BC, rows, maxiter);
    vout(c, p, ps);
}
void ref_mac_bicgstab(void *h, double *ps, const double *rhs, const double *a, const int *ia, const int *ja,
                      int rows, const double *mdiag, int maxiter) {
    RefCtx *c = static_cast<RefCtx *>(h);
    std::vector<double> p = vin(c, ps);
    const int nnz = ia[rows];
    std::vector<double> A(a, a + nnz), M(mdiag, mdiag + rows);
    std::vector<MKL_INT> IA(ia, ia + rows + 1), JA(ja, ja + nnz), MR(rows + 1), MC(rows);
    for (int r = 0; r <= rows; r++) MR[r] = r;
    for (int r = 0; r < rows; r++) MC[r] = r;
    c->mac->m_Poisson->BiCGStab_2FUniform_2D(p, vin(c, rhs), A, JA, IA, M, MC, MR, c->mac->m_BC, rows, maxiter);
    vout(c, p, ps);
}
void ref_mac_update_vel(void *h, const double *uhat, const double *vhat, const double *ps, const double *ls,
                        const double *lsB, const double *H) {
    RefCtx *c = static_cast<RefCtx *>(h);
    c->mac->UpdateVel(c->mac->m_u, c->mac->m_v, vin(c, uhat), vin(c, vhat), vin(c, ps), vin(c, ls), vin(c, lsB),
                      vin(c, H));
}
double ref_mac_update_dt(void *h, const double *u, const double *v) {
    RefCtx *c = static_cast<RefCtx *>(h);
    return c->mac->UpdateDt(vin(c, u), vin(c, v));
}
}
