// LevelSetSolver2D on the B200 (see levelset2d.h).  Each method uploads its
// operands into a session, runs the corresponding asd2g entry point and
// downloads the results; the numerical work is all on the GPU.
#include "levelset2d.h"

#include <cstring>
#include <limits>

#include "asd2g.h"
#include "session.h"

using asd2g_dropin::report;
using asd2g_dropin::SessionCache;

LevelSetSolver2D::LevelSetSolver2D(int nx, int ny, int num_bc_grid, double baseX, double baseY, double dx, double dy)
    : LevelSetSolver2D(nx, ny, num_bc_grid, baseX, baseY, dx, dy, 1.5 * (1.5 * std::min(dx, dy))) {}

LevelSetSolver2D::LevelSetSolver2D(int nx, int ny, int num_bc_grid, double baseX, double baseY, double dx, double dy,
                                   double maxTime)
    : kEps(std::min(dx, dy)), kThickness(1.5 * std::min(dx, dy)), kMaxATime(maxTime), kNx(nx), kNy(ny),
      kNumBCGrid(num_bc_grid), kENOSpatialOrder(2),
      kArrSize(static_cast<int64_t>(nx + 2 * num_bc_grid) * static_cast<int64_t>(ny + 2 * num_bc_grid)),
      kBaseX(baseX), kBaseY(baseY), kDx(dx), kDy(dy), m_atime(0.0), kAdt(std::min(dx, dy) * 0.5),
      m_cache(new SessionCache()) {}

LevelSetSolver2D::~LevelSetSolver2D() = default;

asd2g_session *LevelSetSolver2D::session() {
    if (!m_BC) {
        std::fprintf(stderr, "LevelSetSolver2D: boundary conditions not set (SetBC_P_2D)\n");
        return nullptr;
    }
    asd2g_params p{};
    p.nx = kNx;
    p.ny = kNy;
    p.nbc = kNumBCGrid;
    p.base_x = kBaseX;
    p.base_y = kBaseY;
    p.dx = kDx;
    p.dy = kDy;
    p.rho_h = p.rho_l = 1.0;
    p.mu_h = p.mu_l = 1.0;
    p.cfl = 1.0;
    p.time_order = 2;
    p.ls_max_atime = kMaxATime;
    asd2g_dropin::params_from_bc(*m_BC, p);
    return m_cache->get(p);
}

std::vector<double> LevelSetSolver2D::UpdateHeavisideFuncDeriv(const std::vector<double> &ls) {
    std::vector<double> out(kArrSize, 0.0);
    asd2g_session *s = session();
    if (!s) return out;
    m_cache->up(ASD2G_W0, ls);
    report(asd2g_heaviside_deriv(s, ASD2G_W0, ASD2G_W1), "UpdateHeavisideFuncDeriv");
    m_cache->down(ASD2G_W1, out);
    return out;
}

int LevelSetSolver2D::Solve_LevelSet_2D(std::vector<double> &ls, const std::vector<double> &u,
                                        const std::vector<double> &v, double dt) {
    asd2g_session *s = session();
    if (!s) return -1;
    m_cache->up(ASD2G_LS, ls);
    m_cache->up(ASD2G_U, u);
    m_cache->up(ASD2G_V, v);
    const int rc = report(asd2g_ls_advect(s, dt), "Solve_LevelSet_2D");
    m_cache->down(ASD2G_LS, ls);
    return rc < 0 ? rc : 0;
}

int LevelSetSolver2D::reinit(std::vector<double> &ls, int mode) {
    asd2g_session *s = session();
    if (!s) return -1;
    m_cache->up(ASD2G_LS, ls);
    const int rc = report(asd2g_reinit(s, mode), "reinitialisation");
    m_cache->down(ASD2G_LS, ls);
    // the pseudo-time the reference loop ends at
    double t = 0.0;
    const double tmax = mode == ASD2G_REINIT_FIRSTTIME ? std::max(kDx * kNx, kDy * kNy) : kMaxATime;
    while (t < tmax) t += kAdt;
    m_atime = t;
    return rc < 0 ? rc : 0;
}

int LevelSetSolver2D::Reinit_Original_2D(std::vector<double> &ls) { return reinit(ls, ASD2G_REINIT_ORIGINAL); }
int LevelSetSolver2D::Reinit_Sussman_2D(std::vector<double> &ls) { return reinit(ls, ASD2G_REINIT_SUSSMAN); }
int LevelSetSolver2D::FirstTimeOnlyReinit_Sussman_2D(std::vector<double> &ls) {
    return reinit(ls, ASD2G_REINIT_FIRSTTIME);
}
int LevelSetSolver2D::Reinit_MinRK2_2D(std::vector<double> &ls) { return reinit(ls, ASD2G_REINIT_MINRK2); }
int LevelSetSolver2D::Reinit_MinRK2_Sussman_2D(std::vector<double> &ls) {
    return reinit(ls, ASD2G_REINIT_MINRK2_SUSSMAN);
}

std::vector<double> LevelSetSolver2D::GetSussmanReinitConstraint(const std::vector<double> &ls,
                                                                 const std::vector<double> &lsInit,
                                                                 const std::vector<double> &heavisideDeriv) {
    std::vector<double> out(kArrSize, 0.0);
    asd2g_session *s = session();
    if (!s) return out;
    m_cache->up(ASD2G_W0, ls);
    m_cache->up(ASD2G_W1, lsInit);
    m_cache->up(ASD2G_W2, heavisideDeriv);
    report(asd2g_sussman_constraint(s, ASD2G_W0, ASD2G_W1, ASD2G_W2, ASD2G_W3), "GetSussmanReinitConstraint");
    m_cache->down(ASD2G_W3, out);
    return out;
}

int LevelSetSolver2D::sign(const double &val) { return (val > 0) - (val < 0); }

double LevelSetSolver2D::MinAbs(const double &a, const double &b) { return std::fabs(a) < std::fabs(b) ? a : b; }

double LevelSetSolver2D::MinMod(const double &a, const double &b) {
    if ((std::fabs(a) <= std::fabs(b)) && (a * b > 0)) return a;
    if ((std::fabs(a) > std::fabs(b)) && (a * b > 0)) return b;
    if (a * b <= 0) return 0.0;
    return std::numeric_limits<double>::quiet_NaN();
}

std::vector<int> LevelSetSolver2D::GetSignedLSNormalized(const std::vector<double> &v) {
    // levelset2d.cpp:895-912 (a host-side utility, unused by the solvers)
    std::vector<int> r(v.size());
    for (int i = 0; i < kNx + 2 * kNumBCGrid; i++)
        for (int j = 0; j < kNy + 2 * kNumBCGrid; j++) {
            const double a = v[idx(i, j)];
            if (std::fabs(a) <= kEps) r[idx(i, j)] = static_cast<int>(2.0 * ((0.5 + cos(M_PI * a / kEps)) / kEps - 0.5));
            else if (a > 0) r[idx(i, j)] = 1;
            else if (a < 0) r[idx(i, j)] = -1;
        }
    return r;
}

std::vector<double> LevelSetSolver2D::GetSmoothedSignFunc(const std::vector<double> &ls) {
    std::vector<double> out(ls.size(), 0.0);
    asd2g_session *s = session();
    if (!s) return out;
    m_cache->up(ASD2G_W0, ls);
    report(asd2g_smoothed_sign(s, ASD2G_W0, ASD2G_W1), "GetSmoothedSignFunc");
    m_cache->down(ASD2G_W1, out);
    return out;
}

std::vector<double> LevelSetSolver2D::HJWENO5_LS_2D(std::vector<double> &ls, const std::vector<double> &u,
                                                    const std::vector<double> &v) {
    std::vector<double> out(kArrSize, 0.0);
    asd2g_session *s = session();
    if (!s) return out;
    m_cache->up(ASD2G_LS, ls);
    m_cache->up(ASD2G_W0, u);
    m_cache->up(ASD2G_W1, v);
    report(asd2g_ls_weno_rhs(s, ASD2G_LS, ASD2G_W0, ASD2G_W1, ASD2G_W2), "HJWENO5_LS_2D");
    m_cache->down(ASD2G_W2, out);
    m_cache->down(ASD2G_LS, ls);  // the reference fills ls's ghosts first
    return out;
}

int LevelSetSolver2D::UnitHJWENO5(const std::vector<double> &F, std::vector<double> &FP, std::vector<double> &FM,
                                  const double d, const int n) {
    asd2g_session *s = session();
    if (!s) return -1;
    std::vector<double> fp(n + 2 * kNumBCGrid), fm(n + 2 * kNumBCGrid);
    const int rc = report(asd2g_weno5_line(s, F.data(), fp.data(), fm.data(), d, n), "UnitHJWENO5");
    if (rc < 0) return rc;
    for (int i = kNumBCGrid; i < n + kNumBCGrid; i++) {  // only the points the reference writes
        FP[i] = fp[i];
        FM[i] = fm[i];
    }
    return 0;
}

#define ASD2G_ABSGRAD(NAME, CALL)                                                                             \
    std::vector<double> LevelSetSolver2D::NAME(const std::vector<double> &ls, const std::vector<double> &lsInit) { \
        std::vector<double> out(kArrSize, 0.0);                                                              \
        asd2g_session *s = session();                                                                        \
        if (!s) return out;                                                                                  \
        m_cache->up(ASD2G_W0, ls);                                                                           \
        m_cache->up(ASD2G_W1, lsInit);                                                                       \
        report(CALL(s, ASD2G_W0, ASD2G_W1, ASD2G_W2), #NAME);                                                \
        m_cache->down(ASD2G_W2, out);                                                                        \
        return out;                                                                                          \
    }
ASD2G_ABSGRAD(HJWENO5_DerivAbsLS_2D, asd2g_weno_absgrad)
ASD2G_ABSGRAD(ENO_DerivAbsLS_2D, asd2g_eno)
ASD2G_ABSGRAD(SubcellENO_Min_DerivAbsLS_2D, asd2g_subcell_eno)
#undef ASD2G_ABSGRAD

int LevelSetSolver2D::SetBC_U_2D(std::string W, std::string E, std::string S, std::string N) {
    if (!m_BC) m_BC = std::make_shared<BoundaryCondition2D>(kNx, kNy, kDx, kDy, kNumBCGrid);
    return m_BC->SetBC_U_2D(W, E, S, N);
}
int LevelSetSolver2D::SetBC_V_2D(std::string W, std::string E, std::string S, std::string N) {
    if (!m_BC) m_BC = std::make_shared<BoundaryCondition2D>(kNx, kNy, kDx, kDy, kNumBCGrid);
    return m_BC->SetBC_V_2D(W, E, S, N);
}
int LevelSetSolver2D::SetBC_P_2D(std::string W, std::string E, std::string S, std::string N) {
    if (!m_BC) m_BC = std::make_shared<BoundaryCondition2D>(kNx, kNy, kDx, kDy, kNumBCGrid);
    return m_BC->SetBC_P_2D(W, E, S, N);
}
int LevelSetSolver2D::ApplyBC_U_2D(std::vector<double> &arr) { return m_BC->ApplyBC_U_2D(arr); }
int LevelSetSolver2D::ApplyBC_V_2D(std::vector<double> &arr) { return m_BC->ApplyBC_V_2D(arr); }
int LevelSetSolver2D::ApplyBC_P_2D(std::vector<double> &arr) { return m_BC->ApplyBC_P_2D(arr); }
void LevelSetSolver2D::SetBCConstantUW(double c) { m_BC->SetBCConstantUW(c); }
void LevelSetSolver2D::SetBCConstantUE(double c) { m_BC->SetBCConstantUE(c); }
void LevelSetSolver2D::SetBCConstantUS(double c) { m_BC->SetBCConstantUS(c); }
void LevelSetSolver2D::SetBCConstantUN(double c) { m_BC->SetBCConstantUN(c); }
void LevelSetSolver2D::SetBCConstantVW(double c) { m_BC->SetBCConstantVW(c); }
void LevelSetSolver2D::SetBCConstantVE(double c) { m_BC->SetBCConstantVE(c); }
void LevelSetSolver2D::SetBCConstantVS(double c) { m_BC->SetBCConstantVS(c); }
void LevelSetSolver2D::SetBCConstantVN(double c) { m_BC->SetBCConstantVN(c); }
void LevelSetSolver2D::SetBCConstantPW(double c) { m_BC->SetBCConstantPW(c); }
void LevelSetSolver2D::SetBCConstantPE(double c) { m_BC->SetBCConstantPE(c); }
void LevelSetSolver2D::SetBCConstantPS(double c) { m_BC->SetBCConstantPS(c); }
void LevelSetSolver2D::SetBCConstantPN(double c) { m_BC->SetBCConstantPN(c); }
