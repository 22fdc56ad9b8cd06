// MACSolver2D on the B200 (see mac2d.h).  The session carries the solver's
// physical constants (kRe, kWe, kFr passed as given), its boundary object and
// grid; every numerical method runs through the asd2g C ABI.
#include "mac2d.h"

#include <cstdio>
#include <string>

#include "asd2g.h"
#include "session.h"

using asd2g_dropin::report;
using asd2g_dropin::SessionCache;
using asd2g_dropin::write_zone;

MACSolver2D::MACSolver2D(double Re, double We, double Fr, GAXISENUM2D GAxis, double L, double U, double sigma,
                         double densityRatio, double viscosityRatio, double rhoH, double muH, int nx, int ny,
                         double baseX, double baseY, double lenX, double lenY, TIMEORDERENUM timeOrder, double cfl,
                         double maxtime, int maxIter, int niterskip, int num_bc_grid, bool writeVTK)
    : kNx(nx), kNy(ny), kNumBCGrid(num_bc_grid),
      kArrSize(static_cast<int64_t>(nx + 2 * num_bc_grid) * static_cast<int64_t>(ny + 2 * num_bc_grid)),
      kBaseX(baseX), kBaseY(baseY), kLenX(lenX), kLenY(lenY), kDx(lenX / static_cast<double>(nx)),
      kDy(lenY / static_cast<double>(ny)), kRe(Re), kWe(We), kFr(Fr), kLScale(L), kUScale(U), kSigma(sigma),
      kG(Fr * L / (U * U)), kMuScale((We * sigma / (L * U * U)) * L * U / Re), kRhoScale(We * sigma / (L * U * U)),
      kRhoH(rhoH), kRhoL(rhoH * densityRatio), kRhoRatio(densityRatio), kMuH(muH), kMuL(muH * viscosityRatio),
      kMuRatio(viscosityRatio), kMaxIter(maxIter), kNIterSkip(niterskip), kTimeOrder(timeOrder), kCFL(cfl),
      kMaxTime(maxtime), kWriteVTK(writeVTK), m_PoissonSolverType(POISSONTYPE::CG), m_PLTType(PLTTYPE::NONE),
      kGAxis(GAxis), m_iter(0), m_dt(std::min(0.005, cfl * std::min(lenX / nx, lenY / ny) / U)), m_curTime(0.0),
      m_cache(new SessionCache()) {}

MACSolver2D::MACSolver2D(double rhoH, double rhoL, double muH, double muL, double gConstant, GAXISENUM2D GAxis,
                         double L, double U, double sigma, int nx, int ny, double baseX, double baseY, double lenX,
                         double lenY, TIMEORDERENUM timeOrder, double cfl, double maxtime, int maxIter,
                         int niterskip, int num_bc_grid, bool writeVTK)
    : kNx(nx), kNy(ny), kNumBCGrid(num_bc_grid),
      kArrSize(static_cast<int64_t>(nx + 2 * num_bc_grid) * static_cast<int64_t>(ny + 2 * num_bc_grid)),
      kBaseX(baseX), kBaseY(baseY), kLenX(lenX), kLenY(lenY), kDx(lenX / static_cast<double>(nx)),
      kDy(lenY / static_cast<double>(ny)), kRe(rhoH * L * U / muH), kWe(rhoH * L * U * U / sigma),
      kFr(U * U / (gConstant * L)), kLScale(L), kUScale(U), kSigma(sigma), kG(gConstant), kMuScale(muH),
      kRhoScale(rhoH), kRhoH(rhoH), kRhoL(rhoL), kRhoRatio(rhoL / rhoH), kMuH(muH), kMuL(muL), kMuRatio(muL / muH),
      kMaxIter(maxIter), kNIterSkip(niterskip), kTimeOrder(timeOrder), kCFL(cfl), kMaxTime(maxtime),
      kWriteVTK(writeVTK), m_PoissonSolverType(POISSONTYPE::CG), m_PLTType(PLTTYPE::NONE), kGAxis(GAxis), m_iter(0),
      m_dt(std::min(0.005, cfl * std::min(lenX / nx, lenY / ny) / U)), m_curTime(0.0),
      m_cache(new SessionCache()) {}

MACSolver2D::~MACSolver2D() {
    if (m_BC) m_BC.reset();
}

int MACSolver2D::AllocateVariables() {
    for (std::vector<double> *a : {&m_u, &m_v, &m_rho, &m_kappa, &m_mu, &m_ps, &m_p, &m_J11, &m_J12, &m_J21, &m_J22,
                                   &m_nx, &m_ny, &m_t1x, &m_t1y, &m_t1z, &m_t2x, &m_t2y, &m_t2z})
        *a = std::vector<double>(kArrSize, 0);
    return 0;
}

asd2g_session *MACSolver2D::session() {
    if (!m_BC) {
        std::fprintf(stderr, "MACSolver2D: boundary conditions not set (SetBC_U/V/P_2D)\n");
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
    asd2g_dropin::params_from_bc(*m_BC, p);
    p.rho_h = kRhoH;
    p.rho_l = kRhoL;
    p.mu_h = kMuH;
    p.mu_l = kMuL;
    p.sigma = kSigma;
    p.gravity = kG;
    p.g_axis = static_cast<int>(kGAxis);
    p.time_order = static_cast<int>(kTimeOrder);
    p.cfl = kCFL;
    p.numbers_given = 1;
    p.re = kRe;
    p.we = kWe;
    p.fr = kFr;
    return m_cache->get(p);
}

std::vector<double> MACSolver2D::UpdateHeavisideFunc(const std::vector<double> &ls) {
    std::vector<double> H(kArrSize, 0.0);
    asd2g_session *s = session();
    if (!s) return H;
    m_cache->up(ASD2G_LS, ls);
    report(asd2g_heaviside(s), "UpdateHeavisideFunc");
    m_cache->down(ASD2G_H, H);
    return H;
}

std::vector<double> MACSolver2D::UpdateSmoothHeavisideFunc(const std::vector<double> &ls) {
    std::vector<double> HS(kArrSize, 0.0);
    asd2g_session *s = session();
    if (!s) return HS;
    m_cache->up(ASD2G_LS, ls);
    report(asd2g_heaviside(s), "UpdateSmoothHeavisideFunc");
    m_cache->down(ASD2G_HS, HS);
    return HS;
}

int MACSolver2D::UpdateNTK(const std::shared_ptr<LevelSetSolver2D> &LSolver, const std::vector<double> &ls,
                           std::tuple<std::vector<double> &, std::vector<double> &> normalVec,
                           std::tuple<std::vector<double> &, std::vector<double> &, std::vector<double> &> t1Vec,
                           std::tuple<std::vector<double> &, std::vector<double> &, std::vector<double> &> t2Vec,
                           std::vector<double> &kappa) {
    (void)LSolver, (void)t1Vec, (void)t2Vec, (void)kappa;  // the reference leaves these untouched
    asd2g_session *s = session();
    if (!s) return -1;
    m_cache->up(ASD2G_W0, ls);
    m_cache->up(ASD2G_W1, std::get<0>(normalVec));
    m_cache->up(ASD2G_W2, std::get<1>(normalVec));
    const int rc = report(asd2g_update_ntk(s, ASD2G_W0, ASD2G_W1, ASD2G_W2), "UpdateNTK");
    m_cache->down(ASD2G_W1, std::get<0>(normalVec));
    m_cache->down(ASD2G_W2, std::get<1>(normalVec));
    return rc < 0 ? rc : 0;
}

int MACSolver2D::UpdateKappa(const std::vector<double> &ls) {
    asd2g_session *s = session();
    if (!s) return -1;
    if ((int64_t)m_kappa.size() != kArrSize) m_kappa.assign(kArrSize, 0.0);
    m_cache->up(ASD2G_LS, ls);
    m_cache->up(ASD2G_KAPPA, m_kappa);
    const int rc = report(asd2g_kappa(s), "UpdateKappa");
    m_cache->down(ASD2G_KAPPA, m_kappa);
    return rc < 0 ? rc : 0;
}

// momentum right-hand sides: one device pass computes U and V together
static void mom_pair(asd2g_dropin::SessionCache &c, asd2g_session *s, int which, const std::vector<double> *ls,
                     const std::vector<double> &u, const std::vector<double> &v, const std::vector<double> *H,
                     std::vector<double> &fu, std::vector<double> &fv, const char *what) {
    c.up(ASD2G_U, u);
    c.up(ASD2G_V, v);
    if (ls) c.up(ASD2G_LS, *ls);
    if (H) c.up(ASD2G_HS, *H);
    int rc;
    if (which == 0) rc = asd2g_convection(s, ASD2G_U, ASD2G_V, ASD2G_W0, ASD2G_W1);
    else if (which == 1) rc = asd2g_viscosity(s, ASD2G_U, ASD2G_V, ASD2G_LS, ASD2G_HS, ASD2G_W0, ASD2G_W1);
    else rc = asd2g_momentum_rhs(s, ASD2G_LS, ASD2G_U, ASD2G_V, ASD2G_HS, ASD2G_W0, ASD2G_W1);
    report(rc, what);
    c.down(ASD2G_W0, fu);
    c.down(ASD2G_W1, fv);
}

std::vector<double> MACSolver2D::UpdateFU(const std::shared_ptr<LevelSetSolver2D> &, const std::vector<double> &ls,
                                          const std::vector<double> &u, const std::vector<double> &v,
                                          const std::vector<double> &H) {
    std::vector<double> fu(kArrSize, 0.0), fv(kArrSize, 0.0);
    if (asd2g_session *s = session()) mom_pair(*m_cache, s, 2, &ls, u, v, &H, fu, fv, "UpdateFU");
    return fu;
}

std::vector<double> MACSolver2D::UpdateFV(const std::shared_ptr<LevelSetSolver2D> &, const std::vector<double> &ls,
                                          const std::vector<double> &u, const std::vector<double> &v,
                                          const std::vector<double> &H) {
    std::vector<double> fu(kArrSize, 0.0), fv(kArrSize, 0.0);
    if (asd2g_session *s = session()) mom_pair(*m_cache, s, 2, &ls, u, v, &H, fu, fv, "UpdateFV");
    return fv;
}

std::vector<double> MACSolver2D::AddConvectionFU(const std::vector<double> &u, const std::vector<double> &v) {
    std::vector<double> a(kArrSize, 0.0), b(kArrSize, 0.0);
    if (asd2g_session *s = session()) mom_pair(*m_cache, s, 0, nullptr, u, v, nullptr, a, b, "AddConvectionFU");
    return a;
}

std::vector<double> MACSolver2D::AddConvectionFV(const std::vector<double> &u, const std::vector<double> &v) {
    std::vector<double> a(kArrSize, 0.0), b(kArrSize, 0.0);
    if (asd2g_session *s = session()) mom_pair(*m_cache, s, 0, nullptr, u, v, nullptr, a, b, "AddConvectionFV");
    return b;
}

int MACSolver2D::UnitHJWENO5(const std::vector<double> &F, std::vector<double> &FP, std::vector<double> &FM,
                             const double d, const int n) {
    asd2g_session *s = session();
    if (!s) return -1;
    std::vector<double> fp(n + 2 * kNumBCGrid), fm(n + 2 * kNumBCGrid);
    const int rc = report(asd2g_weno5_line(s, F.data(), fp.data(), fm.data(), d, n), "UnitHJWENO5");
    if (rc < 0) return rc;
    for (int i = kNumBCGrid; i < n + kNumBCGrid; i++) {
        FP[i] = fp[i];
        FM[i] = fm[i];
    }
    return 0;
}

std::vector<double> MACSolver2D::AddViscosityFU(const std::vector<double> &u, const std::vector<double> &v,
                                                const std::vector<double> &ls, const std::vector<double> &H) {
    std::vector<double> a(kArrSize, 0.0), b(kArrSize, 0.0);
    if (asd2g_session *s = session()) mom_pair(*m_cache, s, 1, &ls, u, v, &H, a, b, "AddViscosityFU");
    return a;
}

std::vector<double> MACSolver2D::AddViscosityFV(const std::vector<double> &u, const std::vector<double> &v,
                                                const std::vector<double> &ls, const std::vector<double> &H) {
    std::vector<double> a(kArrSize, 0.0), b(kArrSize, 0.0);
    if (asd2g_session *s = session()) mom_pair(*m_cache, s, 1, &ls, u, v, &H, a, b, "AddViscosityFV");
    return b;
}

// Constant gravity sources (mac2d.cpp:1043-1079): -kG on the U (V) interior
// faces when the axis is X (Y) and kFr is finite; a constant fill.
std::vector<double> MACSolver2D::AddGravityFU() {
    std::vector<double> g(kArrSize, 0.0);
    if ((kFr != 0 || kG != 0.0) && !std::isnan(kFr) && !std::isinf(kFr) && kGAxis == GAXISENUM2D::X)
        for (int i = kNumBCGrid + 1; i < kNx + kNumBCGrid; i++)
            for (int j = kNumBCGrid; j < kNy + kNumBCGrid; j++) g[idx(i, j)] = -kG;
    return g;
}

std::vector<double> MACSolver2D::AddGravityFV() {
    std::vector<double> g(kArrSize, 0.0);
    if ((kFr != 0 || kG != 0.0) && !std::isnan(kFr) && !std::isinf(kFr) && kGAxis == GAXISENUM2D::Y)
        for (int i = kNumBCGrid; i < kNx + kNumBCGrid; i++)
            for (int j = kNumBCGrid + 1; j < kNy + kNumBCGrid; j++) g[idx(i, j)] = -kG;
    return g;
}

int MACSolver2D::GetIntermediateVel(const std::shared_ptr<LevelSetSolver2D> &, const std::vector<double> &ls,
                                    const std::vector<double> &u, const std::vector<double> &v,
                                    std::vector<double> &uhat, std::vector<double> &vhat,
                                    const std::vector<double> &H) {
    asd2g_session *s = session();
    if (!s) return -1;
    m_cache->up(ASD2G_LS, ls);
    m_cache->up(ASD2G_U, u);
    m_cache->up(ASD2G_V, v);
    m_cache->up(ASD2G_UHAT, uhat);
    m_cache->up(ASD2G_VHAT, vhat);
    m_cache->up(ASD2G_HS, H);
    const int rc = report(asd2g_intermediate_vel(s, m_dt, ASD2G_HS), "GetIntermediateVel");
    m_cache->down(ASD2G_UHAT, uhat);
    m_cache->down(ASD2G_VHAT, vhat);
    return rc < 0 ? rc : 0;
}

int MACSolver2D::SetPoissonSolver(POISSONTYPE type) {
    m_PoissonSolverType = type;
    if (!m_Poisson) m_Poisson = std::make_shared<PoissonSolver2D>(kNx, kNy, kNumBCGrid);
    return 0;
}

// GFM assembly + solve on the device (mac2d.cpp:1249-1727).  The operator is
// the reference's, with its all-Neumann pin applied consistently (cell 0 held
// at 0); the iteration is the reference's own CG (poisson2d.cpp:285-400) or
// BiCGStab (:403-575), stopping at its ||r||/||b|| <= 1e-6 or maxiter.
int MACSolver2D::SolvePoisson(std::vector<double> &ps, const std::vector<double> &div, const std::vector<double> &ls,
                              const std::vector<double> &lsB, const std::vector<double> &u,
                              const std::vector<double> &v, const std::vector<double> &H, const int maxiter) {
    (void)lsB, (void)u, (void)v;
    if (!m_Poisson) perror("Solver method for Poisson equations are not set. Please add SetPoissonSolver Method to running code");
    int solver;
    if (m_PoissonSolverType == POISSONTYPE::CG) solver = ASD2G_SOLVER_PCG_REFERENCE;
    else if (m_PoissonSolverType == POISSONTYPE::BICGSTAB) solver = ASD2G_SOLVER_BICGSTAB_REFERENCE;
    else {
        std::fprintf(stderr, "MACSolver2D::SolvePoisson: only POISSONTYPE::CG and ::BICGSTAB are provided\n");
        return -1;
    }
    asd2g_session *s = session();
    if (!s) return -1;
    if ((int64_t)m_kappa.size() != kArrSize) m_kappa.assign(kArrSize, 0.0);
    if ((int64_t)m_p.size() != kArrSize) m_p.assign(kArrSize, 0.0);
    m_cache->up(ASD2G_LS, ls);
    m_cache->up(ASD2G_H, H);
    m_cache->up(ASD2G_DIV, div);
    m_cache->up(ASD2G_KAPPA, m_kappa);
    m_cache->up(ASD2G_P, m_p);
    const bool recompute = kWe != 0.0 && !std::isnan(kWe) && !std::isinf(kWe);
    if (report(asd2g_assemble_gfm(s, m_dt, recompute ? 1 : 0), "GFM assembly") < 0) return -1;
    int iters = 0;
    double res = 0.0;
    const int rc = report(asd2g_solve_pressure(s, solver, 1.0e-6, maxiter, m_dt, &iters, &res), "SolvePoisson");
    std::cout << (solver == ASD2G_SOLVER_PCG_REFERENCE ? "CG : " : "BiCG : ") << iters << " " << maxiter << " Err : " << res
              << std::endl;
    m_cache->down(ASD2G_PS, ps);
    m_cache->down(ASD2G_P, m_p);
    m_cache->down(ASD2G_KAPPA, m_kappa);
    return rc < 0 ? rc : 0;
}

std::vector<double> MACSolver2D::GetDivergence(const std::vector<double> &u, const std::vector<double> &v) {
    std::vector<double> div(kArrSize, 0.0);
    asd2g_session *s = session();
    if (!s) return div;
    m_cache->up(ASD2G_U, u);
    m_cache->up(ASD2G_V, v);
    report(asd2g_divergence(s, ASD2G_U, ASD2G_V, ASD2G_DIV), "GetDivergence");
    m_cache->down(ASD2G_DIV, div);
    return div;
}

int MACSolver2D::UpdateVel(std::vector<double> &u, std::vector<double> &v, const std::vector<double> &us,
                           const std::vector<double> &vs, const std::vector<double> &ps,
                           const std::vector<double> &ls, const std::vector<double> &lsB,
                           const std::vector<double> &H) {
    (void)lsB;
    asd2g_session *s = session();
    if (!s) return -1;
    m_cache->up(ASD2G_U, u);
    m_cache->up(ASD2G_V, v);
    m_cache->up(ASD2G_UHAT, us);
    m_cache->up(ASD2G_VHAT, vs);
    m_cache->up(ASD2G_PS, ps);
    m_cache->up(ASD2G_LS, ls);
    m_cache->up(ASD2G_H, H);
    m_cache->up(ASD2G_KAPPA, m_kappa);
    const int rc = report(asd2g_update_vel(s, m_dt), "UpdateVel");
    m_cache->down(ASD2G_U, u);
    m_cache->down(ASD2G_V, v);
    return rc < 0 ? rc : 0;
}

double MACSolver2D::UpdateDt(const std::vector<double> &u, const std::vector<double> &v) {
    asd2g_session *s = session();
    if (!s) return std::numeric_limits<double>::quiet_NaN();
    m_cache->up(ASD2G_U, u);
    m_cache->up(ASD2G_V, v);
    double dt = 0.0;
    report(asd2g_update_dt(s, &dt), "UpdateDt");
    if (std::isnan(dt) || std::isinf(dt)) std::cout << "dt nan/inf error" << std::endl;
    return dt;
}

int MACSolver2D::SetBC_U_2D(std::string W, std::string E, std::string S, std::string N) {
    if (!m_BC) m_BC = std::make_shared<BoundaryCondition2D>(kNx, kNy, kNumBCGrid);
    return m_BC->SetBC_U_2D(W, E, S, N);
}
int MACSolver2D::SetBC_V_2D(std::string W, std::string E, std::string S, std::string N) {
    if (!m_BC) m_BC = std::make_shared<BoundaryCondition2D>(kNx, kNy, kNumBCGrid);
    return m_BC->SetBC_V_2D(W, E, S, N);
}
int MACSolver2D::SetBC_P_2D(std::string W, std::string E, std::string S, std::string N) {
    if (!m_BC) m_BC = std::make_shared<BoundaryCondition2D>(kNx, kNy, kNumBCGrid);
    return m_BC->SetBC_P_2D(W, E, S, N);
}
int MACSolver2D::ApplyBC_U_2D(std::vector<double> &arr) { return m_BC->ApplyBC_U_2D(arr); }
int MACSolver2D::ApplyBC_V_2D(std::vector<double> &arr) { return m_BC->ApplyBC_V_2D(arr); }
int MACSolver2D::ApplyBC_P_2D(std::vector<double> &arr) { return m_BC->ApplyBC_P_2D(arr); }
void MACSolver2D::SetBCConstantUW(double c) { m_BC->SetBCConstantUW(c); }
void MACSolver2D::SetBCConstantUE(double c) { m_BC->SetBCConstantUE(c); }
void MACSolver2D::SetBCConstantUS(double c) { m_BC->SetBCConstantUS(c); }
void MACSolver2D::SetBCConstantUN(double c) { m_BC->SetBCConstantUN(c); }
void MACSolver2D::SetBCConstantVW(double c) { m_BC->SetBCConstantVW(c); }
void MACSolver2D::SetBCConstantVE(double c) { m_BC->SetBCConstantVE(c); }
void MACSolver2D::SetBCConstantVS(double c) { m_BC->SetBCConstantVS(c); }
void MACSolver2D::SetBCConstantVN(double c) { m_BC->SetBCConstantVN(c); }
void MACSolver2D::SetBCConstantPW(double c) { m_BC->SetBCConstantPW(c); }
void MACSolver2D::SetBCConstantPE(double c) { m_BC->SetBCConstantPE(c); }
void MACSolver2D::SetBCConstantPS(double c) { m_BC->SetBCConstantPS(c); }
void MACSolver2D::SetBCConstantPN(double c) { m_BC->SetBCConstantPN(c); }

int MACSolver2D::sign(const double &val) { return (val > 0) - (val < 0); }

int MACSolver2D::SetPLTType(PLTTYPE type) {
    m_PLTType = type;
    return 0;
}


// Tecplot ASCII output (mac2d.cpp:1990-2063): <vel>_ASCII.plt with X, Y, the
// face velocities averaged to the cell centres, LS and PS; <div>_ASCII.plt
// with X, Y, LS, the divergence of (u, v) and PS.  Both files are created
// with their header when m_iter is 0 and get one zone per call.  The binary
// .szplt output needs the closed TecIO library and is not written.
int MACSolver2D::OutRes(const int iter, const double curTime, const std::string fname_vel_base,
                        const std::string fname_div_base, const std::vector<double> &u, const std::vector<double> &v,
                        const std::vector<double> &ps, const std::vector<double> &ls) {
    if (m_PLTType != PLTTYPE::ASCII && m_PLTType != PLTTYPE::BOTH) return 0;
    const int nbc = kNumBCGrid;
    const int64_t stride = kNy + 2 * nbc;
    std::vector<double> uc(kArrSize, 0.0), vc(kArrSize, 0.0);
    for (int i = nbc; i < kNx + nbc; i++)
        for (int j = nbc; j < kNy + nbc; j++) {
            const int64_t k = j + stride * i;
            uc[k] = (u[k] + u[k + stride]) * 0.5;
            vc[k] = (v[k] + v[k + 1]) * 0.5;
        }
    const std::vector<double> div = GetDivergence(u, v);
    const bool header = m_iter == 0;
    const bool ok =
        write_zone(fname_vel_base + "_ASCII.plt", header, "VEL", "\"X\", \"Y\", \"U\", \"V\", \"LS\", \"PS\"", iter,
                   curTime, kNx, kNy, nbc, kBaseX, kBaseY, kDx, kDy, {&uc, &vc, &ls, &ps}) &&
        write_zone(fname_div_base + "_ASCII.plt", header, "DIV", "\"X\", \"Y\", \"LS\", \"DIV\", \"PS\"", iter,
                   curTime, kNx, kNy, nbc, kBaseX, kBaseY, kDx, kDy, {&ls, &div, &ps});
    if (!ok) perror("MACSolver2D::OutRes");
    return 0;
}

int MACSolver2D::OutResClose() { return 0; }
