// MACSolver2DAxisym on the B200 (see mac2dAxisym.h).  The session carries
// the solver's constants (kRe, kWe, kFr as given), its boundary object and
// the (r, z) grid (x is r, base_x is kBaseR); every numerical method runs
// through the asd2g C ABI.
#include "mac2dAxisym.h"

#include <cstdio>
#include <string>

#include "asd2g.h"
#include "session.h"

using asd2g_dropin::report;
using asd2g_dropin::SessionCache;
using asd2g_dropin::write_zone;

MACSolver2DAxisym::MACSolver2DAxisym(double Re, double We, double Fr, GAXISENUM2DAXISYM GAxis, double L, double U,
                                     double sigma, double densityRatio, double viscosityRatio, double rhoH,
                                     double muH, int nr, int nz, double baseR, double baseZ, double lenR,
                                     double lenZ, double cfl, double maxtime, int maxIter, int niterskip,
                                     int num_bc_grid, bool writeVTK)
    : kNr(nr), kNz(nz), kNumBCGrid(num_bc_grid),
      kArrSize(static_cast<int64_t>(nr + 2 * num_bc_grid) * static_cast<int64_t>(nz + 2 * num_bc_grid)),
      kBaseR(baseR), kBaseZ(baseZ), kLenR(lenR), kLenZ(lenZ), kDr(lenR / static_cast<double>(nr)),
      kDz(lenZ / static_cast<double>(nz)), kRe(Re), kWe(We), kFr(Fr), kLScale(L), kUScale(U), kSigma(sigma),
      kG(Fr * L / (U * U)), kMuScale((We * sigma / (L * U * U)) * L * U / Re), kRhoScale(We * sigma / (L * U * U)),
      kRhoH(rhoH), kRhoL(rhoH * densityRatio), kRhoRatio(densityRatio), kMuH(muH), kMuL(muH * viscosityRatio),
      kMuRatio(viscosityRatio), kMaxIter(maxIter), kNIterSkip(niterskip), kCFL(cfl), kMaxTime(maxtime),
      kWriteVTK(writeVTK), m_PoissonSolverType(POISSONTYPE::CG), m_PLTType(PLTTYPE::NONE), kGAxis(GAxis), m_iter(0),
      m_dt(std::min(0.005, cfl * std::min(lenR / nr, lenZ / nz) / U)), m_curTime(0.0),
      m_cache(new SessionCache()) {}

MACSolver2DAxisym::MACSolver2DAxisym(double rhoH, double rhoL, double muH, double muL, double gConstant,
                                     GAXISENUM2DAXISYM GAxis, double L, double U, double sigma, int nr, int nz,
                                     double baseR, double baseZ, double lenR, double lenZ, double cfl,
                                     double maxtime, int maxIter, int niterskip, int num_bc_grid, bool writeVTK)
    : kNr(nr), kNz(nz), kNumBCGrid(num_bc_grid),
      kArrSize(static_cast<int64_t>(nr + 2 * num_bc_grid) * static_cast<int64_t>(nz + 2 * num_bc_grid)),
      kBaseR(baseR), kBaseZ(baseZ), kLenR(lenR), kLenZ(lenZ), kDr(lenR / static_cast<double>(nr)),
      kDz(lenZ / static_cast<double>(nz)), kRe(rhoH * L * U / muH), kWe(rhoH * L * U * U / sigma),
      kFr(U * U / (gConstant * L)), kLScale(L), kUScale(U), kSigma(sigma), kG(gConstant), kMuScale(muH),
      kRhoScale(rhoH), kRhoH(rhoH), kRhoL(rhoL), kRhoRatio(rhoL / rhoH), kMuH(muH), kMuL(muL), kMuRatio(muL / muH),
      kMaxIter(maxIter), kNIterSkip(niterskip), kCFL(cfl), kMaxTime(maxtime), kWriteVTK(writeVTK),
      m_PoissonSolverType(POISSONTYPE::CG), m_PLTType(PLTTYPE::NONE), kGAxis(GAxis), m_iter(0),
      m_dt(std::min(0.005, cfl * std::min(lenR / nr, lenZ / nz) / U)), m_curTime(0.0),
      m_cache(new SessionCache()) {}

MACSolver2DAxisym::~MACSolver2DAxisym() {
    if (m_BC) m_BC.reset();
}

int MACSolver2DAxisym::AllocateVariables() {
    for (std::vector<double> *a : {&m_u, &m_v, &m_rho, &m_kappa, &m_mu, &m_ps, &m_p, &m_J11, &m_J12, &m_J21, &m_J22,
                                   &m_nr, &m_nz, &m_t1r, &m_t1z, &m_t1t, &m_t2r, &m_t2z, &m_t2t})
        *a = std::vector<double>(kArrSize, 0);
    return 0;
}

asd2g_session *MACSolver2DAxisym::session() {
    if (!m_BC) {
        std::fprintf(stderr, "MACSolver2DAxisym: boundary conditions not set (SetBC_U/V/P_2D)\n");
        return nullptr;
    }
    asd2g_params p{};
    p.nx = kNr;
    p.ny = kNz;
    p.nbc = kNumBCGrid;
    p.base_x = kBaseR;
    p.base_y = kBaseZ;
    p.dx = kDr;
    p.dy = kDz;
    asd2g_dropin::params_from_bc(*m_BC, p);
    p.rho_h = kRhoH;
    p.rho_l = kRhoL;
    p.mu_h = kMuH;
    p.mu_l = kMuL;
    p.sigma = kSigma;
    p.gravity = kG;
    p.g_axis = static_cast<int>(kGAxis);  // R = 0, Z = 1
    p.cfl = kCFL;
    p.numbers_given = 1;
    p.re = kRe;
    p.we = kWe;
    p.fr = kFr;
    return m_cache->get(p);
}

std::vector<double> MACSolver2DAxisym::UpdateHeavisideFunc(const std::vector<double> &ls) {
    std::vector<double> H(kArrSize, 0.0);
    asd2g_session *s = session();
    if (!s) return H;
    m_cache->up(ASD2G_LS, ls);
    report(asd2g_heaviside(s), "UpdateHeavisideFunc");
    m_cache->down(ASD2G_H, H);
    return H;
}

std::vector<double> MACSolver2DAxisym::UpdateSmoothHeavisideFunc(const std::vector<double> &ls) {
    std::vector<double> HS(kArrSize, 0.0);
    asd2g_session *s = session();
    if (!s) return HS;
    m_cache->up(ASD2G_LS, ls);
    report(asd2g_heaviside(s), "UpdateSmoothHeavisideFunc");
    m_cache->down(ASD2G_HS, HS);
    return HS;
}

// The same computation as MACSolver2D::UpdateNTK (mac2dAxisym.cpp:124-219).
int MACSolver2DAxisym::UpdateNTK(const std::shared_ptr<LevelSetSolver2D> &LSolver, const std::vector<double> &ls,
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

int MACSolver2DAxisym::UpdateKappa(const std::vector<double> &ls) {
    asd2g_session *s = session();
    if (!s) return -1;
    if ((int64_t)m_kappa.size() != kArrSize) m_kappa.assign(kArrSize, 0.0);
    m_cache->up(ASD2G_LS, ls);
    m_cache->up(ASD2G_KAPPA, m_kappa);
    const int rc = report(asd2g_axi_kappa(s), "UpdateKappa");
    m_cache->down(ASD2G_KAPPA, m_kappa);
    return rc < 0 ? rc : 0;
}

std::vector<double> MACSolver2DAxisym::GetRHSU(const std::vector<double> &ls, const std::vector<double> &u,
                                               const std::vector<double> &v, const std::vector<double> &H) {
    std::vector<double> out(kArrSize, 0.0);
    asd2g_session *s = session();
    if (!s) return out;
    m_cache->up(ASD2G_LS, ls);
    m_cache->up(ASD2G_U, u);
    m_cache->up(ASD2G_V, v);
    m_cache->up(ASD2G_HS, H);
    report(asd2g_axi_rhs_u(s, m_dt, ASD2G_LS, ASD2G_U, ASD2G_V, ASD2G_HS, ASD2G_W0), "GetRHSU");
    m_cache->down(ASD2G_W0, out);
    return out;
}

std::vector<double> MACSolver2DAxisym::GetRHSV(const std::vector<double> &ls, const std::vector<double> &u,
                                               const std::vector<double> &uhat, const std::vector<double> &v,
                                               const std::vector<double> &H) {
    std::vector<double> out(kArrSize, 0.0);
    asd2g_session *s = session();
    if (!s) return out;
    m_cache->up(ASD2G_LS, ls);
    m_cache->up(ASD2G_U, u);
    m_cache->up(ASD2G_UHAT, uhat);
    m_cache->up(ASD2G_V, v);
    m_cache->up(ASD2G_HS, H);
    report(asd2g_axi_rhs_v(s, m_dt, ASD2G_LS, ASD2G_U, ASD2G_UHAT, ASD2G_V, ASD2G_HS, ASD2G_W0), "GetRHSV");
    m_cache->down(ASD2G_W0, out);
    return out;
}

static void conv_pair(SessionCache &c, asd2g_session *s, const std::vector<double> &u, const std::vector<double> &v,
                      std::vector<double> &cu, std::vector<double> &cv, const char *what) {
    c.up(ASD2G_U, u);
    c.up(ASD2G_V, v);
    report(asd2g_convection(s, ASD2G_U, ASD2G_V, ASD2G_W0, ASD2G_W1), what);
    c.down(ASD2G_W0, cu);
    c.down(ASD2G_W1, cv);
}

std::vector<double> MACSolver2DAxisym::AddConvectionFU(const std::vector<double> &u, const std::vector<double> &v) {
    std::vector<double> a(kArrSize, 0.0), b(kArrSize, 0.0);
    if (asd2g_session *s = session()) conv_pair(*m_cache, s, u, v, a, b, "AddConvectionFU");
    return a;
}

std::vector<double> MACSolver2DAxisym::AddConvectionFV(const std::vector<double> &u, const std::vector<double> &v) {
    std::vector<double> a(kArrSize, 0.0), b(kArrSize, 0.0);
    if (asd2g_session *s = session()) conv_pair(*m_cache, s, u, v, a, b, "AddConvectionFV");
    return b;
}

int MACSolver2DAxisym::UnitHJWENO5(const std::vector<double> &F, std::vector<double> &FP, std::vector<double> &FM,
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

static void visc_pair(SessionCache &c, asd2g_session *s, const std::vector<double> &u, const std::vector<double> &uhat,
                      const std::vector<double> &v, const std::vector<double> &ls, const std::vector<double> &H,
                      std::vector<double> &du, std::vector<double> &dv, const char *what) {
    c.up(ASD2G_LS, ls);
    c.up(ASD2G_U, u);
    c.up(ASD2G_UHAT, uhat);
    c.up(ASD2G_V, v);
    c.up(ASD2G_HS, H);
    report(asd2g_axi_viscosity(s, ASD2G_LS, ASD2G_U, ASD2G_UHAT, ASD2G_V, ASD2G_HS, ASD2G_W0, ASD2G_W1), what);
    c.down(ASD2G_W0, du);
    c.down(ASD2G_W1, dv);
}

std::vector<double> MACSolver2DAxisym::AddExternalViscosityFU(const std::vector<double> &u,
                                                              const std::vector<double> &v,
                                                              const std::vector<double> &ls,
                                                              const std::vector<double> &H) {
    std::vector<double> a(kArrSize, 0.0), b(kArrSize, 0.0);
    if (asd2g_session *s = session()) visc_pair(*m_cache, s, u, u, v, ls, H, a, b, "AddExternalViscosityFU");
    return a;
}

std::vector<double> MACSolver2DAxisym::AddExternalViscosityFV(const std::vector<double> &u,
                                                              const std::vector<double> &uhat,
                                                              const std::vector<double> &v,
                                                              const std::vector<double> &ls,
                                                              const std::vector<double> &H) {
    std::vector<double> a(kArrSize, 0.0), b(kArrSize, 0.0);
    if (asd2g_session *s = session()) visc_pair(*m_cache, s, u, uhat, v, ls, H, a, b, "AddExternalViscosityFV");
    return b;
}

// Constant gravity sources (mac2dAxisym.cpp:912-948): -kG on the U (V)
// interior faces when the axis is R (Z) and kFr is finite.
std::vector<double> MACSolver2DAxisym::AddGravityFU() {
    std::vector<double> g(kArrSize, 0.0);
    if ((kFr != 0 || kG != 0.0) && !std::isnan(kFr) && !std::isinf(kFr) && kGAxis == GAXISENUM2DAXISYM::R)
        for (int i = kNumBCGrid + 1; i < kNr + kNumBCGrid; i++)
            for (int j = kNumBCGrid; j < kNz + kNumBCGrid; j++) g[idx(i, j)] = -kG;
    return g;
}

std::vector<double> MACSolver2DAxisym::AddGravityFV() {
    std::vector<double> g(kArrSize, 0.0);
    if ((kFr != 0 || kG != 0.0) && !std::isnan(kFr) && !std::isinf(kFr) && kGAxis == GAXISENUM2DAXISYM::Z)
        for (int i = kNumBCGrid; i < kNr + kNumBCGrid; i++)
            for (int j = kNumBCGrid + 1; j < kNz + kNumBCGrid; j++) g[idx(i, j)] = -kG;
    return g;
}

static std::vector<double> hat(SessionCache &c, asd2g_session *s, int comp, double dt, int64_t n,
                               const std::vector<double> &ls, const std::vector<double> &rhs,
                               const std::vector<double> &H, const char *what) {
    std::vector<double> out(n, 0.0);
    c.up(ASD2G_LS, ls);
    c.up(ASD2G_W0, rhs);
    c.up(ASD2G_HS, H);
    report(asd2g_axi_hat(s, comp, dt, ASD2G_LS, ASD2G_W0, ASD2G_HS, ASD2G_W1), what);
    c.down(ASD2G_W1, out);
    return out;
}

std::vector<double> MACSolver2DAxisym::GetUHat(const std::vector<double> &ls, const std::vector<double> &u,
                                               const std::vector<double> &rhs, const std::vector<double> &H) {
    (void)u;  // the reference reads only its right side
    asd2g_session *s = session();
    if (!s) return std::vector<double>(kArrSize, 0.0);
    return hat(*m_cache, s, 0, m_dt, kArrSize, ls, rhs, H, "GetUHat");
}

std::vector<double> MACSolver2DAxisym::GetVHat(const std::vector<double> &ls, const std::vector<double> &v,
                                               const std::vector<double> &rhs, const std::vector<double> &H) {
    (void)v;
    asd2g_session *s = session();
    if (!s) return std::vector<double>(kArrSize, 0.0);
    return hat(*m_cache, s, 1, m_dt, kArrSize, ls, rhs, H, "GetVHat");
}

int MACSolver2DAxisym::SetPoissonSolver(POISSONTYPE type) {
    m_PoissonSolverType = type;
    if (!m_Poisson) m_Poisson = std::make_shared<PoissonSolver2D>(kNr, kNz, kNumBCGrid);
    return 0;
}

// The r-weighted GFM assembly + solve on the device (mac2dAxisym.cpp:1488-
// 1978): the reference's own CG (poisson2d.cpp:285-400) or BiCGStab
// (:403-575), stopping at its ||r||/||b|| <= 1e-6 or maxiter.
int MACSolver2DAxisym::SolvePoisson(std::vector<double> &ps, const std::vector<double> &div,
                                    const std::vector<double> &ls, const std::vector<double> &lsB,
                                    const std::vector<double> &u, const std::vector<double> &v,
                                    const std::vector<double> &H, const int maxiter) {
    (void)lsB, (void)u, (void)v;
    if (!m_Poisson) perror("Solver method for Poisson equations are not set. Please add SetPoissonSolver Method to running code");
    int solver;
    if (m_PoissonSolverType == POISSONTYPE::CG) solver = ASD2G_SOLVER_PCG_REFERENCE;
    else if (m_PoissonSolverType == POISSONTYPE::BICGSTAB) solver = ASD2G_SOLVER_BICGSTAB_REFERENCE;
    else {
        std::fprintf(stderr, "MACSolver2DAxisym::SolvePoisson: only POISSONTYPE::CG and ::BICGSTAB are provided\n");
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
    if (report(asd2g_axi_assemble(s, m_dt, recompute ? 1 : 0), "axisymmetric GFM assembly") < 0) return -1;
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

static std::vector<double> axi_div(SessionCache &c, asd2g_session *s, int64_t n, const std::vector<double> &u,
                                   const std::vector<double> &v, int for_poisson, const char *what) {
    std::vector<double> div(n, 0.0);
    c.up(ASD2G_U, u);
    c.up(ASD2G_V, v);
    report(asd2g_axi_divergence(s, ASD2G_U, ASD2G_V, ASD2G_DIV, for_poisson), what);
    c.down(ASD2G_DIV, div);
    return div;
}

std::vector<double> MACSolver2DAxisym::GetDivergence4Poisson(const std::vector<double> &u,
                                                             const std::vector<double> &v) {
    asd2g_session *s = session();
    if (!s) return std::vector<double>(kArrSize, 0.0);
    return axi_div(*m_cache, s, kArrSize, u, v, 1, "GetDivergence4Poisson");
}

std::vector<double> MACSolver2DAxisym::GetDivergence(const std::vector<double> &u, const std::vector<double> &v) {
    asd2g_session *s = session();
    if (!s) return std::vector<double>(kArrSize, 0.0);
    return axi_div(*m_cache, s, kArrSize, u, v, 0, "GetDivergence");
}

// UpdateVel (mac2dAxisym.cpp:2010-2102) is the 2D projection's arithmetic.
int MACSolver2DAxisym::UpdateVel(std::vector<double> &u, std::vector<double> &v, const std::vector<double> &us,
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

double MACSolver2DAxisym::UpdateDt(const std::vector<double> &u, const std::vector<double> &v) {
    asd2g_session *s = session();
    if (!s) return std::numeric_limits<double>::quiet_NaN();
    if ((int64_t)m_kappa.size() != kArrSize) m_kappa.assign(kArrSize, 0.0);
    m_cache->up(ASD2G_U, u);
    m_cache->up(ASD2G_V, v);
    m_cache->up(ASD2G_KAPPA, m_kappa);
    double dt = 0.0;
    report(asd2g_axi_update_dt(s, &dt), "UpdateDt");
    if (std::isnan(dt) || std::isinf(dt)) std::cout << "dt nan/inf error" << std::endl;
    return dt;
}

int MACSolver2DAxisym::CheckCompatibility(const std::vector<double> &u, const std::vector<double> &v,
                                          const std::vector<double> &uhat, const std::vector<double> &vhat) {
    const std::vector<double> div = GetDivergence(u, v), hatDiv = GetDivergence(uhat, vhat);
    double divSum = 0.0, hatDivSum = 0.0;
    for (int i = kNumBCGrid; i < kNr + kNumBCGrid; i++)
        for (int j = kNumBCGrid; j < kNz + kNumBCGrid; j++) {
            divSum += div[idx(i, j)];
            hatDivSum += hatDiv[idx(i, j)];
        }
    std::cout << " Sum of divergence of intermediate velocity : " << hatDivSum << std::endl;
    std::cout << " Sum of divergence of velocity : " << divSum << std::endl;
    return 0;
}

int MACSolver2DAxisym::SetBC_U_2D(std::string W, std::string E, std::string S, std::string N) {
    if (!m_BC) m_BC = std::make_shared<BoundaryCondition2D>(kNr, kNz, kDr, kDz, kNumBCGrid);
    return m_BC->SetBC_U_2D(W, E, S, N);
}
int MACSolver2DAxisym::SetBC_V_2D(std::string W, std::string E, std::string S, std::string N) {
    if (!m_BC) m_BC = std::make_shared<BoundaryCondition2D>(kNr, kNz, kDr, kDz, kNumBCGrid);
    return m_BC->SetBC_V_2D(W, E, S, N);
}
int MACSolver2DAxisym::SetBC_P_2D(std::string W, std::string E, std::string S, std::string N) {
    if (!m_BC) m_BC = std::make_shared<BoundaryCondition2D>(kNr, kNz, kDr, kDz, kNumBCGrid);
    return m_BC->SetBC_P_2D(W, E, S, N);
}
int MACSolver2DAxisym::ApplyBC_U_2D(std::vector<double> &arr) { return m_BC->ApplyBC_U_2D(arr); }
int MACSolver2DAxisym::ApplyBC_V_2D(std::vector<double> &arr) { return m_BC->ApplyBC_V_2D(arr); }
int MACSolver2DAxisym::ApplyBC_P_2D(std::vector<double> &arr) { return m_BC->ApplyBC_P_2D(arr); }
void MACSolver2DAxisym::SetBCConstantUW(double c) { m_BC->SetBCConstantUW(c); }
void MACSolver2DAxisym::SetBCConstantUE(double c) { m_BC->SetBCConstantUE(c); }
void MACSolver2DAxisym::SetBCConstantUS(double c) { m_BC->SetBCConstantUS(c); }
void MACSolver2DAxisym::SetBCConstantUN(double c) { m_BC->SetBCConstantUN(c); }
void MACSolver2DAxisym::SetBCConstantVW(double c) { m_BC->SetBCConstantVW(c); }
void MACSolver2DAxisym::SetBCConstantVE(double c) { m_BC->SetBCConstantVE(c); }
void MACSolver2DAxisym::SetBCConstantVS(double c) { m_BC->SetBCConstantVS(c); }
void MACSolver2DAxisym::SetBCConstantVN(double c) { m_BC->SetBCConstantVN(c); }
void MACSolver2DAxisym::SetBCConstantPW(double c) { m_BC->SetBCConstantPW(c); }
void MACSolver2DAxisym::SetBCConstantPE(double c) { m_BC->SetBCConstantPE(c); }
void MACSolver2DAxisym::SetBCConstantPS(double c) { m_BC->SetBCConstantPS(c); }
void MACSolver2DAxisym::SetBCConstantPN(double c) { m_BC->SetBCConstantPN(c); }

// The pseudo-pressure is p dt, so the ambient pressure enters the pressure
// boundary constants scaled by dt (mac2dAxisym.cpp:2249-2252).
void MACSolver2DAxisym::UpdateAmbientPressure(double ambientPressure) {
    m_BC->SetAmbientPressure(m_dt * ambientPressure);
}

// Host tridiagonal solve with the interface of SolveTDMA (mac2dAxisym.cpp:
// 2255-2306): a, b, c the sub-, main and super-diagonal, d the right side; c
// and d are overwritten, the solution is left in d.  Same elimination order
// as the device sweeps of GetUHat / GetVHat.
int MACSolver2DAxisym::SolveTDMA(std::vector<double> &a, std::vector<double> &b, std::vector<double> &c,
                                 std::vector<double> &d, int n) {
    if (n < 2) return -1;
    c[0] = c[0] / b[0];
    d[0] = d[0] / b[0];
    for (int k = 1; k < n; k++) {
        const double piv = b[k] - a[k] * c[k - 1];
        if (k < n - 1) c[k] = c[k] / piv;
        d[k] = (d[k] - a[k] * d[k - 1]) / piv;
    }
    for (int k = n - 2; k >= 0; k--) d[k] = d[k] - c[k] * d[k + 1];
    return 0;
}

int MACSolver2DAxisym::sign(const double &val) { return (val > 0) - (val < 0); }

int MACSolver2DAxisym::SetPLTType(PLTTYPE type) {
    m_PLTType = type;
    return 0;
}

// Tecplot ASCII output (mac2dAxisym.cpp:2323-2397): <vel>_ASCII.plt with R, Z,
// the face velocities averaged to the cell centres, LS and PS;
// <div>_ASCII.plt with R, Z, LS, GetDivergence(u, v) and PS.  Headers when
// m_iter is 0, one zone per call.  The binary .szplt output needs the closed
// TecIO library and is not written.
int MACSolver2DAxisym::OutRes(const int iter, const double curTime, const std::string fname_vel_base,
                              const std::string fname_div_base, const std::vector<double> &u,
                              const std::vector<double> &v, const std::vector<double> &ps,
                              const std::vector<double> &ls) {
    if (m_PLTType != PLTTYPE::ASCII && m_PLTType != PLTTYPE::BOTH) return 0;
    const int nbc = kNumBCGrid;
    const int64_t stride = kNz + 2 * nbc;
    std::vector<double> uc(kArrSize, 0.0), vc(kArrSize, 0.0);
    for (int i = nbc; i < kNr + nbc; i++)
        for (int j = nbc; j < kNz + nbc; j++) {
            const int64_t k = j + stride * i;
            uc[k] = (u[k] + u[k + stride]) * 0.5;
            vc[k] = (v[k] + v[k + 1]) * 0.5;
        }
    const std::vector<double> div = GetDivergence(u, v);
    const bool header = m_iter == 0;
    const bool ok =
        write_zone(fname_vel_base + "_ASCII.plt", header, "VEL", "\"R\", \"Z\", \"U\", \"V\", \"LS\", \"PS\"", iter,
                   curTime, kNr, kNz, nbc, kBaseR, kBaseZ, kDr, kDz, {&uc, &vc, &ls, &ps}) &&
        write_zone(fname_div_base + "_ASCII.plt", header, "DIV", "\"R\", \"Z\", \"LS\", \"DIV\", \"PS\"", iter,
                   curTime, kNr, kNz, nbc, kBaseR, kBaseZ, kDr, kDz, {&ls, &div, &ps});
    if (!ok) perror("MACSolver2DAxisym::OutRes");
    return 0;
}

int MACSolver2DAxisym::OutResClose() { return 0; }
