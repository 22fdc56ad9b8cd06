// BoundaryCondition2D on the B200: configuration as in the reference
// (bc2d.cpp:16-344, string names, the per-side dispatch), ghost fills through
// the asd2g C ABI.
#include "bc2d.h"

#include <algorithm>
#include <cctype>
#include <iostream>

#include "session.h"

using asd2g_dropin::SessionCache;

BoundaryCondition2D::BoundaryCondition2D(int nx, int ny, int num_bc_grid)
    : kNx(nx), kNy(ny), kNumBCGrid(num_bc_grid), kDx(-1.0), kDy(-1.0), m_AmbientPressure(0.0),
      m_BC_UW(BC2D::CUSTOM), m_BC_UE(BC2D::CUSTOM), m_BC_US(BC2D::CUSTOM), m_BC_UN(BC2D::CUSTOM),
      m_BC_VW(BC2D::CUSTOM), m_BC_VE(BC2D::CUSTOM), m_BC_VS(BC2D::CUSTOM), m_BC_VN(BC2D::CUSTOM),
      m_BC_PW(BC2D::CUSTOM), m_BC_PE(BC2D::CUSTOM), m_BC_PS(BC2D::CUSTOM), m_BC_PN(BC2D::CUSTOM),
      m_BC_DirichletConstantUW(0), m_BC_DirichletConstantUE(0), m_BC_DirichletConstantUS(0),
      m_BC_DirichletConstantUN(0), m_BC_DirichletConstantVW(0), m_BC_DirichletConstantVE(0),
      m_BC_DirichletConstantVS(0), m_BC_DirichletConstantVN(0), m_BC_DirichletConstantPW(0),
      m_BC_DirichletConstantPE(0), m_BC_DirichletConstantPS(0), m_BC_DirichletConstantPN(0),
      m_cache(new SessionCache()) {}

BoundaryCondition2D::BoundaryCondition2D(int nx, int ny, double dx, double dy, int num_bc_grid)
    : BoundaryCondition2D(nx, ny, num_bc_grid) {
    const_cast<double &>(kDx) = dx;
    const_cast<double &>(kDy) = dy;
}

BoundaryCondition2D::~BoundaryCondition2D() = default;

namespace {
std::string lower(std::string s) {
    std::transform(s.begin(), s.end(), s.begin(), ::tolower);
    return s;
}
// Name -> kind of one side.  `axisym_dirichlet` selects whether "axisym"
// also sets the constant to 0 (bc2d.cpp:32-36 vs :84-88).
BC2D parse(const std::string &n, bool pressure_ok) {
    if (n == "periodic") return BC2D::PERIODIC;
    if (n == "neumann") return BC2D::NEUMANN;
    if (n == "axisym") return BC2D::AXISYM;
    if (n == "wall") return BC2D::WALL;
    if (n == "dirichlet") return BC2D::DIRICHLET;
    if (n == "inlet") return BC2D::INLET;
    if (n == "outlet") return BC2D::OUTLET;
    if (pressure_ok && n == "pressure") return BC2D::PRESSURE;
    if (pressure_ok && n == "lsfree") return BC2D::LSFREE;
    return BC2D::CUSTOM;
}
}  // namespace

int BoundaryCondition2D::SetBC_U_2D(std::string W, std::string E, std::string S, std::string N) {
    W = lower(W), E = lower(E), S = lower(S), N = lower(N);
    if (W == "pressure" || E == "pressure" || S == "pressure" || N == "pressure") {
        std::cout << "Boundary Condition Error : constant pressure BC is not allowed at velocity" << std::endl;
        exit(1);
    }
    m_BC_UW = parse(W, false);
    m_BC_UE = parse(E, false);
    m_BC_US = parse(S, false);
    m_BC_UN = parse(N, false);
    // constants forced to 0 (bc2d.cpp:32-41, :58-67, :80-82, :98-100)
    if (m_BC_UW == BC2D::AXISYM || m_BC_UW == BC2D::WALL) SetBCConstantUW(0.0);
    if (m_BC_UE == BC2D::AXISYM || m_BC_UE == BC2D::WALL) SetBCConstantUE(0.0);
    if (m_BC_US == BC2D::WALL) SetBCConstantUS(0.0);
    if (m_BC_UN == BC2D::WALL) SetBCConstantUN(0.0);
    return 0;
}

int BoundaryCondition2D::SetBC_V_2D(std::string W, std::string E, std::string S, std::string N) {
    W = lower(W), E = lower(E), S = lower(S), N = lower(N);
    if (W == "pressure" || E == "pressure" || S == "pressure" || N == "pressure") {
        std::cout << "Boundary Condition Error : constant pressure BC is not allowed at velocity" << std::endl;
        exit(1);
    }
    m_BC_VW = parse(W, false);
    m_BC_VE = parse(E, false);
    m_BC_VS = parse(S, false);
    m_BC_VN = parse(N, false);
    // (bc2d.cpp:150-153, :171-174, :188-196, :214-222)
    if (m_BC_VW == BC2D::WALL) SetBCConstantVW(0.0);
    if (m_BC_VE == BC2D::WALL) SetBCConstantVE(0.0);
    if (m_BC_VS == BC2D::AXISYM || m_BC_VS == BC2D::WALL) SetBCConstantVS(0.0);
    if (m_BC_VN == BC2D::AXISYM || m_BC_VN == BC2D::WALL) SetBCConstantVN(0.0);
    return 0;
}

int BoundaryCondition2D::SetBC_P_2D(std::string W, std::string E, std::string S, std::string N) {
    m_BC_PW = parse(lower(W), true);
    m_BC_PE = parse(lower(E), true);
    m_BC_PS = parse(lower(S), true);
    m_BC_PN = parse(lower(N), true);
    return 0;
}

void BoundaryCondition2D::side_fill(std::vector<double> &arr, char grid, int side, int fill) {
    asd2g_params p{};
    p.nx = kNx;
    p.ny = kNy;
    p.nbc = kNumBCGrid;
    p.dx = kDx > 0.0 ? kDx : 1.0;  // the LS-free fill divides by dx (bc2d.cpp:863-900)
    p.dy = kDy > 0.0 ? kDy : 1.0;
    p.rho_h = p.rho_l = 1.0;
    p.mu_h = p.mu_l = 1.0;
    p.cfl = 1.0;
    p.time_order = 2;
    asd2g_dropin::params_from_bc(*this, p);
    if ((fill == ASD2G_FILL_LSFREE || (grid == 'P' && side >= 0 && fill == ASD2G_FILL_CONFIGURED)) && kDx < 0.0) {
        const BC2D q[4] = {m_BC_PW, m_BC_PE, m_BC_PS, m_BC_PN};
        if (fill == ASD2G_FILL_LSFREE || q[side] == BC2D::LSFREE)
            std::cout << "BC Initialization Error : kDx not set" << std::endl;
    }
    asd2g_session *s = m_cache->get(p);
    if (!s) return;
    m_cache->up(ASD2G_W0, arr);
    if (side < 0) asd2g_dropin::report(asd2g_apply_bc(s, ASD2G_W0, grid), "ApplyBC");
    else asd2g_dropin::report(asd2g_apply_bc_side(s, ASD2G_W0, grid, side, fill), "BC side fill");
    m_cache->down(ASD2G_W0, arr);
}

int BoundaryCondition2D::ApplyBC_U_2D(std::vector<double> &arr) { side_fill(arr, 'U', -1, 0); return 0; }
int BoundaryCondition2D::ApplyBC_V_2D(std::vector<double> &arr) { side_fill(arr, 'V', -1, 0); return 0; }
int BoundaryCondition2D::ApplyBC_P_2D(std::vector<double> &arr) { side_fill(arr, 'P', -1, 0); return 0; }

#define ASD2G_SIDE(NAME, GRID, SIDE, FILL) \
    void BoundaryCondition2D::NAME(std::vector<double> &arr) { side_fill(arr, GRID, SIDE, FILL); }
ASD2G_SIDE(BC_UW, 'U', 0, ASD2G_FILL_CONFIGURED)
ASD2G_SIDE(BC_UE, 'U', 1, ASD2G_FILL_CONFIGURED)
ASD2G_SIDE(BC_US, 'U', 2, ASD2G_FILL_CONFIGURED)
ASD2G_SIDE(BC_UN, 'U', 3, ASD2G_FILL_CONFIGURED)
ASD2G_SIDE(BC_VW, 'V', 0, ASD2G_FILL_CONFIGURED)
ASD2G_SIDE(BC_VE, 'V', 1, ASD2G_FILL_CONFIGURED)
ASD2G_SIDE(BC_VS, 'V', 2, ASD2G_FILL_CONFIGURED)
ASD2G_SIDE(BC_VN, 'V', 3, ASD2G_FILL_CONFIGURED)
ASD2G_SIDE(BC_PW, 'P', 0, ASD2G_FILL_CONFIGURED)
ASD2G_SIDE(BC_PE, 'P', 1, ASD2G_FILL_CONFIGURED)
ASD2G_SIDE(BC_PS, 'P', 2, ASD2G_FILL_CONFIGURED)
ASD2G_SIDE(BC_PN, 'P', 3, ASD2G_FILL_CONFIGURED)
ASD2G_SIDE(BC_PeriodicUW, 'U', 0, ASD2G_FILL_PERIODIC)
ASD2G_SIDE(BC_PeriodicUE, 'U', 1, ASD2G_FILL_PERIODIC)
ASD2G_SIDE(BC_PeriodicUS, 'U', 2, ASD2G_FILL_PERIODIC)
ASD2G_SIDE(BC_PeriodicUN, 'U', 3, ASD2G_FILL_PERIODIC)
ASD2G_SIDE(BC_PeriodicVW, 'V', 0, ASD2G_FILL_PERIODIC)
ASD2G_SIDE(BC_PeriodicVE, 'V', 1, ASD2G_FILL_PERIODIC)
ASD2G_SIDE(BC_PeriodicVS, 'V', 2, ASD2G_FILL_PERIODIC)
ASD2G_SIDE(BC_PeriodicVN, 'V', 3, ASD2G_FILL_PERIODIC)
ASD2G_SIDE(BC_PeriodicPW, 'P', 0, ASD2G_FILL_PERIODIC)
ASD2G_SIDE(BC_PeriodicPE, 'P', 1, ASD2G_FILL_PERIODIC)
ASD2G_SIDE(BC_PeriodicPS, 'P', 2, ASD2G_FILL_PERIODIC)
ASD2G_SIDE(BC_PeriodicPN, 'P', 3, ASD2G_FILL_PERIODIC)
ASD2G_SIDE(BC_NeumannUW, 'U', 0, ASD2G_FILL_NEUMANN)
ASD2G_SIDE(BC_NeumannUE, 'U', 1, ASD2G_FILL_NEUMANN)
ASD2G_SIDE(BC_NeumannUS, 'U', 2, ASD2G_FILL_NEUMANN)
ASD2G_SIDE(BC_NeumannUN, 'U', 3, ASD2G_FILL_NEUMANN)
ASD2G_SIDE(BC_NeumannVW, 'V', 0, ASD2G_FILL_NEUMANN)
ASD2G_SIDE(BC_NeumannVE, 'V', 1, ASD2G_FILL_NEUMANN)
ASD2G_SIDE(BC_NeumannVS, 'V', 2, ASD2G_FILL_NEUMANN)
ASD2G_SIDE(BC_NeumannVN, 'V', 3, ASD2G_FILL_NEUMANN)
ASD2G_SIDE(BC_NeumannPW, 'P', 0, ASD2G_FILL_NEUMANN)
ASD2G_SIDE(BC_NeumannPE, 'P', 1, ASD2G_FILL_NEUMANN)
ASD2G_SIDE(BC_NeumannPS, 'P', 2, ASD2G_FILL_NEUMANN)
ASD2G_SIDE(BC_NeumannPN, 'P', 3, ASD2G_FILL_NEUMANN)
ASD2G_SIDE(BC_DirichletUW, 'U', 0, ASD2G_FILL_DIRICHLET)
ASD2G_SIDE(BC_DirichletUE, 'U', 1, ASD2G_FILL_DIRICHLET)
ASD2G_SIDE(BC_DirichletUS, 'U', 2, ASD2G_FILL_DIRICHLET)
ASD2G_SIDE(BC_DirichletUN, 'U', 3, ASD2G_FILL_DIRICHLET)
ASD2G_SIDE(BC_DirichletVW, 'V', 0, ASD2G_FILL_DIRICHLET)
ASD2G_SIDE(BC_DirichletVE, 'V', 1, ASD2G_FILL_DIRICHLET)
ASD2G_SIDE(BC_DirichletVS, 'V', 2, ASD2G_FILL_DIRICHLET)
ASD2G_SIDE(BC_DirichletVN, 'V', 3, ASD2G_FILL_DIRICHLET)
ASD2G_SIDE(BC_DirichletPW, 'P', 0, ASD2G_FILL_DIRICHLET)
ASD2G_SIDE(BC_DirichletPE, 'P', 1, ASD2G_FILL_DIRICHLET)
ASD2G_SIDE(BC_DirichletPS, 'P', 2, ASD2G_FILL_DIRICHLET)
ASD2G_SIDE(BC_DirichletPN, 'P', 3, ASD2G_FILL_DIRICHLET)
ASD2G_SIDE(BC_LSFreeBoundaryPW, 'P', 0, ASD2G_FILL_LSFREE)
ASD2G_SIDE(BC_LSFreeBoundaryPE, 'P', 1, ASD2G_FILL_LSFREE)
ASD2G_SIDE(BC_LSFreeBoundaryPS, 'P', 2, ASD2G_FILL_LSFREE)
ASD2G_SIDE(BC_LSFreeBoundaryPN, 'P', 3, ASD2G_FILL_LSFREE)
#undef ASD2G_SIDE

void BoundaryCondition2D::SetBCConstantUW(double c) { m_BC_DirichletConstantUW = c; }
void BoundaryCondition2D::SetBCConstantUE(double c) { m_BC_DirichletConstantUE = c; }
void BoundaryCondition2D::SetBCConstantUS(double c) { m_BC_DirichletConstantUS = c; }
void BoundaryCondition2D::SetBCConstantUN(double c) { m_BC_DirichletConstantUN = c; }
void BoundaryCondition2D::SetBCConstantVW(double c) { m_BC_DirichletConstantVW = c; }
void BoundaryCondition2D::SetBCConstantVE(double c) { m_BC_DirichletConstantVE = c; }
void BoundaryCondition2D::SetBCConstantVS(double c) { m_BC_DirichletConstantVS = c; }
void BoundaryCondition2D::SetBCConstantVN(double c) { m_BC_DirichletConstantVN = c; }
void BoundaryCondition2D::SetBCConstantPW(double c) { m_BC_DirichletConstantPW = c; }
void BoundaryCondition2D::SetBCConstantPE(double c) { m_BC_DirichletConstantPE = c; }
void BoundaryCondition2D::SetBCConstantPS(double c) { m_BC_DirichletConstantPS = c; }
void BoundaryCondition2D::SetBCConstantPN(double c) { m_BC_DirichletConstantPN = c; }

void BoundaryCondition2D::SetAmbientPressure(double ambientPressure) {
    // bc2d.cpp:822-833
    m_AmbientPressure = ambientPressure;
    auto amb = [](BC2D b) { return b == BC2D::INLET || b == BC2D::OUTLET || b == BC2D::PRESSURE; };
    if (amb(m_BC_PW)) SetBCConstantPW(ambientPressure);
    if (amb(m_BC_PE)) SetBCConstantPE(ambientPressure);
    if (amb(m_BC_PS)) SetBCConstantPS(ambientPressure);
    if (amb(m_BC_PN)) SetBCConstantPN(ambientPressure);
}
