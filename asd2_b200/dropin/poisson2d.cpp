// PoissonSolver2D on the B200 (see poisson2d.h).  The CSR solvers keep the
// reference's conventions: x starts at 0, the stopping test is the hard-coded
// ||r||/||b|| <= 1e-6 (poisson2d.cpp:311) and the iteration is the
// reference's own (CG first-step direction and err_tol^2 term; BiCGStab with
// rho_2 never updated).  The pinned all-Neumann gather/scatter of
// CG_2FUniformP_2D (:239-275) is reproduced.
#include "poisson2d.h"

#include <cstdio>

#include "asd2g.h"
#include "session.h"

using asd2g_dropin::report;
using asd2g_dropin::SessionCache;

PoissonSolver2D::PoissonSolver2D(int nx, int ny, int num_bc_grid)
    : kNx(nx), kNy(ny), kNumBCGrid(num_bc_grid), m_cache(new SessionCache()) {}

PoissonSolver2D::~PoissonSolver2D() = default;

int PoissonSolver2D::GS_2FUniform_2D(std::vector<double> &, const std::vector<double> &, std::vector<double> &,
                                     std::vector<MKL_INT> &, std::vector<MKL_INT> &, const double, const double,
                                     const double, const double, const std::shared_ptr<BoundaryCondition2D> &,
                                     const int) {
    std::fprintf(stderr, "PoissonSolver2D::GS_2FUniform_2D is not provided by the B200 build\n");
    return -1;
}

int PoissonSolver2D::MKL_2FUniform_2D(std::vector<double> &, const std::vector<double> &, double, double, double,
                                      double, std::shared_ptr<BoundaryCondition2D>) {
    std::fprintf(stderr, "PoissonSolver2D::MKL_2FUniform_2D (MKL FFT Helmholtz) is not provided by the B200 build\n");
    return -1;
}

std::vector<double> PoissonSolver2D::InvertMatrixDiagonal(const std::vector<double> &M) {
    std::vector<double> inv(M.size(), 0.0);
    for (size_t i = 0; i < M.size(); i++) inv[i] = 1.0 / M[i];
    return inv;
}

int PoissonSolver2D::csr(int solver, double *x, const double *b, std::vector<double> &AVals,
                         std::vector<MKL_INT> &ACols, std::vector<MKL_INT> &ARowIdx, std::vector<double> &MVals,
                         std::vector<MKL_INT> &MRowIdx, int64_t size, int maxIter, const char *name) {
    asd2g_params p{};
    p.nx = kNx;
    p.ny = kNy;
    p.nbc = kNumBCGrid;
    p.dx = p.dy = 1.0;
    p.rho_h = p.rho_l = p.mu_h = p.mu_l = 1.0;
    p.cfl = 1.0;
    p.time_order = 2;
    for (int k = 0; k < 4; k++) p.bc_u[k] = p.bc_v[k] = p.bc_p[k] = ASD2G_BC_NEUMANN;
    asd2g_session *s = m_cache->get(p);
    if (!s) return -1;
    const int rows = static_cast<int>(size);
    std::vector<double> diag(rows);
    for (int r = 0; r < rows; r++) diag[r] = MVals[MRowIdx[r]];
    int iters = 0;
    double res = 0.0;
    const int rc = report(asd2g_csr_solve(s, solver, rows, ARowIdx.data(), ACols.data(), AVals.data(), diag.data(), b,
                                          x, 1.0e-6, maxIter, &iters, &res),
                          name);
    std::cout << (solver == ASD2G_SOLVER_PCG_REFERENCE ? "CG : " : "BiCG : ") << iters << " " << maxIter
              << " Err : " << res << std::endl;
    return rc < 0 ? rc : 0;
}

int PoissonSolver2D::CG_2FUniform_2D(double *x, double *b, std::vector<double> &AVals, std::vector<MKL_INT> &ACols,
                                     std::vector<MKL_INT> &ARowIdx, std::vector<double> &MVals,
                                     std::vector<MKL_INT> &MCols, std::vector<MKL_INT> &MRowIdx,
                                     const std::shared_ptr<BoundaryCondition2D> &, int64_t size, const int maxIter) {
    (void)MCols;
    return csr(ASD2G_SOLVER_PCG_REFERENCE, x, b, AVals, ACols, ARowIdx, MVals, MRowIdx, size, maxIter,
               "CG_2FUniform_2D");
}

static bool all_neumann(const BoundaryCondition2D &bc) {
    auto n = [](BC2D b) { return b == BC2D::NEUMANN || b == BC2D::AXISYM || b == BC2D::WALL; };
    return n(bc.m_BC_PW) && n(bc.m_BC_PE) && n(bc.m_BC_PS) && n(bc.m_BC_PN);
}

int PoissonSolver2D::CG_2FUniformP_2D(std::vector<double> &ps, const std::vector<double> &rhs,
                                      std::vector<double> &AVals, std::vector<MKL_INT> &ACols,
                                      std::vector<MKL_INT> &ARowIdx, std::vector<double> &MVals,
                                      std::vector<MKL_INT> &MCols, std::vector<MKL_INT> &MRowIdx,
                                      const std::shared_ptr<BoundaryCondition2D> &PBC, int64_t size,
                                      const int maxIter) {
    std::vector<double> b(size, 0.0), x(size, 0.0);
    const bool pin = all_neumann(*PBC);
    for (int j = 0; j < kNy; j++)
        for (int i = 0; i < kNx; i++) {
            int64_t k = i + (int64_t)j * kNx;
            if (pin) {
                if (i == 0 && j == 0) continue;
                k--;
            }
            b[k] = rhs[idx(i + kNumBCGrid, j + kNumBCGrid)];
        }
    const int rc = CG_2FUniform_2D(x.data(), b.data(), AVals, ACols, ARowIdx, MVals, MCols, MRowIdx, PBC, size,
                                   maxIter);
    for (int j = 0; j < kNy; j++)
        for (int i = 0; i < kNx; i++) {
            int64_t k = i + (int64_t)j * kNx;
            if (pin) {
                if (i == 0 && j == 0) continue;
                k--;
            }
            const double val = x[k];
            ps[idx(i + kNumBCGrid, j + kNumBCGrid)] = val;
            if (std::isnan(val) || std::isinf(val)) {
                std::cout << "poisson equation nan/inf error : " << i + kNumBCGrid << " " << j + kNumBCGrid << " "
                          << val << std::endl;
                exit(1);
            }
        }
    return rc;
}

int PoissonSolver2D::BiCGStab_2FUniform_2D(std::vector<double> &ps, const std::vector<double> &rhs,
                                           std::vector<double> &AVals, std::vector<MKL_INT> &ACols,
                                           std::vector<MKL_INT> &ARowIdx, std::vector<double> &M,
                                           std::vector<MKL_INT> &MCols, std::vector<MKL_INT> &MRowIdx,
                                           const std::shared_ptr<BoundaryCondition2D> &, int64_t size,
                                           const int maxiter) {
    (void)MCols;
    // poisson2d.cpp:427-440: b is gathered without the pin shift
    std::vector<double> b(size, 0.0), x(size, 0.0);
    for (int j = 0; j < kNy; j++)
        for (int i = 0; i < kNx; i++) {
            const int64_t k = i + (int64_t)j * kNx;
            if (k < size) b[k] = rhs[idx(i + kNumBCGrid, j + kNumBCGrid)];
        }
    const int rc = csr(ASD2G_SOLVER_BICGSTAB_REFERENCE, x.data(), b.data(), AVals, ACols, ARowIdx, M, MRowIdx, size,
                       maxiter, "BiCGStab_2FUniform_2D");
    for (int j = 0; j < kNy; j++)
        for (int i = 0; i < kNx; i++) {
            const int64_t k = i + (int64_t)j * kNx;
            if (k >= size) continue;
            ps[idx(i + kNumBCGrid, j + kNumBCGrid)] = x[k];
            if (std::isnan(x[k]) || std::isinf(x[k])) {
                std::cout << "poisson equation nan/inf error : " << i + kNumBCGrid << " " << j + kNumBCGrid << " "
                          << x[k] << std::endl;
                exit(1);
            }
        }
    return rc;
}
