// PoissonSolver2D with the interface of the reference's include/poisson2d.h
// (poisson2d.h:31-61).  The CSR-input Krylov solvers run on the B200
// (asd2g_csr_solve); MKL is not needed (MKL_INT comes from mkl_types.h).
#ifndef __POISSON2D_H_
#define __POISSON2D_H_

#define _USE_MATH_DEFINES
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "bc2d.h"
#include "common.h"
#include "mkl_types.h"

namespace asd2g_dropin {
struct SessionCache;
}

class PoissonSolver2D {
    int kNx, kNy, kNumBCGrid;

public:
    PoissonSolver2D(int nx, int ny, int num_bc_grid);
    ~PoissonSolver2D();

    // SOR and the MKL FFT Helmholtz solver are not provided (not on any
    // solver path of the droplet step; the latter is closed MKL code): both
    // report an error and return -1.
    int GS_2FUniform_2D(std::vector<double>& ps, const std::vector<double>& rhs, std::vector<double>& AVals,
                        std::vector<MKL_INT>& ACols, std::vector<MKL_INT>& ARowIdx, const double lenX,
                        const double lenY, const double dx, const double dy,
                        const std::shared_ptr<BoundaryCondition2D>& PBC, const int maxiter);
    int MKL_2FUniform_2D(std::vector<double>& phi, const std::vector<double>& rhs, double lenX, double lenY,
                         double dx, double dy, std::shared_ptr<BoundaryCondition2D> PBC);

    int CG_2FUniformP_2D(std::vector<double>& ps, const std::vector<double>& rhs, std::vector<double>& AVals,
                         std::vector<MKL_INT>& ACols, std::vector<MKL_INT>& ARowIdx, std::vector<double>& MVals,
                         std::vector<MKL_INT>& MCols, std::vector<MKL_INT>& MRowIdx,
                         const std::shared_ptr<BoundaryCondition2D>& PBC, int64_t size, const int maxIter);
    int CG_2FUniform_2D(double* x, double* b, std::vector<double>& AVals, std::vector<MKL_INT>& ACols,
                        std::vector<MKL_INT>& ARowIdx, std::vector<double>& MVals, std::vector<MKL_INT>& MCols,
                        std::vector<MKL_INT>& MRowIdx, const std::shared_ptr<BoundaryCondition2D>& PBC, int64_t size,
                        const int maxIter);

    int BiCGStab_2FUniform_2D(std::vector<double>& ps, const std::vector<double>& rhs, std::vector<double>& AVals,
                              std::vector<MKL_INT>& ACols, std::vector<MKL_INT>& ARowIdx, std::vector<double>& M,
                              std::vector<MKL_INT>& MCols, std::vector<MKL_INT>& MRowIdx,
                              const std::shared_ptr<BoundaryCondition2D>& PBC, int64_t size, const int maxiter);

    // declared and never defined by the reference either
    bool IsSymmetric(std::vector<double>& AVals, std::vector<MKL_INT>& ACols, std::vector<MKL_INT>& ARowIdx);

    std::vector<double> InvertMatrixDiagonal(const std::vector<double>& M);
    int idx(int i, int j) { return j + (kNy + 2 * kNumBCGrid) * i; }

private:
    int csr(int solver, double* x, const double* b, std::vector<double>& AVals, std::vector<MKL_INT>& ACols,
            std::vector<MKL_INT>& ARowIdx, std::vector<double>& MVals, std::vector<MKL_INT>& MRowIdx, int64_t size,
            int maxIter, const char* name);
    std::unique_ptr<asd2g_dropin::SessionCache> m_cache;
};

#endif
