// Serial, fixed-order definitions of the MKL routines declared in mkl.h, used
// only to build the reference sources as a CPU oracle.  Summation runs left
// to right so that a reference run is reproducible bit for bit.  The CSR SpMV
// skips columns outside [0, m): the reference's all-Neumann pin (mac2d.cpp
// :1585-1607) emits zero-valued entries with column indices >= m, which real
// MKL would read out of bounds.
//
// Capture hook: after ref_shim_capture_arm(), the first SpMV records its CSR
// operand and the first dcopy records its source vector.  Inside
// PoissonSolver2D::CG_2FUniform_2D (poisson2d.cpp:320-329) those are exactly
// the assembled matrix A and the right-hand side b.
//
// With ASD2_SHIM_EXTERNAL_CBLAS (the threaded build for the timed CPU
// baseline, not for parity) the cblas_d* calls go to a real CBLAS linked in
// (OpenBLAS, its own threads), the SpMV rows are split over OpenMP threads
// (each row still summed in order) and dcopy captures nothing.
#include "mkl.h"
#include <cmath>
#include <vector>

namespace {
struct Capture {
    bool armed = false, have_a = false, have_b = false;
    std::vector<double> a, b;
    std::vector<MKL_INT> ia, ja;
    MKL_INT m = 0;
} g_cap;
}  // namespace

extern "C" {
#ifndef ASD2_SHIM_EXTERNAL_CBLAS
void cblas_dcopy(const MKL_INT n, const double *x, const MKL_INT incx, double *y, const MKL_INT incy) {
    if (g_cap.armed && g_cap.have_a && !g_cap.have_b) {
        g_cap.b.assign(n, 0.0);
        for (MKL_INT i = 0; i < n; i++) g_cap.b[i] = x[(int64_t)i * incx];
        g_cap.have_b = true;
    }
    for (MKL_INT i = 0; i < n; i++) y[(int64_t)i * incy] = x[(int64_t)i * incx];
}

void cblas_daxpy(const MKL_INT n, const double a, const double *x, const MKL_INT incx, double *y,
                 const MKL_INT incy) {
    for (MKL_INT i = 0; i < n; i++) y[(int64_t)i * incy] += a * x[(int64_t)i * incx];
}

double cblas_ddot(const MKL_INT n, const double *x, const MKL_INT incx, const double *y, const MKL_INT incy) {
    double s = 0.0;
    for (MKL_INT i = 0; i < n; i++) s += x[(int64_t)i * incx] * y[(int64_t)i * incy];
    return s;
}

double cblas_dnrm2(const MKL_INT n, const double *x, const MKL_INT incx) {
    double s = 0.0;
    for (MKL_INT i = 0; i < n; i++) s += x[(int64_t)i * incx] * x[(int64_t)i * incx];
    return std::sqrt(s);
}

void cblas_dscal(const MKL_INT n, const double a, double *x, const MKL_INT incx) {
    for (MKL_INT i = 0; i < n; i++) x[(int64_t)i * incx] *= a;
}
#endif

void mkl_cspblas_dcsrgemv(const char *, const MKL_INT *m, const double *a, const MKL_INT *ia,
                          const MKL_INT *ja, const double *x, double *y) {
    const MKL_INT rows = *m;
    if (g_cap.armed && !g_cap.have_a) {
        g_cap.m = rows;
        g_cap.ia.assign(ia, ia + rows + 1);
        g_cap.ja.assign(ja, ja + ia[rows]);
        g_cap.a.assign(a, a + ia[rows]);
        g_cap.have_a = true;
    }
#ifdef ASD2_SHIM_EXTERNAL_CBLAS
#pragma omp parallel for schedule(static)
#endif
    for (MKL_INT r = 0; r < rows; r++) {
        double s = 0.0;
        for (MKL_INT k = ia[r]; k < ia[r + 1]; k++) {
            const MKL_INT c = ja[k];
            if (c < 0 || c >= rows) continue;
            s += a[k] * x[c];
        }
        y[r] = s;
    }
}

void MKL_Free_Buffers(void) {}
void mkl_set_num_threads(int) {}

// ---- capture control (called by ref_driver.cpp) ----
void ref_shim_capture_arm(void) {
    g_cap = Capture();
    g_cap.armed = true;
}
int ref_shim_capture_sizes(int *m, int *nnz, int *nb) {
    if (!g_cap.have_a || !g_cap.have_b) return -1;
    *m = g_cap.m;
    *nnz = (int)g_cap.a.size();
    *nb = (int)g_cap.b.size();
    return 0;
}
int ref_shim_capture_copy(double *a, int *ia, int *ja, double *b) {
    if (!g_cap.have_a || !g_cap.have_b) return -1;
    for (size_t k = 0; k < g_cap.a.size(); k++) { a[k] = g_cap.a[k]; ja[k] = g_cap.ja[k]; }
    for (size_t k = 0; k < g_cap.ia.size(); k++) ia[k] = g_cap.ia[k];
    for (size_t k = 0; k < g_cap.b.size(); k++) b[k] = g_cap.b[k];
    g_cap.armed = false;
    return 0;
}
}
