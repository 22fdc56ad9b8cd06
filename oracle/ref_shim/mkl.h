/* Minimal stand-in for the Intel MKL headers that the reference's
 * src/poisson2d.cpp and src/mac2d.cpp include.  It declares only what those
 * files call: the five CBLAS level-1 routines, the 0-based CSR SpMV and the
 * (unused, aborting) FFT Helmholtz solver entry points.  The definitions live
 * in shim.cpp: serial, fixed summation order, so that reference runs are
 * reproducible, plus a capture hook that records the first CSR matrix and
 * right-hand side handed to the Jacobi-PCG solver.
 * Test infrastructure only: nothing in the product links this. */
#ifndef ASD2_REF_SHIM_MKL_H
#define ASD2_REF_SHIM_MKL_H
#include <cstdlib>
#include <cstdint>

typedef int MKL_INT;
typedef void *DFTI_DESCRIPTOR_HANDLE;

extern "C" {
void cblas_dcopy(const MKL_INT n, const double *x, const MKL_INT incx, double *y, const MKL_INT incy);
void cblas_daxpy(const MKL_INT n, const double a, const double *x, const MKL_INT incx, double *y, const MKL_INT incy);
double cblas_ddot(const MKL_INT n, const double *x, const MKL_INT incx, const double *y, const MKL_INT incy);
double cblas_dnrm2(const MKL_INT n, const double *x, const MKL_INT incx);
void cblas_dscal(const MKL_INT n, const double a, double *x, const MKL_INT incx);
void mkl_cspblas_dcsrgemv(const char *transa, const MKL_INT *m, const double *a, const MKL_INT *ia,
                          const MKL_INT *ja, const double *x, double *y);
void MKL_Free_Buffers(void);
void mkl_set_num_threads(int n);
}

/* The FFT Helmholtz path (POISSONTYPE::MKL) is closed MKL code and is not on
 * any path this project reproduces: calling it aborts. */
template <class... A> inline void d_init_Helmholtz_2D(A...) { std::abort(); }
template <class... A> inline void d_commit_Helmholtz_2D(A...) { std::abort(); }
template <class... A> inline void d_Helmholtz_2D(A...) { std::abort(); }
template <class... A> inline void free_Helmholtz_2D(A...) { std::abort(); }
#endif
