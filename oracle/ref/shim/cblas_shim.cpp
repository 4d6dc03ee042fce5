// Naive CBLAS routines (row/col-major GEMM, copy, axpy) used only to link the
// reference's CPU FMM path for the oracle build. OpenBLAS is not in the image.
#include "cblas.h"
#include <complex>

namespace {
template <class T>
inline T at(const T* a, enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE t, blasint ld, blasint i, blasint j)
{
   // element (i, j) of op(A)
   bool tr = (t != CblasNoTrans);
   blasint r = tr ? j : i, c = tr ? i : j;
   T v = (o == CblasRowMajor) ? a[(long)r * ld + c] : a[(long)c * ld + r];
   return v;
}
template <class T>
inline T conjIf(T v, enum CBLAS_TRANSPOSE) { return v; }
template <class R>
inline std::complex<R> conjIf(std::complex<R> v, enum CBLAS_TRANSPOSE t)
{ return t == CblasConjTrans ? std::conj(v) : v; }

template <class T>
void gemm(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, blasint m, blasint n, blasint k,
          T alpha, const T* a, blasint lda, const T* b, blasint ldb, T beta, T* c, blasint ldc)
{
   for(blasint i = 0; i < m; i++)
      for(blasint j = 0; j < n; j++)
      {
         T s = T(0);
         for(blasint p = 0; p < k; p++)
            s += conjIf(at(a, o, ta, lda, i, p), ta) * conjIf(at(b, o, tb, ldb, p, j), tb);
         T& dst = (o == CblasRowMajor) ? c[(long)i * ldc + j] : c[(long)j * ldc + i];
         dst = (beta == T(0)) ? alpha * s : alpha * s + beta * dst;
      }
}
}

extern "C" {
void cblas_sgemm(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, blasint m, blasint n,
                 blasint k, float al, const float* a, blasint lda, const float* b, blasint ldb, float be, float* c,
                 blasint ldc)
{ gemm<float>(o, ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc); }
void cblas_dgemm(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, blasint m, blasint n,
                 blasint k, double al, const double* a, blasint lda, const double* b, blasint ldb, double be,
                 double* c, blasint ldc)
{ gemm<double>(o, ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc); }
void cblas_cgemm(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, blasint m, blasint n,
                 blasint k, const void* al, const void* a, blasint lda, const void* b, blasint ldb, const void* be,
                 void* c, blasint ldc)
{
   typedef std::complex<float> C;
   gemm<C>(o, ta, tb, m, n, k, *(const C*)al, (const C*)a, lda, (const C*)b, ldb, *(const C*)be, (C*)c, ldc);
}
void cblas_zgemm(enum CBLAS_ORDER o, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb, blasint m, blasint n,
                 blasint k, const void* al, const void* a, blasint lda, const void* b, blasint ldb, const void* be,
                 void* c, blasint ldc)
{
   typedef std::complex<double> C;
   gemm<C>(o, ta, tb, m, n, k, *(const C*)al, (const C*)a, lda, (const C*)b, ldb, *(const C*)be, (C*)c, ldc);
}
void cblas_scopy(blasint n, const float* x, blasint ix, float* y, blasint iy)
{ for(blasint i = 0; i < n; i++) y[(long)i * iy] = x[(long)i * ix]; }
void cblas_dcopy(blasint n, const double* x, blasint ix, double* y, blasint iy)
{ for(blasint i = 0; i < n; i++) y[(long)i * iy] = x[(long)i * ix]; }
void cblas_saxpy(blasint n, float a, const float* x, blasint ix, float* y, blasint iy)
{ for(blasint i = 0; i < n; i++) y[(long)i * iy] += a * x[(long)i * ix]; }
void cblas_daxpy(blasint n, double a, const double* x, blasint ix, double* y, blasint iy)
{ for(blasint i = 0; i < n; i++) y[(long)i * iy] += a * x[(long)i * ix]; }
}
