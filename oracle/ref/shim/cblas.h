// Minimal CBLAS declarations (OpenBLAS-compatible names) so that the reference
// FMM sources compile without OpenBLAS. Implemented naively in cblas_shim.cpp.
// Only the routines the reference's CPU path calls are provided.
#pragma once
typedef int blasint;
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
#ifdef __cplusplus
extern "C" {
#endif
void cblas_sgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE, blasint, blasint, blasint,
                 float, const float*, blasint, const float*, blasint, float, float*, blasint);
void cblas_dgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE, blasint, blasint, blasint,
                 double, const double*, blasint, const double*, blasint, double, double*, blasint);
void cblas_cgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE, blasint, blasint, blasint,
                 const void*, const void*, blasint, const void*, blasint, const void*, void*, blasint);
void cblas_zgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE, blasint, blasint, blasint,
                 const void*, const void*, blasint, const void*, blasint, const void*, void*, blasint);
void cblas_scopy(blasint, const float*, blasint, float*, blasint);
void cblas_dcopy(blasint, const double*, blasint, double*, blasint);
void cblas_saxpy(blasint, float, const float*, blasint, float*, blasint);
void cblas_daxpy(blasint, double, const double*, blasint, double*, blasint);
#ifdef __cplusplus
}
#endif
