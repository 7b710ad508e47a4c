/*
 * Declaration-only CBLAS header used when compiling the reference's own
 * sources (lu2.c, lu2tlib.c, lu2lib.c) into oracle/_ref/.  The reference
 * includes <cblas.h> and calls only cblas_dgemm and cblas_idamax; the
 * definitions come from the OpenBLAS shared library shipped in the image.
 * Test infrastructure only.
 */
#ifndef LU2_ORACLE_CBLAS_DECL_H
#define LU2_ORACLE_CBLAS_DECL_H
#include <stddef.h>
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb,
                 int m, int n, int k, double alpha, const double *a, int lda,
                 const double *b, int ldb, double beta, double *c, int ldc);
size_t cblas_idamax(int n, const double *x, int incx);
#endif
