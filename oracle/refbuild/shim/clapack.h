/* clapack.h -- the CLAPACK prototypes SFbox calls (sfnewton.cpp:4,
 * MPS.cpp:4), with f2c's calling convention (every argument by pointer).
 * Test infrastructure; implemented in lapack_bridge.c. */
#ifndef CLAPACK_SHIM_H
#define CLAPACK_SHIM_H
#include "f2c.h"
#ifdef __cplusplus
extern "C" {
#endif
int dgemm_(char *transa, char *transb, integer *m, integer *n, integer *k, doublereal *alpha, doublereal *a,
           integer *lda, doublereal *b, integer *ldb, doublereal *beta, doublereal *c, integer *ldc);
int dgemv_(char *trans, integer *m, integer *n, doublereal *alpha, doublereal *a, integer *lda, doublereal *x,
           integer *incx, doublereal *beta, doublereal *y, integer *incy);
int dgeqrf_(integer *m, integer *n, doublereal *a, integer *lda, doublereal *tau, doublereal *work, integer *lwork,
            integer *info);
int dgesvd_(char *jobu, char *jobvt, integer *m, integer *n, doublereal *a, integer *lda, doublereal *s,
            doublereal *u, integer *ldu, doublereal *vt, integer *ldvt, doublereal *work, integer *lwork,
            integer *info);
int dgetrf_(integer *m, integer *n, doublereal *a, integer *lda, integer *ipiv, integer *info);
int dgetri_(integer *n, doublereal *a, integer *lda, integer *ipiv, doublereal *work, integer *lwork, integer *info);
int dorgqr_(integer *m, integer *n, integer *k, doublereal *a, integer *lda, doublereal *tau, doublereal *work,
            integer *lwork, integer *info);
int dposvx_(char *fact, char *uplo, integer *n, integer *nrhs, doublereal *a, integer *lda, doublereal *af,
            integer *ldaf, char *equed, doublereal *s, doublereal *b, integer *ldb, doublereal *x, integer *ldx,
            doublereal *rcond, doublereal *ferr, doublereal *berr, doublereal *work, integer *iwork, integer *info);
#ifdef __cplusplus
}
#endif
#endif
