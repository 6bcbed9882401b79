/* lapack_bridge.c -- serves the CLAPACK routines SFbox calls from the LAPACK
 * bundled with scipy (libscipy_openblas, 32-bit integers, symbols prefixed
 * "scipy_"), passing the hidden Fortran string lengths explicitly.
 * Test infrastructure for the oracle's build of the reference sources. */
#include <stddef.h>
#include "clapack.h"

#define STR1 ((size_t)1)
void scipy_dgemm_(char *, char *, integer *, integer *, integer *, doublereal *, doublereal *, integer *,
                  doublereal *, integer *, doublereal *, doublereal *, integer *, size_t, size_t);
void scipy_dgemv_(char *, integer *, integer *, doublereal *, doublereal *, integer *, doublereal *, integer *,
                  doublereal *, doublereal *, integer *, size_t);
void scipy_dgeqrf_(integer *, integer *, doublereal *, integer *, doublereal *, doublereal *, integer *, integer *);
void scipy_dgesvd_(char *, char *, integer *, integer *, doublereal *, integer *, doublereal *, doublereal *,
                   integer *, doublereal *, integer *, doublereal *, integer *, integer *, size_t, size_t);
void scipy_dgetrf_(integer *, integer *, doublereal *, integer *, integer *, integer *);
void scipy_dgetri_(integer *, doublereal *, integer *, integer *, doublereal *, integer *, integer *);
void scipy_dorgqr_(integer *, integer *, integer *, doublereal *, integer *, doublereal *, doublereal *, integer *,
                   integer *);
void scipy_dposvx_(char *, char *, integer *, integer *, doublereal *, integer *, doublereal *, integer *, char *,
                   doublereal *, doublereal *, integer *, doublereal *, integer *, doublereal *, doublereal *,
                   doublereal *, doublereal *, integer *, integer *, size_t, size_t, size_t);

int dgemm_(char *ta, char *tb, integer *m, integer *n, integer *k, doublereal *al, doublereal *a, integer *lda,
           doublereal *b, integer *ldb, doublereal *be, doublereal *c, integer *ldc) {
    scipy_dgemm_(ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc, STR1, STR1);
    return 0;
}
int dgemv_(char *t, integer *m, integer *n, doublereal *al, doublereal *a, integer *lda, doublereal *x,
           integer *incx, doublereal *be, doublereal *y, integer *incy) {
    scipy_dgemv_(t, m, n, al, a, lda, x, incx, be, y, incy, STR1);
    return 0;
}
int dgeqrf_(integer *m, integer *n, doublereal *a, integer *lda, doublereal *tau, doublereal *w, integer *lw,
            integer *info) {
    scipy_dgeqrf_(m, n, a, lda, tau, w, lw, info);
    return 0;
}
int dgesvd_(char *ju, char *jv, integer *m, integer *n, doublereal *a, integer *lda, doublereal *s, doublereal *u,
            integer *ldu, doublereal *vt, integer *ldvt, doublereal *w, integer *lw, integer *info) {
    scipy_dgesvd_(ju, jv, m, n, a, lda, s, u, ldu, vt, ldvt, w, lw, info, STR1, STR1);
    return 0;
}
int dgetrf_(integer *m, integer *n, doublereal *a, integer *lda, integer *ipiv, integer *info) {
    scipy_dgetrf_(m, n, a, lda, ipiv, info);
    return 0;
}
int dgetri_(integer *n, doublereal *a, integer *lda, integer *ipiv, doublereal *w, integer *lw, integer *info) {
    scipy_dgetri_(n, a, lda, ipiv, w, lw, info);
    return 0;
}
int dorgqr_(integer *m, integer *n, integer *k, doublereal *a, integer *lda, doublereal *tau, doublereal *w,
            integer *lw, integer *info) {
    scipy_dorgqr_(m, n, k, a, lda, tau, w, lw, info);
    return 0;
}
int dposvx_(char *f, char *ul, integer *n, integer *nrhs, doublereal *a, integer *lda, doublereal *af,
            integer *ldaf, char *eq, doublereal *s, doublereal *b, integer *ldb, doublereal *x, integer *ldx,
            doublereal *rcond, doublereal *ferr, doublereal *berr, doublereal *w, integer *iw, integer *info) {
    scipy_dposvx_(f, ul, n, nrhs, a, lda, af, ldaf, eq, s, b, ldb, x, ldx, rcond, ferr, berr, w, iw, info, STR1,
                  STR1, STR1);
    return 0;
}
