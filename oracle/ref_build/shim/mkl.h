/* Shim for the reference build: the LAPACKE subset the reference calls
   (Cluster.cpp:1254,1260; Matrix.cpp:1489,1526,2352), implemented in
   oracle/ref_build/lapack_standin.cpp. */
#ifndef HTF_SHIM_MKL_H
#define HTF_SHIM_MKL_H
#include <stdint.h>
#include "mkl_types.h"
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
#ifdef __cplusplus
extern "C" {
#endif
int LAPACKE_dpotrf(int layout, char uplo, int n, double *a, int lda);
int LAPACKE_dpotri(int layout, char uplo, int n, double *a, int lda);
int LAPACKE_dspev(int layout, char jobz, char uplo, int n, double *ap, double *w, double *z, int ldz);
int LAPACKE_dgesvd(int layout, char jobu, char jobvt, int m, int n, double *a, int lda,
                   double *s, double *u, int ldu, double *vt, int ldvt, double *superb);
#ifdef __cplusplus
}
#endif
#endif
