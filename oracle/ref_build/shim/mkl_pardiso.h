/* Shim for the reference build: PARDISO prototype; the implementation is the
   dense stand-in in oracle/ref_build/pardiso_standin.cpp. */
#ifndef HTF_SHIM_MKL_PARDISO_H
#define HTF_SHIM_MKL_PARDISO_H
#include "mkl_types.h"
#ifdef __cplusplus
extern "C" {
#endif
void pardiso(void *pt, const MKL_INT *maxfct, const MKL_INT *mnum, const MKL_INT *mtype,
             const MKL_INT *phase, const MKL_INT *n, const void *a, const MKL_INT *ia,
             const MKL_INT *ja, MKL_INT *perm, const MKL_INT *nrhs, MKL_INT *iparm,
             const MKL_INT *msglvl, void *b, void *x, MKL_INT *error);
#ifdef __cplusplus
}
#endif
#define PARDISO pardiso
#endif
