/* Shim for the reference build: the MKL integer type (LP64 interface). */
#ifndef HTF_SHIM_MKL_TYPES_H
#define HTF_SHIM_MKL_TYPES_H
#define MKL_INT int
#endif
