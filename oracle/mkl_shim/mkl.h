/*
 * Oracle test infrastructure: a self-written stand-in for the two Intel MKL
 * entry points the reference calls.  Intel MKL is not installed here, so the
 * reference's compiled oracle (oracle/_ref) is linked against this shim.
 *
 *  - cblas_zgemm: only the row-major NoTrans/NoTrans case used by
 *    G12KBA-GW/src/headers/commutators.h:39-40 (hG_commutator).
 *  - MKL_Complex8 / LAPACKE_cheev: see mkl_lapacke.h (init_G.h:28-54).
 *
 * MKL's own blocking and FMA order are unknown, so results at the zgemm
 * boundary agree with MKL to round-off only ("parity unpinned at the MKL
 * boundary").  Nothing in the product links this file.
 */
#ifndef G12_ORACLE_MKL_SHIM_H
#define G12_ORACLE_MKL_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MKL_INT;
typedef struct { float real, imag; } MKL_Complex8;
typedef struct { double real, imag; } MKL_Complex16;

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

/* C = alpha*A*B + beta*C, complex128, row-major, no transposes (other
 * layouts/transposes abort: the reference never uses them). */
void cblas_zgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 MKL_INT m, MKL_INT n, MKL_INT k, const void *alpha,
                 const void *a, MKL_INT lda, const void *b, MKL_INT ldb,
                 const void *beta, void *c, MKL_INT ldc);

#ifdef __cplusplus
}
#endif

#include "mkl_lapacke.h"

#endif
