/*
 * Oracle test infrastructure: stand-in for LAPACKE_cheev as called by
 * G12KBA-GW/src/headers/init_G.h:38 (jobz='V', uplo='L', row-major).
 *
 * Contract reproduced (LAPACK cheev): on entry the lower triangle of the
 * complex64 matrix `a` holds a Hermitian matrix; on exit `w` holds the
 * eigenvalues in ascending order and column k of `a` (a[i*lda+k]) the
 * matching orthonormal eigenvector.  Returns 0.
 *
 * Algorithm (not MKL's, which is unavailable here): cyclic complex Jacobi
 * rotations carried out in FP64 on the float-rounded input, eigenpairs sorted
 * ascending, each eigenvector's phase fixed so that its first component of
 * largest modulus is real and positive, then rounded to complex64.  The
 * framework's host G0 code implements the same published method with the same
 * operation order, so both produce bit-identical complex64 eigenvectors.
 */
#ifndef G12_ORACLE_MKL_LAPACKE_SHIM_H
#define G12_ORACLE_MKL_LAPACKE_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

#ifndef G12_ORACLE_MKL_SHIM_H
typedef int MKL_INT;
typedef struct { float real, imag; } MKL_Complex8;
#endif
typedef MKL_INT lapack_int;

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

lapack_int LAPACKE_cheev(int matrix_layout, char jobz, char uplo, lapack_int n,
                         MKL_Complex8 *a, lapack_int lda, float *w);

#ifdef __cplusplus
}
#endif

#endif
