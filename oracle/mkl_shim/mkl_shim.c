/*
 * Oracle test infrastructure: implementations of the MKL stand-ins declared in
 * mkl.h / mkl_lapacke.h.  Linked only into the compiled reference oracle
 * (oracle/_ref) and never into the product.
 */
#include "mkl.h"
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

void cblas_zgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 MKL_INT m, MKL_INT n, MKL_INT k, const void *alpha,
                 const void *a, MKL_INT lda, const void *b, MKL_INT ldb,
                 const void *beta, void *c, MKL_INT ldc)
{
    /* commutators.h:39-40 only uses RowMajor, NoTrans, NoTrans. */
    if (layout != CblasRowMajor || ta != CblasNoTrans || tb != CblasNoTrans) {
        fprintf(stderr, "mkl shim: unsupported cblas_zgemm form\n");
        abort();
    }
    const double *A = (const double *)a, *B = (const double *)b;
    const double *al = (const double *)alpha, *be = (const double *)beta;
    double *C = (double *)c;
    for (MKL_INT i = 0; i < m; ++i) {
        for (MKL_INT j = 0; j < n; ++j) {
            double sr = 0.0, si = 0.0;
            for (MKL_INT p = 0; p < k; ++p) {
                double ar = A[2 * (i * lda + p)], ai = A[2 * (i * lda + p) + 1];
                double br = B[2 * (p * ldb + j)], bi = B[2 * (p * ldb + j) + 1];
                sr += ar * br - ai * bi;
                si += ar * bi + ai * br;
            }
            double rr, ri;
            if (al[0] == 1.0 && al[1] == 0.0) { rr = sr; ri = si; }
            else { rr = al[0] * sr - al[1] * si; ri = al[0] * si + al[1] * sr; }
            if (!(be[0] == 0.0 && be[1] == 0.0)) {
                double cr = C[2 * (i * ldc + j)], ci = C[2 * (i * ldc + j) + 1];
                rr += be[0] * cr - be[1] * ci;
                ri += be[0] * ci + be[1] * cr;
            }
            C[2 * (i * ldc + j)] = rr;
            C[2 * (i * ldc + j) + 1] = ri;
        }
    }
}

/*
 * Cyclic complex Jacobi eigen-solver (Jacobi 1846; the real-symmetric update
 * formulas as in Rutishauser's Handbook algorithm, made Hermitian by first
 * rotating the phase of a_pq to the real axis).  A and V are n*n row-major,
 * stored as interleaved re/im doubles.  On return diag(A) holds eigenvalues
 * and the columns of V the eigenvectors.
 */
static void jacobi_hermitian(int n, double *A, double *V)
{
#define RE(M, r, c) (M)[2 * ((r) * n + (c))]
#define IM(M, r, c) (M)[2 * ((r) * n + (c)) + 1]
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) { RE(V, r, c) = (r == c) ? 1.0 : 0.0; IM(V, r, c) = 0.0; }
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int p = 0; p < n; ++p) {
            tot += RE(A, p, p) * RE(A, p, p);
            for (int q = p + 1; q < n; ++q)
                off += RE(A, p, q) * RE(A, p, q) + IM(A, p, q) * IM(A, p, q);
        }
        tot += 2.0 * off;
        if (off == 0.0 || off <= 1e-36 * tot) break;
        for (int p = 0; p < n - 1; ++p) {
            for (int q = p + 1; q < n; ++q) {
                double apr = RE(A, p, q), api = IM(A, p, q);
                double mag = hypot(apr, api);
                if (mag == 0.0) continue;
                double er = apr / mag, ei = api / mag;          /* e = a_pq/|a_pq| */
                double theta = (RE(A, q, q) - RE(A, p, p)) / (2.0 * mag);
                double t;
                if (fabs(theta) > 1e150) t = 0.5 / theta;
                else t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double cs = 1.0 / sqrt(t * t + 1.0);
                double sn = t * cs;
                /* s*conj(e) and c*conj(e) */
                double sr = sn * er, si = -sn * ei;
                double cr = cs * er, ci = -cs * ei;
                for (int r = 0; r < n; ++r) {
                    if (r == p || r == q) continue;
                    double xr = RE(A, r, p), xi = IM(A, r, p);
                    double yr = RE(A, r, q), yi = IM(A, r, q);
                    double nrp_r = cs * xr - (sr * yr - si * yi);
                    double nrp_i = cs * xi - (sr * yi + si * yr);
                    double nrq_r = sn * xr + (cr * yr - ci * yi);
                    double nrq_i = sn * xi + (cr * yi + ci * yr);
                    RE(A, r, p) = nrp_r; IM(A, r, p) = nrp_i;
                    RE(A, r, q) = nrq_r; IM(A, r, q) = nrq_i;
                    RE(A, p, r) = nrp_r; IM(A, p, r) = -nrp_i;
                    RE(A, q, r) = nrq_r; IM(A, q, r) = -nrq_i;
                }
                RE(A, p, p) = RE(A, p, p) - t * mag; IM(A, p, p) = 0.0;
                RE(A, q, q) = RE(A, q, q) + t * mag; IM(A, q, q) = 0.0;
                RE(A, p, q) = 0.0; IM(A, p, q) = 0.0;
                RE(A, q, p) = 0.0; IM(A, q, p) = 0.0;
                for (int r = 0; r < n; ++r) {
                    double xr = RE(V, r, p), xi = IM(V, r, p);
                    double yr = RE(V, r, q), yi = IM(V, r, q);
                    RE(V, r, p) = cs * xr - (sr * yr - si * yi);
                    IM(V, r, p) = cs * xi - (sr * yi + si * yr);
                    RE(V, r, q) = sn * xr + (cr * yr - ci * yi);
                    IM(V, r, q) = sn * xi + (cr * yi + ci * yr);
                }
            }
        }
    }
#undef RE
#undef IM
}

lapack_int LAPACKE_cheev(int matrix_layout, char jobz, char uplo, lapack_int n,
                         MKL_Complex8 *a, lapack_int lda, float *w)
{
    /* init_G.h:38 only uses (LAPACK_ROW_MAJOR, 'V', 'L'). */
    if (matrix_layout != LAPACK_ROW_MAJOR || jobz != 'V' || uplo != 'L') {
        fprintf(stderr, "mkl shim: unsupported LAPACKE_cheev form\n");
        abort();
    }
    if (n <= 0) return 0;
    double *A = (double *)malloc(sizeof(double) * 2 * n * n);
    double *V = (double *)malloc(sizeof(double) * 2 * n * n);
    int *ord = (int *)malloc(sizeof(int) * n);
    /* Hermitian matrix from the lower triangle; LAPACK ignores Im(diag). */
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j <= i; ++j) {
            double re = (double)a[i * lda + j].real, im = (double)a[i * lda + j].imag;
            if (i == j) im = 0.0;
            A[2 * (i * n + j)] = re; A[2 * (i * n + j) + 1] = im;
            A[2 * (j * n + i)] = re; A[2 * (j * n + i) + 1] = -im;
        }
    }
    jacobi_hermitian(n, A, V);
    /* stable ascending order of eigenvalues */
    for (int i = 0; i < n; ++i) ord[i] = i;
    for (int i = 1; i < n; ++i) {
        int key = ord[i];
        double kv = A[2 * (key * n + key)];
        int j = i - 1;
        while (j >= 0 && A[2 * (ord[j] * n + ord[j])] > kv) { ord[j + 1] = ord[j]; --j; }
        ord[j + 1] = key;
    }
    for (int k = 0; k < n; ++k) {
        int src = ord[k];
        w[k] = (float)A[2 * (src * n + src)];
        /* phase: first component of largest modulus made real positive */
        int m = 0; double best = -1.0;
        for (int i = 0; i < n; ++i) {
            double mr = V[2 * (i * n + src)], mi = V[2 * (i * n + src) + 1];
            double mm = mr * mr + mi * mi;
            if (mm > best) { best = mm; m = i; }
        }
        double pr = V[2 * (m * n + src)], pi = V[2 * (m * n + src) + 1];
        double pm = hypot(pr, pi);
        double ur = pr / pm, ui = -pi / pm;                 /* conj(v_m)/|v_m| */
        for (int i = 0; i < n; ++i) {
            double vr = V[2 * (i * n + src)], vi = V[2 * (i * n + src) + 1];
            double nr = vr * ur - vi * ui, ni = vr * ui + vi * ur;
            a[i * lda + k].real = (float)nr;
            a[i * lda + k].imag = (float)ni;
        }
    }
    free(A); free(V); free(ord);
    return 0;
}
