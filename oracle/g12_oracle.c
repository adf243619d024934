/*
 * Oracle test infrastructure: plain-C FP64 restatement of the reference
 * algorithm (VlcekGroup/G12KBA, G12KBA-GW/src).  Each function cites the
 * reference lines it restates.  Loops are the reference's naive ones (the
 * O(n^5) commutator, the O(n^4 * Ns * Nb) Psi/Pi), so this file is a checker,
 * not a fast path.  Pinned against the compiled reference (oracle/_ref) by
 * tests/test_oracle.py and against the committed golden vectors.
 */
#include "g12_oracle.h"
#include "mkl_shim/mkl_lapacke.h"
#include <complex.h>
#include <errno.h>
#include <limits.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;
static const cplx IM = 1.0 * _Complex_I;

#define C(p) ((cplx *)(p))
#define CC(p) ((const cplx *)(p))

/* IDX_4D / IDX_8D (commutators.h:59-60) */
#define IDX4(x, y, z, t) ((size_t)((x) + (y) * Ns) + (size_t)((z) + (t) * Ns) * (size_t)(Nb * Ns))
#define IDX8(x, y, z, t, m, nn, q, w)                                                            \
    ((size_t)((x) + (y) * Ns) + (size_t)((z) + (t) * Nb) * Ns2 + (size_t)((m) + (nn) * Ns) * Ns2 * Nb2 + \
     (size_t)((q) + (w) * Nb) * Ns2 * Ns2 * Nb2)

/* fermi_func.h:21-24 */
double oracle_fermi(double t, double t0, double tau) { return 1.0 / (1 + exp((t0 - t) / tau)); }

/* HF.h:57-104: h is zeroed here (the reference always passes a fresh vector). */
void oracle_h_HFx_quench(double *hp, const double *G1p, int Ns, int Nb, double U, double t1,
                         double t2, double w, const double *V, int nV, int Nq)
{
    int n = Ns * Nb;
    cplx *h = C(hp);
    const cplx *G = CC(G1p);
    for (int x = 0; x < n * n; ++x) h[x] = 0;
    for (int i = 0; i < Ns; ++i) {
        for (int a = 0; a < Nb; ++a) {
            int mu = i + a * Ns;
            h[mu * n + mu] += 0.0; /* epsilon[a] is always zero (read_input.h:43) */
            if (i < Nq) h[mu * n + mu] += w;
            if (i < Ns - 1) {
                h[((i + 1) + a * Ns) * n + mu] += -t1;
                h[mu * n + (i + 1) + a * Ns] += -t1;
            }
            if (a < Nb - 1) {
                h[mu * n + (i + (a + 1) * Ns)] += -t2;
                h[(i + (a + 1) * Ns) * n + mu] += -t2;
            }
            h[mu * n + mu] += -IM * U * G[mu * n + mu];
            for (int g = 0; g < Nb; ++g) {
                int ig = i + g * Ns;
                if (g != a) h[mu * n + ig] += IM * U * G[ig * n + mu];
                if (g != a) h[mu * n + mu] += -2.0 * IM * U * G[ig * n + ig];
            }
            for (int m = 1; m <= nV; ++m) {
                if (i + m < Ns) {
                    for (int d = 0; d < Nb; ++d) {
                        int pd = (i + m) + d * Ns, pa = (i + m) + a * Ns, id = i + d * Ns;
                        h[mu * n + mu] += -2.0 * IM * V[m - 1] * G[pd * n + pd];
                        h[pa * n + id] += IM * V[m - 1] * G[pa * n + id];
                        h[mu * n + pd] += IM * V[m - 1] * G[mu * n + pd];
                    }
                }
                if (i - m >= 0) {
                    for (int d = 0; d < Nb; ++d) {
                        int qd = (i - m) + d * Ns;
                        h[mu * n + mu] += -2.0 * IM * V[m - 1] * G[qd * n + qd];
                    }
                }
            }
        }
    }
}

/* commutators.h:28-51: comm = hG - Gh */
void oracle_hG_commutator(const double *Gp, const double *hp, double *commp, int n)
{
    const cplx *G = CC(Gp), *h = CC(hp);
    cplx *comm = C(commp);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            cplx hg = 0, gh = 0;
            for (int k = 0; k < n; ++k) {
                hg += h[i * n + k] * G[k * n + j];
                gh += G[i * n + k] * h[k * n + j];
            }
            comm[i * n + j] = hg - gh;
        }
}

/* commutators.h:53-99 */
void oracle_h2_commutator(const double *G2p, const double *hp, double *commp, int Ns, int Nb)
{
    const cplx *G2 = CC(G2p), *h = CC(hp);
    cplx *comm = C(commp);
    size_t Ns2 = (size_t)Ns * Ns, Nb2 = (size_t)Nb * Nb;
#pragma omp parallel for collapse(4) schedule(static)
    for (int b = 0; b < Nb; ++b)
        for (int a = 0; a < Nb; ++a)
            for (int j = 0; j < Ns; ++j)
                for (int i = 0; i < Ns; ++i)
                    for (int d = 0; d < Nb; ++d)
                        for (int g = 0; g < Nb; ++g)
                            for (int l = 0; l < Ns; ++l)
                                for (int k = 0; k < Ns; ++k) {
                                    cplx acc = 0;
                                    for (int r = 0; r < Nb; ++r)
                                        for (int p = 0; p < Ns; ++p) {
                                            acc += h[IDX4(p, r, j, b)] * G2[IDX8(k, l, g, d, i, p, a, r)];
                                            acc += h[IDX4(p, r, i, a)] * G2[IDX8(k, l, g, d, p, j, r, b)];
                                            acc -= h[IDX4(l, d, p, r)] * G2[IDX8(k, p, g, r, i, j, a, b)];
                                            acc -= h[IDX4(k, g, p, r)] * G2[IDX8(p, l, r, d, i, j, a, b)];
                                        }
                                    comm[IDX8(k, l, g, d, i, j, a, b)] = acc;
                                }
}

/* The long-range (n >= 1) part shared by psi.h:74-142 (xyxy) and psi.h:198-266 (xxxx). */
static cplx psi_long_range(const cplx *G1, int Ns, int Nb, const double *V, int nV, int i, int j,
                           int k, int l, int a, int b, int g, int d)
{
    cplx g2 = G1[IDX4(k, g, i, a)], g3 = G1[IDX4(l, d, j, b)];
    cplx s = 0;
    for (int m = 1; m <= nV; ++m) {
        double v = V[m - 1];
        if (abs(k - l) == m) s += -v * g2 * g3;
        if (abs(i - j) == m) s += v * g2 * g3;
        for (int sgn = 1; sgn >= -1; sgn -= 2) {
            int lp = l + sgn * m, jp = j + sgn * m, kp = k + sgn * m, ip = i + sgn * m;
            if (lp >= 0 && lp < Ns)
                for (int r = 0; r < Nb; ++r) s += -IM * v * G1[IDX4(lp, r, i, a)] * G1[IDX4(k, g, lp, r)] * g3;
            if (jp >= 0 && jp < Ns)
                for (int r = 0; r < Nb; ++r) s += IM * v * G1[IDX4(jp, r, i, a)] * G1[IDX4(k, g, jp, r)] * g3;
            if (kp >= 0 && kp < Ns)
                for (int r = 0; r < Nb; ++r) s += -IM * v * G1[IDX4(kp, r, j, b)] * G1[IDX4(l, d, kp, r)] * g2;
            if (ip >= 0 && ip < Ns)
                for (int r = 0; r < Nb; ++r) s += IM * v * G1[IDX4(ip, r, j, b)] * G1[IDX4(l, d, ip, r)] * g2;
        }
    }
    return s;
}

/* psi.h:26-154 (xy = 1) and psi.h:157-276 (xy = 0) */
static void psi_common(double *psip, const double *G1p, int Ns, int Nb, double U, const double *V,
                       int nV, int xy)
{
    const cplx *G1 = CC(G1p);
    cplx *psi = C(psip);
    size_t Ns2 = (size_t)Ns * Ns, Nb2 = (size_t)Nb * Nb;
#pragma omp parallel for collapse(4) schedule(static)
    for (int i = 0; i < Ns; ++i)
        for (int j = 0; j < Ns; ++j)
            for (int k = 0; k < Ns; ++k)
                for (int l = 0; l < Ns; ++l)
                    for (int a = 0; a < Nb; ++a)
                        for (int b = 0; b < Nb; ++b)
                            for (int g = 0; g < Nb; ++g)
                                for (int d = 0; d < Nb; ++d) {
                                    cplx g2 = G1[IDX4(k, g, i, a)], g3 = G1[IDX4(l, d, j, b)];
                                    double dmask = (double)(i == j) * (double)(a != b) -
                                                   (double)(l == k) * (double)(g != d);
                                    cplx s = U * g2 * g3 * dmask;
                                    for (int r = 0; r < Nb; ++r) {
                                        s += IM * U * (g2 * ((double)(r != a) * G1[IDX4(i, r, j, b)] * G1[IDX4(l, d, i, r)] -
                                                             (double)(r != g) * G1[IDX4(k, r, j, b)] * G1[IDX4(l, d, k, r)]));
                                        s += IM * U * (g3 * ((double)(r != b) * G1[IDX4(j, r, i, a)] * G1[IDX4(k, g, j, r)] -
                                                             (double)(r != d) * G1[IDX4(l, r, i, a)] * G1[IDX4(k, g, l, r)]));
                                    }
                                    if (xy) {
                                        cplx g12 = G1[IDX4(l, d, i, a)], g13 = G1[IDX4(k, g, j, b)];
                                        cplx g14 = G1[IDX4(l, d, k, g)], g15 = G1[IDX4(i, a, j, b)];
                                        cplx g16 = G1[IDX4(k, g, l, d)], g17 = G1[IDX4(j, b, i, a)];
                                        double dd = (double)(k == l) * (double)(d == g) -
                                                    (double)(i == j) * (double)(a == b);
                                        s += -g2 * U * g3 * dd;
                                        s += -IM * g2 * U * (g13 * g14 - g15 * g12);
                                        s += -IM * g3 * U * (g12 * g16 - g17 * g13);
                                    }
                                    s += psi_long_range(G1, Ns, Nb, V, nV, i, j, k, l, a, b, g, d);
                                    psi[IDX8(k, l, g, d, i, j, a, b)] = s;
                                }
}

void oracle_psi_xxxx(double *psi, const double *G1, int Ns, int Nb, double U, const double *V, int nV)
{
    psi_common(psi, G1, Ns, Nb, U, V, nV, 0);
}

void oracle_psi_xyxy(double *psi, const double *G1, int Ns, int Nb, double U, const double *V, int nV)
{
    psi_common(psi, G1, Ns, Nb, U, V, nV, 1);
}

/* pi.h:25-95.  G2a is the routine's third argument ("G2xyxy"), G2b the fourth. */
void oracle_pi(double *pip, const double *G1p, const double *G2ap, const double *G2bp, double U,
               int Ns, int Nb, const double *V, int nV)
{
    const cplx *G1 = CC(G1p), *A = CC(G2ap), *B = CC(G2bp);
    cplx *pi = C(pip);
    size_t Ns2 = (size_t)Ns * Ns, Nb2 = (size_t)Nb * Nb;
#pragma omp parallel for collapse(4) schedule(static)
    for (int i = 0; i < Ns; ++i)
        for (int j = 0; j < Ns; ++j)
            for (int k = 0; k < Ns; ++k)
                for (int l = 0; l < Ns; ++l)
                    for (int a = 0; a < Nb; ++a)
                        for (int b = 0; b < Nb; ++b)
                            for (int g = 0; g < Nb; ++g)
                                for (int d = 0; d < Nb; ++d) {
                                    cplx gy = G1[IDX4(l, d, j, b)];
                                    cplx s = 0;
                                    for (int r = 0; r < Nb; ++r) {
                                        size_t x3 = IDX8(k, j, g, r, i, j, a, r), x4 = IDX8(k, l, g, r, i, l, a, r);
                                        s += -IM * U * gy * (B[x3] * (double)(r != b) - (double)(r != d) * B[x4]);
                                        s += -IM * U * gy * (A[x3] * (double)(r != b) - (double)(r != d) * A[x4]);
                                    }
                                    s += -IM * U * gy * (A[IDX8(k, j, g, b, i, j, a, b)] - A[IDX8(k, l, g, d, i, l, a, d)]);
                                    for (int m = 1; m <= nV; ++m) {
                                        double v = V[m - 1];
                                        if (l + m < Ns)
                                            for (int r = 0; r < Nb; ++r) {
                                                size_t x = IDX8(k, l + m, g, r, i, l + m, a, r);
                                                s += IM * v * gy * (A[x] + B[x]);
                                            }
                                        if (l - m >= 0)
                                            for (int r = 0; r < Nb; ++r) {
                                                size_t x = IDX8(k, l - m, g, r, i, l - m, a, r);
                                                s += IM * v * gy * (A[x] + B[x]);
                                            }
                                        if (j + m < Ns)
                                            for (int r = 0; r < Nb; ++r) {
                                                size_t x = IDX8(k, j + m, g, r, i, j + m, a, r);
                                                s += -IM * v * gy * (A[x] + B[x]);
                                            }
                                        if (j - m >= 0)
                                            for (int r = 0; r < Nb; ++r) {
                                                size_t x = IDX8(k, j - m, g, r, i, j - m, a, r);
                                                s += -IM * v * gy * (A[x] + B[x]);
                                            }
                                    }
                                    pi[IDX8(k, l, g, d, i, j, a, b)] = s;
                                }
}

/* collision_integral.h:27-69 */
void oracle_collision(double *Ip, const double *G2xyp, const double *G2xxp, int Ns, int Nb, double U,
                      const double *V, int nV)
{
    const cplx *XY = CC(G2xyp), *XX = CC(G2xxp);
    cplx *Ix = C(Ip);
    size_t Ns2 = (size_t)Ns * Ns, Nb2 = (size_t)Nb * Nb;
    for (int i = 0; i < Ns; ++i)
        for (int j = 0; j < Ns; ++j)
            for (int a = 0; a < Nb; ++a)
                for (int b = 0; b < Nb; ++b) {
                    cplx s = -IM * U * XY[IDX8(j, i, b, a, i, i, a, a)];
                    for (int m = 0; m < Nb; ++m)
                        if (m != a) {
                            size_t x = IDX8(j, i, b, m, i, i, a, m);
                            s += -IM * U * XX[x];
                            s += -IM * U * XY[x];
                        }
                    for (int m = 1; m <= nV; ++m) {
                        if (i + m < Ns)
                            for (int g = 0; g < Nb; ++g) {
                                size_t x = IDX8(j, i + m, b, g, i, i + m, a, g);
                                s += -IM * V[m - 1] * (XY[x] + XX[x]);
                            }
                        if (i - m >= 0)
                            for (int g = 0; g < Nb; ++g) {
                                size_t x = IDX8(j, i - m, b, g, i, i - m, a, g);
                                s += -IM * V[m - 1] * (XY[x] + XX[x]);
                            }
                    }
                    Ix[IDX4(j, b, i, a)] = s;
                }
}

/* G1_G2_t_step.h:24-47 */
void oracle_G1_step(const double *commp, const double *Ip, double *Kp, double *RKp, double w, int n)
{
    const cplx *comm = CC(commp), *Ix = CC(Ip);
    cplx *K = C(Kp), *RK = C(RKp);
    for (int mu = 0; mu < n; ++mu)
        for (int nu = 0; nu < n; ++nu) {
            K[mu * n + nu] = -IM * (comm[mu * n + nu] + Ix[mu * n + nu] + conj(Ix[nu * n + mu]));
            RK[mu * n + nu] += w * K[mu * n + nu];
        }
}

/* G1_G2_t_step.h:55-86 */
void oracle_G2_step(const double *commp, const double *psip, const double *pip, double *Kp, double *RKp,
                    double w, int Ns, int Nb)
{
    const cplx *comm = CC(commp), *psi = CC(psip), *pi = CC(pip);
    cplx *K = C(Kp), *RK = C(RKp);
    size_t Ns2 = (size_t)Ns * Ns, Nb2 = (size_t)Nb * Nb;
#pragma omp parallel for collapse(4) schedule(static)
    for (int a = 0; a < Nb; ++a)
        for (int b = 0; b < Nb; ++b)
            for (int i = 0; i < Ns; ++i)
                for (int j = 0; j < Ns; ++j)
                    for (int d = 0; d < Nb; ++d)
                        for (int g = 0; g < Nb; ++g)
                            for (int l = 0; l < Ns; ++l)
                                for (int k = 0; k < Ns; ++k) {
                                    size_t x1 = IDX8(k, l, g, d, i, j, a, b);
                                    size_t x2 = IDX8(j, i, b, a, l, k, d, g);
                                    K[x1] = -IM * (comm[x1] + psi[x1] + pi[x1] - conj(pi[x2]));
                                    RK[x1] += w * K[x1];
                                }
}

/* init_G.h:28-75 (eigenstates + make_G0) with the shim's complex64 cheev. */
void oracle_make_G0(double *G1p, int Ns, int Nb, int p_number, double t1, double t2)
{
    int n = Ns * Nb;
    cplx *G1 = C(G1p);
    cplx *h = (cplx *)calloc((size_t)n * n, sizeof(cplx));
    cplx *ev = (cplx *)calloc((size_t)n * n, sizeof(cplx));
    MKL_Complex8 *a = (MKL_Complex8 *)calloc((size_t)n * n, sizeof(MKL_Complex8));
    float *w = (float *)calloc((size_t)n, sizeof(float));
    oracle_h_HFx_quench((double *)h, G1p, Ns, Nb, 0.0, t1, t2, 0.0, NULL, 0, 0);
    for (int j = 0; j < n; ++j)
        for (int i = j; i < n; ++i) {
            a[i * n + j].real = (float)creal(h[i * n + j]);
            a[i * n + j].imag = (float)cimag(h[i * n + j]);
        }
    LAPACKE_cheev(LAPACK_ROW_MAJOR, 'V', 'L', n, a, n, w);
    for (int x = 0; x < n * n; ++x) ev[x] = (double)a[x].real + IM * (double)a[x].imag;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            cplx s = 0;
            for (int k = 0; k < p_number; ++k) s += ev[i * n + k] * conj(ev[j * n + k]) * IM;
            G1[i * n + j] = s;
        }
    free(h); free(ev); free(a); free(w);
}

/* dipole.h:25-32 */
void oracle_dipole(double *p, const double *trajp, int64_t T, int n)
{
    const cplx *traj = CC(trajp);
    int N = n * n;
    double sq = sqrt((double)N);
    for (int64_t t = 0; t < T; ++t) p[t] = 0.0;
    for (int i = 0; i < (int)(sq / 2); ++i)
        for (int64_t t = 0; t < T; ++t)
            p[t] += 2 * (sq / 2 - i - .5) *
                    (cimag(traj[t * N + i * ((int)sq + 1)]) - cimag(traj[t * N + N - i * ((int)sq + 1) - 1])) / sq;
}

/* AS.h:96-100,114-121: the loop runs until |U_AS - U| <= 0 has held at 20 loop
 * heads; U_AS at a loop head is the previous step's last-stage value. */
int64_t oracle_as_steps(const oracle_params *p)
{
    double t = 0, u_as = NAN;
    int count = 0;
    int64_t steps = 0;
    while (count < 20) {
        if (fabs(u_as - p->U) <= 0) count += 1;
        u_as = oracle_fermi(t + .1, p->AS_midpoint, p->AS_rate) * p->U;
        t += .1;
        ++steps;
        if (steps > 100000000) return -1;
    }
    return steps;
}

/* RK_solver.h:66,96,216 */
int64_t oracle_rk_iterations(const oracle_params *p)
{
    double tmax = (double)p->time_steps * p->dt, t = 0;
    int64_t it = 0;
    while (t < tmax) { ++it; t += p->dt; }
    return it;
}

static double vlaw(const oracle_params *p, int r)
{
    if (p->vlaw == 1) return 1.0 / (1.0 + (double)r);
    return exp(-.7 * r);
}

/* One step of AS.h:102-170 (phase 0) or RK_solver.h:112-214 (phase 1). */
void oracle_step(const oracle_params *p, int phase, double t, double *t_temp, double *G1p,
                 double *G2xxp, double *G2xyp)
{
    int Ns = p->Ns, Nb = p->Nb, n = Ns * Nb;
    size_t n2 = (size_t)n * n, n4 = n2 * n2;
    int nV = p->EHM ? Ns - 1 : 0;
    double *V = (double *)calloc(nV > 0 ? nV : 1, sizeof(double));
    cplx *G1 = C(G1p), *XX = C(G2xxp), *XY = C(G2xyp);
    cplx *K1 = calloc(n2, sizeof(cplx)), *RK1 = calloc(n2, sizeof(cplx)), *T1 = calloc(n2, sizeof(cplx));
    cplx *h = calloc(n2, sizeof(cplx)), *c1 = calloc(n2, sizeof(cplx)), *Ix = calloc(n2, sizeof(cplx));
    cplx *Kxx = calloc(n4, sizeof(cplx)), *Kxy = calloc(n4, sizeof(cplx));
    cplx *RKxx = calloc(n4, sizeof(cplx)), *RKxy = calloc(n4, sizeof(cplx));
    cplx *Txx = calloc(n4, sizeof(cplx)), *Txy = calloc(n4, sizeof(cplx));
    cplx *Cxx = calloc(n4, sizeof(cplx)), *Cxy = calloc(n4, sizeof(cplx));
    cplx *Pxx = calloc(n4, sizeof(cplx)), *Pxy = calloc(n4, sizeof(cplx));
    cplx *Qxx = calloc(n4, sizeof(cplx)), *Qxy = calloc(n4, sizeof(cplx));
    double dt_full = phase == 0 ? .1 : p->dt, dt = dt_full;
    int gate = (p->U != 0 && !p->HF);
    for (int k = 0; k < 4; ++k) {
        double w;
        if (k == 1 || k == 2) { dt = dt_full / 2; w = 2; }
        else { dt = dt_full; w = 1; }
        double tk;
        if (phase == 0) tk = (k != 0) ? t + dt : t;
        else { if (k != 0) *t_temp = t + dt; tk = *t_temp; }
        for (size_t x = 0; x < n2; ++x) T1[x] = G1[x] + K1[x] * dt;
        for (size_t x = 0; x < n4; ++x) { Txx[x] = XX[x] + Kxx[x] * dt; Txy[x] = XY[x] + Kxy[x] * dt; }
        double ueff, wq = 0;
        int nq = 0;
        if (phase == 0) {
            ueff = oracle_fermi(tk, p->AS_midpoint, p->AS_rate) * p->U;
            for (int r = 0; r < nV; ++r) V[r] = ueff * vlaw(p, r + 1);
        } else {
            ueff = p->U;
            for (int r = 0; r < nV; ++r) V[r] = p->U * vlaw(p, r + 1);
            if (tk < 50) { wq = 0 * oracle_fermi(tk, p->quench_on_midpoint, p->quench_rate) * p->quench_strength; nq = 0; }
            else if (!p->q_pulse) { wq = oracle_fermi(tk, p->quench_on_midpoint, p->quench_rate) * p->quench_strength; nq = p->Nq; }
            else {
                wq = (oracle_fermi(tk, p->quench_on_midpoint, p->quench_rate) *
                      (1 - oracle_fermi(tk, p->quench_off_midpoint, p->quench_rate))) * p->quench_strength;
                nq = p->Nq;
            }
        }
        oracle_h_HFx_quench((double *)h, (double *)T1, Ns, Nb, ueff, p->t1, p->t2, wq, V, nV, nq);
        oracle_hG_commutator((double *)T1, (double *)h, (double *)c1, n);
        if (gate) {
            oracle_collision((double *)Ix, (double *)Txy, (double *)Txx, Ns, Nb, ueff, V, nV);
            oracle_h2_commutator((double *)Txx, (double *)h, (double *)Cxx, Ns, Nb);
            oracle_h2_commutator((double *)Txy, (double *)h, (double *)Cxy, Ns, Nb);
            oracle_psi_xxxx((double *)Pxx, (double *)T1, Ns, Nb, ueff, V, nV);
            oracle_psi_xyxy((double *)Pxy, (double *)T1, Ns, Nb, ueff, V, nV);
            oracle_pi((double *)Qxx, (double *)T1, (double *)Txy, (double *)Txx, ueff, Ns, Nb, V, nV);
            oracle_pi((double *)Qxy, (double *)T1, (double *)Txx, (double *)Txy, ueff, Ns, Nb, V, nV);
            oracle_G2_step((double *)Cxx, (double *)Pxx, (double *)Qxx, (double *)Kxx, (double *)RKxx, w, Ns, Nb);
            oracle_G2_step((double *)Cxy, (double *)Pxy, (double *)Qxy, (double *)Kxy, (double *)RKxy, w, Ns, Nb);
        }
        oracle_G1_step((double *)c1, (double *)Ix, (double *)K1, (double *)RK1, w, n);
    }
    for (size_t x = 0; x < n2; ++x) G1[x] += RK1[x] * dt / 6.0;
    for (size_t x = 0; x < n4; ++x) { XX[x] += RKxx[x] * dt / 6.0; XY[x] += RKxy[x] * dt / 6.0; }
    free(V); free(K1); free(RK1); free(T1); free(h); free(c1); free(Ix);
    free(Kxx); free(Kxy); free(RKxx); free(RKxy); free(Txx); free(Txy);
    free(Cxx); free(Cxy); free(Pxx); free(Pxy); free(Qxx); free(Qxy);
}

/* Main.cpp:47-58 from a given G0 (AS.h:63-214 then RK_solver.h:64-226). */
int64_t oracle_run(const oracle_params *p, const double *G0, int skip_as, double *traj, int64_t max_T,
                   double *G1_out, double *G2xx_out, double *G2xy_out)
{
    int n = p->Ns * p->Nb;
    size_t n2 = (size_t)n * n, n4 = n2 * n2;
    double *G1 = (double *)malloc(sizeof(double) * 2 * n2);
    double *XX = (double *)calloc(2 * n4, sizeof(double));
    double *XY = (double *)calloc(2 * n4, sizeof(double));
    memcpy(G1, G0, sizeof(double) * 2 * n2);
    if (!skip_as) {
        int64_t steps = oracle_as_steps(p);
        double t = 0, tt = 0;
        for (int64_t s = 0; s < steps; ++s) { oracle_step(p, 0, t, &tt, G1, XX, XY); t += .1; }
    }
    double tmax = (double)p->time_steps * p->dt, t = 0, t_temp = 0;
    int64_t T = 0;
    while (t < tmax) {
        if (T < max_T) memcpy(traj + 2 * n2 * T, G1, sizeof(double) * 2 * n2);
        ++T;
        double num_dens = 2 * G1[1];
        if (fabs(num_dens) > 3 || isnan(num_dens)) break;
        oracle_step(p, 1, t, &t_temp, G1, XX, XY);
        t += p->dt;
    }
    if (G1_out) memcpy(G1_out, G1, sizeof(double) * 2 * n2);
    if (G2xx_out) memcpy(G2xx_out, XX, sizeof(double) * 2 * n4);
    if (G2xy_out) memcpy(G2xy_out, XY, sizeof(double) * 2 * n4);
    free(G1); free(XX); free(XY);
    return T;
}

/* ---- input file (read_input.h:53-146) ---------------------------------- */

typedef struct { char **line; int count; int last_nl; int exists; } lines_t;

static void load_lines(const char *path, lines_t *L)
{
    memset(L, 0, sizeof(*L));
    FILE *f = fopen(path, "rb");
    if (!f) return;
    L->exists = 1;
    size_t cap = 0, len = 0;
    char *buf = NULL;
    int ch, cap_lines = 0;
    int pending = 0;
    while ((ch = fgetc(f)) != EOF) {
        pending = 1;
        if (len + 1 >= cap) { cap = cap ? cap * 2 : 64; buf = (char *)realloc(buf, cap); }
        if (ch == '\n') {
            buf[len] = 0;
            if (L->count == cap_lines) { cap_lines = cap_lines ? cap_lines * 2 : 16; L->line = (char **)realloc(L->line, sizeof(char *) * cap_lines); }
            L->line[L->count++] = strdup(buf);
            len = 0;
            pending = 0;
            L->last_nl = 1;
        } else {
            buf[len++] = (char)ch;
            L->last_nl = 0;
        }
    }
    if (pending) {
        if (!buf) buf = (char *)calloc(1, 1);
        buf[len] = 0;
        if (L->count == cap_lines) { cap_lines = cap_lines ? cap_lines * 2 : 16; L->line = (char **)realloc(L->line, sizeof(char *) * cap_lines); }
        L->line[L->count++] = strdup(buf);
        L->last_nl = 0;
    }
    free(buf);
    fclose(f);
}

static void free_lines(lines_t *L)
{
    for (int i = 0; i < L->count; ++i) free(L->line[i]);
    free(L->line);
}

typedef struct { char *log; int cap; int len; } logbuf_t;

static void logf_(logbuf_t *lb, const char *fmt, ...)
{
    if (!lb->log || lb->cap <= 0) return;
    va_list ap;
    va_start(ap, fmt);
    int r = vsnprintf(lb->log + lb->len, (size_t)(lb->cap - lb->len), fmt, ap);
    va_end(ap);
    if (r > 0) lb->len += r;
    if (lb->len >= lb->cap) lb->len = lb->cap - 1;
}

/* read_input.h:53-83: the line after the first line containing `var`
 * (substring match); past the end of the file std::getline leaves the last
 * extracted string in place, which is "" unless the file lacks a final
 * newline.  An empty result reads as "0" with a message. */
static const char *read_var_val(const lines_t *L, const char *var, logbuf_t *lb)
{
    int counter = 0;
    for (int i = 0; i < L->count; ++i) {
        counter++;
        if (strstr(L->line[i], var)) break;
    }
    const char *s = "";
    if (counter + 1 <= L->count) s = L->line[counter];
    else if (L->exists && L->count > 0 && !L->last_nl) s = L->line[L->count - 1];
    if (s[0] == 0) {
        logf_(lb, "Missing value for %s initialising to 0\n", var);
        return "0";
    }
    return s;
}

static int to_double(const char *s, double *out)
{
    char *end;
    errno = 0;
    double v = strtod(s, &end);
    if (end == s) return -1;
    if (errno == ERANGE) return -2;
    *out = v;
    return 0;
}

static int to_int(const char *s, int *out)
{
    char *end;
    errno = 0;
    long v = strtol(s, &end, 10);
    if (end == s) return -1;
    if (errno == ERANGE || v < INT_MIN || v > INT_MAX) return -2;
    *out = (int)v;
    return 0;
}

/* read_input.h:85-146.  Returns 0, or -1 where the reference's stod/stoi
 * would throw (the reference terminates). */
int oracle_read_input(const char *path, oracle_params *p, char *log, int logcap)
{
    lines_t L;
    logbuf_t lb = {log, logcap, 0};
    if (log && logcap > 0) log[0] = 0;
    load_lines(path, &L);
    /* defaults, read_input.h:27-49 */
    memset(p, 0, sizeof(*p));
    p->t1 = 1; p->U = .5; p->time_steps = 1000; p->dt = .02; p->quench_strength = 1; p->Ns = 2; p->Nb = 1;
    p->AS_rate = 3; p->AS_midpoint = 25; p->quench_rate = .2; p->quench_on_midpoint = 50; p->quench_off_midpoint = 55;
    int rc = 0;
#define RD(key, field) do { if (!rc && to_double(read_var_val(&L, key, &lb), &p->field)) rc = -1; } while (0)
#define RI(key, field) do { if (!rc && to_int(read_var_val(&L, key, &lb), &p->field)) rc = -1; } while (0)
    RD("t1", t1); RD("t2", t2); RD("t3", t3); RD("U", U);
    RI("time_steps", time_steps); RD("dt", dt); RD("quench_strength", quench_strength);
    RI("Ns", Ns); RI("Nb", Nb); RI("Nq", Nq);
    RD("AS_rate", AS_rate); RD("AS_midpoint", AS_midpoint);
    RD("quench_on_midpoint", quench_on_midpoint); RD("quench_off_midpoint", quench_off_midpoint);
    RD("quench_rate", quench_rate);
#undef RD
#undef RI
    if (rc) { free_lines(&L); return -1; }
    if (!strcmp(read_var_val(&L, "HF", &lb), "true")) p->HF = 1;
    else if (!strcmp(read_var_val(&L, "HF", &lb), "false")) p->HF = 0;
    else { logf_(&lb, "Invalid specification of HF calculation parameter, performing full HF-GKBA calculation.\n"); p->HF = 0; }
    if (!strcmp(read_var_val(&L, "EHM", &lb), "true")) p->EHM = 1;
    else if (!strcmp(read_var_val(&L, "EHM", &lb), "false")) p->EHM = 0;
    else { logf_(&lb, "Invalid specification for EHM parameter. performing full calculation for onsite model.\n"); p->EHM = 0; }
    if (!strcmp(read_var_val(&L, "q_type", &lb), "full")) p->q_pulse = 0;
    else if (!strcmp(read_var_val(&L, "q_type", &lb), "pulse")) p->q_pulse = 1;
    else if (!strcmp(read_var_val(&L, "q_type", &lb), "none")) { p->quench_strength = 0; p->Nq = 0; }
    else logf_(&lb, "Invalid specification of quench type, no quench initiated\n");
    free_lines(&L);
    return 0;
}
