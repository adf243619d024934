/*
 * Oracle test infrastructure: plain-C FP64 restatement of the reference's
 * HF-GKBA G1-G2 propagation (VlcekGroup/G12KBA, G12KBA-GW/src/headers).
 * Used only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg as the checker.  The product never links it.
 *
 * Arrays are interleaved (re, im) doubles.  G1 is n x n row-major, n = Ns*Nb,
 * orbital index mu = site + band*Ns (IDX_4D, commutators.h:59).  G2 tensors use
 * the reference layout IDX_8D(k,l,g,d,i,j,a,b) (commutators.h:60).
 */
#ifndef G12_ORACLE_H
#define G12_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Parameters as produced by read_input.h:85-146 (assign_vals). */
typedef struct {
    int Ns, Nb, Nq, time_steps;
    int HF, EHM;            /* booleans */
    int q_pulse;            /* 0: "full", 1: "pulse" (q_type "none" maps to full, qs=0, Nq=0) */
    int vlaw;               /* 0: U*exp(-0.7 r) (AS.h:138), 1: U/(1+r) */
    double t1, t2, t3, U, dt, quench_strength;
    double AS_rate, AS_midpoint, quench_rate, quench_on_midpoint, quench_off_midpoint;
} oracle_params;

double oracle_fermi(double t, double t0, double tau);
int oracle_read_input(const char *path, oracle_params *p, char *log, int logcap);

void oracle_h_HFx_quench(double *h, const double *G1, int Ns, int Nb, double U, double t1,
                         double t2, double w, const double *V, int nV, int Nq);
void oracle_hG_commutator(const double *G, const double *h, double *comm, int n);
void oracle_h2_commutator(const double *G2, const double *h, double *comm, int Ns, int Nb);
void oracle_psi_xxxx(double *psi, const double *G1, int Ns, int Nb, double U, const double *V, int nV);
void oracle_psi_xyxy(double *psi, const double *G1, int Ns, int Nb, double U, const double *V, int nV);
void oracle_pi(double *pi, const double *G1, const double *G2a, const double *G2b, double U,
               int Ns, int Nb, const double *V, int nV);
void oracle_collision(double *I, const double *G2xy, const double *G2xx, int Ns, int Nb, double U,
                      const double *V, int nV);
void oracle_G1_step(const double *comm, const double *I, double *K, double *RK, double w, int n);
void oracle_G2_step(const double *comm, const double *psi, const double *pi, double *K, double *RK,
                    double w, int Ns, int Nb);
void oracle_make_G0(double *G1, int Ns, int Nb, int p_number, double t1, double t2);
void oracle_dipole(double *p, const double *traj, int64_t T, int n);

/* Number of AS steps (AS.h:96-100) and RK4 iterations (RK_solver.h:96,216). */
int64_t oracle_as_steps(const oracle_params *p);
int64_t oracle_rk_iterations(const oracle_params *p);

/* One RK4 step of either phase (AS.h:102-170 / RK_solver.h:112-214).
 * phase 0: adiabatic switching at AS time t; phase 1: RK4 at time t with the
 * quench schedule; *t_temp carries RK_solver.h's stage time across steps. */
void oracle_step(const oracle_params *p, int phase, double t, double *t_temp,
                 double *G1, double *G2xx, double *G2xy);

/* Full Main.cpp pipeline from a given G0: AS then RK4.  traj must hold
 * max_T*n*n complex entries; returns the number of snapshots written (the
 * density guard of RK_solver.h:101-110 stops early). */
int64_t oracle_run(const oracle_params *p, const double *G0, int skip_as, double *traj, int64_t max_T,
                   double *G1_out, double *G2xx_out, double *G2xy_out);

#ifdef __cplusplus
}
#endif
#endif
