/*
 * g12kba - B200-native HF-GKBA G1-G2 propagation with GW self-energy.
 *
 * C ABI of libg12kba.so.  Plain pointers and sizes only.  Complex numbers are
 * interleaved (re, im) doubles.  G1 is n x n row-major with orbital index
 * mu = site + band*Ns (n = Ns*Nb).  G2 tensors handed across this boundary use
 * the reference's flat layout IDX_8D(k,l,g,d,i,j,a,b) =
 *   k + l*Ns + (g + d*Nb)*Ns^2 + (i + j*Ns)*Ns^2*Nb^2 + (a + b*Nb)*Ns^4*Nb^2
 * (G12KBA-GW/src/headers/commutators.h:60), n^4 complex entries each.
 *
 * The reference (VlcekGroup/G12KBA) has no library API: its surface is the
 * `input` file and the text outputs of G12KBA-GW/src/main/Main.cpp:44-62.  The
 * seams these entry points replace are the free functions that Main.cpp calls;
 * each declaration names the one it stands for.
 *
 * Conventions: the caller owns every host buffer, a context owns its device
 * memory; one context per host thread; functions return G12_OK (0), a
 * positive status (G12_GUARD_TRIPPED) or a negative error code, and never
 * throw across the ABI.
 */
#ifndef G12KBA_H
#define G12KBA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define G12_OK 0
#define G12_GUARD_TRIPPED 1       /* RK_solver.h:106-110 density guard (outputs still valid) */
#define G12_ERR_INVALID (-1)      /* bad argument or unsupported size */
#define G12_ERR_CUDA (-2)         /* CUDA runtime failure; see g12_last_error */
#define G12_ERR_NOMEM (-3)
#define G12_ERR_PARSE (-4)        /* input value the reference's stod/stoi rejects */
#define G12_ERR_NO_DEVICE (-5)    /* no CUDA device: there is no CPU fallback */

#define G12_MAX_N 64              /* n = Ns*Nb supported by the kernels */

enum g12_quench { G12_QUENCH_FULL = 0, G12_QUENCH_PULSE = 1 };
enum g12_vlaw { G12_VLAW_EXP = 0, G12_VLAW_INV = 1 };
enum g12_precision {
    G12_PREC_FP64 = 0,    /* plain FP64 path (parity with the reference) */
    G12_PREC_TF32X3 = 1,  /* two-body commutator on tcgen05 kind::tf32: 2 tf32 pieces, 3 products */
    G12_PREC_BF16OZ = 2,  /* tcgen05 kind::f16: exact 8-bit integer digits in bf16 (4 per operand,
                             10 products, exact FP32 partial sums), unbiased; the accurate mixed mode */
    G12_PREC_FP32 = 3,    /* symmetric engine with an FP32 CUDA-core contraction (checker) */
    G12_PREC_TF32X6 = 4,  /* tcgen05 kind::tf32: 3 tf32 pieces per operand, 6 products */
    G12_PREC_FP64SYM = 5  /* symmetric engine entirely in FP64 (FP64 CUDA-core contraction,
                             FP64 stage input and intermediate): the symmetric formulation
                             without any reduced precision */
};
/* The mixed modes (BF16OZ, TF32X3, TF32X6, FP32) and FP64SYM use the symmetric engine: they
 * require the physical G2 symmetries G2[mu2 mu1; nu2 nu1] = G2[mu1 mu2; nu1 nu2]
 * and G2[nu1 nu2; mu1 mu2] = conj(G2[mu1 mu2; nu1 nu2]) (every state reached
 * from G2 = 0 has them; set_state keeps the upper 32 x 32 blocks of G2 seen as
 * an n^2 x n^2 matrix) and keep the RK4 state in FP64.  n = Ns*Nb must be 16 or
 * 32 for the tensor-core modes, 8, 16, 32 or 64 for FP32 and 8, 16 or 32 for
 * FP64SYM.  TF32X3/TF32X6
 * inherit the tensor cores' biased FP32 accumulation (about -4e-8 relative per
 * contraction on B200), which accumulates into a linear phase drift of G1;
 * BF16OZ keeps every partial sum an exact integer and has no such bias. */

/* Run parameters: the globals of read_input.h:27-49 plus the extensions that
 * the reference hard-codes (all defaults reproduce the reference). */
typedef struct g12_params {
    int32_t Ns, Nb, Nq;
    int32_t time_steps;
    int32_t HF, EHM;             /* booleans */
    int32_t q_type;              /* g12_quench; input "none" gives FULL with qs=0, Nq=0 */
    int32_t v_law;               /* g12_vlaw; EXP = U*exp(-0.7 r) as in AS.h:138 */
    double t1, t2, t3, U, dt, quench_strength;
    double AS_rate, AS_midpoint, quench_rate, quench_on_midpoint, quench_off_midpoint;
    double quench_gate;          /* quench off while t < gate (RK_solver.h:141: 50) */
    double as_dt;                /* AS step (AS.h:114-121: 0.1) */
    double decay_rate;           /* EXP law rate (read_input.h:29: 0.7) */
} g12_params;

typedef struct g12_ctx g12_ctx;
typedef struct g12_batch g12_batch;

/* ---- host side: input, schedule, initial state, outputs ---------------- */

/* read_input.h:29-49 defaults. */
void g12_params_default(g12_params *p);

/* read_input.h:53-146 (read_var_val + assign_vals): alternating key/value
 * lines, first line containing the key as a substring.  The messages the
 * reference prints go to `log` (may be NULL).  Extension keys: V_law (exp|inv),
 * quench_gate, AS_dt. */
int g12_read_input(const char *path, g12_params *p, char *log, int32_t logcap);

/* AS.h:96-100 loop count and RK_solver.h:96,216 iteration count. */
int64_t g12_as_steps(const g12_params *p);
int64_t g12_rk_iterations(const g12_params *p);

/* init_G.h:57-75 make_G0(..., p_number = Ns/2, U = 0): complex64 Hermitian
 * eigen-solve of the hopping Hamiltonian, G1 = i * sum_{k<p} v_k v_k^H. */
int g12_make_G0(const g12_params *p, int32_t p_number, double *G1_out);

/* dipole.h:25-32 over T snapshots (host). */
int g12_dipole(const double *traj, int64_t T, int32_t n, double *p_out);

/* Particle number N = 2 Tr Im G1 per snapshot (host).  No counterpart in the
 * reference, which only guards the site-0 density (RK_solver.h:101-110); the
 * equations conserve N exactly, so it checks a propagation. */
int g12_particle_number(const double *traj, int64_t T, int32_t n, double *N_out);

/* write_to_file.h:52-69 (real_/imag_<name>) and :26-34; std::ostream default
 * formatting (6 significant digits). */
int g12_write_cfile2D(const char *name, const double *traj, int64_t T, int32_t n2);
int g12_write_rfile(const char *name, const double *data, int64_t count);

/* ---- device context: one system ---------------------------------------- */

int g12_create(const g12_params *p, int32_t precision, int32_t device, g12_ctx **out);
int g12_destroy(g12_ctx *ctx);
const char *g12_last_error(const g12_ctx *ctx);  /* NULL ctx: last creation error */

/* State in/out (host buffers).  NULL G2 pointers on set mean zero; NULL on
 * get skips that tensor.  set_state also resets the RK4 clock to t = 0. */
int g12_set_state(g12_ctx *ctx, const double *G1, const double *G2xx, const double *G2xy);
int g12_get_state(g12_ctx *ctx, double *G1, double *G2xx, double *G2xy);

/* Adiabatic_switching (AS.h:63-214): all g12_as_steps() steps. */
int g12_adiabatic_switch(g12_ctx *ctx, int64_t *steps_done);

/* RK4 (RK_solver.h:64-226), continued from the context's clock: up to
 * nsteps steps; traj_out (nullable) receives the snapshot of G1 taken at the
 * start of each step (nsteps * n*n complex).  Returns G12_GUARD_TRIPPED when
 * the site-0 density guard stops the run (*steps_done snapshots written, the
 * last one the offending state). */
int g12_propagate(g12_ctx *ctx, int64_t nsteps, double *traj_out, int64_t *steps_done);

/* Same, with the trajectory left on the device: dipole_out (nullable, host)
 * receives dipole.h:25-32 per snapshot, reduced on the GPU. */
int g12_propagate_dipole(g12_ctx *ctx, int64_t nsteps, double *dipole_out, int64_t *steps_done);

/* One right-hand-side evaluation on the given state (host buffers, G2 in the
 * reference layout) with explicit stage scalars; returns the terms the
 * reference computes in one RK stage (RK_solver.h:141-169):
 *   h (HF.h:57), comm1 (commutators.h:28), Ix (collision_integral.h:27),
 *   K1 (G1_G2_t_step.h:24), K2xx / K2xy (G1_G2_t_step.h:55, which combine
 *   commutators.h:53, psi.h:26/157 and pi.h:25).
 * V is U_eff * law(r) for r = 1..Ns-1 when EHM.  Any output may be NULL. */
int g12_rhs(g12_ctx *ctx, const double *G1, const double *G2xx, const double *G2xy,
            double U_eff, double w_quench, int32_t Nq_eff,
            double *h, double *comm1, double *Ix, double *K1, double *K2xx, double *K2xy);

/* Total energy of the context's current state, reduced on the GPU in FP64.
 * No counterpart in the reference; it is the energy the G1-G2 equations
 * conserve while h0 and U are constant (no quench ramp, after adiabatic
 * switching):
 *   E = 2 Tr[h0 rho] + Tr[(h - h0) rho]
 *       - Re sum_{p,q} (w_xx(p,q) G2xx[p q; p q] + w_xy(p,q) G2xy[p q; p q]),
 * rho = -i G1, h = HF.h:57-104 at (U_eff, w_quench, Nq_eff), h0 = h at U = 0,
 * w the pair interaction of collision_integral.h:41-62 (U on one site, 0
 * for the same orbital in xx; V_m = U_eff law(m) between sites m apart).
 * E_out[4] = {E, 2 Tr[h0 rho], Tr[(h - h0) rho], correlation part}. */
int g12_total_energy(g12_ctx *ctx, double U_eff, double w_quench, int32_t Nq_eff, double *E_out);

/* Device time of the last g12_propagate* call's kernels (CUDA events, ms). */
double g12_last_device_ms(const g12_ctx *ctx);

/* Number of kernel launches one RK4 step issues (graph nodes). */
int32_t g12_launches_per_step(const g12_ctx *ctx);

/* Profiling: runs `nsteps` RK4 steps kernel by kernel (no graph) with CUDA
 * events around every launch on the context's stream and returns the number
 * of kernel kinds; avg_ms[i] (i < cap) receives kind i's mean launch time and
 * calls_per_step[i] (nullable) its launches per step.  Advances the state. */
int32_t g12_kernel_times(g12_ctx *ctx, int32_t nsteps, double *avg_ms, int32_t *calls_per_step, int32_t cap);
const char *g12_kernel_name(const g12_ctx *ctx, int32_t kind);

/* Measurement aid: with bytes > 0, g12_propagate* and g12_adiabatic_switch
 * time every RK4 step on its own (CUDA events around the step's graph) and, after
 * each step's end event, write `bytes` bytes of a private device buffer, so that
 * every timed step starts with the state evicted from L2 (126 MB on B200) and the
 * eviction write itself is not timed (g12_last_device_ms sums the steps);
 * g12_kernel_times writes it between steps.  0 (the default) switches it off.  No
 * counterpart in the reference. */
int32_t g12_set_l2_eviction(g12_ctx *ctx, int64_t bytes);

/* Measured FP64 FMA throughput of `device` (TFLOP/s, 2 flops per FMA): the
 * FP64 roofline denominator, which the tensor-core peaks do not cover. */
double g12_fp64_peak_tflops(int32_t device);

/* ---- batched ensembles ---------------------------------------------------
 * Many independent systems (each with its own g12_params: Ns, Nb, U, t2,
 * quench, ...) advanced together by the FP64 engine: every RK4 stage is one
 * launch per kernel kind for the whole ensemble, each step one CUDA graph.
 * Each system's results equal what a single-system context computes.  The
 * row/column-mixing tile (matrices per block) is autotuned per n at creation.
 * No counterpart in the reference (which runs one system per process); the
 * per-system semantics are those of AS.h:63 / RK_solver.h:64. */
int g12_batch_create(const g12_params *systems, int32_t nsys, int32_t precision, int32_t device,
                     g12_batch **out);
int g12_batch_destroy(g12_batch *b);
const char *g12_batch_last_error(const g12_batch *b);  /* NULL: last creation error */
int g12_batch_set_state(g12_batch *b, int32_t i, const double *G1, const double *G2xx, const double *G2xy);
int g12_batch_get_state(g12_batch *b, int32_t i, double *G1, double *G2xx, double *G2xy);
/* each system runs its own g12_as_steps() steps; the ensemble takes the maximum */
int g12_batch_adiabatic_switch(g12_batch *b, int64_t *steps_done);
/* nsteps RK4 steps of every system; dipole_out (nullable) is nsys x nsteps */
int g12_batch_propagate(g12_batch *b, int64_t nsteps, double *dipole_out, int64_t *steps_done);
double g12_batch_last_device_ms(const g12_batch *b);
int32_t g12_batch_tile(const g12_batch *b, int32_t i);  /* autotuned matrices per block of system i */

/* ---- allocation-free entry point ----------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * code whose device memory is owned by another allocator (a caching or arena
 * allocator that already reserved it) and latency-critical loops that cannot
 * afford cudaMalloc's implicit synchronisation.  Computes what g12_rhs returns
 * as K1, K2xx, K2xy, on caller-provided device buffers (G2 in the reference
 * layout, interleaved complex128), enqueued on `stream` (NULL: the legacy
 * default stream) on the current device.  All scratch lives in one static
 * device array of about 6.4 MiB that every GPU loading the library holds until
 * exit; n = Ns*Nb above G12_NOALLOC_MAX_N is rejected (G12_ERR_INVALID, message
 * in `err`).  Calls share that array: calls whose GPU work overlaps race and
 * must be serialised by the caller.  The first call on a device performs a
 * one-time set-up (symbol address lookup, kernel attributes) and should come
 * before any stream capture; that set-up is kept per device ordinal and does
 * not survive cudaDeviceReset.  A CUDA error left pending by earlier work is
 * reported as such (G12_ERR_CUDA, nothing launched). */
#define G12_NOALLOC_MAX_N 16
int g12_rhs_noalloc(const g12_params *p, const double *G1_dev, const double *G2xx_dev,
                    const double *G2xy_dev, double U_eff, double w_quench, int32_t Nq_eff,
                    double *K1_dev, double *K2xx_dev, double *K2xy_dev, void *stream,
                    char *err, int32_t errcap);

/* ---- learned G1 extrapolator ---------------------------------------------
 * No counterpart in the reference (it has no learned component).  An MLP
 * dims[0] -> dims[1] -> dims[2] -> dims[3] -> dims[4] (GELU after the first
 * three layers) maps a window of K past G1 snapshots to the next M snapshots.
 * Snapshot features: rho = -i G1, upper triangle (mu <= nu, row-major), the
 * n(n+1)/2 real parts then the imaginary parts: F = n(n+1) floats.
 * Input slots k < K-1 hold (x_{t-K+1+k} - x_t)/s_in, slot K-1 (x_t - mean)/s_abs;
 * outputs are (x_{t+1+m} - x_t)/s_out.  Weights are FP32 masters rounded to
 * bf16 in every tcgen05 GEMM (FP32 accumulation); training is Adam on MSE.
 * Widths must be multiples of 128; batches multiples of 128 (rollouts pad).
 * Pointers named *_dev are device memory; everything else is host memory. */
typedef struct g12_mlp g12_mlp;
int g12_mlp_create(const int32_t *dims, int32_t max_batch, uint64_t seed, int32_t device, g12_mlp **out);
int g12_mlp_destroy(g12_mlp *m);
const char *g12_mlp_last_error(const g12_mlp *m);  /* NULL: last creation error */
int64_t g12_mlp_param_count(const g12_mlp *m);
/* parameters / gradients, per layer W ([out][in]) then b, FP32 */
int g12_mlp_set_params(g12_mlp *m, const float *params);
int g12_mlp_get_params(g12_mlp *m, float *params);
int g12_mlp_get_grads(g12_mlp *m, float *grads);
int g12_mlp_forward(g12_mlp *m, const float *X_dev, int32_t batch, float *Y_dev);
/* mean squared error of forward(X) against Y and all parameter gradients */
int g12_mlp_loss_grad(g12_mlp *m, const float *X_dev, const float *Y_dev, int32_t batch, double *loss);
int g12_mlp_adam(g12_mlp *m, float lr, float beta1, float beta2, float eps, float weight_decay);
int g12_mlp_set_norm(g12_mlp *m, int32_t K, int32_t M, int32_t F, const float *mean, float s_in, float s_abs,
                     float s_out);
/* windows of feat_dev [ntraj][snaps][F]: idx = batch pairs (trajectory, t),
 * t the window's last snapshot (K-1 <= t, t+M < snaps) */
int g12_mlp_windows(g12_mlp *m, const float *feat_dev, int32_t ntraj, int64_t snaps, const int64_t *idx,
                    int32_t batch, float *X_dev, float *Y_dev);
int g12_mlp_train_windows(g12_mlp *m, const float *feat_dev, int32_t ntraj, int64_t snaps, const int64_t *idx,
                          int32_t batch, float lr, float weight_decay, double *loss);
/* windows, loss and gradients of one batch without the Adam step (returns
 * once the gradients are complete on the device) */
int g12_mlp_grad_windows(g12_mlp *m, const float *feat_dev, int32_t ntraj, int64_t snaps, const int64_t *idx,
                         int32_t batch, double *loss);
/* the device block holding every weight and bias gradient (segments padded to
 * 64 floats, padding zero): data-parallel training reduces it across ranks
 * between g12_mlp_grad_windows and g12_mlp_adam */
int g12_mlp_grad_buffer(g12_mlp *m, float **grads_dev, int64_t *count);
/* one step after r blocks of the network's own rollout from windows ending at
 * idx's t (targets: the true snapshots that follow); noise: Gaussian input
 * noise in normalised units (0: none) */
int g12_mlp_train_pushforward(g12_mlp *m, const float *feat_dev, int32_t ntraj, int64_t snaps, const int64_t *idx,
                              int32_t batch, int32_t r, float noise, float lr, float weight_decay, double *loss);
/* in place: snapshots t0+1 .. snaps-1 of every trajectory from blocks of M
 * predictions ((snaps-1-t0) % M == 0); device time in *elapsed_ms */
int g12_mlp_rollout(g12_mlp *m, float *feat_dev, int32_t ntraj, int64_t snaps, int64_t t0, float *elapsed_ms);
/* The plain-RK4 judge of a rollout: pred_dev and ref_dev [ntraj][snaps][F]
 * (the network's and the RK4 snapshot features of the same trajectories, F as
 * set by g12_mlp_set_norm); the dipole (dipole.h:25-32) of both after t0, the
 * running maximum of |p_pred - p_ref| / max |p_ref| (the RK4 maximum after
 * t0), and accepted_out[b] (host) = the snapshots after t0 up to the last
 * checkpoint (every `every` snapshots) at which it is still <= tol (all
 * snapshots after t0 when every full checkpoint passes). */
int g12_mlp_judge(g12_mlp *m, const float *pred_dev, const float *ref_dev, int32_t ntraj, int64_t snaps, int64_t t0,
                  int32_t every, double tol, int64_t *accepted_out);

/* Batched propagation recording snapshot features (the layout above) of every
 * system after every `every`-th step into feat_dev [nsys][nsteps/every][F]
 * (device memory); all systems must share n.  dipole_out as g12_batch_propagate. */
int g12_batch_propagate_features(g12_batch *b, int64_t nsteps, int32_t every, float *feat_dev, double *dipole_out,
                                 int64_t *steps_done);

#ifdef __cplusplus
}
#endif

#endif /* G12KBA_H */
