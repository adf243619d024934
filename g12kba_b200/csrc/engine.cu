// Device context of libg12kba.so: buffers, the per-step CUDA graph, the
// schedule of stage scalars, and the C-ABI entry points that drive them.
#include "g12kba.h"
#include "internal.h"
#include "fp64_kernels.cuh"
#include "mixed.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

using namespace g12;

namespace {

thread_local std::string g_create_error;

struct LaunchCfg {
    ApplyCfg ab, cd;
    bool tc = false;         // FP64 tensor-core (DMMA) two-body halves
    ApplyTcCfg tcc{};
    size_t tc_ab_smem = 0, tc_cd_smem = 0;
    dim3 tc_grid;
    int ab_threads, cd_threads;
    size_t ab_smem, cd_smem, prep_smem, g1_smem;
    dim3 apply_grid;
    int prep_blocks, g1_blocks;
    int prep_wide_blocks;    // k_prep_wide (mixed engine, n = 32)
    size_t prep_wide_smem;
    int steps_per_graph;
};

}  // namespace

struct g12_ctx {
    g12_params P{};
    int prec = G12_PREC_FP64;
    int device = 0;
    std::string err;
    int Ns = 0, Nb = 0, n = 0;
    long long n2 = 0, n3 = 0, n4 = 0;
    Dev d{};
    LaunchCfg lc{};
    MixedState mixed{};
    cudaStream_t s = nullptr;
    cudaStream_t s2 = nullptr;                 // side branch of the captured step (k_g1)
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaGraphExec_t graph = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // snapshot copies of a finished half of the trajectory ring, overlapped with
    // the next half's steps: copy stream, per-half events (start and end of the
    // half's steps, end of its copy) and the guard status after each half (pinned)
    cudaStream_t s_copy = nullptr;
    cudaEvent_t ev_hs[2] = {}, ev_he[2] = {}, ev_hc[2] = {};
    int *status_h = nullptr;
    StepP *sched_dev = nullptr;
    long long sched_cap = 0;
    StepP *sched_host = nullptr;  // pinned
    long long traj_cap = 0;
    double t_rk = 0, t_temp = 0;   // RK4 clock (RK_solver.h:78-80)
    float last_ms = 0;
    std::vector<void *> allocs;
    void *evict_buf = nullptr;      // g12_set_l2_eviction: written after every step
    size_t evict_bytes = 0;
    double *energy_dev = nullptr;   // g12_total_energy result (4 doubles)
    std::vector<cudaEvent_t> ring;  // per-step event pairs of the eviction timing
};

namespace {

bool ck(g12_ctx *c, cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return true;
    if (c) c->err = std::string(what) + ": " + cudaGetErrorString(e);
    else g_create_error = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}

#define CK(call)                                   \
    do {                                           \
        if (!ck(ctx, (call), #call)) return G12_ERR_CUDA; \
    } while (0)

template <typename T>
bool dalloc(g12_ctx *ctx, T **p, size_t count)
{
    void *q = nullptr;
    if (!ck(ctx, cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)), "cudaMalloc")) return false;
    cudaMemset(q, 0, std::max<size_t>(count, 1) * sizeof(T));
    ctx->allocs.push_back(q);
    *p = (T *)q;
    return true;
}

double vlaw(const g12_params &P, int r)
{
    // AS.h:138 / RK_solver.h:74: U*exp(-decay_rate*(i+1)); extension: U/(1+r)
    if (P.v_law == G12_VLAW_INV) return 1.0 / (1.0 + double(r));
    return std::exp(-P.decay_rate * r);
}

ApplyCfg make_apply_cfg(int n, bool cd, size_t *smem, int *threads)
{
    ApplyCfg c;
    c.NP = (n + 3) / 4 * 4;
    c.S = c.NP / 4;
    c.LD = c.NP + 1;
    const int per = c.S * c.S;
    c.NB = std::max(1, std::min(n * n, 256 / per));
    auto bytes = [&](int nb) {
        size_t b = (size_t(2) * c.NP * c.LD + size_t(nb) * c.NP * c.LD) * sizeof(double2);
        if (cd) b += size_t(n) * n * sizeof(double2);
        return b;
    };
    while (c.NB > 1 && bytes(c.NB) > 200 * 1024) c.NB--;
    *smem = bytes(c.NB);
    *threads = c.NB * per;
    return c;
}

void stage_dt(double dt_full, int k, double *dtk, double *w)
{
    if (k == 1 || k == 2) {
        *dtk = dt_full / 2;
        *w = 2;
    } else {
        *dtk = dt_full;
        *w = 1;
    }
}

// AS.h:102-141 scalars for `steps` steps from AS time 0.
void build_as_sched(const g12_params &P, long long steps, StepP *out)
{
    double t = 0;
    for (long long s = 0; s < steps; ++s) {
        StepP sp{};
        sp.record = 0;
        for (int k = 0; k < 4; ++k) {
            double dtk, w;
            stage_dt(P.as_dt, k, &dtk, &w);
            const double t_rk = (k != 0) ? t + dtk : t;
            StageP &st = sp.st[k];
            st.U = fermi(t_rk, P.AS_midpoint, P.AS_rate) * P.U;
            st.wq = 0;
            st.nq = 0;
            st.w = w;
            st.dt = P.as_dt;
            double dn = 0, wn = 0;
            if (k < 3) stage_dt(P.as_dt, k + 1, &dn, &wn);
            st.c_next = dn;
        }
        out[s] = sp;
        t += P.as_dt;
    }
}

// RK_solver.h:120-151 scalars, continuing the context's clock.
void build_rk_sched(const g12_params &P, long long steps, double *t_io, double *t_temp_io, StepP *out)
{
    double t = *t_io, t_temp = *t_temp_io;
    for (long long s = 0; s < steps; ++s) {
        StepP sp{};
        sp.record = 1;
        for (int k = 0; k < 4; ++k) {
            double dtk, w;
            stage_dt(P.dt, k, &dtk, &w);
            if (k != 0) t_temp = t + dtk;
            StageP &st = sp.st[k];
            st.U = P.U;
            st.w = w;
            st.dt = P.dt;
            if (t_temp < P.quench_gate) {
                st.wq = 0 * fermi(t_temp, P.quench_on_midpoint, P.quench_rate) * P.quench_strength;
                st.nq = 0;
            } else if (P.q_type == G12_QUENCH_PULSE) {
                st.wq = (fermi(t_temp, P.quench_on_midpoint, P.quench_rate) *
                         (1 - fermi(t_temp, P.quench_off_midpoint, P.quench_rate))) *
                        P.quench_strength;
                st.nq = P.Nq;
            } else {
                st.wq = fermi(t_temp, P.quench_on_midpoint, P.quench_rate) * P.quench_strength;
                st.nq = P.Nq;
            }
            double dn = 0, wn = 0;
            if (k < 3) stage_dt(P.dt, k + 1, &dn, &wn);
            st.c_next = dn;
        }
        out[s] = sp;
        t += P.dt;
    }
    *t_io = t;
    *t_temp_io = t_temp;
}

int ensure_sched(g12_ctx *ctx, long long steps)
{
    if (steps <= ctx->sched_cap) return G12_OK;
    if (ctx->sched_dev) cudaFree(ctx->sched_dev);
    if (ctx->sched_host) cudaFreeHost(ctx->sched_host);
    ctx->sched_dev = nullptr;
    ctx->sched_host = nullptr;
    long long cap = std::max<long long>(steps, 1024);
    CK(cudaMalloc(&ctx->sched_dev, cap * sizeof(StepP)));
    CK(cudaMallocHost(&ctx->sched_host, cap * sizeof(StepP)));
    ctx->sched_cap = cap;
    // the graph bakes the Dev struct by value: rebuild it with the new pointer
    ctx->d.sched = ctx->sched_dev;
    if (ctx->graph) {
        cudaGraphExecDestroy(ctx->graph);
        ctx->graph = nullptr;
    }
    return G12_OK;
}

// The two halves of the FP64 two-body commutator with the fused epilogue:
// q = 0 rows (particle indices), q = 1 columns + epilogue; -1 both.
void enqueue_apply(const LaunchCfg &lc, const Dev &d, int k, cudaStream_t s, int q = -1)
{
    if (lc.tc) {
        if (q != 1) launch_apply_tc<false>(lc.tc_grid, lc.tc_ab_smem, s, d, k, lc.tcc);
        if (q != 0) launch_apply_tc<true>(lc.tc_grid, lc.tc_cd_smem, s, d, k, lc.tcc);
    } else {
        if (q != 1) k_apply<false><<<lc.apply_grid, lc.ab_threads, lc.ab_smem, s>>>(d, k, lc.ab);
        if (q != 0) k_apply<true><<<lc.apply_grid, lc.cd_threads, lc.cd_smem, s>>>(d, k, lc.cd);
    }
}

// The stage tables.  On the mixed engine at n = 32 in 16-warp blocks: 66 blocks
// instead of 264 leave SMs free, so that the digit GEMM (launched
// programmatically after it) starts its first CTAs, those with a fourth tile,
// while k_prep runs (a GEMM CTA does not fit beside a k_prep block).
inline bool prep_is_wide(bool mixed_path, const Dev &d) { return mixed_path && d.n == 32; }

inline void enqueue_prep(const LaunchCfg &lc, const Dev &d, int k, cudaStream_t s, bool mixed_path)
{
    if (prep_is_wide(mixed_path, d))
        k_prep_wide<<<lc.prep_wide_blocks, kPrepWarpsWide * 32, lc.prep_wide_smem, s>>>(d, k);
    else
        k_prep<<<lc.prep_blocks, kPrepWarps * 32, lc.prep_smem, s>>>(d, k);
}

// One RK4 step.  k_g1 of stage k only feeds k_prep of stage k+1, so it runs
// on a side branch (s2) concurrently with the two-body kernels of stage k.
void enqueue_step(g12_ctx *ctx, const Dev &d, cudaStream_t s)
{
    const LaunchCfg &lc = ctx->lc;
    k_step_begin<<<1, 256, 0, s>>>(d);
    const bool mixed_path = ctx->prec != G12_PREC_FP64 && d.gate && mixed_fuses_g1(ctx->mixed);
    for (int k = 0; k < 4; ++k) {
        enqueue_prep(lc, d, k, s, mixed_path);
        if (mixed_path) {
            // digit GEMM, then the epilogue with the G1 side as extra blocks of
            // its launch (two launches per stage after k_prep).  (Running
            // k_prep's table blocks on a side stream beside the GEMM was
            // measured slower: the join before the epilogue costs it its
            // programmatic launch.)
            mixed_enqueue_kind(ctx->mixed, d, k, ctx->prec, 0, s);
            mixed_enqueue_kind(ctx->mixed, d, k, ctx->prec, 1, s, true);
            continue;
        }
        if (ctx->prec != G12_PREC_FP64 && d.gate) {
            // symmetric engine: k_g1 forks after the GEMM (one 201 KB CTA per SM,
            // which k_g1's blocks would keep off their SMs) and overlaps the epilogue
            mixed_enqueue_kind(ctx->mixed, d, k, ctx->prec, 0, s);
            cudaEventRecord(ctx->ev_fork, s);
            cudaStreamWaitEvent(ctx->s2, ctx->ev_fork, 0);
            k_g1<<<lc.g1_blocks, kG1Threads, lc.g1_smem, ctx->s2>>>(d, k);
            cudaEventRecord(ctx->ev_join, ctx->s2);
            mixed_enqueue_kind(ctx->mixed, d, k, ctx->prec, 1, s);
            cudaStreamWaitEvent(s, ctx->ev_join, 0);
            continue;
        }
        cudaEventRecord(ctx->ev_fork, s);
        cudaStreamWaitEvent(ctx->s2, ctx->ev_fork, 0);
        k_g1<<<lc.g1_blocks, kG1Threads, lc.g1_smem, ctx->s2>>>(d, k);
        cudaEventRecord(ctx->ev_join, ctx->s2);
        if (d.gate) {
            if (ctx->prec == G12_PREC_FP64) {
                enqueue_apply(lc, d, k, s);
            } else {
                mixed_enqueue_stage(ctx->mixed, d, k, ctx->prec, s);
            }
        }
        cudaStreamWaitEvent(s, ctx->ev_join, 0);
    }
}

int build_graph(g12_ctx *ctx)
{
    if (ctx->graph) return G12_OK;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(ctx->s, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < ctx->lc.steps_per_graph; ++i) enqueue_step(ctx, ctx->d, ctx->s);
    CK(cudaStreamEndCapture(ctx->s, &g));
    cudaError_t e = cudaGraphInstantiate(&ctx->graph, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    return G12_OK;
}

// Runs `steps` scheduled steps (already in sched_host) through the graph.
// traj_out / dip_out (host, nullable) receive one entry per recorded step.
// The steps in halves of the snapshot ring: while half h's steps run, the
// previous half's snapshots and dipoles are copied to the caller's buffers on
// the copy stream; a half's steps wait (on the device) for the copy of the
// half that used the same ring slots two halves earlier.  The guard status is
// read after each half (pinned word); a tripped guard ends the call there.
int run_steps_overlapped(g12_ctx *ctx, long long steps, double *traj_out, double *dip_out, bool recorded,
                         long long *done)
{
    const long long G = ctx->lc.steps_per_graph;
    const long long half = std::max<long long>(G, (ctx->traj_cap / 2) / G * G);
    CK(cudaMemcpyAsync(ctx->d.limit, &steps, sizeof(long long), cudaMemcpyHostToDevice, ctx->s));
    const long long nh = (steps + half - 1) / half;
    float total_ms = 0;
    // finish half c: its status, its time, its copies
    auto finish = [&](long long c, long long *got_out) -> int {
        const int h = int(c & 1);
        const long long b = c * half, len = std::min(half, steps - b);
        CK(cudaEventSynchronize(ctx->ev_he[h]));
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev_hs[h], ctx->ev_he[h]);
        total_ms += ms;
        const int status = ctx->status_h[h];
        long long got = len;
        if (status > 0) got = std::min(len, (long long)status - b);  // guard at step status-1
        if (recorded && got > 0) {
            const long long off = b % ctx->traj_cap;
            CK(cudaStreamWaitEvent(ctx->s_copy, ctx->ev_he[h], 0));
            if (traj_out)
                CK(cudaMemcpyAsync(traj_out + 2 * b * ctx->n2, ctx->d.traj + off * ctx->n2,
                                   got * ctx->n2 * sizeof(double2), cudaMemcpyDeviceToHost, ctx->s_copy));
            if (dip_out)
                CK(cudaMemcpyAsync(dip_out + b, ctx->d.dip + off, got * sizeof(double), cudaMemcpyDeviceToHost,
                                   ctx->s_copy));
        }
        CK(cudaEventRecord(ctx->ev_hc[h], ctx->s_copy));
        if (ctx->prec != G12_PREC_FP64) {
            const int me = mixed_error(ctx->mixed);
            if (me) {
                ctx->err = "tensor-core pipeline wait expired (code " + std::to_string(me) + ")";
                return G12_ERR_CUDA;
            }
        }
        *got_out = got;
        return status > 0 ? G12_GUARD_TRIPPED : G12_OK;
    };
    long long base = 0;
    int rc = G12_OK;
    for (long long c = 0; c < nh && rc == G12_OK; ++c) {
        const int h = int(c & 1);
        const long long len = std::min(half, steps - c * half);
        // ring slots of this half: free once the copy of half c - 2 is done
        if (c >= 2) CK(cudaStreamWaitEvent(ctx->s, ctx->ev_hc[h], 0));
        CK(cudaEventRecord(ctx->ev_hs[h], ctx->s));
        for (long long q = 0; q < len; q += G) CK(cudaGraphLaunch(ctx->graph, ctx->s));
        CK(cudaMemcpyAsync(&ctx->status_h[h], ctx->d.status, sizeof(int), cudaMemcpyDeviceToHost, ctx->s));
        CK(cudaEventRecord(ctx->ev_he[h], ctx->s));
        if (c >= 1) {
            long long got = 0;
            rc = finish(c - 1, &got);
            base += got;
        }
    }
    if (rc == G12_OK) {
        long long got = 0;
        rc = finish(nh - 1, &got);
        base += got;
    }
    // a tripped guard leaves the queued half inert (its steps return at once)
    CK(cudaStreamSynchronize(ctx->s));
    CK(cudaStreamSynchronize(ctx->s_copy));
    *done = base;
    ctx->last_ms = total_ms;
    return rc;
}

int run_steps(g12_ctx *ctx, long long steps, double *traj_out, double *dip_out, long long *done)
{
    *done = 0;
    if (steps <= 0) return G12_OK;
    int rc = build_graph(ctx);
    if (rc) return rc;
    CK(cudaMemcpyAsync(ctx->sched_dev, ctx->sched_host, steps * sizeof(StepP), cudaMemcpyHostToDevice, ctx->s));
    const long long zero = 0;
    CK(cudaMemcpyAsync(ctx->d.counter, &zero, sizeof(long long), cudaMemcpyHostToDevice, ctx->s));
    CK(cudaMemsetAsync(ctx->d.status, 0, sizeof(int), ctx->s));
    const bool recorded = ctx->sched_host[0].record != 0;
    float total_ms = 0;
    long long base = 0;
    if (!ctx->evict_bytes && ctx->traj_cap >= 2 * ctx->lc.steps_per_graph)
        return run_steps_overlapped(ctx, steps, traj_out, dip_out, recorded, done);
    while (base < steps) {
        const long long chunk = std::min(steps - base, ctx->traj_cap);
        const long long lim = base + chunk;
        CK(cudaMemcpyAsync(ctx->d.limit, &lim, sizeof(long long), cudaMemcpyHostToDevice, ctx->s));
        CK(cudaStreamSynchronize(ctx->s));
        const int G = ctx->lc.steps_per_graph;
        if (ctx->evict_bytes) {
            // L2 eviction between timed graph launches: each launch is timed on
            // its own (an event pair around it) and the eviction write follows
            // its end event.  The launches are queued ahead of the device (a ring
            // of event pairs, read back every kRing launches), so no host
            // submission gap falls inside a timed span.
            constexpr int kRing = 32;
            if (ctx->ring.empty()) {
                ctx->ring.resize(2 * kRing);
                for (auto &e : ctx->ring) CK(cudaEventCreate(&e));
            }
            int used = 0;
            auto drain = [&]() -> bool {
                if (!used) return true;
                if (!ck(ctx, cudaEventSynchronize(ctx->ring[2 * used - 1]), "cudaEventSynchronize")) return false;
                for (int j = 0; j < used; ++j) {
                    float ms = 0;
                    cudaEventElapsedTime(&ms, ctx->ring[2 * j], ctx->ring[2 * j + 1]);
                    total_ms += ms;
                }
                used = 0;
                return true;
            };
            for (long long q = 0; q < chunk; q += G) {
                CK(cudaEventRecord(ctx->ring[2 * used], ctx->s));
                CK(cudaGraphLaunch(ctx->graph, ctx->s));
                CK(cudaEventRecord(ctx->ring[2 * used + 1], ctx->s));
                CK(cudaMemsetAsync(ctx->evict_buf, 0, ctx->evict_bytes, ctx->s));
                if (++used == kRing && !drain()) return G12_ERR_CUDA;
            }
            if (!drain()) return G12_ERR_CUDA;
        } else {
            CK(cudaEventRecord(ctx->ev0, ctx->s));
            for (long long q = 0; q < chunk; q += G) CK(cudaGraphLaunch(ctx->graph, ctx->s));
            CK(cudaEventRecord(ctx->ev1, ctx->s));
        }
        int status = 0;
        CK(cudaMemcpyAsync(&status, ctx->d.status, sizeof(int), cudaMemcpyDeviceToHost, ctx->s));
        CK(cudaStreamSynchronize(ctx->s));
        if (!ctx->evict_bytes) {
            float ms = 0;
            cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
            total_ms += ms;
        }
        long long got = chunk;
        if (status > 0) got = (long long)status - base;  // guard at step status-1
        if (recorded) {
            const long long off = base % ctx->traj_cap;
            if (traj_out && got > 0)
                CK(cudaMemcpy(traj_out + 2 * base * ctx->n2, ctx->d.traj + off * ctx->n2,
                              got * ctx->n2 * sizeof(double2), cudaMemcpyDeviceToHost));
            if (dip_out && got > 0)
                CK(cudaMemcpy(dip_out + base, ctx->d.dip + off, got * sizeof(double), cudaMemcpyDeviceToHost));
        }
        if (ctx->prec != G12_PREC_FP64) {
            const int me = mixed_error(ctx->mixed);
            if (me) {
                ctx->err = "tensor-core pipeline wait expired (code " + std::to_string(me) + ")";
                return G12_ERR_CUDA;
            }
        }
        base += got;
        if (status > 0) {
            *done = base;
            ctx->last_ms = total_ms;
            return G12_GUARD_TRIPPED;
        }
    }
    *done = base;
    ctx->last_ms = total_ms;
    return G12_OK;
}

}  // namespace

extern "C" int g12_create(const g12_params *p, int32_t precision, int32_t device, g12_ctx **out)
{
    g_create_error.clear();
    if (!p || !out) return G12_ERR_INVALID;
    *out = nullptr;
    const int n = p->Ns * p->Nb;
    if (p->Ns < 1 || p->Nb < 1 || n > G12_MAX_N) {
        g_create_error = "unsupported size: need 1 <= Ns*Nb <= 64";
        return G12_ERR_INVALID;
    }
    if (precision < G12_PREC_FP64 || precision > G12_PREC_FP64SYM) {
        g_create_error = "unknown precision mode";
        return G12_ERR_INVALID;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        g_create_error = "no CUDA device (libg12kba has no CPU path)";
        return G12_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) {
        g_create_error = "bad device ordinal";
        return G12_ERR_INVALID;
    }
    auto ctx = new g12_ctx();
    ctx->P = *p;
    ctx->prec = precision;
    ctx->device = device;
    ctx->Ns = p->Ns;
    ctx->Nb = p->Nb;
    ctx->n = n;
    ctx->n2 = (long long)n * n;
    ctx->n3 = ctx->n2 * n;
    ctx->n4 = ctx->n2 * ctx->n2;
    auto fail = [&](int rc) {
        g_create_error = ctx->err;
        g12_destroy(ctx);
        return rc;
    };
    if (!ck(ctx, cudaSetDevice(device), "cudaSetDevice")) return fail(G12_ERR_CUDA);
    cudaDeviceProp prop;
    if (!ck(ctx, cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties")) return fail(G12_ERR_CUDA);
    if (prop.major < 10) {
        ctx->err = "libg12kba is built for sm_100a (B200)";
        return fail(G12_ERR_NO_DEVICE);
    }
    if (!ck(ctx, cudaStreamCreateWithFlags(&ctx->s, cudaStreamNonBlocking), "cudaStreamCreate") ||
        !ck(ctx, cudaStreamCreateWithFlags(&ctx->s2, cudaStreamNonBlocking), "cudaStreamCreate") ||
        !ck(ctx, cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming), "cudaEventCreate") ||
        !ck(ctx, cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming), "cudaEventCreate"))
        return fail(G12_ERR_CUDA);
    cudaEventCreate(&ctx->ev0);
    cudaEventCreate(&ctx->ev1);
    if (!ck(ctx, cudaStreamCreateWithFlags(&ctx->s_copy, cudaStreamNonBlocking), "cudaStreamCreate") ||
        !ck(ctx, cudaMallocHost(&ctx->status_h, 2 * sizeof(int)), "cudaMallocHost"))
        return fail(G12_ERR_CUDA);
    for (int h = 0; h < 2; ++h)
        if (!ck(ctx, cudaEventCreate(&ctx->ev_hs[h]), "cudaEventCreate") ||
            !ck(ctx, cudaEventCreate(&ctx->ev_he[h]), "cudaEventCreate") ||
            !ck(ctx, cudaEventCreateWithFlags(&ctx->ev_hc[h], cudaEventDisableTiming), "cudaEventCreate"))
            return fail(G12_ERR_CUDA);

    Dev &d = ctx->d;
    d.Ns = p->Ns;
    d.Nb = p->Nb;
    d.n = n;
    d.nv = p->EHM ? std::max(0, p->Ns - 1) : 0;
    d.gate = (p->U != 0 && !p->HF) ? 1 : 0;  // RK_solver.h:154, AS.h:144 (global U)
    d.debug = 0;
    d.n2 = ctx->n2;
    d.n3 = ctx->n3;
    d.n4 = ctx->n4;
    d.t1 = p->t1;
    d.t2 = p->t2;
    for (int r = 0; r < kMaxN; ++r) d.law[r] = (r < d.nv) ? vlaw(*p, r + 1) : 0.0;
    const long long n2 = ctx->n2, n3 = ctx->n3, n4 = ctx->n4;
    bool ok = dalloc(ctx, &d.Y1, n2) && dalloc(ctx, &d.G1t0, n2) && dalloc(ctx, &d.G1t1, n2) &&
              dalloc(ctx, &d.RK1, n2) && dalloc(ctx, &d.h, n2) && dalloc(ctx, &d.Ix, n2) &&
              dalloc(ctx, &d.comm_dbg, n2) && dalloc(ctx, &d.K1_dbg, n2) && dalloc(ctx, &d.Y2, 2 * n4) &&
              dalloc(ctx, &d.RK2, 2 * n4) && dalloc(ctx, &d.TMP0, 2 * n4) && dalloc(ctx, &d.TMP1, 2 * n4) &&
              dalloc(ctx, &d.TAB, 2 * n4) && dalloc(ctx, &d.D, 2 * n3) && dalloc(ctx, &d.Q, 2 * n3) &&
              dalloc(ctx, &d.Rt, n2 * p->Ns) && dalloc(ctx, &d.counter, 1) && dalloc(ctx, &d.limit, 1) &&
              dalloc(ctx, &d.status, 1) && dalloc(ctx, &d.active, 1) && dalloc(ctx, &d.cur, 1) &&
              dalloc(ctx, &ctx->energy_dev, 4);
    if (!ok) return fail(G12_ERR_NOMEM);
    // trajectory ring: up to 4096 snapshots or 1 GiB
    ctx->traj_cap = std::max<long long>(1, std::min<long long>(4096, (1LL << 30) / (n2 * 16)));
    d.traj_cap = ctx->traj_cap;
    d.dip_cap = ctx->traj_cap;
    if (!dalloc(ctx, &d.traj, ctx->traj_cap * n2) || !dalloc(ctx, &d.dip, ctx->traj_cap)) return fail(G12_ERR_NOMEM);

    LaunchCfg &lc = ctx->lc;
    lc.ab = make_apply_cfg(n, false, &lc.ab_smem, &lc.ab_threads);
    lc.cd = make_apply_cfg(n, true, &lc.cd_smem, &lc.cd_threads);
    lc.cd.NB = lc.ab.NB = std::min(lc.ab.NB, lc.cd.NB);
    lc.ab_threads = lc.cd_threads = lc.ab.NB * lc.ab.S * lc.ab.S;
    lc.ab_smem = (size_t(2) * lc.ab.NP * lc.ab.LD + size_t(lc.ab.NB) * lc.ab.NP * lc.ab.LD) * sizeof(double2);
    lc.cd_smem = lc.ab_smem + size_t(n) * n * sizeof(double2);
    lc.apply_grid = dim3(unsigned((n2 + lc.ab.NB - 1) / lc.ab.NB), 2, 1);
    lc.prep_blocks = prep_blocks(n2);
    lc.prep_smem = prep_smem();
    lc.prep_wide_blocks = prep_blocks<kPrepWarpsWide>(n2);
    lc.prep_wide_smem = prep_smem<kPrepWarpsWide>();
    lc.g1_blocks = g1_blocks(n2);
    lc.g1_smem = g1_smem(n2);
    lc.steps_per_graph = n <= 8 ? 8 : (n <= 32 ? 4 : 1);
    lc.tc = apply_tc_ok(n);
    if (lc.tc) {
        lc.tcc = make_apply_tc_cfg(n, &lc.tc_ab_smem, &lc.tc_cd_smem);
        lc.tc_grid = dim3(unsigned((n2 + lc.tcc.NB - 1) / lc.tcc.NB), 2, 1);
        if (!ck(ctx, apply_tc_smem_attr<false>(lc.tcc, lc.tc_ab_smem), "attr") ||
            !ck(ctx, apply_tc_smem_attr<true>(lc.tcc, lc.tc_cd_smem), "attr"))
            return fail(G12_ERR_CUDA);
    }
    if (!ck(ctx, cudaFuncSetAttribute(k_apply<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(lc.ab_smem)), "attr") ||
        !ck(ctx, cudaFuncSetAttribute(k_apply<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(lc.cd_smem)), "attr") ||
        !ck(ctx, cudaFuncSetAttribute(k_prep, cudaFuncAttributeMaxDynamicSharedMemorySize, int(lc.prep_smem)), "attr") ||
        !ck(ctx, cudaFuncSetAttribute(k_prep_wide, cudaFuncAttributeMaxDynamicSharedMemorySize, int(lc.prep_wide_smem)),
            "attr") ||
        !ck(ctx, cudaFuncSetAttribute(k_g1, cudaFuncAttributeMaxDynamicSharedMemorySize, int(lc.g1_smem)), "attr"))
        return fail(G12_ERR_CUDA);
    if (precision != G12_PREC_FP64) {
        int rc = mixed_init(ctx->mixed, d, precision, &ctx->err);
        if (rc) return fail(rc);
        if (ctx->mixed.epip) {
            d.Zt = ctx->mixed.Zt;  // k_prep writes the combined table the persistent epilogue reads
        } else {
            d.Qt = ctx->mixed.s.Qt;  // k_prep writes the transposed tables the epilogue reads
            d.Rtt = ctx->mixed.s.Rtt;
        }
        d.ozb = ctx->mixed.ozb;  // k_prep also writes the digits of h for the tcgen05 GEMM
    }
    if (ensure_sched(ctx, 1024)) return fail(G12_ERR_CUDA);
    *out = ctx;
    return G12_OK;
}

extern "C" int g12_destroy(g12_ctx *ctx)
{
    if (!ctx) return G12_OK;
    cudaSetDevice(ctx->device);
    if (ctx->s) cudaStreamSynchronize(ctx->s);
    if (ctx->graph) cudaGraphExecDestroy(ctx->graph);
    if (ctx->evict_buf) cudaFree(ctx->evict_buf);
    mixed_free(ctx->mixed);
    for (void *p : ctx->allocs) cudaFree(p);
    if (ctx->sched_dev) cudaFree(ctx->sched_dev);
    if (ctx->sched_host) cudaFreeHost(ctx->sched_host);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->s_copy) cudaStreamSynchronize(ctx->s_copy);
    for (int h = 0; h < 2; ++h) {
        if (ctx->ev_hs[h]) cudaEventDestroy(ctx->ev_hs[h]);
        if (ctx->ev_he[h]) cudaEventDestroy(ctx->ev_he[h]);
        if (ctx->ev_hc[h]) cudaEventDestroy(ctx->ev_hc[h]);
    }
    if (ctx->status_h) cudaFreeHost(ctx->status_h);
    if (ctx->s_copy) cudaStreamDestroy(ctx->s_copy);
    for (cudaEvent_t e : ctx->ring) cudaEventDestroy(e);
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    if (ctx->s2) cudaStreamDestroy(ctx->s2);
    if (ctx->s) cudaStreamDestroy(ctx->s);
    delete ctx;
    return G12_OK;
}

extern "C" const char *g12_last_error(const g12_ctx *ctx)
{
    if (!ctx) return g_create_error.c_str();
    return ctx->err.c_str();
}

namespace {

int upload_g2(g12_ctx *ctx, const double *src, double2 *dst)
{
    if (!src) {
        CK(cudaMemsetAsync(dst, 0, ctx->n4 * sizeof(double2), ctx->s));
        return G12_OK;
    }
    CK(cudaMemcpyAsync(ctx->d.TAB, src, ctx->n4 * sizeof(double2), cudaMemcpyHostToDevice, ctx->s));
    k_from_ref<<<592, 256, 0, ctx->s>>>(ctx->d.TAB, dst, ctx->Ns, ctx->Nb, ctx->n4);
    CK(cudaGetLastError());
    return G12_OK;
}

int download_g2(g12_ctx *ctx, const double2 *src, double *dst)
{
    if (!dst) return G12_OK;
    k_to_ref<<<592, 256, 0, ctx->s>>>(src, ctx->d.TAB, ctx->Ns, ctx->Nb, ctx->n4);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dst, ctx->d.TAB, ctx->n4 * sizeof(double2), cudaMemcpyDeviceToHost, ctx->s));
    return G12_OK;
}

}  // namespace

extern "C" int g12_set_state(g12_ctx *ctx, const double *G1, const double *G2xx, const double *G2xy)
{
    if (!ctx || !G1) return G12_ERR_INVALID;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(ctx->d.Y1, G1, ctx->n2 * sizeof(double2), cudaMemcpyHostToDevice, ctx->s));
    int rc = upload_g2(ctx, G2xx, ctx->d.Y2);
    if (!rc) rc = upload_g2(ctx, G2xy, ctx->d.Y2 + ctx->n4);
    if (rc) return rc;
    k_init_D<<<592, 256, 0, ctx->s>>>(ctx->d);
    CK(cudaGetLastError());
    if (ctx->prec != G12_PREC_FP64) {
        rc = mixed_on_state(ctx->mixed, ctx->d, ctx->s);
        if (rc) return rc;
    }
    CK(cudaStreamSynchronize(ctx->s));
    ctx->t_rk = 0;
    ctx->t_temp = 0;
    return G12_OK;
}

extern "C" int g12_get_state(g12_ctx *ctx, double *G1, double *G2xx, double *G2xy)
{
    if (!ctx) return G12_ERR_INVALID;
    CK(cudaSetDevice(ctx->device));
    if (G1) CK(cudaMemcpyAsync(G1, ctx->d.Y1, ctx->n2 * sizeof(double2), cudaMemcpyDeviceToHost, ctx->s));
    if (ctx->prec != G12_PREC_FP64 && (G2xx || G2xy)) {
        if (mixed_to_full(ctx->mixed, ctx->d, ctx->s)) {
            ctx->err = "state expansion failed";
            return G12_ERR_CUDA;
        }
    }
    int rc = download_g2(ctx, ctx->d.Y2, G2xx);
    if (!rc) {
        CK(cudaStreamSynchronize(ctx->s));
        rc = download_g2(ctx, ctx->d.Y2 + ctx->n4, G2xy);
    }
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->s));
    return G12_OK;
}

extern "C" int g12_adiabatic_switch(g12_ctx *ctx, int64_t *steps_done)
{
    if (!ctx) return G12_ERR_INVALID;
    CK(cudaSetDevice(ctx->device));
    const long long steps = g12_as_steps(&ctx->P);
    if (steps < 0) {
        ctx->err = "adiabatic switching does not terminate for these parameters";
        return G12_ERR_INVALID;
    }
    int rc = ensure_sched(ctx, steps);
    if (rc) return rc;
    build_as_sched(ctx->P, steps, ctx->sched_host);
    long long done = 0;
    rc = run_steps(ctx, steps, nullptr, nullptr, &done);
    if (steps_done) *steps_done = done;
    return rc;
}

static int propagate_impl(g12_ctx *ctx, int64_t nsteps, double *traj_out, double *dip_out, int64_t *steps_done)
{
    if (!ctx || nsteps < 0) return G12_ERR_INVALID;
    CK(cudaSetDevice(ctx->device));
    int rc = ensure_sched(ctx, nsteps);
    if (rc) return rc;
    double t = ctx->t_rk, tt = ctx->t_temp;
    build_rk_sched(ctx->P, nsteps, &t, &tt, ctx->sched_host);
    long long done = 0;
    rc = run_steps(ctx, nsteps, traj_out, dip_out, &done);
    // advance the clock by the steps actually taken
    double t2 = ctx->t_rk, tt2 = ctx->t_temp;
    if (done == nsteps) {
        t2 = t;
        tt2 = tt;
    } else if (done > 0) {
        std::vector<StepP> scratch((size_t)done);
        build_rk_sched(ctx->P, done, &t2, &tt2, scratch.data());
    }
    ctx->t_rk = t2;
    ctx->t_temp = tt2;
    if (steps_done) *steps_done = done;
    return rc;
}

extern "C" int g12_propagate(g12_ctx *ctx, int64_t nsteps, double *traj_out, int64_t *steps_done)
{
    return propagate_impl(ctx, nsteps, traj_out, nullptr, steps_done);
}

extern "C" int g12_propagate_dipole(g12_ctx *ctx, int64_t nsteps, double *dipole_out, int64_t *steps_done)
{
    return propagate_impl(ctx, nsteps, nullptr, dipole_out, steps_done);
}

extern "C" int g12_rhs(g12_ctx *ctx, const double *G1, const double *G2xx, const double *G2xy, double U_eff,
                       double w_quench, int32_t Nq_eff, double *h, double *comm1, double *Ix, double *K1,
                       double *K2xx, double *K2xy)
{
    if (!ctx || !G1) return G12_ERR_INVALID;
    int rc = g12_set_state(ctx, G1, G2xx, G2xy);
    if (rc) return rc;
    StepP sp{};
    for (int k = 0; k < 4; ++k) {
        sp.st[k].U = U_eff;
        sp.st[k].wq = w_quench;
        sp.st[k].nq = Nq_eff;
        sp.st[k].w = 1;
    }
    Dev dd = ctx->d;
    dd.debug = 1;
    if (ctx->prec != G12_PREC_FP64) {
        // the per-pair epilogue (the one with the K output) reads the transposed tables
        dd.Qt = ctx->mixed.s.Qt;
        dd.Rtt = ctx->mixed.s.Rtt;
        dd.Zt = nullptr;
    }
    const int one = 1;
    CK(cudaMemcpyAsync(dd.cur, &sp, sizeof(StepP), cudaMemcpyHostToDevice, ctx->s));
    CK(cudaMemcpyAsync(dd.active, &one, sizeof(int), cudaMemcpyHostToDevice, ctx->s));
    CK(cudaMemcpyAsync(dd.G1t0, dd.Y1, ctx->n2 * sizeof(double2), cudaMemcpyDeviceToDevice, ctx->s));
    CK(cudaMemsetAsync(dd.TMP0, 0, 2 * ctx->n4 * sizeof(double2), ctx->s));
    const LaunchCfg &lc = ctx->lc;
    k_prep<<<lc.prep_blocks, kPrepWarps * 32, lc.prep_smem, ctx->s>>>(dd, 0);
    k_g1<<<lc.g1_blocks, kG1Threads, lc.g1_smem, ctx->s>>>(dd, 0);
    if (dd.gate) {
        if (ctx->prec == G12_PREC_FP64) {
            enqueue_apply(lc, dd, 0, ctx->s);
        } else {
            mixed_enqueue_stage(ctx->mixed, dd, 0, ctx->prec, ctx->s);
        }
    }
    CK(cudaGetLastError());
    const size_t b2 = ctx->n2 * sizeof(double2);
    if (h) CK(cudaMemcpyAsync(h, dd.h, b2, cudaMemcpyDeviceToHost, ctx->s));
    if (comm1) CK(cudaMemcpyAsync(comm1, dd.comm_dbg, b2, cudaMemcpyDeviceToHost, ctx->s));
    if (Ix) CK(cudaMemcpyAsync(Ix, dd.Ix, b2, cudaMemcpyDeviceToHost, ctx->s));
    if (K1) CK(cudaMemcpyAsync(K1, dd.K1_dbg, b2, cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    // FP64: K2 in TMP0; symmetric engine: K2 in Y2 (its full-state staging buffer)
    double2 *K2src = (ctx->prec == G12_PREC_FP64) ? dd.TMP0 : dd.Y2;
    rc = download_g2(ctx, K2src, K2xx);
    if (!rc) {
        CK(cudaStreamSynchronize(ctx->s));
        rc = download_g2(ctx, K2src + ctx->n4, K2xy);
    }
    CK(cudaStreamSynchronize(ctx->s));
    if (ctx->prec != G12_PREC_FP64 && mixed_error(ctx->mixed)) {
        ctx->err = "tensor-core pipeline wait expired";
        return G12_ERR_CUDA;
    }
    return rc;
}

extern "C" int g12_total_energy(g12_ctx *ctx, double U_eff, double w_quench, int32_t Nq_eff, double *E_out)
{
    if (!ctx || !E_out || Nq_eff < 0) return G12_ERR_INVALID;
    CK(cudaSetDevice(ctx->device));
    StageP st{};
    st.U = U_eff;
    st.wq = w_quench;
    st.nq = Nq_eff;
    // Y1 and D (the particle-2 diagonal of G2) hold the current state on both engines
    k_energy<<<1, kEnergyThreads, 0, ctx->s>>>(ctx->d, st, ctx->energy_dev);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(E_out, ctx->energy_dev, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->s));
    CK(cudaStreamSynchronize(ctx->s));
    return G12_OK;
}

extern "C" double g12_last_device_ms(const g12_ctx *ctx) { return ctx ? ctx->last_ms : 0.0; }

extern "C" int32_t g12_set_l2_eviction(g12_ctx *ctx, int64_t bytes)
{
    if (!ctx || bytes < 0) return G12_ERR_INVALID;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->s));
    if (ctx->graph) {
        cudaGraphExecDestroy(ctx->graph);
        ctx->graph = nullptr;
    }
    if (ctx->evict_buf) cudaFree(ctx->evict_buf);
    ctx->evict_buf = nullptr;
    ctx->evict_bytes = 0;
    ctx->lc.steps_per_graph = ctx->n <= 8 ? 8 : (ctx->n <= 32 ? 4 : 1);
    if (bytes == 0) return G12_OK;
    if (cudaMalloc(&ctx->evict_buf, size_t(bytes)) != cudaSuccess) {
        cudaGetLastError();
        ctx->evict_buf = nullptr;
        ctx->err = "out of device memory (L2 eviction buffer)";
        return G12_ERR_NOMEM;
    }
    ctx->evict_bytes = size_t(bytes);
    ctx->lc.steps_per_graph = 1;  // evict between every step
    return G12_OK;
}

namespace {

const char *kFp64Names[] = {"k_step_begin", "k_prep", "k_g1", "k_apply<rows>", "k_apply<cols+epilogue>"};
const char *kFp64TcNames[] = {"k_step_begin", "k_prep", "k_g1", "k_apply_tc<rows>", "k_apply_tc<cols+epilogue>"};

}  // namespace

extern "C" const char *g12_kernel_name(const g12_ctx *ctx, int32_t kind)
{
    if (!ctx) return "";
    if (ctx->prec != G12_PREC_FP64 && kind >= 3) return mixed_kernel_name(ctx->mixed, kind - 3);
    if (kind < 0 || kind >= 5) return "";
    if (kind == 1 &&
        prep_is_wide(ctx->prec != G12_PREC_FP64 && ctx->d.gate && mixed_fuses_g1(ctx->mixed), ctx->d))
        return "k_prep_wide";
    return ctx->lc.tc ? kFp64TcNames[kind] : kFp64Names[kind];
}

extern "C" int32_t g12_kernel_times(g12_ctx *ctx, int32_t nsteps, double *avg_ms, int32_t *calls_per_step, int32_t cap)
{
    if (!ctx || nsteps <= 0) return G12_ERR_INVALID;
    CK(cudaSetDevice(ctx->device));
    int rc = ensure_sched(ctx, nsteps);
    if (rc) return rc;
    double t = ctx->t_rk, tt = ctx->t_temp;
    build_rk_sched(ctx->P, nsteps, &t, &tt, ctx->sched_host);
    ctx->t_rk = t;
    ctx->t_temp = tt;
    CK(cudaMemcpyAsync(ctx->sched_dev, ctx->sched_host, nsteps * sizeof(StepP), cudaMemcpyHostToDevice, ctx->s));
    const long long zero = 0, lim = nsteps;
    CK(cudaMemcpyAsync(ctx->d.counter, &zero, sizeof(long long), cudaMemcpyHostToDevice, ctx->s));
    CK(cudaMemcpyAsync(ctx->d.limit, &lim, sizeof(long long), cudaMemcpyHostToDevice, ctx->s));
    CK(cudaMemsetAsync(ctx->d.status, 0, sizeof(int), ctx->s));
    const int nk = (ctx->prec == G12_PREC_FP64) ? 5 : 3 + mixed_kernel_kinds(ctx->mixed);
    std::vector<double> tot(nk, 0.0);
    std::vector<int> calls(nk, 0);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const LaunchCfg &lc = ctx->lc;
    const Dev &d = ctx->d;
    auto timed = [&](int kind, auto &&launch) {
        cudaEventRecord(a, ctx->s);
        launch();
        cudaEventRecord(b, ctx->s);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        tot[kind] += ms;
        calls[kind] += 1;
    };
    for (int s = 0; s < nsteps; ++s) {
        timed(0, [&] { k_step_begin<<<1, 256, 0, ctx->s>>>(d); });
        for (int k = 0; k < 4; ++k) {
            // the digit-GEMM path runs the G1 side inside its epilogue launch
            const bool fused = ctx->prec != G12_PREC_FP64 && d.gate && mixed_fuses_g1(ctx->mixed);
            timed(1, [&] { enqueue_prep(lc, d, k, ctx->s, fused); });
            if (!fused) timed(2, [&] { k_g1<<<lc.g1_blocks, kG1Threads, lc.g1_smem, ctx->s>>>(d, k); });
            if (!d.gate) continue;
            if (ctx->prec == G12_PREC_FP64) {
                timed(3, [&] { enqueue_apply(lc, d, k, ctx->s, 0); });
                timed(4, [&] { enqueue_apply(lc, d, k, ctx->s, 1); });
            } else {
                for (int q = 0; q < mixed_kernel_kinds(ctx->mixed); ++q)
                    timed(3 + q, [&] { mixed_enqueue_kind(ctx->mixed, d, k, ctx->prec, q, ctx->s, fused); });
            }
        }
        if (ctx->evict_bytes) cudaMemsetAsync(ctx->evict_buf, 0, ctx->evict_bytes, ctx->s);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CK(cudaGetLastError());
    for (int i = 0; i < nk && i < cap; ++i) {
        avg_ms[i] = calls[i] ? tot[i] / calls[i] : 0.0;
        if (calls_per_step) calls_per_step[i] = calls[i] / nsteps;
    }
    return nk;
}

namespace {

// Independent FMA chains per thread: throughput, not latency, bound.
__global__ void k_fp64_peak(double *out, int iters, double a, double b)
{
    double x[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) x[q] = threadIdx.x * 1e-9 + q;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int q = 0; q < 8; ++q) x[q] = fma(x[q], a, b);
    }
    double s = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) s += x[q];
    if (s == 12345.678) out[0] = s;
}

}  // namespace

extern "C" double g12_fp64_peak_tflops(int32_t device)
{
    if (cudaSetDevice(device) != cudaSuccess) return 0.0;
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    double *out = nullptr;
    if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) return 0.0;
    const int blocks = prop.multiProcessorCount * 8, threads = 256, iters = 4096;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    k_fp64_peak<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < 5; ++r) {
        cudaEventRecord(a);
        k_fp64_peak<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        best = std::min(best, ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    const double flops = 2.0 * 8.0 * double(iters) * blocks * threads;
    return flops / (best * 1e-3) / 1e12;
}

extern "C" int32_t g12_launches_per_step(const g12_ctx *ctx)
{
    if (!ctx) return 0;
    int per_stage = 2;  // k_prep, k_g1
    if (ctx->d.gate) {
        per_stage += (ctx->prec == G12_PREC_FP64) ? 2 : mixed_launches_per_stage(ctx->mixed);
        if (ctx->prec != G12_PREC_FP64 && mixed_fuses_g1(ctx->mixed)) per_stage -= 1;  // k_g1 in k_sym_epi
    }
    return 1 + 4 * per_stage;
}
