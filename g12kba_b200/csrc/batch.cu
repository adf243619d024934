// Batched ensembles: many independent systems with different Ns, Nb, U, t2,
// quench strength ... advanced together, one launch per kernel kind and RK
// stage for the whole ensemble (RK_solver.h's step, per system), captured in
// one CUDA graph per step.  Each block finds its system from prefix offsets
// and runs the same device code as the single-system engine on that system's
// buffers, so every system's result is bit-identical to running it alone.
// The row/column-mixing tile shape (matrices per block) is chosen per
// orbital count n by timing the candidates at batch creation.
#include "g12kba.h"
#include "internal.h"
#include "fp64_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

using namespace g12;

namespace {

thread_local std::string g_batch_error;

struct BatchDev {
    const Dev *devs;
    const ApplyCfg *cfg;
    const ApplyTcCfg *tcfg;
    const int *off_prep, *off_g1, *off_apply, *off_tc;  // nsys + 1 prefix offsets (blocks)
    int nsys;
};

// threads of a block of the batched FP64 tensor-core halves (every system's
// tile shape fits: warps past its matrices stay idle)
constexpr int kTcThreads = 512;

// largest i with off[i] <= b
__device__ __forceinline__ int find_sys(const int *off, int nsys, int b)
{
    int lo = 0, hi = nsys - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void load_dev(Dev &dst, const Dev &src)
{
    const int words = int(sizeof(Dev) / 4);
    const uint32_t *s = reinterpret_cast<const uint32_t *>(&src);
    uint32_t *d = reinterpret_cast<uint32_t *>(&dst);
    for (int w = threadIdx.x; w < words; w += blockDim.x) d[w] = s[w];
    __syncthreads();
}

__global__ void __launch_bounds__(256) kb_step_begin(BatchDev b)
{
    __shared__ Dev sd;
    load_dev(sd, b.devs[blockIdx.x]);
    step_begin_body(sd);
}

__global__ void __launch_bounds__(kPrepWarps * 32) kb_prep(BatchDev b, int k)
{
    __shared__ Dev sd;
    __shared__ int sys;
    if (threadIdx.x == 0) sys = find_sys(b.off_prep, b.nsys, blockIdx.x);
    __syncthreads();
    load_dev(sd, b.devs[sys]);
    prep_body(sd, k, blockIdx.x - b.off_prep[sys]);
}

__global__ void __launch_bounds__(kG1Threads) kb_g1(BatchDev b, int k)
{
    __shared__ Dev sd;
    __shared__ int sys;
    if (threadIdx.x == 0) sys = find_sys(b.off_g1, b.nsys, blockIdx.x);
    __syncthreads();
    load_dev(sd, b.devs[sys]);
    g1_body(sd, k, blockIdx.x - b.off_g1[sys]);
}

template <bool CD>
__global__ void __launch_bounds__(256) kb_apply(BatchDev b, int k)
{
    __shared__ Dev sd;
    __shared__ int sys;
    if (threadIdx.x == 0) sys = find_sys(b.off_apply, b.nsys, blockIdx.x);
    __syncthreads();
    load_dev(sd, b.devs[sys]);
    const ApplyCfg cfg = b.cfg[sys];
    const int local = blockIdx.x - b.off_apply[sys];
    const int chunks = int((sd.n2 + cfg.NB - 1) / cfg.NB);
    apply_body<CD>(sd, k, cfg, local % chunks, local / chunks);
}

// systems with 16 <= n <= 48: the FP64 tensor-core (DMMA) halves, the same
// device code as a single-system context of that n
template <bool CD>
__global__ void __launch_bounds__(kTcThreads) kb_apply_tc(BatchDev b, int k)
{
    __shared__ Dev sd;
    __shared__ int sys;
    if (threadIdx.x == 0) sys = find_sys(b.off_tc, b.nsys, blockIdx.x);
    __syncthreads();
    load_dev(sd, b.devs[sys]);
    const ApplyTcCfg cfg = b.tcfg[sys];
    const int local = blockIdx.x - b.off_tc[sys];
    const int chunks = int((sd.n2 + cfg.NB - 1) / cfg.NB);
    apply_tc_body<CD>(sd, k, cfg, local % chunks, local / chunks);
}

__global__ void kb_reset(BatchDev b, const long long *limits)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.nsys) return;
    const Dev &d = b.devs[i];
    *d.counter = 0;
    *d.limit = limits[i];
    *d.status = 0;
}

// dip rings of all systems -> out[sys][0..steps)
__global__ void kb_gather_dip(BatchDev b, int steps, double *out)
{
    const int i = blockIdx.y;
    const Dev &d = b.devs[i];
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < steps; s += gridDim.x * blockDim.x)
        out[(long long)i * steps + s] = d.dip[s % d.dip_cap];
}

// snapshot features of every system (state after the step just run):
// rho = -i G1, upper triangle (mu <= nu, row-major), real parts then imaginary
// parts -> feat[sys][snap][n(n+1)]
__global__ void kb_features(BatchDev b, long long snap, long long nsnap, float *feat)
{
    const int i = blockIdx.y;
    const Dev &d = b.devs[i];
    const int n = d.n, nt = n * (n + 1) / 2;
    float *out = feat + ((long long)i * nsnap + snap) * (2 * nt);
    for (int x = threadIdx.x; x < nt; x += blockDim.x) {
        int mu = 0, r = x;
        while (r >= n - mu) {
            r -= n - mu;
            ++mu;
        }
        const double2 g = d.Y1[mu * n + mu + r];
        out[x] = float(g.y);
        out[nt + x] = float(-g.x);
    }
}

ApplyCfg apply_cfg_nb(int n, int nb)
{
    ApplyCfg c;
    c.NP = (n + 3) / 4 * 4;
    c.S = c.NP / 4;
    c.LD = c.NP + 1;
    c.NB = nb;
    return c;
}

size_t apply_smem(const ApplyCfg &c, int n, bool cd)
{
    size_t b = (size_t(2) * c.NP * c.LD + size_t(c.NB) * c.NP * c.LD) * sizeof(double2);
    if (cd) b += size_t(n) * n * sizeof(double2);
    return b;
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

void as_sched(const g12_params &P, long long s0, long long steps, StepP *out)
{
    double t = 0;
    for (long long s = 0; s < s0; ++s) t += P.as_dt;
    for (long long s = 0; s < steps; ++s) {
        StepP sp{};
        for (int k = 0; k < 4; ++k) {
            double dtk, w;
            stage_dt(P.as_dt, k, &dtk, &w);
            const double t_rk = (k != 0) ? t + dtk : t;
            StageP &st = sp.st[k];
            st.U = fermi(t_rk, P.AS_midpoint, P.AS_rate) * P.U;
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

void rk_sched(const g12_params &P, long long steps, double *t_io, double *tt_io, StepP *out)
{
    double t = *t_io, t_temp = *tt_io;
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
    *tt_io = t_temp;
}

double vlaw(const g12_params &P, int r)
{
    if (P.v_law == G12_VLAW_INV) return 1.0 / (1.0 + double(r));
    return std::exp(-P.decay_rate * r);
}

constexpr long long kChunk = 512;  // steps per schedule upload

}  // namespace

struct g12_batch {
    int device = 0;
    int nsys = 0;
    std::string err;
    std::vector<g12_params> P;
    std::vector<Dev> dev;
    std::vector<ApplyCfg> cfg;
    std::vector<ApplyTcCfg> tcfg;
    std::vector<int> off_prep, off_g1, off_apply, off_tc;
    BatchDev bd{};
    void *pool = nullptr;
    Dev *devs_d = nullptr;
    ApplyCfg *cfg_d = nullptr;
    ApplyTcCfg *tcfg_d = nullptr;
    int *offs_d = nullptr;
    long long *limits_d = nullptr;
    double *dip_d = nullptr;
    StepP *sched_h = nullptr;  // pinned: nsys x kChunk
    StepP *sched_d = nullptr;
    size_t smem_prep = 0, smem_g1 = 0, smem_ab = 0, smem_cd = 0, smem_tab = 0, smem_tcd = 0;
    cudaStream_t s = nullptr, s2 = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, fork = nullptr, join = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::vector<double> t_rk, t_temp;
    std::map<int, int> tuned_nb;  // n -> matrices per block (of the kernel kind that n uses)
    float last_ms = 0;
};

namespace {

#define BCK(call)                                                                      \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            b->err = std::string(#call) + ": " + cudaGetErrorString(e_);               \
            return G12_ERR_CUDA;                                                       \
        }                                                                              \
    } while (0)

int batch_enqueue_step(g12_batch *b, cudaStream_t s)
{
    const BatchDev &bd = b->bd;
    kb_step_begin<<<b->nsys, 256, 0, s>>>(bd);
    const int tp = b->off_prep.back(), tg = b->off_g1.back(), ta = b->off_apply.back(), tt = b->off_tc.back();
    for (int k = 0; k < 4; ++k) {
        kb_prep<<<tp, kPrepWarps * 32, b->smem_prep, s>>>(bd, k);
        cudaEventRecord(b->fork, s);
        cudaStreamWaitEvent(b->s2, b->fork, 0);
        kb_g1<<<tg, kG1Threads, b->smem_g1, b->s2>>>(bd, k);
        cudaEventRecord(b->join, b->s2);
        if (ta > 0) kb_apply<false><<<ta, 256, b->smem_ab, s>>>(bd, k);
        if (tt > 0) kb_apply_tc<false><<<tt, kTcThreads, b->smem_tab, s>>>(bd, k);
        if (ta > 0) kb_apply<true><<<ta, 256, b->smem_cd, s>>>(bd, k);
        if (tt > 0) kb_apply_tc<true><<<tt, kTcThreads, b->smem_tcd, s>>>(bd, k);
        cudaStreamWaitEvent(s, b->join, 0);
    }
    return G12_OK;
}

// times the row/column-mixing kernels of one system for each admissible
// matrices-per-block value and keeps the fastest
ApplyTcCfg tc_cfg_nb(int n, int nb, size_t *sab, size_t *scd)
{
    ApplyTcCfg c = make_apply_tc_cfg(n, sab, scd);
    const size_t plane = size_t(apply_tc_plane(c.NP, c.LDD)) * sizeof(double);
    c.NB = nb;
    c.threads = kTcThreads;
    *sab = (4 + 2 * size_t(nb)) * plane;
    *scd = *sab + size_t(n) * (n + 1) * sizeof(double2);
    return c;
}

int autotune_tc(g12_batch *b, int sys);

int autotune(g12_batch *b, int sys)
{
    const Dev &d = b->dev[sys];
    const int n = d.n;
    if (b->tuned_nb.count(n)) return b->tuned_nb[n];
    if (apply_tc_ok(n)) return autotune_tc(b, sys);
    const int S = ((n + 3) / 4 * 4) / 4;
    std::vector<int> cands;
    for (int nb = 1; nb <= 64; nb *= 2) {
        const ApplyCfg c = apply_cfg_nb(n, nb);
        if (nb * S * S > 256 || nb > n * n || apply_smem(c, n, true) > 200 * 1024) break;
        cands.push_back(nb);
    }
    if (cands.empty()) cands.push_back(1);
    // a throwaway active stage on this system's buffers
    StepP sp{};
    for (int k = 0; k < 4; ++k) sp.st[k].w = 1;
    const int one = 1;
    cudaMemcpy(d.cur, &sp, sizeof(StepP), cudaMemcpyHostToDevice);
    cudaMemcpy(d.active, &one, sizeof(int), cudaMemcpyHostToDevice);
    float best = 1e30f;
    int best_nb = cands[0];
    for (int nb : cands) {
        const ApplyCfg c = apply_cfg_nb(n, nb);
        const dim3 grid(unsigned((d.n2 + nb - 1) / nb), 2);
        const size_t sab = apply_smem(c, n, false), scd = apply_smem(c, n, true);
        cudaFuncSetAttribute(k_apply<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sab));
        cudaFuncSetAttribute(k_apply<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(scd));
        Dev dd = d;
        dd.debug = 1;  // results go to the scratch tensors only
        for (int rep = 0; rep < 4; ++rep) {
            cudaEventRecord(b->ev0, b->s);
            k_apply<false><<<grid, 256, sab, b->s>>>(dd, 0, c);
            k_apply<true><<<grid, 256, scd, b->s>>>(dd, 0, c);
            cudaEventRecord(b->ev1, b->s);
            cudaEventSynchronize(b->ev1);
            float ms = 0;
            cudaEventElapsedTime(&ms, b->ev0, b->ev1);
            if (rep > 0 && ms < best) {
                best = ms;
                best_nb = nb;
            }
        }
    }
    b->tuned_nb[n] = best_nb;
    return best_nb;
}

// the tensor-core halves: matrices per block over {1, 2, 4, ...} within one
// block of kTcThreads threads and 200 KB of shared memory, timed like the FMA path
int autotune_tc(g12_batch *b, int sys)
{
    const Dev &d = b->dev[sys];
    const int n = d.n;
    size_t sab = 0, scd = 0;
    const ApplyTcCfg base = make_apply_tc_cfg(n, &sab, &scd);
    const int tpm = apply_tc_tpm(base);
    std::vector<int> cands;
    for (int nb = 1; nb * tpm * 32 <= kTcThreads && nb <= n * n; nb *= 2) {
        tc_cfg_nb(n, nb, &sab, &scd);
        if (scd > 200 * 1024) break;
        cands.push_back(nb);
    }
    StepP sp{};
    for (int k = 0; k < 4; ++k) sp.st[k].w = 1;
    const int one = 1;
    cudaMemcpy(d.cur, &sp, sizeof(StepP), cudaMemcpyHostToDevice);
    cudaMemcpy(d.active, &one, sizeof(int), cudaMemcpyHostToDevice);
    float best = 1e30f;
    int best_nb = cands[0];
    for (int nb : cands) {
        const ApplyTcCfg c = tc_cfg_nb(n, nb, &sab, &scd);
        const dim3 grid(unsigned((d.n2 + nb - 1) / nb), 2);
        apply_tc_smem_attr<false>(c, sab);
        apply_tc_smem_attr<true>(c, scd);
        Dev dd = d;
        dd.debug = 1;  // results go to the scratch tensors only
        for (int rep = 0; rep < 4; ++rep) {
            cudaEventRecord(b->ev0, b->s);
            launch_apply_tc<false>(grid, sab, b->s, dd, 0, c);
            launch_apply_tc<true>(grid, scd, b->s, dd, 0, c);
            cudaEventRecord(b->ev1, b->s);
            cudaEventSynchronize(b->ev1);
            float ms = 0;
            cudaEventElapsedTime(&ms, b->ev0, b->ev1);
            if (rep > 0 && ms < best) {
                best = ms;
                best_nb = nb;
            }
        }
    }
    b->tuned_nb[n] = best_nb;
    return best_nb;
}

int upload_sched_and_reset(g12_batch *b, const std::vector<long long> &lim)
{
    BCK(cudaMemcpyAsync(b->sched_d, b->sched_h, sizeof(StepP) * b->nsys * kChunk, cudaMemcpyHostToDevice, b->s));
    BCK(cudaMemcpyAsync(b->limits_d, lim.data(), sizeof(long long) * b->nsys, cudaMemcpyHostToDevice, b->s));
    kb_reset<<<(b->nsys + 127) / 128, 128, 0, b->s>>>(b->bd, b->limits_d);
    BCK(cudaGetLastError());
    return G12_OK;
}

int build_batch_graph(g12_batch *b)
{
    if (b->graph) return G12_OK;
    cudaGraph_t g;
    BCK(cudaStreamBeginCapture(b->s, cudaStreamCaptureModeThreadLocal));
    batch_enqueue_step(b, b->s);
    BCK(cudaStreamEndCapture(b->s, &g));
    cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    BCK(e);
    return G12_OK;
}

// runs `steps` steps of each system's schedule (filled chunk by chunk by
// `fill`); after(step) may enqueue work after each step's graph
template <typename Fill, typename After>
int batch_run(g12_batch *b, long long steps, double *dip_out, Fill fill, After after)
{
    int rc = build_batch_graph(b);
    if (rc) return rc;
    float total = 0;
    std::vector<double> chunk_dip;
    for (long long base = 0; base < steps; base += kChunk) {
        const long long n = std::min(kChunk, steps - base);
        std::vector<long long> lim(b->nsys, n);
        fill(base, n);
        rc = upload_sched_and_reset(b, lim);
        if (rc) return rc;
        BCK(cudaStreamSynchronize(b->s));
        BCK(cudaEventRecord(b->ev0, b->s));
        for (long long q = 0; q < n; ++q) {
            BCK(cudaGraphLaunch(b->graph, b->s));
            after(base + q);
        }
        BCK(cudaGetLastError());
        BCK(cudaEventRecord(b->ev1, b->s));
        BCK(cudaStreamSynchronize(b->s));
        float ms = 0;
        cudaEventElapsedTime(&ms, b->ev0, b->ev1);
        total += ms;
        if (dip_out) {
            kb_gather_dip<<<dim3(8, b->nsys), 128, 0, b->s>>>(b->bd, int(n), b->dip_d);
            chunk_dip.resize(size_t(b->nsys) * n);
            BCK(cudaMemcpyAsync(chunk_dip.data(), b->dip_d, sizeof(double) * chunk_dip.size(), cudaMemcpyDeviceToHost, b->s));
            BCK(cudaStreamSynchronize(b->s));
            for (int i = 0; i < b->nsys; ++i)
                std::memcpy(dip_out + size_t(i) * steps + base, chunk_dip.data() + size_t(i) * n, sizeof(double) * n);
        }
    }
    b->last_ms = total;
    return G12_OK;
}

}  // namespace

extern "C" int g12_batch_create(const g12_params *systems, int32_t nsys, int32_t precision, int32_t device,
                                g12_batch **out)
{
    g_batch_error.clear();
    if (!systems || nsys < 1 || !out) return G12_ERR_INVALID;
    *out = nullptr;
    if (precision != G12_PREC_FP64) {
        g_batch_error = "batched ensembles run the FP64 engine";
        return G12_ERR_INVALID;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        g_batch_error = "no CUDA device (libg12kba has no CPU path)";
        return G12_ERR_NO_DEVICE;
    }
    auto b = new g12_batch();
    b->device = device;
    b->nsys = nsys;
    b->P.assign(systems, systems + nsys);
    auto fail = [&](int rc, const std::string &msg) {
        g_batch_error = msg.empty() ? b->err : msg;
        g12_batch_destroy(b);
        return rc;
    };
    for (int i = 0; i < nsys; ++i) {
        const int n = systems[i].Ns * systems[i].Nb;
        if (systems[i].Ns < 1 || systems[i].Nb < 1 || n > G12_MAX_N) return fail(G12_ERR_INVALID, "unsupported size in batch");
    }
    if (cudaSetDevice(device) != cudaSuccess) return fail(G12_ERR_INVALID, "bad device");
    cudaStreamCreateWithFlags(&b->s, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&b->s2, cudaStreamNonBlocking);
    cudaEventCreate(&b->ev0);
    cudaEventCreate(&b->ev1);
    cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming);
    // one pool, 256-byte aligned sub-buffers per system
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    std::vector<size_t> base(nsys);
    size_t total = 0;
    for (int i = 0; i < nsys; ++i) {
        const long long n = systems[i].Ns * systems[i].Nb, n2 = n * n, n3 = n2 * n, n4 = n2 * n2;
        base[i] = total;
        total += al(8 * n2 * 16) + al(5 * 2 * n4 * 16) + al(2 * 2 * n3 * 16) + al(n2 * systems[i].Ns * 16) +
                 al(n2 * 16) + al(kChunk * 8) + al(4 * 8 + sizeof(StepP));
    }
    if (cudaMalloc(&b->pool, total) != cudaSuccess) return fail(G12_ERR_NOMEM, "out of device memory (batch)");
    cudaMemset(b->pool, 0, total);
    b->dev.resize(nsys);
    b->cfg.resize(nsys);
    b->t_rk.assign(nsys, 0.0);
    b->t_temp.assign(nsys, 0.0);
    if (cudaMallocHost(&b->sched_h, sizeof(StepP) * nsys * kChunk) != cudaSuccess)
        return fail(G12_ERR_NOMEM, "out of pinned host memory (batch)");
    for (int i = 0; i < nsys; ++i) {
        const g12_params &p = systems[i];
        const long long n = p.Ns * p.Nb, n2 = n * n, n3 = n2 * n, n4 = n2 * n2;
        unsigned char *q = static_cast<unsigned char *>(b->pool) + base[i];
        auto take = [&](size_t bytes) {
            unsigned char *r = q;
            q += al(bytes);
            return r;
        };
        Dev &d = b->dev[i];
        std::memset(&d, 0, sizeof(Dev));
        d.Ns = p.Ns;
        d.Nb = p.Nb;
        d.n = int(n);
        d.nv = p.EHM ? std::max(0, p.Ns - 1) : 0;
        d.gate = (p.U != 0 && !p.HF) ? 1 : 0;
        d.n2 = n2;
        d.n3 = n3;
        d.n4 = n4;
        d.t1 = p.t1;
        d.t2 = p.t2;
        for (int r = 0; r < kMaxN; ++r) d.law[r] = (r < d.nv) ? vlaw(p, r + 1) : 0.0;
        double2 *g1 = reinterpret_cast<double2 *>(take(8 * n2 * 16));
        d.Y1 = g1;
        d.G1t0 = g1 + n2;
        d.G1t1 = g1 + 2 * n2;
        d.RK1 = g1 + 3 * n2;
        d.h = g1 + 4 * n2;
        d.Ix = g1 + 5 * n2;
        d.comm_dbg = g1 + 6 * n2;
        d.K1_dbg = g1 + 7 * n2;
        double2 *g2 = reinterpret_cast<double2 *>(take(5 * 2 * n4 * 16));
        d.Y2 = g2;
        d.RK2 = g2 + 2 * n4;
        d.TMP0 = g2 + 4 * n4;
        d.TMP1 = g2 + 6 * n4;
        d.TAB = g2 + 8 * n4;
        double2 *tb = reinterpret_cast<double2 *>(take(2 * 2 * n3 * 16));
        d.D = tb;
        d.Q = tb + 2 * n3;
        d.Rt = reinterpret_cast<double2 *>(take(n2 * p.Ns * 16));
        d.traj = reinterpret_cast<double2 *>(take(n2 * 16));
        d.traj_cap = 1;
        d.dip = reinterpret_cast<double *>(take(kChunk * 8));
        d.dip_cap = kChunk;
        unsigned char *words = take(4 * 8 + sizeof(StepP));
        d.counter = reinterpret_cast<long long *>(words);
        d.limit = reinterpret_cast<long long *>(words + 8);
        d.status = reinterpret_cast<int *>(words + 16);
        d.active = reinterpret_cast<int *>(words + 20);
        d.cur = reinterpret_cast<StepP *>(words + 32);
    }
    // every system's schedule chunk lives in one device array (one upload per chunk)
    if (cudaMalloc(&b->sched_d, sizeof(StepP) * nsys * kChunk) != cudaSuccess) return fail(G12_ERR_NOMEM, "");
    for (int i = 0; i < nsys; ++i) b->dev[i].sched = b->sched_d + size_t(i) * kChunk;
    // tile shapes (autotuned per n) and block offsets
    int maxn = 0;
    b->off_prep.assign(1, 0);
    b->off_g1.assign(1, 0);
    b->off_apply.assign(1, 0);
    b->off_tc.assign(1, 0);
    b->tcfg.resize(nsys);
    for (int i = 0; i < nsys; ++i) {
        const int n = b->dev[i].n;
        maxn = std::max(maxn, n);
        b->off_prep.push_back(b->off_prep.back() + prep_blocks(b->dev[i].n2));
        b->off_g1.push_back(b->off_g1.back() + g1_blocks(b->dev[i].n2));
    }
    if (cudaMalloc(&b->devs_d, sizeof(Dev) * nsys) != cudaSuccess) return fail(G12_ERR_NOMEM, "");
    for (int i = 0; i < nsys; ++i) {
        const int n = b->dev[i].n;
        const int nb = autotune(b, i);
        const int chunks = int((b->dev[i].n2 + nb - 1) / nb);
        const int blocks = b->dev[i].gate ? 2 * chunks : 0;
        if (apply_tc_ok(n)) {
            size_t sab = 0, scd = 0;
            b->tcfg[i] = tc_cfg_nb(n, nb, &sab, &scd);
            b->cfg[i] = apply_cfg_nb(n, 1);
            b->off_apply.push_back(b->off_apply.back());
            b->off_tc.push_back(b->off_tc.back() + blocks);
            b->smem_tab = std::max(b->smem_tab, sab);
            b->smem_tcd = std::max(b->smem_tcd, scd);
        } else {
            b->cfg[i] = apply_cfg_nb(n, nb);
            b->tcfg[i] = ApplyTcCfg{};
            b->off_apply.push_back(b->off_apply.back() + blocks);
            b->off_tc.push_back(b->off_tc.back());
            b->smem_ab = std::max(b->smem_ab, apply_smem(b->cfg[i], n, false));
            b->smem_cd = std::max(b->smem_cd, apply_smem(b->cfg[i], n, true));
        }
    }
    b->smem_prep = prep_smem();
    b->smem_g1 = g1_smem((long long)maxn * maxn);
    cudaFuncSetAttribute(kb_apply<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(b->smem_ab));
    cudaFuncSetAttribute(kb_apply<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(b->smem_cd));
    cudaFuncSetAttribute(kb_apply_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(b->smem_tab));
    cudaFuncSetAttribute(kb_apply_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(b->smem_tcd));
    cudaFuncSetAttribute(kb_prep, cudaFuncAttributeMaxDynamicSharedMemorySize, int(b->smem_prep));
    cudaFuncSetAttribute(kb_g1, cudaFuncAttributeMaxDynamicSharedMemorySize, int(b->smem_g1));
    cudaMemcpy(b->devs_d, b->dev.data(), sizeof(Dev) * nsys, cudaMemcpyHostToDevice);
    if (cudaMalloc(&b->cfg_d, sizeof(ApplyCfg) * nsys) != cudaSuccess ||
        cudaMalloc(&b->tcfg_d, sizeof(ApplyTcCfg) * nsys) != cudaSuccess ||
        cudaMalloc(&b->offs_d, sizeof(int) * 4 * (nsys + 1)) != cudaSuccess ||
        cudaMalloc(&b->limits_d, sizeof(long long) * nsys) != cudaSuccess ||
        cudaMalloc(&b->dip_d, sizeof(double) * nsys * kChunk) != cudaSuccess)
        return fail(G12_ERR_NOMEM, "out of device memory (batch)");
    cudaMemcpy(b->cfg_d, b->cfg.data(), sizeof(ApplyCfg) * nsys, cudaMemcpyHostToDevice);
    cudaMemcpy(b->offs_d, b->off_prep.data(), sizeof(int) * (nsys + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(b->offs_d + nsys + 1, b->off_g1.data(), sizeof(int) * (nsys + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(b->offs_d + 2 * (nsys + 1), b->off_apply.data(), sizeof(int) * (nsys + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(b->offs_d + 3 * (nsys + 1), b->off_tc.data(), sizeof(int) * (nsys + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(b->tcfg_d, b->tcfg.data(), sizeof(ApplyTcCfg) * nsys, cudaMemcpyHostToDevice);
    b->bd.tcfg = b->tcfg_d;
    b->bd.off_tc = b->offs_d + 3 * (nsys + 1);
    b->bd.devs = b->devs_d;
    b->bd.cfg = b->cfg_d;
    b->bd.off_prep = b->offs_d;
    b->bd.off_g1 = b->offs_d + nsys + 1;
    b->bd.off_apply = b->offs_d + 2 * (nsys + 1);
    b->bd.nsys = nsys;
    if (cudaGetLastError() != cudaSuccess) return fail(G12_ERR_CUDA, "batch set-up failed");
    *out = b;
    return G12_OK;
}

extern "C" int g12_batch_destroy(g12_batch *b)
{
    if (!b) return G12_OK;
    cudaSetDevice(b->device);
    if (b->s) cudaStreamSynchronize(b->s);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    cudaFree(b->pool);
    cudaFree(b->devs_d);
    cudaFree(b->cfg_d);
    cudaFree(b->tcfg_d);
    cudaFree(b->offs_d);
    cudaFree(b->limits_d);
    cudaFree(b->dip_d);
    cudaFree(b->sched_d);
    if (b->sched_h) cudaFreeHost(b->sched_h);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->join) cudaEventDestroy(b->join);
    if (b->s2) cudaStreamDestroy(b->s2);
    if (b->s) cudaStreamDestroy(b->s);
    delete b;
    return G12_OK;
}

extern "C" const char *g12_batch_last_error(const g12_batch *b) { return b ? b->err.c_str() : g_batch_error.c_str(); }

extern "C" int g12_batch_set_state(g12_batch *b, int32_t i, const double *G1, const double *G2xx, const double *G2xy)
{
    if (!b || i < 0 || i >= b->nsys || !G1) return G12_ERR_INVALID;
    BCK(cudaSetDevice(b->device));
    const Dev &d = b->dev[i];
    BCK(cudaMemcpyAsync(d.Y1, G1, d.n2 * sizeof(double2), cudaMemcpyHostToDevice, b->s));
    const double *src[2] = {G2xx, G2xy};
    for (int t = 0; t < 2; ++t) {
        if (!src[t]) {
            BCK(cudaMemsetAsync(d.Y2 + t * d.n4, 0, d.n4 * sizeof(double2), b->s));
            continue;
        }
        BCK(cudaMemcpyAsync(d.TAB, src[t], d.n4 * sizeof(double2), cudaMemcpyHostToDevice, b->s));
        k_from_ref<<<256, 256, 0, b->s>>>(d.TAB, d.Y2 + t * d.n4, d.Ns, d.Nb, d.n4);
    }
    k_init_D<<<256, 256, 0, b->s>>>(d);
    BCK(cudaGetLastError());
    BCK(cudaStreamSynchronize(b->s));
    b->t_rk[i] = 0;
    b->t_temp[i] = 0;
    return G12_OK;
}

extern "C" int g12_batch_get_state(g12_batch *b, int32_t i, double *G1, double *G2xx, double *G2xy)
{
    if (!b || i < 0 || i >= b->nsys) return G12_ERR_INVALID;
    BCK(cudaSetDevice(b->device));
    const Dev &d = b->dev[i];
    if (G1) BCK(cudaMemcpyAsync(G1, d.Y1, d.n2 * sizeof(double2), cudaMemcpyDeviceToHost, b->s));
    double *dst[2] = {G2xx, G2xy};
    for (int t = 0; t < 2; ++t) {
        if (!dst[t]) continue;
        k_to_ref<<<256, 256, 0, b->s>>>(d.Y2 + t * d.n4, d.TAB, d.Ns, d.Nb, d.n4);
        BCK(cudaMemcpyAsync(dst[t], d.TAB, d.n4 * sizeof(double2), cudaMemcpyDeviceToHost, b->s));
        BCK(cudaStreamSynchronize(b->s));
    }
    BCK(cudaStreamSynchronize(b->s));
    return G12_OK;
}

extern "C" int g12_batch_adiabatic_switch(g12_batch *b, int64_t *steps_done)
{
    if (!b) return G12_ERR_INVALID;
    BCK(cudaSetDevice(b->device));
    std::vector<long long> nas(b->nsys);
    long long mx = 0;
    for (int i = 0; i < b->nsys; ++i) {
        nas[i] = g12_as_steps(&b->P[i]);
        if (nas[i] < 0) {
            b->err = "adiabatic switching does not terminate for system " + std::to_string(i);
            return G12_ERR_INVALID;
        }
        mx = std::max(mx, nas[i]);
    }
    int rc = build_batch_graph(b);
    if (rc) return rc;
    for (long long base = 0; base < mx; base += kChunk) {
        const long long n = std::min(kChunk, mx - base);
        std::vector<long long> lim(b->nsys);
        for (int i = 0; i < b->nsys; ++i) {
            lim[i] = std::max(0LL, std::min(n, nas[i] - base));
            as_sched(b->P[i], base, lim[i], b->sched_h + size_t(i) * kChunk);
        }
        rc = upload_sched_and_reset(b, lim);
        if (rc) return rc;
        for (long long q = 0; q < n; ++q) BCK(cudaGraphLaunch(b->graph, b->s));
        BCK(cudaStreamSynchronize(b->s));
    }
    if (steps_done) *steps_done = mx;
    return G12_OK;
}

extern "C" int g12_batch_propagate(g12_batch *b, int64_t nsteps, double *dipole_out, int64_t *steps_done)
{
    if (!b || nsteps < 0) return G12_ERR_INVALID;
    BCK(cudaSetDevice(b->device));
    int rc = batch_run(
        b, nsteps, dipole_out,
        [&](long long, long long n) {
            for (int i = 0; i < b->nsys; ++i)
                rk_sched(b->P[i], n, &b->t_rk[i], &b->t_temp[i], b->sched_h + size_t(i) * kChunk);
        },
        [](long long) {});
    if (steps_done) *steps_done = rc == G12_OK ? nsteps : 0;
    return rc;
}

extern "C" int g12_batch_propagate_features(g12_batch *b, int64_t nsteps, int32_t every, float *feat_dev,
                                            double *dipole_out, int64_t *steps_done)
{
    if (!b || nsteps < 0 || every < 1 || !feat_dev) return G12_ERR_INVALID;
    const int n = b->P[0].Ns * b->P[0].Nb;
    for (int i = 1; i < b->nsys; ++i)
        if (b->P[i].Ns * b->P[i].Nb != n) {
            b->err = "feature recording needs one n for all systems";
            return G12_ERR_INVALID;
        }
    BCK(cudaSetDevice(b->device));
    const long long nsnap = nsteps / every;
    int rc = batch_run(
        b, nsteps, dipole_out,
        [&](long long, long long nn) {
            for (int i = 0; i < b->nsys; ++i)
                rk_sched(b->P[i], nn, &b->t_rk[i], &b->t_temp[i], b->sched_h + size_t(i) * kChunk);
        },
        [&](long long step) {
            if ((step + 1) % every == 0 && (step + 1) / every <= nsnap)
                kb_features<<<dim3(1, b->nsys), 128, 0, b->s>>>(b->bd, (step + 1) / every - 1, nsnap, feat_dev);
        });
    if (steps_done) *steps_done = rc == G12_OK ? nsteps : 0;
    return rc;
}

extern "C" double g12_batch_last_device_ms(const g12_batch *b) { return b ? b->last_ms : 0.0; }

extern "C" int32_t g12_batch_tile(const g12_batch *b, int32_t i)
{
    if (!b || i < 0 || i >= b->nsys) return 0;
    return apply_tc_ok(b->dev[i].n) ? b->tcfg[i].NB : b->cfg[i].NB;
}
