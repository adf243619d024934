// g12_rhs_noalloc: one right-hand-side evaluation that allocates no device
// memory.  Everything g12_rhs keeps in context buffers (the row-mixing half of
// the two-body commutator, the particle-2 diagonals, the Pi/Psi factor
// tables, h, the collision integral, the layout-converted inputs and outputs)
// lives instead in one file-scope __device__ array of fixed size.
//
// Who needs this: code that runs inside a host application whose device
// memory is owned by another allocator (a caching or arena allocator that has
// already reserved the memory, so a raw cudaMalloc would fail or fragment the
// pool), and code in latency-critical loops, where cudaMalloc/cudaFree would
// add implicit device synchronisation.  Such callers hand in device buffers for
// the inputs and outputs only.
//
// Limits and sharing rules:
//   - n = Ns*Nb <= G12_NOALLOC_MAX_N (16); larger systems are rejected.
//   - The scratch array (kScratchBytes, about 6.4 MiB) exists once per GPU that
//     loads the library and is held until the process exits.
//   - Every call on a device shares that one array and leaves the last call's
//     contents in it; calls whose work overlaps on the GPU (other streams,
//     other host threads) race on it and must be serialised by the caller.
//   - The first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) and sets kernel attributes; make that first call
//     before any stream capture.  That set-up is cached per device ordinal for
//     the life of the process and does not survive cudaDeviceReset: do not
//     call this entry point after resetting a device it was used on.
#include "g12kba.h"
#include "internal.h"

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>

// Kernels compiled privately for this translation unit (internal linkage), so
// this file shares no code path with the context engine.
namespace {
namespace priv {
using ::g12::StageP;
using ::g12::StepP;
#include "fp64_kernels.cuh"
}  // namespace priv
namespace K = priv::g12;
using ::g12::StepP;
}  // namespace

namespace {

constexpr int kMax = G12_NOALLOC_MAX_N;
constexpr size_t kN2 = size_t(kMax) * kMax, kN3 = kN2 * kMax, kN4 = kN2 * kN2;
// double2 slots: 8 n^2 arrays, 3 x (2 n^4) tensors, 2 x (2 n^3) tables, Rt (n^2 Ns)
constexpr size_t kSlots = 8 * kN2 + 6 * kN4 + 4 * kN3 + kN2 * kMax;
constexpr size_t kScratchBytes = kSlots * sizeof(double2) + 512;  // + StepP and the active flag

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct DeviceSetup {
    void *base = nullptr;
    bool ready = false;
};

std::mutex g_mu;
DeviceSetup g_setup[256];

void set_err(char *err, int32_t cap, const std::string &msg)
{
    if (err && cap > 0) std::snprintf(err, size_t(cap), "%s", msg.c_str());
}

__global__ void k_noalloc_params(StepP sp, StepP *cur, int *active)
{
    *cur = sp;
    *active = 1;
}

struct Cfg {
    K::ApplyCfg a;
    int threads;
    size_t ab_smem, cd_smem;
};

Cfg apply_cfg(int n)
{
    Cfg c;
    c.a.NP = (n + 3) / 4 * 4;
    c.a.S = c.a.NP / 4;
    c.a.LD = c.a.NP + 1;
    const int per = c.a.S * c.a.S;
    c.a.NB = std::max(1, std::min(n * n, 256 / per));
    c.threads = c.a.NB * per;
    c.ab_smem = (size_t(2) * c.a.NP * c.a.LD + size_t(c.a.NB) * c.a.NP * c.a.LD) * sizeof(double2);
    c.cd_smem = c.ab_smem + size_t(n) * n * sizeof(double2);
    return c;
}

// Once per device, with that device current: the array's device address and
// the kernels' shared-memory limits.
int setup_device(int dev, void **base, std::string *msg)
{
    std::lock_guard<std::mutex> lock(g_mu);
    if (dev < 0 || dev >= 256) {
        *msg = "device ordinal out of range";
        return G12_ERR_INVALID;
    }
    DeviceSetup &s = g_setup[dev];
    if (!s.ready) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            *msg = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return G12_ERR_CUDA;
        }
        const Cfg c = apply_cfg(kMax);
        const size_t prep = K::prep_smem();
        if ((e = cudaFuncSetAttribute(K::k_apply<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(c.ab_smem))) ||
            (e = cudaFuncSetAttribute(K::k_apply<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(c.cd_smem))) ||
            (e = cudaFuncSetAttribute(K::k_prep, cudaFuncAttributeMaxDynamicSharedMemorySize, int(prep))) ||
            (e = cudaFuncSetAttribute(K::k_g1, cudaFuncAttributeMaxDynamicSharedMemorySize, int(K::g1_smem(kN2))))) {
            *msg = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
            return G12_ERR_CUDA;
        }
        s.base = p;
        s.ready = true;
    }
    *base = s.base;
    return G12_OK;
}

}  // namespace

extern "C" int g12_rhs_noalloc(const g12_params *p, const double *G1_dev, const double *G2xx_dev,
                               const double *G2xy_dev, double U_eff, double w_quench, int32_t Nq_eff,
                               double *K1_dev, double *K2xx_dev, double *K2xy_dev, void *stream, char *err,
                               int32_t errcap)
{
    if (!p || !G1_dev || !G2xx_dev || !G2xy_dev || !K1_dev || !K2xx_dev || !K2xy_dev) {
        set_err(err, errcap, "g12_rhs_noalloc: null argument");
        return G12_ERR_INVALID;
    }
    const int Ns = p->Ns, Nb = p->Nb, n = Ns * Nb;
    if (Ns < 1 || Nb < 1) {
        set_err(err, errcap, "g12_rhs_noalloc: invalid Ns = " + std::to_string(Ns) + ", Nb = " + std::to_string(Nb) +
                                 " (both must be >= 1)");
        return G12_ERR_INVALID;
    }
    if (n > kMax) {
        set_err(err, errcap, "g12_rhs_noalloc: n = Ns*Nb = " + std::to_string(n) +
                                 " exceeds the static scratch limit G12_NOALLOC_MAX_N = " + std::to_string(kMax));
        return G12_ERR_INVALID;
    }
    // an error left pending by earlier, unrelated work of the caller is reported
    // as such (and cleared), not blamed on this call's launches
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_err(err, errcap, std::string("g12_rhs_noalloc: a CUDA error from earlier work was pending on entry "
                                         "(nothing was launched): ") + cudaGetErrorString(e));
        return G12_ERR_CUDA;
    }
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_err(err, errcap, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        return G12_ERR_NO_DEVICE;
    }
    void *basev = nullptr;
    std::string msg;
    int rc = setup_device(dev, &basev, &msg);
    if (rc) {
        set_err(err, errcap, "g12_rhs_noalloc: " + msg);
        return rc;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long n2 = (long long)n * n, n3 = n2 * n, n4 = n2 * n2;

    // carve the scratch array (sized for kMax, used for n)
    double2 *b = static_cast<double2 *>(basev);
    auto take = [&](size_t count) {
        double2 *q = b;
        b += count;
        return q;
    };
    K::Dev d{};
    d.Ns = Ns;
    d.Nb = Nb;
    d.n = n;
    d.nv = p->EHM ? std::max(0, Ns - 1) : 0;
    d.gate = (p->U != 0 && !p->HF) ? 1 : 0;
    d.debug = 1;
    d.n2 = n2;
    d.n3 = n3;
    d.n4 = n4;
    d.t1 = p->t1;
    d.t2 = p->t2;
    for (int r = 0; r < K::kMaxN; ++r) {
        double law = 0.0;
        if (r < d.nv) law = (p->v_law == G12_VLAW_INV) ? 1.0 / (1.0 + double(r + 1)) : std::exp(-p->decay_rate * (r + 1));
        d.law[r] = law;
    }
    d.G1t0 = const_cast<double2 *>(reinterpret_cast<const double2 *>(G1_dev));
    d.G1t1 = take(kN2);
    d.Y1 = take(kN2);
    d.RK1 = take(kN2);
    d.h = take(kN2);
    d.Ix = take(kN2);
    d.comm_dbg = take(kN2);
    take(kN2);
    take(kN2);
    d.K1_dbg = reinterpret_cast<double2 *>(K1_dev);
    d.Y2 = take(2 * kN4);
    d.TMP0 = take(2 * kN4);
    d.TAB = take(2 * kN4);
    d.D = take(2 * kN3);
    d.Q = take(2 * kN3);
    d.Rt = take(kN2 * kMax);
    d.TMP1 = d.TMP0;  // not touched by a single debug stage
    d.RK2 = d.TMP0;
    unsigned char *tail = reinterpret_cast<unsigned char *>(b);
    d.cur = reinterpret_cast<StepP *>(tail);
    d.active = reinterpret_cast<int *>(tail + 256);

    StepP sp{};
    for (int k = 0; k < 4; ++k) {
        sp.st[k].U = U_eff;
        sp.st[k].wq = w_quench;
        sp.st[k].nq = Nq_eff;
        sp.st[k].w = 1;
    }
    const Cfg c = apply_cfg(n);
    const int prep_blocks = K::prep_blocks(n2);
    const size_t prep_smem = K::prep_smem();
    const dim3 grid(unsigned((n2 + c.a.NB - 1) / c.a.NB), 2, 1);

    k_noalloc_params<<<1, 1, 0, s>>>(sp, d.cur, d.active);
    K::k_from_ref<<<64, 256, 0, s>>>(reinterpret_cast<const double2 *>(G2xx_dev), d.Y2, Ns, Nb, n4);
    K::k_from_ref<<<64, 256, 0, s>>>(reinterpret_cast<const double2 *>(G2xy_dev), d.Y2 + n4, Ns, Nb, n4);
    K::k_init_D<<<64, 256, 0, s>>>(d);
    K::k_prep<<<prep_blocks, K::kPrepWarps * 32, prep_smem, s>>>(d, 0);
    K::k_g1<<<K::g1_blocks(n2), K::kG1Threads, K::g1_smem(n2), s>>>(d, 0);
    if (d.gate) {
        K::k_apply<false><<<grid, c.threads, c.ab_smem, s>>>(d, 0, c.a);
        K::k_apply<true><<<grid, c.threads, c.cd_smem, s>>>(d, 0, c.a);
        K::k_to_ref<<<64, 256, 0, s>>>(d.TMP0, reinterpret_cast<double2 *>(K2xx_dev), Ns, Nb, n4);
        K::k_to_ref<<<64, 256, 0, s>>>(d.TMP0 + n4, reinterpret_cast<double2 *>(K2xy_dev), Ns, Nb, n4);
    } else {
        // no two-body terms (RK_solver.h:154): K2 is zero
        if ((e = cudaMemsetAsync(K2xx_dev, 0, size_t(n4) * sizeof(double2), s)) != cudaSuccess ||
            (e = cudaMemsetAsync(K2xy_dev, 0, size_t(n4) * sizeof(double2), s)) != cudaSuccess) {
            cudaGetLastError();
            set_err(err, errcap, std::string("g12_rhs_noalloc: cudaMemsetAsync of K2: ") + cudaGetErrorString(e));
            return G12_ERR_CUDA;
        }
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_err(err, errcap, std::string("g12_rhs_noalloc launch: ") + cudaGetErrorString(e));
        return G12_ERR_CUDA;
    }
    return G12_OK;
}
