// Learned G1 extrapolator: an MLP that maps a window of K past G1 snapshots to
// the next M snapshots, trained and run on the GPU by the kernels in this file.
// No counterpart in the reference (G12KBA-GW has no learned component); the
// trajectories it learns from come from the propagation engine.
//
// Features of a snapshot: rho = -i G1 (Hermitian), its upper triangle
// (mu <= nu, row-major) as nt = n(n+1)/2 real parts followed by nt imaginary
// parts: F = n(n+1) floats.
// Network input (D0 = K F):   slot k < K-1: (x_{t-K+1+k} - x_t) / s_in
//                             slot K-1:     (x_t - mean) / s_abs
// Network output (D4 = M F):  (x_{t+1+m} - x_t) / s_out,  m = 0..M-1
// Layers: D0 -> D1 -> D2 -> D3 -> D4, exact GELU after the first three.
// Weights W_l are [out][in] FP32 masters; every GEMM rounds its operands to
// bf16 (round to nearest even) while staging them in shared memory and
// accumulates in FP32 in tensor memory (tcgen05.mma kind::f16, M = N = 128).
//
// GEMM forms (B = batch rows):
//   forward   Z_l  = A_{l-1} W_l^T        (A: K-contiguous, W: K-contiguous)
//   backward  dA   = dZ_l W_l             (W: N-contiguous)
//             dW_l = dZ_l^T A_{l-1}       (dZ: M-contiguous, A: N-contiguous)
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "g12kba.h"
#include "internal.h"

// The tcgen05 helpers (descriptors, mbarriers, TMEM loads) are compiled
// privately for this translation unit (internal linkage).
namespace {
namespace priv {
using ::g12::StageP;
using ::g12::StepP;
#include "sym_oz.cuh"
}  // namespace priv
}  // namespace

namespace {

using namespace priv::g12;

constexpr int kBM = 128, kBN = 128, kBK = 64;
constexpr int kGemmThreads = 128;
constexpr int kTileBytes = 128 * 128;  // 128 rows x 64 bf16
constexpr int kStages = 2;
constexpr int kGemmSmem = kStages * 2 * kTileBytes + 1024 + 64;

struct GemmArgs {
    const float *A;
    long long sam, sak;  // A(m, k) = A[m*sam + k*sak]
    const float *B;
    long long sbk, sbn;  // B(k, n) = B[k*sbk + n*sbn]
    float *C;
    long long ldc;       // C(m, n) = C[m*ldc + n]
    int M, N, K;
    int kchunks_per_split;
    int *err;
};

// stage one 128 x 64 operand tile (rows r, K columns) into a 128-byte swizzled
// K-major bf16 tile; element (r, k) is src[r*srow + k] when KC (K contiguous,
// sk unused) and src[k*sk + r] otherwise (rows contiguous, srow unused).
template <bool KC>
__device__ __forceinline__ void stage_tile(unsigned char *dst, const float *src, long long srow, long long sk, int r0,
                                           int k0, int tid)
{
    if constexpr (KC) {
        // 16 float4 per row; thread -> (row group, float4 column)
        const int c4 = tid & 15, rg = tid >> 4;
        float4 v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int r = rg + 8 * i;
            v[i] = *reinterpret_cast<const float4 *>(src + (long long)(r0 + r) * srow + (k0 + 4 * c4));
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int r = rg + 8 * i;
            const __nv_bfloat162 lo = __floats2bfloat162_rn(v[i].x, v[i].y);
            const __nv_bfloat162 hi = __floats2bfloat162_rn(v[i].z, v[i].w);
            uint2 w;
            w.x = *reinterpret_cast<const uint32_t *>(&lo);
            w.y = *reinterpret_cast<const uint32_t *>(&hi);
            *reinterpret_cast<uint2 *>(dst + swz_byte(r, 4 * c4)) = w;
        }
    } else {
        // rows contiguous: thread -> (4 consecutive rows, 2 consecutive k); 8 passes
#pragma unroll
        for (int it = 0; it < 8; ++it) {
            const int idx = tid + kGemmThreads * it;
            const int rq = idx & 31, kp = idx >> 5;  // 32 row quads x 32 k pairs
            const int r = 4 * rq, k = 2 * kp;
            const float4 a = *reinterpret_cast<const float4 *>(src + (long long)(k0 + k) * sk + (r0 + r));
            const float4 b = *reinterpret_cast<const float4 *>(src + (long long)(k0 + k + 1) * sk + (r0 + r));
            const __nv_bfloat162 p0 = __floats2bfloat162_rn(a.x, b.x);
            const __nv_bfloat162 p1 = __floats2bfloat162_rn(a.y, b.y);
            const __nv_bfloat162 p2 = __floats2bfloat162_rn(a.z, b.z);
            const __nv_bfloat162 p3 = __floats2bfloat162_rn(a.w, b.w);
            *reinterpret_cast<__nv_bfloat162 *>(dst + swz_byte(r + 0, k)) = p0;
            *reinterpret_cast<__nv_bfloat162 *>(dst + swz_byte(r + 1, k)) = p1;
            *reinterpret_cast<__nv_bfloat162 *>(dst + swz_byte(r + 2, k)) = p2;
            *reinterpret_cast<__nv_bfloat162 *>(dst + swz_byte(r + 3, k)) = p3;
        }
    }
}

// C(m, n) (+)= sum_k A(m, k) B(k, n) over this CTA's K range.  Grid: (N/128,
// M/128, splits).  ATOMIC: add into C (split-K; C zeroed by the caller).
template <bool AKC, bool BKC, bool ATOMIC>
__global__ void __launch_bounds__(kGemmThreads) k_mlp_gemm(GemmArgs g)
{
    extern __shared__ unsigned char smraw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + kStages * 2 * kTileBytes);  // kStages barriers
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + kStages);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n0 = blockIdx.x * kBN, m0 = blockIdx.y * kBM;
    const int kc_total = g.K / kBK;
    const int c_begin = blockIdx.z * g.kchunks_per_split;
    const int c_end = min(kc_total, c_begin + g.kchunks_per_split);
    if (c_begin >= c_end) return;  // uniform over the CTA

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(128)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = umma_idesc_bf16(kBN);
    uint32_t uses[kStages] = {0, 0};
    bool ok = true;
    for (int c = c_begin; c < c_end; ++c) {
        const int st = (c - c_begin) % kStages;
        unsigned char *As = sm + st * 2 * kTileBytes;
        unsigned char *Bs = As + kTileBytes;
        if (c - c_begin >= kStages) {  // the MMAs that last read this stage must be done
            ok = mbar_wait(&bars[st], (uses[st] - 1) & 1);
            ok = __syncthreads_and(ok);
            if (!ok) break;
        }
        const int k0 = c * kBK;
        // A tile rows are m; B tile rows are n (B(k, n): row stride sbn, K stride sbk)
        stage_tile<AKC>(As, g.A, g.sam, g.sak, m0, k0, tid);
        stage_tile<BKC>(Bs, g.B, g.sbn, g.sbk, n0, k0, tid);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            const uint32_t ab = smem_u32(As), bb = smem_u32(Bs);
#pragma unroll
            for (int ks = 0; ks < kBK / 16; ++ks)
                umma_bf16(tmem, umma_desc_sw128(ab + ks * 32), umma_desc_sw128(bb + ks * 32), idesc,
                          (c > c_begin || ks > 0) ? 1u : 0u);
            umma_commit(&bars[st]);
        }
        uses[st] += 1;
    }
    // wait for the last commit of every stage in use
    if (ok) {
        for (int s = 0; s < kStages; ++s)
            if (uses[s]) ok = ok && mbar_wait(&bars[s], (uses[s] - 1) & 1);
        ok = __syncthreads_and(ok);
    }
    if (!ok) {
        if (tid == 0) atomicExch(g.err, 1);
        for (int s = 0; s < kStages; ++s)
            if (uses[s]) mbar_wait(&bars[s], (uses[s] - 1) & 1);
    } else {
        tc_fence_after();
        // TMEM -> shared (rows of 64 columns, padded) -> coalesced global writes,
        // in two column halves (128 x 65 floats = 33 KB of the stage buffers)
        float *S = reinterpret_cast<float *>(sm);
        const int row = warp * 32 + lane;
        for (int h = 0; h < 2; ++h) {
            for (int cb = 0; cb < 64; cb += 32) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + h * 64 + cb, v);
#pragma unroll
                for (int i = 0; i < 32; ++i) S[row * 65 + cb + i] = v[i];
            }
            __syncthreads();
            for (int x = tid; x < kBM * 64; x += kGemmThreads) {
                const int r = x >> 6, cc = x & 63;
                float *dst = g.C + (long long)(m0 + r) * g.ldc + (n0 + h * 64 + cc);
                if constexpr (ATOMIC) atomicAdd(dst, S[r * 65 + cc]);
                else *dst = S[r * 65 + cc];
            }
            __syncthreads();
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128) : "memory");
}

__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x)
{
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// Z += bias (pre-activation kept for the backward pass); A = gelu(Z) or Z
__global__ void k_bias_act(float *Z, const float *bias, float *A, int rows, int cols, int act)
{
    const long long total = (long long)rows * cols;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const float z = Z[i] + bias[i % cols];
        Z[i] = z;
        if (A) A[i] = act ? gelu_f(z) : z;
    }
}

__global__ void k_gelu_back(const float *dA, const float *Z, float *dZ, long long total)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        dZ[i] = dA[i] * gelu_grad(Z[i]);
}

// db[c] = sum_r dZ[r][c]
__global__ void k_colsum(const float *dZ, int rows, int cols, float *db)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.f;
    for (int r = 0; r < rows; ++r) s += dZ[(long long)r * cols + c];
    db[c] = s;
}

// loss = mean (Yh - Y)^2; dY = 2 (Yh - Y) / count
__global__ void k_mse(const float *Yh, const float *Y, float *dY, long long count, double *loss)
{
    __shared__ double red[256];
    double acc = 0.0;
    const float sc = 2.0f / float(count);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x) {
        const float d = Yh[i] - Y[i];
        dY[i] = sc * d;
        acc += double(d) * d;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0] / double(count));
}

// Adam (Kingma and Ba 2015) with decoupled weight decay on the weights
__global__ void k_adam(float *w, const float *g, float *m, float *v, long long count, float lr, float b1, float b2,
                       float eps, float wd, float bc1, float bc2)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * ((mi / bc1) / (sqrtf(vi / bc2) + eps) + wd * w[i]);
    }
}

struct Norm {
    int K, M, F;
    float s_in, s_abs, s_out;
    const float *mean;  // F
};

// windows -> network input/target.  feat: [traj][snap][F]; idx[b] = (traj, t)
// with t the last snapshot of the window.  Y may be null (inference).
__device__ __forceinline__ uint32_t hash32(uint64_t x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return uint32_t(x);
}

// standard normal deviate from a counter (Box-Muller on two hashed uniforms)
__device__ __forceinline__ float gauss(uint64_t seed, uint64_t ctr)
{
    const float u1 = (hash32(seed ^ (2 * ctr)) + 1.0f) * 2.3283064e-10f;   // (0, 1]
    const float u2 = hash32(seed ^ (2 * ctr + 1)) * 2.3283064e-10f;
    return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

// noise > 0 adds noise * N(0, 1) to every input (training only)
__global__ void k_windows(const float *feat, long long snaps, const long long *idx, int batch, Norm nm, float *X,
                          float *Y, float noise = 0.f, unsigned long long seed = 0)
{
    const int b = blockIdx.y;
    if (b >= batch) return;
    const long long tr = idx[2 * b], t = idx[2 * b + 1];
    const float *base = feat + tr * snaps * nm.F;
    const float *xt = base + t * nm.F;
    const long long D0 = (long long)nm.K * nm.F, D4 = (long long)nm.M * nm.F;
    for (long long i = blockIdx.x * blockDim.x + threadIdx.x; i < D0; i += (long long)gridDim.x * blockDim.x) {
        const int k = int(i / nm.F), f = int(i % nm.F);
        float v;
        if (k == nm.K - 1) v = (xt[f] - nm.mean[f]) / nm.s_abs;
        else v = (base[(t - nm.K + 1 + k) * nm.F + f] - xt[f]) / nm.s_in;
        if (noise > 0.f) v += noise * gauss(seed, (uint64_t)b * D0 + i);
        X[b * D0 + i] = v;
    }
    if (!Y) return;
    for (long long i = blockIdx.x * blockDim.x + threadIdx.x; i < D4; i += (long long)gridDim.x * blockDim.x) {
        const int m = int(i / nm.F), f = int(i % nm.F);
        Y[b * D4 + i] = (base[(t + 1 + m) * nm.F + f] - xt[f]) / nm.s_out;
    }
}

// rollout: the network output of trajectory b (rows b) -> snapshots
// out[b][t+1+m] = x_t + s_out * y[m]  (t = the window's last snapshot)
__global__ void k_emit(const float *Yh, long long snaps, const long long *idx, int batch, Norm nm, float *feat)
{
    const int b = blockIdx.y;
    if (b >= batch) return;
    const long long tr = idx[2 * b], t = idx[2 * b + 1];
    float *base = feat + tr * snaps * nm.F;
    const float *xt = base + t * nm.F;
    const long long D4 = (long long)nm.M * nm.F;
    for (long long i = blockIdx.x * blockDim.x + threadIdx.x; i < D4; i += (long long)gridDim.x * blockDim.x) {
        const int m = int(i / nm.F), f = int(i % nm.F);
        base[(t + 1 + m) * nm.F + f] = xt[f] + nm.s_out * Yh[b * D4 + i];
    }
}

// scratch[b][j] = feat[traj_b][t_b + j], j < L  (idx = (traj, t) pairs)
__global__ void k_gather_seq(const float *feat, long long snaps, const long long *idx, int batch, int L, int F,
                             float *scratch)
{
    const int b = blockIdx.y;
    if (b >= batch) return;
    const float *src = feat + (idx[2 * b] * snaps + idx[2 * b + 1]) * F;
    float *dst = scratch + (long long)b * L * F;
    for (long long i = blockIdx.x * blockDim.x + threadIdx.x; i < (long long)L * F; i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

__global__ void k_seq_idx(long long *idx, int batch, long long t)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < batch) {
        idx[2 * b] = b;
        idx[2 * b + 1] = t;
    }
}

__global__ void k_advance_idx(long long *idx, int batch, int M)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < batch) idx[2 * b + 1] += M;
}

std::string g_mlp_error;

}  // namespace

struct g12_mlp {
    int device = 0;
    int dims[5] = {};
    int max_batch = 0;
    std::string err;
    cudaStream_t s = nullptr;
    std::vector<float *> W, b, gW, gb, mW, vW, mb, vb;  // per layer
    std::vector<float *> Z, A, dA;                      // per layer, max_batch rows
    float *dY = nullptr;
    float *Xbuf = nullptr, *Ybuf = nullptr;
    double *loss_d = nullptr;
    int *err_d = nullptr;
    long long *idx_d = nullptr;
    float *mean_d = nullptr;
    Norm norm{};
    bool has_norm = false;
    long long adam_t = 0;
    float *scratch = nullptr;
    long long scratch_floats = 0;
    float *grad_all = nullptr;     // every gW / gb segment, each padded to 64 floats
    long long grad_floats = 0;
    long long *idx2_d = nullptr;
    unsigned long long noise_ctr = 0;
    std::vector<void *> allocs;
};

namespace {

#define MCK(call)                                                                   \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            m->err = std::string(#call) + ": " + cudaGetErrorString(e_);            \
            return G12_ERR_CUDA;                                                    \
        }                                                                           \
    } while (0)

template <typename T>
bool malloc_zero(g12_mlp *m, T **p, size_t count)
{
    void *q = nullptr;
    if (cudaMalloc(&q, count * sizeof(T)) != cudaSuccess) return false;
    cudaMemset(q, 0, count * sizeof(T));
    m->allocs.push_back(q);
    *p = reinterpret_cast<T *>(q);
    return true;
}

int grid_for(long long count) { return int(std::min<long long>((count + 255) / 256, 148LL * 16)); }

// C = op(A) op(B) with the layouts of the header comment
template <bool AKC, bool BKC>
int gemm(g12_mlp *m, const float *A, long long sam, long long sak, const float *B, long long sbk, long long sbn, float *C,
         long long ldc, int M, int N, int K)
{
    if (M % kBM || N % kBN || K % kBK) {
        m->err = "MLP GEMM sizes must be multiples of 128 (M, N) and 64 (K)";
        return G12_ERR_INVALID;
    }
    GemmArgs g{A, sam, sak, B, sbk, sbn, C, ldc, M, N, K, 0, m->err_d};
    const int tiles = (M / kBM) * (N / kBN);
    const int kc = K / kBK;
    int splits = std::max(1, std::min(kc, (2 * 148 + tiles - 1) / tiles));
    g.kchunks_per_split = (kc + splits - 1) / splits;
    splits = (kc + g.kchunks_per_split - 1) / g.kchunks_per_split;
    const dim3 grid(N / kBN, M / kBM, splits);
    if (splits > 1) {
        MCK(cudaMemsetAsync(C, 0, sizeof(float) * size_t(M) * ldc, m->s));  // ldc == N for every call
        k_mlp_gemm<AKC, BKC, true><<<grid, kGemmThreads, kGemmSmem, m->s>>>(g);
    } else {
        k_mlp_gemm<AKC, BKC, false><<<grid, kGemmThreads, kGemmSmem, m->s>>>(g);
    }
    MCK(cudaGetLastError());
    return G12_OK;
}

// forward over `batch` rows of X (D0 wide); output in A[3] (pre-activation Z[3])
int forward(g12_mlp *m, const float *X, int batch)
{
    const float *in = X;
    for (int l = 0; l < 4; ++l) {
        const int din = m->dims[l], dout = m->dims[l + 1];
        int rc = gemm<true, true>(m, in, din, 1, m->W[l], 1, din, m->Z[l], dout, batch, dout, din);
        if (rc) return rc;
        const long long cnt = (long long)batch * dout;
        k_bias_act<<<grid_for(cnt), 256, 0, m->s>>>(m->Z[l], m->b[l], m->A[l], batch, dout, l < 3 ? 1 : 0);
        MCK(cudaGetLastError());
        in = m->A[l];
    }
    return G12_OK;
}

int backward(g12_mlp *m, const float *X, int batch)
{
    // dZ_3 = dY (in m->dY)
    const float *dZ = m->dY;
    for (int l = 3; l >= 0; --l) {
        const int din = m->dims[l], dout = m->dims[l + 1];
        const float *Ain = (l == 0) ? X : m->A[l - 1];
        // dW_l[o][i] = sum_b dZ[b][o] Ain[b][i]: A(m=o, k=b) = dZ[b*dout + o] (rows contiguous)
        int rc = gemm<false, false>(m, dZ, 1, dout, Ain, din, 1, m->gW[l], din, dout, din, batch);
        if (rc) return rc;
        k_colsum<<<(dout + 127) / 128, 128, 0, m->s>>>(dZ, batch, dout, m->gb[l]);
        MCK(cudaGetLastError());
        if (l == 0) break;
        // dA_{l-1}[b][i] = sum_o dZ[b][o] W_l[o][i]: B(k=o, n=i) = W[o*din + i] (n contiguous)
        rc = gemm<true, false>(m, dZ, dout, 1, m->W[l], din, 1, m->dA[l - 1], din, batch, din, dout);
        if (rc) return rc;
        const long long cnt = (long long)batch * din;
        k_gelu_back<<<grid_for(cnt), 256, 0, m->s>>>(m->dA[l - 1], m->Z[l - 1], m->dA[l - 1], cnt);
        MCK(cudaGetLastError());
        dZ = m->dA[l - 1];
    }
    return G12_OK;
}

int check_err(g12_mlp *m)
{
    int e = 0;
    MCK(cudaMemcpyAsync(&e, m->err_d, sizeof(int), cudaMemcpyDeviceToHost, m->s));
    MCK(cudaStreamSynchronize(m->s));
    if (e) {
        m->err = "tensor-core pipeline wait expired in the MLP GEMM";
        return G12_ERR_CUDA;
    }
    return G12_OK;
}

long long layer_params(const int *dims, int l) { return (long long)dims[l] * dims[l + 1] + dims[l + 1]; }

}  // namespace

extern "C" int g12_mlp_create(const int32_t *dims, int32_t max_batch, uint64_t seed, int32_t device, g12_mlp **out)
{
    g_mlp_error.clear();
    if (!dims || !out || max_batch < 128 || max_batch % 128) {
        g_mlp_error = "need 5 layer widths and max_batch a positive multiple of 128";
        return G12_ERR_INVALID;
    }
    *out = nullptr;
    if (dims[0] % kBN || dims[4] % kBN) {
        g_mlp_error = "input and output widths must be multiples of 128";
        return G12_ERR_INVALID;
    }
    for (int l = 0; l < 5; ++l)
        if (dims[l] <= 0 || dims[l] % kBN) {
            g_mlp_error = "layer widths must be positive multiples of 128";
            return G12_ERR_INVALID;
        }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        g_mlp_error = "no CUDA device (libg12kba has no CPU path)";
        return G12_ERR_NO_DEVICE;
    }
    auto m = new g12_mlp();
    m->device = device;
    m->max_batch = max_batch;
    std::memcpy(m->dims, dims, sizeof(m->dims));
    auto fail = [&](int rc, const char *msg) {
        g_mlp_error = msg;
        g12_mlp_destroy(m);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return fail(G12_ERR_CUDA, "cudaSetDevice failed");
    cudaStreamCreateWithFlags(&m->s, cudaStreamNonBlocking);
    m->W.resize(4);
    m->b.resize(4);
    m->gW.resize(4);
    m->gb.resize(4);
    m->mW.resize(4);
    m->vW.resize(4);
    m->mb.resize(4);
    m->vb.resize(4);
    m->Z.resize(4);
    m->A.resize(4);
    m->dA.resize(4);
    std::mt19937_64 rng(seed);
    // the gradients live in one block (one collective reduces all of them in
    // data-parallel training); segments start on 256-byte boundaries and the
    // padding stays zero
    auto pad64 = [](size_t x) { return (x + 63) / 64 * 64; };
    size_t gtot = 0;
    for (int l = 0; l < 4; ++l) gtot += pad64(size_t(dims[l]) * dims[l + 1]) + pad64(size_t(dims[l + 1]));
    if (!malloc_zero(m, &m->grad_all, gtot)) return fail(G12_ERR_NOMEM, "out of device memory (MLP)");
    m->grad_floats = (long long)gtot;
    size_t goff = 0;
    for (int l = 0; l < 4; ++l) {
        const size_t nw = size_t(dims[l]) * dims[l + 1], nb = dims[l + 1];
        m->gW[l] = m->grad_all + goff;
        goff += pad64(nw);
        m->gb[l] = m->grad_all + goff;
        goff += pad64(nb);
    }
    for (int l = 0; l < 4; ++l) {
        const size_t nw = size_t(dims[l]) * dims[l + 1], nb = dims[l + 1];
        if (!malloc_zero(m, &m->W[l], nw) || !malloc_zero(m, &m->b[l], nb) ||
            !malloc_zero(m, &m->mW[l], nw) || !malloc_zero(m, &m->vW[l], nw) ||
            !malloc_zero(m, &m->mb[l], nb) || !malloc_zero(m, &m->vb[l], nb) ||
            !malloc_zero(m, &m->Z[l], size_t(max_batch) * dims[l + 1]) ||
            !malloc_zero(m, &m->A[l], size_t(max_batch) * dims[l + 1]) ||
            !malloc_zero(m, &m->dA[l], size_t(max_batch) * dims[l + 1]))
            return fail(G12_ERR_NOMEM, "out of device memory (MLP)");
        // He-style uniform init, bound sqrt(3 / fan_in) (x 0.5 on the last layer)
        std::vector<float> w(nw);
        const double bound = std::sqrt(3.0 / dims[l]) * (l == 3 ? 0.5 : 1.0);
        std::uniform_real_distribution<double> u(-bound, bound);
        for (auto &x : w) x = float(u(rng));
        cudaMemcpy(m->W[l], w.data(), nw * sizeof(float), cudaMemcpyHostToDevice);
    }
    if (!malloc_zero(m, &m->dY, size_t(max_batch) * dims[4]) || !malloc_zero(m, &m->Xbuf, size_t(max_batch) * dims[0]) ||
        !malloc_zero(m, &m->Ybuf, size_t(max_batch) * dims[4]) || !malloc_zero(m, &m->loss_d, 1) ||
        !malloc_zero(m, &m->err_d, 1) || !malloc_zero(m, &m->idx_d, size_t(2) * max_batch) ||
        !malloc_zero(m, &m->idx2_d, size_t(2) * max_batch))
        return fail(G12_ERR_NOMEM, "out of device memory (MLP)");
    cudaFuncSetAttribute(k_mlp_gemm<true, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
    cudaFuncSetAttribute(k_mlp_gemm<true, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
    cudaFuncSetAttribute(k_mlp_gemm<true, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
    cudaFuncSetAttribute(k_mlp_gemm<true, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
    cudaFuncSetAttribute(k_mlp_gemm<false, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
    cudaFuncSetAttribute(k_mlp_gemm<false, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
    if (cudaDeviceSynchronize() != cudaSuccess) return fail(G12_ERR_CUDA, "MLP setup failed");
    *out = m;
    return G12_OK;
}

extern "C" int g12_mlp_destroy(g12_mlp *m)
{
    if (!m) return G12_OK;
    cudaSetDevice(m->device);
    if (m->s) cudaStreamSynchronize(m->s);
    for (void *p : m->allocs) cudaFree(p);
    if (m->scratch) cudaFree(m->scratch);
    if (m->s) cudaStreamDestroy(m->s);
    delete m;
    return G12_OK;
}

extern "C" const char *g12_mlp_last_error(const g12_mlp *m) { return m ? m->err.c_str() : g_mlp_error.c_str(); }

extern "C" int64_t g12_mlp_param_count(const g12_mlp *m)
{
    if (!m) return 0;
    long long c = 0;
    for (int l = 0; l < 4; ++l) c += layer_params(m->dims, l);
    return c;
}

// host layout: for each layer, W ([out][in]) then b
extern "C" int g12_mlp_set_params(g12_mlp *m, const float *params)
{
    if (!m || !params) return G12_ERR_INVALID;
    MCK(cudaSetDevice(m->device));
    const float *p = params;
    for (int l = 0; l < 4; ++l) {
        const size_t nw = size_t(m->dims[l]) * m->dims[l + 1], nb = m->dims[l + 1];
        MCK(cudaMemcpy(m->W[l], p, nw * sizeof(float), cudaMemcpyHostToDevice));
        MCK(cudaMemcpy(m->b[l], p + nw, nb * sizeof(float), cudaMemcpyHostToDevice));
        p += nw + nb;
    }
    return G12_OK;
}

static int copy_out(g12_mlp *m, const std::vector<float *> &W, const std::vector<float *> &b, float *out)
{
    float *p = out;
    for (int l = 0; l < 4; ++l) {
        const size_t nw = size_t(m->dims[l]) * m->dims[l + 1], nb = m->dims[l + 1];
        MCK(cudaMemcpy(p, W[l], nw * sizeof(float), cudaMemcpyDeviceToHost));
        MCK(cudaMemcpy(p + nw, b[l], nb * sizeof(float), cudaMemcpyDeviceToHost));
        p += nw + nb;
    }
    return G12_OK;
}

extern "C" int g12_mlp_get_params(g12_mlp *m, float *params)
{
    if (!m || !params) return G12_ERR_INVALID;
    MCK(cudaSetDevice(m->device));
    MCK(cudaStreamSynchronize(m->s));
    return copy_out(m, m->W, m->b, params);
}

extern "C" int g12_mlp_get_grads(g12_mlp *m, float *grads)
{
    if (!m || !grads) return G12_ERR_INVALID;
    MCK(cudaSetDevice(m->device));
    MCK(cudaStreamSynchronize(m->s));
    return copy_out(m, m->gW, m->gb, grads);
}

// Y (batch x D4, device) = network(X (batch x D0, device))
extern "C" int g12_mlp_forward(g12_mlp *m, const float *X_dev, int32_t batch, float *Y_dev)
{
    if (!m || !X_dev || !Y_dev || batch < 1 || batch > m->max_batch || batch % 128) return G12_ERR_INVALID;
    MCK(cudaSetDevice(m->device));
    int rc = forward(m, X_dev, batch);
    if (rc) return rc;
    MCK(cudaMemcpyAsync(Y_dev, m->A[3], sizeof(float) * size_t(batch) * m->dims[4], cudaMemcpyDeviceToDevice, m->s));
    return check_err(m);
}

// loss (mean squared error) and gradients of all parameters (kept on the device)
extern "C" int g12_mlp_loss_grad(g12_mlp *m, const float *X_dev, const float *Y_dev, int32_t batch, double *loss)
{
    if (!m || !X_dev || !Y_dev || batch < 1 || batch > m->max_batch || batch % 128) return G12_ERR_INVALID;
    MCK(cudaSetDevice(m->device));
    int rc = forward(m, X_dev, batch);
    if (rc) return rc;
    MCK(cudaMemsetAsync(m->loss_d, 0, sizeof(double), m->s));
    const long long cnt = (long long)batch * m->dims[4];
    k_mse<<<std::min(grid_for(cnt), 592), 256, 0, m->s>>>(m->A[3], Y_dev, m->dY, cnt, m->loss_d);
    MCK(cudaGetLastError());
    rc = backward(m, X_dev, batch);
    if (rc) return rc;
    double l = 0;
    MCK(cudaMemcpyAsync(&l, m->loss_d, sizeof(double), cudaMemcpyDeviceToHost, m->s));
    rc = check_err(m);
    if (loss) *loss = l;
    return rc;
}

extern "C" int g12_mlp_adam(g12_mlp *m, float lr, float beta1, float beta2, float eps, float weight_decay)
{
    if (!m) return G12_ERR_INVALID;
    MCK(cudaSetDevice(m->device));
    m->adam_t += 1;
    const float bc1 = 1.f - std::pow(beta1, float(m->adam_t)), bc2 = 1.f - std::pow(beta2, float(m->adam_t));
    for (int l = 0; l < 4; ++l) {
        const long long nw = (long long)m->dims[l] * m->dims[l + 1], nb = m->dims[l + 1];
        k_adam<<<grid_for(nw), 256, 0, m->s>>>(m->W[l], m->gW[l], m->mW[l], m->vW[l], nw, lr, beta1, beta2, eps,
                                               weight_decay, bc1, bc2);
        k_adam<<<grid_for(nb), 256, 0, m->s>>>(m->b[l], m->gb[l], m->mb[l], m->vb[l], nb, lr, beta1, beta2, eps, 0.f,
                                               bc1, bc2);
    }
    MCK(cudaGetLastError());
    return G12_OK;
}

extern "C" int g12_mlp_set_norm(g12_mlp *m, int32_t K, int32_t M, int32_t F, const float *mean, float s_in, float s_abs,
                                float s_out)
{
    if (!m || !mean || K < 2 || M < 1 || (long long)K * F != m->dims[0] || (long long)M * F != m->dims[4] ||
        !(s_in > 0) || !(s_abs > 0) || !(s_out > 0))
        return G12_ERR_INVALID;
    MCK(cudaSetDevice(m->device));
    if (!m->mean_d && !malloc_zero(m, &m->mean_d, size_t(F))) return G12_ERR_NOMEM;
    MCK(cudaMemcpy(m->mean_d, mean, sizeof(float) * F, cudaMemcpyHostToDevice));
    m->norm = Norm{K, M, F, s_in, s_abs, s_out, m->mean_d};
    m->has_norm = true;
    return G12_OK;
}

// one optimisation step on windows of a device feature array:
// feat [ntraj][snaps][F], idx (host) = batch pairs (traj, t)
static bool windows_in_range(const g12_mlp *m, int32_t ntraj, int64_t snaps, const int64_t *idx, int32_t batch)
{
    for (int b = 0; b < batch; ++b)
        if (idx[2 * b] < 0 || idx[2 * b] >= ntraj || idx[2 * b + 1] < m->norm.K - 1 || idx[2 * b + 1] + m->norm.M >= snaps)
            return false;
    return true;
}

extern "C" int g12_mlp_train_windows(g12_mlp *m, const float *feat_dev, int32_t ntraj, int64_t snaps, const int64_t *idx,
                                     int32_t batch, float lr, float weight_decay, double *loss)
{
    if (!m || !m->has_norm || !feat_dev || !idx || batch < 128 || batch % 128 || batch > m->max_batch)
        return G12_ERR_INVALID;
    MCK(cudaSetDevice(m->device));
    if (!windows_in_range(m, ntraj, snaps, idx, batch)) {
        m->err = "window out of the trajectory";
        return G12_ERR_INVALID;
    }
    MCK(cudaMemcpyAsync(m->idx_d, idx, sizeof(long long) * 2 * batch, cudaMemcpyHostToDevice, m->s));
    k_windows<<<dim3(64, batch), 256, 0, m->s>>>(feat_dev, snaps, m->idx_d, batch, m->norm, m->Xbuf, m->Ybuf);
    MCK(cudaGetLastError());
    int rc = g12_mlp_loss_grad(m, m->Xbuf, m->Ybuf, batch, loss);
    if (rc) return rc;
    return g12_mlp_adam(m, lr, 0.9f, 0.999f, 1e-8f, weight_decay);
}

// windows, loss and gradients without the Adam step (data-parallel training
// reduces the gradients across ranks in between)
extern "C" int g12_mlp_grad_windows(g12_mlp *m, const float *feat_dev, int32_t ntraj, int64_t snaps, const int64_t *idx,
                                    int32_t batch, double *loss)
{
    if (!m || !m->has_norm || !feat_dev || !idx || batch < 128 || batch % 128 || batch > m->max_batch)
        return G12_ERR_INVALID;
    MCK(cudaSetDevice(m->device));
    if (!windows_in_range(m, ntraj, snaps, idx, batch)) {
        m->err = "window out of the trajectory";
        return G12_ERR_INVALID;
    }
    MCK(cudaMemcpyAsync(m->idx_d, idx, sizeof(long long) * 2 * batch, cudaMemcpyHostToDevice, m->s));
    k_windows<<<dim3(64, batch), 256, 0, m->s>>>(feat_dev, snaps, m->idx_d, batch, m->norm, m->Xbuf, m->Ybuf);
    MCK(cudaGetLastError());
    return g12_mlp_loss_grad(m, m->Xbuf, m->Ybuf, batch, loss);
}

extern "C" int g12_mlp_grad_buffer(g12_mlp *m, float **grads_dev, int64_t *count)
{
    if (!m || !grads_dev || !count) return G12_ERR_INVALID;
    *grads_dev = m->grad_all;
    *count = m->grad_floats;
    return G12_OK;
}

// network inputs and targets of windows (host copies; for tests)
extern "C" int g12_mlp_windows(g12_mlp *m, const float *feat_dev, int32_t ntraj, int64_t snaps, const int64_t *idx,
                               int32_t batch, float *X_dev, float *Y_dev)
{
    if (!m || !m->has_norm || !feat_dev || !idx || batch < 1 || batch > m->max_batch) return G12_ERR_INVALID;
    if (!windows_in_range(m, ntraj, snaps, idx, batch)) {
        m->err = "window out of the trajectory";
        return G12_ERR_INVALID;
    }
    MCK(cudaSetDevice(m->device));
    MCK(cudaMemcpyAsync(m->idx_d, idx, sizeof(long long) * 2 * batch, cudaMemcpyHostToDevice, m->s));
    k_windows<<<dim3(64, batch), 256, 0, m->s>>>(feat_dev, snaps, m->idx_d, batch, m->norm, X_dev, Y_dev);
    MCK(cudaGetLastError());
    MCK(cudaStreamSynchronize(m->s));
    return G12_OK;
}

// Autoregressive rollout of `ntraj` trajectories in place: feat_dev [ntraj][snaps][F]
// holds snapshots 0..t0 of each trajectory; blocks of M snapshots are appended
// after t0 until `snaps` is reached (the last block is clipped by the caller's
// choice of snaps: snaps - 1 - t0 must be a multiple of M).
extern "C" int g12_mlp_rollout(g12_mlp *m, float *feat_dev, int32_t ntraj, int64_t snaps, int64_t t0, float *elapsed_ms)
{
    if (!m || !m->has_norm || !feat_dev || ntraj < 1 || ntraj > m->max_batch || t0 < m->norm.K - 1 || t0 >= snaps ||
        (snaps - 1 - t0) % m->norm.M)
        return G12_ERR_INVALID;
    MCK(cudaSetDevice(m->device));
    const int rows = (ntraj + 127) / 128 * 128;  // GEMM rows (padding rows hold zeros)
    std::vector<long long> idx(size_t(2) * ntraj);
    for (int b = 0; b < ntraj; ++b) {
        idx[2 * b] = b;
        idx[2 * b + 1] = t0;
    }
    MCK(cudaMemcpyAsync(m->idx_d, idx.data(), sizeof(long long) * idx.size(), cudaMemcpyHostToDevice, m->s));
    MCK(cudaMemsetAsync(m->Xbuf, 0, sizeof(float) * size_t(rows) * m->dims[0], m->s));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, m->s);
    const long long nblocks = (snaps - 1 - t0) / m->norm.M;
    int rc = G12_OK;
    for (long long q = 0; q < nblocks && !rc; ++q) {
        k_windows<<<dim3(64, ntraj), 256, 0, m->s>>>(feat_dev, snaps, m->idx_d, ntraj, m->norm, m->Xbuf, nullptr);
        rc = forward(m, m->Xbuf, rows);
        if (rc) break;
        k_emit<<<dim3(32, ntraj), 256, 0, m->s>>>(m->A[3], snaps, m->idx_d, ntraj, m->norm, feat_dev);
        k_advance_idx<<<(ntraj + 127) / 128, 128, 0, m->s>>>(m->idx_d, ntraj, m->norm.M);
    }
    cudaEventRecord(e1, m->s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (elapsed_ms) *elapsed_ms = ms;
    if (rc) return rc;
    MCK(cudaGetLastError());
    return check_err(m);
}

namespace {

// dipole.h:25-32 of one snapshot's features (Im G1_ii = Re rho_ii sits at the
// upper-triangle index i n - i (i - 1) / 2 of the real parts)
__device__ __forceinline__ double feat_dipole(const float *f, int n)
{
    double p = 0.0;
    for (int i = 0; i < n / 2; ++i) {
        const int a = i * n - i * (i - 1) / 2, j = n - 1 - i, b2 = j * n - j * (j - 1) / 2;
        p += 2.0 * (n / 2.0 - i - 0.5) * (double(f[a]) - double(f[b2])) / n;
    }
    return p;
}

// One block per trajectory: max |p_ref| after t0, then the maximum of
// |p_pred - p_ref| / max |p_ref| over each checkpoint interval (atomicMax on
// the bits of nonnegative doubles), then the first failing checkpoint.
__global__ void __launch_bounds__(256) k_judge(const float *pred, const float *ref, long long snaps, long long t0, int n,
                                               int every, int nck, double tol, long long *accepted)
{
    extern __shared__ unsigned long long ivmax[];  // nck interval maxima
    __shared__ double red[256];
    const int F = n * (n + 1);
    const float *P = pred + (long long)blockIdx.x * snaps * F;
    const float *Rf = ref + (long long)blockIdx.x * snaps * F;
    const long long T = snaps - 1 - t0;
    double amp = 0.0;
    for (long long s = threadIdx.x; s < T; s += blockDim.x) amp = fmax(amp, fabs(feat_dipole(Rf + (t0 + 1 + s) * F, n)));
    red[threadIdx.x] = amp;
    for (int x = threadIdx.x; x < nck; x += blockDim.x) ivmax[x] = 0ull;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    amp = fmax(red[0], 1e-12);
    for (long long s = threadIdx.x; s < (long long)nck * every; s += blockDim.x) {
        const long long q = (t0 + 1 + s) * F;
        const double e = fabs(feat_dipole(P + q, n) - feat_dipole(Rf + q, n)) / amp;
        atomicMax(&ivmax[s / every], (unsigned long long)__double_as_longlong(e));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        long long acc = T;
        double run = 0.0;
        for (int j = 0; j < nck; ++j) {
            run = fmax(run, __longlong_as_double((long long)ivmax[j]));
            if (run > tol) {
                acc = (long long)j * every;
                break;
            }
        }
        accepted[blockIdx.x] = acc;
    }
}

}  // namespace

extern "C" int g12_mlp_judge(g12_mlp *m, const float *pred_dev, const float *ref_dev, int32_t ntraj, int64_t snaps,
                             int64_t t0, int32_t every, double tol, int64_t *accepted_out)
{
    if (!m || !m->has_norm || !pred_dev || !ref_dev || !accepted_out || ntraj < 1 || every < 1 || t0 < 0 ||
        t0 >= snaps - 1)
        return G12_ERR_INVALID;
    const int F = m->norm.F;
    int n = 0;
    while ((n + 1) * (n + 2) <= F) ++n;
    if (n * (n + 1) != F) return G12_ERR_INVALID;
    const long long nck = (snaps - 1 - t0) / every;  // full checkpoint intervals
    if (nck > 6000) {
        m->err = "g12_mlp_judge: more than 6000 checkpoints";
        return G12_ERR_INVALID;
    }
    MCK(cudaSetDevice(m->device));
    long long *acc_d = nullptr;
    MCK(cudaMallocAsync(&acc_d, sizeof(long long) * ntraj, m->s));
    k_judge<<<ntraj, 256, sizeof(unsigned long long) * std::max<long long>(nck, 1), m->s>>>(
        pred_dev, ref_dev, snaps, t0, n, every, int(nck), tol, acc_d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(accepted_out, acc_d, sizeof(long long) * ntraj, cudaMemcpyDeviceToHost, m->s);
    cudaFreeAsync(acc_d, m->s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->s);
    if (e != cudaSuccess) {
        m->err = std::string("g12_mlp_judge: ") + cudaGetErrorString(e);
        return G12_ERR_CUDA;
    }
    return G12_OK;
}

// One optimisation step after `r` blocks of the network's own rollout
// ("pushforward" training): windows start at (traj, t) of feat_dev, the network
// predicts r blocks of M snapshots from them (no gradient through those), and
// the step trains the prediction of the next M true snapshots from the window
// that now ends in predicted snapshots.  noise > 0 adds Gaussian noise of that
// size (in normalised units) to every network input of the step.
extern "C" int g12_mlp_train_pushforward(g12_mlp *m, const float *feat_dev, int32_t ntraj, int64_t snaps,
                                         const int64_t *idx, int32_t batch, int32_t r, float noise, float lr,
                                         float weight_decay, double *loss)
{
    if (!m || !m->has_norm || !feat_dev || !idx || r < 0 || batch < 128 || batch % 128 || batch > m->max_batch)
        return G12_ERR_INVALID;
    const Norm &nm = m->norm;
    const int L = nm.K + (r + 1) * nm.M;
    for (int b = 0; b < batch; ++b)
        if (idx[2 * b] < 0 || idx[2 * b] >= ntraj || idx[2 * b + 1] < nm.K - 1 ||
            idx[2 * b + 1] - (nm.K - 1) + L > snaps) {
            m->err = "window out of the trajectory";
            return G12_ERR_INVALID;
        }
    MCK(cudaSetDevice(m->device));
    const long long need = (long long)batch * L * nm.F;
    if (need > m->scratch_floats) {
        MCK(cudaStreamSynchronize(m->s));
        if (m->scratch) cudaFree(m->scratch);
        m->scratch = nullptr;
        m->scratch_floats = 0;
        MCK(cudaMalloc(&m->scratch, sizeof(float) * need));
        m->scratch_floats = need;
    }
    std::vector<long long> first(size_t(2) * batch);
    for (int b = 0; b < batch; ++b) {
        first[2 * b] = idx[2 * b];
        first[2 * b + 1] = idx[2 * b + 1] - (nm.K - 1);
    }
    MCK(cudaMemcpyAsync(m->idx_d, first.data(), sizeof(long long) * first.size(), cudaMemcpyHostToDevice, m->s));
    k_gather_seq<<<dim3(32, batch), 256, 0, m->s>>>(feat_dev, snaps, m->idx_d, batch, L, nm.F, m->scratch);
    k_seq_idx<<<(batch + 127) / 128, 128, 0, m->s>>>(m->idx2_d, batch, nm.K - 1);
    MCK(cudaGetLastError());
    for (int q = 0; q < r; ++q) {
        k_windows<<<dim3(64, batch), 256, 0, m->s>>>(m->scratch, L, m->idx2_d, batch, nm, m->Xbuf, nullptr);
        int rc = forward(m, m->Xbuf, batch);
        if (rc) return rc;
        k_emit<<<dim3(32, batch), 256, 0, m->s>>>(m->A[3], L, m->idx2_d, batch, nm, m->scratch);
        k_advance_idx<<<(batch + 127) / 128, 128, 0, m->s>>>(m->idx2_d, batch, nm.M);
    }
    k_windows<<<dim3(64, batch), 256, 0, m->s>>>(m->scratch, L, m->idx2_d, batch, nm, m->Xbuf, m->Ybuf, noise,
                                                 0x9E3779B97F4A7C15ULL + m->noise_ctr++);
    MCK(cudaGetLastError());
    int rc = g12_mlp_loss_grad(m, m->Xbuf, m->Ybuf, batch, loss);
    if (rc) return rc;
    return g12_mlp_adam(m, lr, 0.9f, 0.999f, 1e-8f, weight_decay);
}
