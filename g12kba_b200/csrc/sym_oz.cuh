// tcgen05 (sm_100a) W contraction with exact integer-digit products
// (error-free splitting after Ozaki, Ogita, Oishi and Rump, "Error-free
// transformations of matrix multiplication by using fast routines of matrix
// multiplication and its applications", Numer. Algorithms 59 (2012)).
//
// Why: tcgen05 kind::tf32 / kind::f16 accumulate in FP32 with a rounding that
// is biased toward zero (measured on B200: about -4e-8 relative per W
// element).  A uniformly shrunk commutator acts like a rescaled Hamiltonian,
// so the phase error of G1 grows linearly in time (1.5e-5 after the 10,000-step
// n = 32 run).  Here every partial sum is an integer below 2^24, so the FP32
// accumulation is exact whatever its rounding mode.
//
// Each A row m (and each B row j) is written as
//   a = 2^(e_m - 6) * (d0 + d1 2^-7 + d2 2^-14 + d3 2^-21),
// with e_m = floor(log2 max_k |a|), |d0| <= 128 and |d1..d3| <= 64 obtained by
// successive round-to-nearest (so the truncation after d3, <= 2^-28 of the row
// maximum, is unbiased).  The digits are held exactly in bf16.  The products
// with digit-level i + j = L (L = 0..3) accumulate in TMEM accumulator L:
//   |sum| <= (L+1) * K * 128 * 128 <= 4 * 64 * 2^14 = 2^22 < 2^24  (exact).
// T1 = 2^(e_m - 6) 2^(e_j - 6) sum_L 2^(-7L) P_L is formed in FP64.
//
// Tile and operands as in sym_tc.cuh, except that the FP32 rows are read by the
// threads (two rows per warp per load, coalesced) and digit-split straight into
// 128-byte-swizzled bf16 rows; K = 2n bf16 = 128 (n = 32) or 64 (n = 16) bytes.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "sym_tc.cuh"

namespace g12 {

constexpr int kOzDigits = 4;
constexpr int kOzLevels = 4;

// D f32, A/B bf16, K-major, M = 128, N = n_cols
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n_cols)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n_cols >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}

// digits of x (already scaled so that |x| < 2^21): x = d0 2^14 + d1 2^7 + d2 + d3 2^-7 + r
__device__ __forceinline__ void oz_digits(float x, float (&d)[kOzDigits])
{
    float r = x;
    d[0] = rintf(r * (1.0f / 16384.0f));
    r -= d[0] * 16384.0f;
    d[1] = rintf(r * (1.0f / 128.0f));
    r -= d[1] * 128.0f;
    d[2] = rintf(r);
    r -= d[2];
    d[3] = rintf(r * 128.0f);
}

template <int NN>
struct OzShape {
    static constexpr int N = 2 * NN;           // UMMA N
    static constexpr int K = 2 * NN;           // real K (bf16 elements per row)
    static constexpr int KS = K / 16;          // 32-byte K steps per product
    static constexpr int CPT = 128 / NN;
    static constexpr int ROW_BYTES = 128;      // one 128-byte swizzled row (zero-padded for n = 16)
    static constexpr int A_BYTES = 128 * ROW_BYTES;
    static constexpr int B_BYTES = N * ROW_BYTES;
    static constexpr int TMEM_COLS = kOzLevels * N;  // 256 (n = 32) or 128 (n = 16)
    static constexpr int OFF_A = 0;                               // kOzDigits x A_BYTES
    static constexpr int OFF_B = kOzDigits * A_BYTES;             // kOzDigits x B_BYTES
    static constexpr int OFF_EA = OFF_B + kOzDigits * B_BYTES;    // 128 ints
    static constexpr int OFF_EB = OFF_EA + 128 * 4;               // N ints
    static constexpr int OFF_BAR = OFF_EB + 256 * 4;
    static constexpr int SMEM = OFF_BAR + 64 + 1024;
    static constexpr int S_LD = N + 1;
    static constexpr int LPR = K * 4 / 16;    // lanes per FP32 row (16-byte loads): 16 or 8
    static constexpr int RPW = 32 / LPR;      // rows per warp load: 2 or 4
    static_assert(128 * S_LD * 4 <= kOzDigits * A_BYTES, "staging must fit in the digit buffers");
    static_assert(TMEM_COLS <= 256, "two CTAs per SM share 512 TMEM columns");
};

__device__ __forceinline__ int swz_byte(int row, int kk2)  // bf16 element kk2 of a 128-byte swizzled row
{
    return row * 128 + ((((kk2 >> 3) ^ (row & 7)) << 4) | ((kk2 & 7) << 1));
}

template <int NN>
__global__ void __launch_bounds__(128) k_sym_gemm_oz(SymDev s, int k)
{
    using Sh = OzShape<NN>;
    if (!*s.d.active) return;
    extern __shared__ unsigned char smraw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
    unsigned char *Ad = sm + Sh::OFF_A;
    unsigned char *Bd = sm + Sh::OFF_B;
    int *eA = reinterpret_cast<int *>(sm + Sh::OFF_EA);
    int *eB = reinterpret_cast<int *>(sm + Sh::OFF_EB);
    uint64_t *bar_mma = reinterpret_cast<uint64_t *>(sm + Sh::OFF_BAR);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar_mma + 1);
    float *S = reinterpret_cast<float *>(Ad);  // staging reuses the A digit buffers after the MMAs
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long n2 = (long long)NN * NN;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(Sh::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(bar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // zero the digit buffers once (the n = 16 rows use half of each 128-byte row)
    for (int i = tid; i < (Sh::OFF_EA) / 16; i += blockDim.x) reinterpret_cast<uint4 *>(sm)[i] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    // B digits: rows j of the real form of h^T (FP64), one thread per row
    for (int j = tid; j < Sh::N; j += blockDim.x) {
        const int po = j / NN, mu1 = j % NN;
        double mx = 0.0;
        for (int kk = 0; kk < Sh::K; ++kk) {
            const int pi = kk / NN, rho = kk % NN;
            const double2 hv = s.d.h[mu1 * NN + rho];
            const double v = (po == 0) ? ((pi == 0) ? hv.x : -hv.y) : ((pi == 0) ? hv.y : hv.x);
            mx = fmax(mx, fabs(v));
        }
        const int e = (mx > 0.0) ? ilogb(mx) : 0;
        eB[j] = e;
        for (int kk = 0; kk < Sh::K; ++kk) {
            const int pi = kk / NN, rho = kk % NN;
            const double2 hv = s.d.h[mu1 * NN + rho];
            const double v = (po == 0) ? ((pi == 0) ? hv.x : -hv.y) : ((pi == 0) ? hv.y : hv.x);
            // |v * 2^(20-e)| < 2^21; the first digit and remainders are exact in FP64 before rounding to FP32
            double r = ldexp(v, 20 - e);
            float d[kOzDigits];
            d[0] = float(rint(r / 16384.0));
            r -= double(d[0]) * 16384.0;
            d[1] = float(rint(r / 128.0));
            r -= double(d[1]) * 128.0;
            d[2] = float(rint(r));
            r -= double(d[2]);
            d[3] = float(rint(r * 128.0));
#pragma unroll
            for (int q = 0; q < kOzDigits; ++q)
                *reinterpret_cast<__nv_bfloat16 *>(Bd + q * Sh::B_BYTES + swz_byte(j, kk)) = __float2bfloat16_rn(d[q]);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = umma_idesc_bf16(Sh::N);
    const int ntiles = 2 * s.gemm_tiles;
    uint32_t phase = 0;
    bool ok = true;
    const int sub = lane / Sh::LPR, sl = lane % Sh::LPR;  // row within the warp load, lane within the row
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int t = tile / s.gemm_tiles, g = tile % s.gemm_tiles;
        const float *Xg = sym_in(s, k) + t * 2 * s.n4;
        // A digits: rows m = slot*NN + mu2, 4 floats per lane, row maximum by shuffles
        for (int base = warp * Sh::RPW; base < 128; base += 4 * Sh::RPW) {
            const int m = base + sub;
            const int slot = m / NN, mu2 = m % NN;
            const int c = s.gemm_c[g * Sh::CPT + slot];
            const float4 v = reinterpret_cast<const float4 *>(Xg + ((long long)mu2 * n2 + c) * Sh::K)[sl];
            float mx = fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w)));
#pragma unroll
            for (int o = Sh::LPR / 2; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            const int e = (mx > 0.f) ? ilogbf(mx) : 0;
            if (sl == 0) eA[m] = e;
            const float vv[4] = {v.x, v.y, v.z, v.w};
            __nv_bfloat16 dq[kOzDigits][4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                float d[kOzDigits];
                oz_digits(ldexpf(vv[i], 20 - e), d);
#pragma unroll
                for (int q = 0; q < kOzDigits; ++q) dq[q][i] = __float2bfloat16_rn(d[q]);
            }
            const int kk0 = sl * 4;
#pragma unroll
            for (int q = 0; q < kOzDigits; ++q) {
                uint2 w;
                w.x = uint32_t(__bfloat16_as_ushort(dq[q][0])) | (uint32_t(__bfloat16_as_ushort(dq[q][1])) << 16);
                w.y = uint32_t(__bfloat16_as_ushort(dq[q][2])) | (uint32_t(__bfloat16_as_ushort(dq[q][3])) << 16);
                *reinterpret_cast<uint2 *>(Ad + q * Sh::A_BYTES + swz_byte(m, kk0)) = w;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            const uint32_t ab = smem_u32(Ad), bb = smem_u32(Bd);
            for (int L = 0; L < kOzLevels; ++L) {
                uint32_t acc = 0;
                for (int i = 0; i <= L; ++i) {
                    const int j = L - i;
                    for (int ks = 0; ks < Sh::KS; ++ks) {
                        umma_bf16(tmem + L * Sh::N, umma_desc_sw128(ab + i * Sh::A_BYTES + ks * 32),
                                  umma_desc_sw128(bb + j * Sh::B_BYTES + ks * 32), idesc, acc);
                        acc = 1;
                    }
                }
            }
            umma_commit(bar_mma);
        }
        ok = mbar_wait(bar_mma, phase);
        ok = __syncthreads_and(ok);
        if (!ok) {
            if (tid == 0) atomicExch(s.err, 3);
            break;
        }
        tc_fence_after();
        // TMEM -> FP64 combination -> FP32 staging S[row][j]
        const int row = warp * 32 + lane;
        const double sa = ldexp(1.0, eA[row] - 6);
#pragma unroll 1
        for (int cc = 0; cc < Sh::N / 32; ++cc) {
            double accd[32];
#pragma unroll
            for (int i = 0; i < 32; ++i) accd[i] = 0.0;
#pragma unroll
            for (int L = kOzLevels - 1; L >= 0; --L) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + L * Sh::N + cc * 32, v);
                const double w = ldexp(1.0, -7 * L);
#pragma unroll
                for (int i = 0; i < 32; ++i) accd[i] += w * double(v[i]);
            }
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const int j = cc * 32 + i;
                S[row * Sh::S_LD + j] = float(accd[i] * sa * ldexp(1.0, eB[j] - 6));
            }
        }
        tc_fence_before();
        __syncthreads();
        float *Wg = s.W + t * 2 * s.n4;
        for (int e = tid; e < Sh::CPT * 2 * NN * NN; e += blockDim.x) {
            const int r = e % (NN * NN), part = (e / (NN * NN)) % 2, slot = e / (2 * NN * NN);
            const int mu1 = r % NN, mu2 = r / NN;
            const int ps = s.gemm_partner[g * Sh::CPT + slot];
            const float v = S[(slot * NN + mu2) * Sh::S_LD + part * NN + mu1] + S[(ps * NN + mu1) * Sh::S_LD + part * NN + mu2];
            const int c = s.gemm_c[g * Sh::CPT + slot];
            Wg[((long long)c * 2 + part) * n2 + r] = v;
        }
        // (the staging overwrote the digit buffers; the MMAs read only the K steps
        // the next tile rewrites, so no clearing is needed)
        __syncthreads();
        phase ^= 1;
    }
    if (!ok) mbar_wait(bar_mma, phase);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Sh::TMEM_COLS) : "memory");
}

}  // namespace g12
