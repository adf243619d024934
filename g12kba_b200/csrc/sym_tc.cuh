// tcgen05 (sm_100a) W contraction for the symmetric engine, TF32x3.
//
// Per tile: rows m = (slot, mu2) of G2 (128 rows = 128/n values of c, each with
// all n values of mu2), K = (part, rho) = 2n, N = (part, mu1) = 2n.
//   A[m][k]  = TMP (FP32, K-major rows of 2n floats), fetched by TMA with
//              128-byte swizzle, split in shared memory into hi = tf32(a) and
//              lo = tf32(a - hi);
//   Bt[j][k] = the real form of h (built per CTA), split the same way;
//   D = A_hi B_hi + A_hi B_lo + A_lo B_hi accumulated in FP32 in TMEM
//       (tcgen05.mma kind::tf32, M = 128, N = 2n, K = 8 per instruction).
// The accumulator tile is T1 = (h (x) 1) M on these rows; W = T1 + e(T1) is
// formed from the staged tile (each c's exchange partner cbar is in the same
// tile) and stored as in k_sym_gemm_simt.
//
// Every wait is bounded (about one second of clock cycles); on expiry the
// kernel records a code in s.err, waits a bounded time for its own copies,
// frees its TMEM and returns.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "sym_kernels.cuh"

namespace g12 {

constexpr long long kWaitCycles = 2000000000LL;  // ~1 s at 2 GHz

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// one hardware-suspended wait for phase `parity` (returns false when the
// hardware's time window ends first; the thread wakes as soon as the phase completes)
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// bounded wait on phase `parity`; false when the cycle budget runs out
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    const long long t0 = clock64();
    while (!mbar_try(bar, parity)) {
        if (clock64() - t0 > kWaitCycles) return false;
    }
    return true;
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2,
                                            int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
        "[%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}

// 1-D bulk copy global -> shared, completing bytes on an mbarrier (both
// addresses 16-byte aligned, bytes a multiple of 16)
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ uint32_t tf32_round(float v)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return r;
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;            // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;  // stride byte offset
    d |= (uint64_t)1 << 46;            // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;            // SWIZZLE_128B
    return d;
}

// instruction descriptor: D f32, A/B tf32, both K-major, M = 128, N = n_cols
__host__ __device__ constexpr uint32_t umma_idesc_tf32(int n_cols)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n_cols >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// PIECES = 2: a = a0 + a1 (tf32 each), products a0 b0 + a0 b1 + a1 b0 ("x3");
// PIECES = 3: a = a0 + a1 + a2, products with piece-index sum <= 2 ("x6").
template <int NN, int PIECES>
struct TcShape {
    static constexpr int N = 2 * NN;       // UMMA N
    static constexpr int KB = 2 * NN / 32; // 128-byte K blocks
    static constexpr int CPT = 128 / NN;   // c values per tile
    static constexpr int A_BYTES = 128 * 128;
    static constexpr int B_BYTES = N * 128;
    static constexpr int TMEM_COLS = N < 32 ? 32 : N;
    static constexpr int OFF_A = 0;                             // PIECES x KB x A_BYTES
    static constexpr int OFF_B = PIECES * KB * A_BYTES;         // PIECES x KB x B_BYTES
    static constexpr int OFF_BAR = OFF_B + PIECES * KB * B_BYTES;
    static constexpr int SMEM = OFF_BAR + 64 + 1024;            // + alignment slack
    static constexpr int S_LD = N + 1;                          // staging row stride (floats)
    static constexpr int NPROD = PIECES == 2 ? 3 : 6;
    static_assert(128 * S_LD * 4 <= 2 * KB * A_BYTES, "staging must fit in the A buffers");
};

template <int NN, int PIECES>
__global__ void __launch_bounds__(128) k_sym_gemm_tc(SymDev s, int k, const __grid_constant__ CUtensorMap tmap)
{
    using Sh = TcShape<NN, PIECES>;
    if (!*s.d.active) return;
    extern __shared__ unsigned char smraw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
    float *Ahi = reinterpret_cast<float *>(sm + Sh::OFF_A);  // piece 0 (TMA lands here)
    uint32_t *Bp = reinterpret_cast<uint32_t *>(sm + Sh::OFF_B);
    uint64_t *bar_tma = reinterpret_cast<uint64_t *>(sm + Sh::OFF_BAR);
    uint64_t *bar_mma = bar_tma + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar_tma + 2);
    float *S = Ahi;  // staging reuses both A buffers once the MMAs are done
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n = NN;
    const long long n2 = (long long)n * n;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(Sh::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(bar_tma, 1);
        mbar_init(bar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // B = real form of h^T, split into tf32 pieces, 128-byte swizzled K-major
    for (int e = tid; e < Sh::N * 2 * NN; e += blockDim.x) {
        const int j = e / (2 * NN), kk = e % (2 * NN);
        const int po = j / NN, mu1 = j % NN, pi = kk / NN, rho = kk % NN;
        const double2 hv = s.d.h[mu1 * n + rho];
        double vd;
        if (po == 0) vd = (pi == 0) ? hv.x : -hv.y;
        else vd = (pi == 0) ? hv.y : hv.x;
        const int kb = kk >> 5, kin = kk & 31;
        const int word = kb * (Sh::B_BYTES / 4) + j * 32 + ((((kin >> 2) ^ (j & 7)) << 2) | (kin & 3));
        // pieces of the FP64 value (h is FP64): each a tf32-rounded remainder
        double rem = vd;
#pragma unroll
        for (int q = 0; q < PIECES; ++q) {
            const uint32_t pq = tf32_round(float(rem));
            Bp[q * Sh::KB * (Sh::B_BYTES / 4) + word] = pq;
            rem -= double(__uint_as_float(pq));
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = umma_idesc_tf32(Sh::N);
    const int ntiles = 2 * s.gemm_tiles;
    uint32_t phase = 0;
    bool ok = true;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int t = tile / s.gemm_tiles, g = tile % s.gemm_tiles;
        if (tid == 0) {
            mbar_expect_tx(bar_tma, Sh::KB * Sh::A_BYTES);
            for (int slot = 0; slot < Sh::CPT; ++slot) {
                const int c = s.gemm_c[g * Sh::CPT + slot];
                for (int kb = 0; kb < Sh::KB; ++kb)
                    tma_load_4d(reinterpret_cast<unsigned char *>(Ahi) + kb * Sh::A_BYTES + slot * NN * 128, &tmap,
                                bar_tma, kb * 32, c, 0, t);
            }
        }
        ok = mbar_wait(bar_tma, phase);
        ok = __syncthreads_and(ok);
        if (!ok) {
            if (tid == 0) atomicExch(s.err, 1);
            break;
        }
        // split A into tf32 pieces: piece 0 in place, then the exact FP32 remainders
        float4 *a4 = reinterpret_cast<float4 *>(Ahi);
        constexpr int A4 = Sh::KB * Sh::A_BYTES / 16;
        for (int i = tid; i < A4; i += blockDim.x) {
            float4 v = a4[i];
#pragma unroll
            for (int q = 0; q < PIECES; ++q) {
                uint4 h;
                h.x = tf32_round(v.x);
                h.y = tf32_round(v.y);
                h.z = tf32_round(v.z);
                h.w = tf32_round(v.w);
                v.x -= __uint_as_float(h.x);
                v.y -= __uint_as_float(h.y);
                v.z -= __uint_as_float(h.z);
                v.w -= __uint_as_float(h.w);
                reinterpret_cast<uint4 *>(a4)[q * A4 + i] = h;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            const uint32_t abase = smem_u32(Ahi), bbase = smem_u32(Bp);
            // (A piece, B piece) pairs, smallest terms first
            constexpr int PA[6] = {2, 1, 0, 1, 0, 0}, PB[6] = {0, 1, 2, 0, 1, 0};
            constexpr int first = Sh::NPROD == 3 ? 3 : 0;
            uint32_t acc = 0;
            for (int pr = first; pr < 6; ++pr) {
                const uint32_t pa = abase + PA[pr] * Sh::KB * Sh::A_BYTES, pb = bbase + PB[pr] * Sh::KB * Sh::B_BYTES;
                for (int kb = 0; kb < Sh::KB; ++kb) {
                    for (int ks = 0; ks < 4; ++ks) {
                        const uint32_t oa = kb * Sh::A_BYTES + ks * 32, ob = kb * Sh::B_BYTES + ks * 32;
                        umma_tf32(tmem, umma_desc_sw128(pa + oa), umma_desc_sw128(pb + ob), idesc, acc);
                        acc = 1;
                    }
                }
            }
            umma_commit(bar_mma);
        }
        ok = mbar_wait(bar_mma, phase);
        ok = __syncthreads_and(ok);
        if (!ok) {
            if (tid == 0) atomicExch(s.err, 2);
            break;
        }
        tc_fence_after();
        // TMEM -> registers -> staging S[row][j]
        const int row = warp * 32 + lane;
#pragma unroll
        for (int cc = 0; cc < Sh::N / 32; ++cc) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + cc * 32, v);
#pragma unroll
            for (int i = 0; i < 32; ++i) S[row * Sh::S_LD + cc * 32 + i] = v[i];
        }
        tc_fence_before();
        __syncthreads();
        // W[mu1][mu2][c] = T1[mu1][mu2][c] + T1[mu2][mu1][cbar]
        float *Wg = s.W + t * 2 * s.n4;
        for (int e = tid; e < Sh::CPT * 2 * NN * NN; e += blockDim.x) {
            const int r = e % (NN * NN), part = (e / (NN * NN)) % 2, slot = e / (2 * NN * NN);
            const int mu1 = r % NN, mu2 = r / NN;
            const int ps = s.gemm_partner[g * Sh::CPT + slot];
            const float v = S[(slot * NN + mu2) * Sh::S_LD + part * NN + mu1] + S[(ps * NN + mu1) * Sh::S_LD + part * NN + mu2];
            const int c = s.gemm_c[g * Sh::CPT + slot];
            Wg[((long long)c * 2 + part) * n2 + r] = v;
        }
        __syncthreads();
        phase ^= 1;
    }
    if (!ok) {
        // let in-flight copies and MMAs land (bounded) before the TMEM is released
        mbar_wait(bar_tma, phase);
        mbar_wait(bar_mma, phase);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Sh::TMEM_COLS) : "memory");
}

}  // namespace g12
