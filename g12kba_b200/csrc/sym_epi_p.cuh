// Persistent stage epilogue of the symmetric engine at n = 32 (FP32 W and stage
// input; the digit-GEMM path).  Same arithmetic as k_sym_epi<32, float> (C = W -
// W^H on a tile pair, Psi, Pi, K2, RK4 bookkeeping, next-stage input), organised
// for the B200 memory system instead of one short-lived block per tile pair:
//   * one 512-thread CTA per SM walks its tile pairs (u = blockIdx.x + i G);
//   * the next pair's inputs are copied into a second shared-memory buffer while
//     the current pair is computed (double buffering, 81 KB per buffer): one
//     thread issues 1-D bulk copies of the FP64 state tile and RK4 sum, the two
//     16 KB slices of the combined Psi/Pi table Zt and the pair's Rt and Q rows
//     (completion on an mbarrier per buffer); every thread copies one 16-byte
//     chunk of each W tile with cp.async into a bank-swizzled layout;
//   * G1 is staged once per CTA, not once per tile pair;
//   * the table terms i g22 (Rtt[site mu2] - Rtt[site nu2]) + g22 (Qt[mu2] -
//     Qt[nu2]) of the per-pair kernel are read as g22 (Zt[mu2] - Zt[nu2]), two
//     shared-memory reads instead of four L2 reads per element;
//   * the next-stage input is rounded to FP32 once, into a padded staging tile
//     that both output tiles (R, C) and (C, R) are written from.
// CTAs past the pair CTAs (s.g1x of them) run the stage's G1 side (g1_body).
// Every mbarrier wait is bounded; on expiry the kernel records code 91 in the
// error word, lets its copies in flight land (bounded) and returns.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sym_tc.cuh"

namespace g12 {

constexpr int kEpiPThreads = 512;
constexpr int kEpiPMaxUnits = 16;  // tile pairs per CTA (the host keeps the grid at >= 2 npairs / 16)

struct EpiPBuf {
    // W tiles as 64 rows (c_l * 2 + part) of 32 floats (r_l), 16-byte chunks
    // swizzled by row: chunk q of row rho sits at q ^ ((rho >> 1) & 7), so both the
    // row reads and the column reads of the transposed tile spread over the banks
    float Wrc[2 * kTB * kTB];              // row (c_l, part) = W[R0 + .][C0 + c_l]
    float Wcr[2 * kTB * kTB];              // row (r_l, part) = W[C0 + .][R0 + r_l]
    double2 Yc[kTB * kTB], Ac[kTB * kTB];  // the pair's compressed state and RK4 sum
    double2 Zm[kTB * kTB], Zn[kTB * kTB];  // Zt[t][mu2], Zt[t][nu2] ([nu1][mu1])
    double2 Rt[kTB];                       // Rt[(mu2, nu2)][s], s < Ns
    double2 Qr[kTB];                       // Q[t][nu2][mu2][x], x < n
};
constexpr size_t kEpiPSmem = 2 * sizeof(double2) * 32 * 33 + 2 * sizeof(EpiPBuf) + sizeof(float2) * 32 * 33;

// float index of element (row rho, column c) of a swizzled W tile
__device__ __forceinline__ int epip_wsw(int rho, int c) { return rho * kTB + ((((c >> 2) ^ (rho >> 1)) & 7) << 2) + (c & 3); }

__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// one thread: bulk copies of tile pair u's state tiles, table slices and rows, completing on bar
__device__ __forceinline__ void epip_issue_bulk(const SymDev &s, int k, int u, int Rb, int Cb, EpiPBuf &b, uint64_t *bar)
{
    constexpr int n = 32, n2 = n * n, n3 = n2 * n;
    const int t = u / s.npairs;
    const bool diag = Rb == Cb;
    const uint32_t tile = kTB * kTB * sizeof(double2);
    mbar_expect_tx(bar, tile * (1 + (k > 0) + 2 * !diag) + s.d.Ns * sizeof(double2) + n * sizeof(double2));
    bulk_load(b.Yc, s.Yc + (long long)u * (kTB * kTB), tile, bar);
    if (k > 0) bulk_load(b.Ac, s.Ac + (long long)u * (kTB * kTB), tile, bar);
    if (!diag) {
        bulk_load(b.Zm, s.d.Zt + t * n3 + Rb * n2, tile, bar);
        bulk_load(b.Zn, s.d.Zt + t * n3 + Cb * n2, tile, bar);
    }
    bulk_load(b.Rt, s.d.Rt + (Rb * n + Cb) * s.d.Ns, s.d.Ns * sizeof(double2), bar);
    bulk_load(b.Qr, s.d.Q + t * n3 + (Cb * n + Rb) * n, n * sizeof(double2), bar);
}

// copies of tile pair (t; mu2 = Rb, nu2 = Cb)'s W tiles, table slices and rows
// (produced by this stage's GEMM and k_prep)
__device__ __forceinline__ void epip_issue_stage(const SymDev &s, int t, int Rb, int Cb, EpiPBuf &b)
{
    constexpr int n = 32;
    constexpr int n2 = n * n;
    static_assert(2 * kTB * kTB / 4 == kEpiPThreads, "one 16-byte chunk of each W tile per thread");
    const float *Wg = s.W + (long long)t * 2 * s.n4;
    const int R0 = Rb * kTB, C0 = Cb * kTB;
    const int x = threadIdx.x, rho = x >> 3, q = x & 7;  // 8 threads per 128-byte row
    const int dst = rho * kTB + (((q ^ (rho >> 1)) & 7) << 2);
    cp_async16(&b.Wrc[dst], Wg + (2 * C0 + rho) * n2 + R0 + 4 * q);
    cp_async16(&b.Wcr[dst], Wg + (2 * R0 + rho) * n2 + C0 + 4 * q);
}

__global__ void __launch_bounds__(kEpiPThreads, 1) k_sym_epi_p(SymDev s, int k)
{
    if (!*s.d.active) return;
    const Dev &d = s.d;
    const int G = int(gridDim.x) - s.g1x;  // pair CTAs
    if (int(blockIdx.x) >= G) {
        // the stage's G1 side (h and Ix come from k_prep)
        grid_dep_wait();
        g1_body(d, k, int(blockIdx.x) - G);
        return;
    }
    constexpr int n = 32, GLD = n + 1, KLD = kTB + 1;
    constexpr int n3 = n * n * n;
    extern __shared__ __align__(16) unsigned char smp[];
    double2 *Gs = reinterpret_cast<double2 *>(smp);  // n x GLD
    double2 *Ks = Gs + n * GLD;                       // [c_l][r_l] K or next input, rows of KLD
    EpiPBuf *buf = reinterpret_cast<EpiPBuf *>(Ks + kTB * KLD);
    float2 *KF = reinterpret_cast<float2 *>(buf + 2);  // [c_l][r_l] next-stage input (FP32), rows of KLD
    __shared__ int site[n];
    __shared__ double wtab[n];  // pair weight by site distance m: U (m = 0), V_m (m <= nv), 0
    __shared__ int2 urc[kEpiPMaxUnits];
    __shared__ __align__(8) uint64_t bar[2];
    const int units = 2 * s.npairs;
    const int nu = (units - int(blockIdx.x) + G - 1) / G;
    if (nu <= 0) return;
    if (nu > kEpiPMaxUnits) {
        // grid too small for the unit table (the host sizes it): report, skip the stage
        if (threadIdx.x == 0) atomicExch(s.err, 90);
        return;
    }
    // step scalars (k_step_begin finished before k_prep started)
    const StageP st = d.cur->st[k];
    const double U = st.U;
    if (int(threadIdx.x) < nu) urc[threadIdx.x] = s.pairs[(int(blockIdx.x) + int(threadIdx.x) * G) % s.npairs];
    if (threadIdx.x < n) {
        const int m = threadIdx.x;
        site[m] = m % d.Ns;
        // the reference's weights U (same site) and V_m (|i - j| = m <= nv): U * double(si == sj) + V
        wtab[m] = m == 0 ? U : (m <= d.nv ? U * d.law[m - 1] : 0.0);
    }
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const double2 *G1 = (k & 1) ? d.G1t1 : d.G1t0;
#pragma unroll
    for (int q = 0; q < n * n / kEpiPThreads; ++q) {
        const int x = threadIdx.x + q * kEpiPThreads;
        Gs[(x / n) * GLD + x % n] = G1[x];
    }
    __syncthreads();
    // W comes from the GEMM launched just before this kernel, the tables from
    // k_prep before it (G1 was complete before k_prep started)
    grid_dep_wait();
    if (threadIdx.x == 0) epip_issue_bulk(s, k, blockIdx.x, urc[0].x, urc[0].y, buf[0], &bar[0]);
    epip_issue_stage(s, int(blockIdx.x) / s.npairs, urc[0].x, urc[0].y, buf[0]);
    cp_async_commit();

    const int rl = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int mu1 = rl, si = site[mu1];
    float *const Out0 = sym_out<float>(s, k);
    for (int i = 0; i < nu; ++i) {
        if (i + 1 < nu) {
            const int u1 = int(blockIdx.x) + (i + 1) * G;
            EpiPBuf &b1 = buf[(i + 1) & 1];
            if (threadIdx.x == 0) epip_issue_bulk(s, k, u1, urc[i + 1].x, urc[i + 1].y, b1, &bar[(i + 1) & 1]);
            epip_issue_stage(s, u1 / s.npairs, urc[i + 1].x, urc[i + 1].y, b1);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        const bool ok = mbar_wait(&bar[i & 1], (i >> 1) & 1);
        if (!__syncthreads_and(ok)) {
            // copies did not arrive in time: report, let the ones in flight land, return
            cp_async_wait<0>();
            if (threadIdx.x == 0) {
                atomicExch(s.err, 91);
                if (i + 1 < nu) mbar_wait(&bar[(i + 1) & 1], ((i + 1) >> 1) & 1);
            }
            return;
        }
        const EpiPBuf &b = buf[i & 1];
        const int u = int(blockIdx.x) + i * G, t = u / s.npairs;
        const int mu2 = urc[i].x, nu2 = urc[i].y;  // n = 32: one mu2 per row block, one nu2 per column block
        const bool diag = mu2 == nu2;
        const int sj = site[mu2], sl = site[nu2];
        // per-row (mu1 = lane) values of this pair
        const double wa = wtab[abs(si - sj)];
        const double2 ra = b.Rt[si], qa = b.Qr[mu1];
        const double2 g22 = Gs[mu2 * GLD + nu2];
        double2 a1 = make_double2(0.0, 0.0), a2 = a1, fa = a1;
        if (t == 0) {
            a1 = c_mul(g22, Gs[mu1 * GLD + mu2]);
            a2 = c_mul(g22, Gs[mu1 * GLD + nu2]);
            fa = c_mul(Gs[mu2 * GLD + mu1], Gs[mu1 * GLD + nu2]);
        }
        const double dmu = U * double(mu1 == mu2);
        // loads of both elements first (the stores below go to other buffers)
        double2 C[2], g11[2], gT[2], zd[2], acs[2], ycs[2];
        double wb[2];
        double2 rb[2], qb[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int cl = w + 16 * j, e = cl * kTB + rl;
            const float w1x = b.Wrc[epip_wsw(2 * cl, rl)], w1y = b.Wrc[epip_wsw(2 * cl + 1, rl)];
            const float w2x = b.Wcr[epip_wsw(2 * rl, cl)], w2y = b.Wcr[epip_wsw(2 * rl + 1, cl)];
            C[j] = make_double2(double(w1x) - double(w2x), double(w1y) + double(w2y));
            g11[j] = Gs[mu1 * GLD + cl];
            gT[j] = Gs[cl * GLD + mu1];
            zd[j] = diag ? make_double2(0.0, 0.0) : c_sub(b.Zm[e], b.Zn[e]);
            acs[j] = b.Ac[e];
            ycs[j] = b.Yc[e];
            const int sk = site[cl];
            wb[j] = wtab[abs(sk - sl)];
            rb[j] = b.Rt[sk];
            qb[j] = b.Qr[cl];
        }
        double2 Kv[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int cl = w + 16 * j, nu1 = cl;
            const double2 g1122 = c_mul(g11[j], g22);
            double2 psi = c_scale(g1122, wa - wb[j]);
            psi = c_add(psi, c_i(c_mul(g11[j], c_sub(ra, rb[j]))));
            if (t == 0) {
                psi = c_sub(psi, c_scale(g1122, dmu - U * double(nu1 == nu2)));
                const double2 y1 = Gs[mu2 * GLD + nu1], y2 = Gs[nu2 * GLD + nu1];
                const double2 e1 = c_sub(c_mul(a1, y1), c_mul(a2, y2));  // g22 (x1 y1 - x2 y2)
                const double2 e2 = c_sub(fa, c_mul(y1, Gs[nu1 * GLD + nu2]));
                psi = c_add(psi, c_scale(c_mi(c_add(e1, c_mul(g11[j], e2))), U));
            }
            // the Rtt and Qt terms; Zt[mu2] - Zt[nu2] vanishes on the diagonal pairs
            const double2 acc = c_add(c_add(C[j], psi), c_mul(g22, zd[j]));
            const double2 piP = c_mul(gT[j], c_sub(qb[j], qa));
            Kv[j] = c_mi(c_sub(acc, c_conj(piP)));
        }
        double2 *Ycg = s.Yc + (long long)u * (kTB * kTB), *Acg = s.Ac + (long long)u * (kTB * kTB);
        // RK4 bookkeeping of one element (RK_solver.h:137-139, 209-213) on the compressed state
        auto rk4 = [&](double2 K, double2 ac, double2 yc, int e) -> double2 {
            const double2 rk = c_add(k == 0 ? make_double2(0.0, 0.0) : ac, c_scale(K, st.w));
            double2 v;
            if (k < 3) {
                Acg[e] = rk;
                v = c_add(yc, c_scale(K, st.c_next));
            } else {
                v = c_add(yc, c_scale(c_scale(rk, st.dt), 1.0 / 6.0));
                Ycg[e] = v;
            }
            return v;
        };
        if (!diag) {
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int cl = w + 16 * j;
                const double2 v = rk4(Kv[j], acs[j], ycs[j], cl * kTB + rl);
                KF[cl * KLD + rl] = make_float2(float(v.x), float(v.y));
            }
            __syncthreads();
        } else {
            // keep the diagonal block exactly Hermitian: K <- (K + K^H) / 2, then the
            // bookkeeping and the particle-2 diagonal D (mu2 == nu2 on these pairs)
#pragma unroll
            for (int j = 0; j < 2; ++j) Ks[(w + 16 * j) * KLD + rl] = Kv[j];
            __syncthreads();
            double2 sym[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int cl = w + 16 * j;
                const double2 a = Ks[cl * KLD + rl], bb = c_conj(Ks[rl * KLD + cl]);
                sym[j] = make_double2(0.5 * (a.x + bb.x), 0.5 * (a.y + bb.y));
            }
            __syncthreads();
            double2 *Dt = d.D + t * n3;
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int cl = w + 16 * j;
                const double2 v = rk4(sym[j], acs[j], ycs[j], cl * kTB + rl);
                KF[cl * KLD + rl] = make_float2(float(v.x), float(v.y));
                Dt[(mu1 * n + cl) * n + mu2] = v;
            }
            __syncthreads();
        }
        float *Out = Out0 + (long long)t * 2 * s.n4;
        // tile (R, C): tmp_index(n, r_l, mu2, nu2 * 32 + c_l, part), fastest index mu1 = r_l
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int cl = w + 16 * j;
            const float2 v = KF[cl * KLD + rl];
            const int o = ((mu2 * n * n + nu2 * kTB + cl) * 2) * n + rl;
            Out[o] = v.x;
            Out[o + n] = v.y;
        }
        if (!diag) {
            // tile (C, R): element (c, r) = conj(v) at tmp_index(n, c_l, nu2, mu2 * 32 + r_l, part),
            // fastest index nu1 = c_l (the lane)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int rr = w + 16 * j;
                const float2 v = KF[rl * KLD + rr];
                const int o = ((nu2 * n * n + mu2 * kTB + rr) * 2) * n + rl;
                Out[o] = v.x;
                Out[o + n] = -v.y;
            }
        }
    }
}

}  // namespace g12
