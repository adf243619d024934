// Persistent stage epilogue of the symmetric engine at n = 32 (FP32 W and stage
// input; the digit-GEMM path).  Same arithmetic as k_sym_epi<32, float> (C = W -
// W^H on a tile pair, Psi, Pi, K2, RK4 bookkeeping, next-stage input), organised
// for the B200 memory system instead of one short-lived block per tile pair:
//   * one 512-thread CTA per SM walks its tile pairs (u = blockIdx.x + i G);
//   * the next pair's inputs are copied into a second shared-memory buffer while
//     the current pair is computed (double buffering, 81 KB per buffer): lane 0
//     of warps 0, 1 and 2 issue 1-D bulk copies of the FP64 state tile and RK4
//     sum, the two 16 KB slices of the combined Psi/Pi table Zt and the pair's
//     Rt and Q rows (completion on an mbarrier per buffer; one thread issuing
//     all six took 0.37 us per pair, while the other warps waited for it);
//     every thread copies one 16-byte chunk of each W tile with cp.async into a
//     bank-swizzled layout;
//   * G1 is staged once per CTA, not once per tile pair, and the first pair's
//     bulk copies are issued before the wait for the GEMM (only W comes from it);
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
constexpr int kEpiPWarps = kEpiPThreads / 32;
constexpr int kEpiPEJ = kTB / kEpiPWarps;  // elements per thread and tile pair: (lane, w + kEpiPWarps j)
constexpr int kEpiPChunks = 2 * kTB * kTB / 4;  // 16-byte chunks of one W tile
static_assert(kEpiPChunks == 512 && (kEpiPThreads == 512 || kEpiPThreads == 1024), "chunk and element mapping");
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

__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// a tile pair of this CTA: row block Rb = mu2, column block Cb = nu2 (n = 32),
// tensor t, unit index u = t npairs + pair index
struct EpiPUnit {
    int Rb, Cb, t, u;
};

// bulk copies of a tile pair's state tiles, table slices and rows, completing on
// bar, issued by lane 0 of warps 0, 1 and 2 in parallel (each bulk copy takes
// about 0.06 us to issue).  Warp 0's single arrival carries the whole byte
// count, so the phase completes only when it has happened and every copy has
// landed, in whatever order the warps run (the transaction count may go
// below zero meanwhile).
__device__ __forceinline__ void epip_issue_bulk(const SymDev &s, int k, const EpiPUnit &un, EpiPBuf &b, uint64_t *bar)
{
    constexpr int n = 32, n2 = n * n, n3 = n2 * n;
    const bool diag = un.Rb == un.Cb;
    const uint32_t tile = kTB * kTB * sizeof(double2);
    const int w = threadIdx.x >> 5;
    if (w == 0) {
        mbar_expect_tx(bar, tile * (1 + (k > 0) + 2 * !diag) + s.d.Ns * sizeof(double2) + n * sizeof(double2));
        bulk_load(b.Yc, s.Yc + (long long)un.u * (kTB * kTB), tile, bar);
        if (k > 0) bulk_load(b.Ac, s.Ac + (long long)un.u * (kTB * kTB), tile, bar);
    } else if (w == 1) {
        if (!diag) {
            bulk_load(b.Zm, s.d.Zt + un.t * n3 + un.Rb * n2, tile, bar);
            bulk_load(b.Zn, s.d.Zt + un.t * n3 + un.Cb * n2, tile, bar);
        }
    } else {
        bulk_load(b.Rt, s.d.Rt + (un.Rb * n + un.Cb) * s.d.Ns, s.d.Ns * sizeof(double2), bar);
        bulk_load(b.Qr, s.d.Q + un.t * n3 + (un.Cb * n + un.Rb) * n, n * sizeof(double2), bar);
    }
}

// every thread: its 16-byte chunk (source offset src, swizzled destination dst)
// of both W tiles of a tile pair (512 threads) or of one of them (1024 threads:
// the first half the direct tile); Wt = W of the pair's tensor
__device__ __forceinline__ void epip_issue_w(const float *Wt, const EpiPUnit &un, EpiPBuf &b, int dst, int src)
{
    constexpr int n2 = 32 * 32;
    if (kEpiPThreads == 512 || int(threadIdx.x) < kEpiPChunks)
        cp_async16(&b.Wrc[dst], Wt + (2 * un.Cb * kTB) * n2 + un.Rb * kTB + src);
    if (kEpiPThreads == 512 || int(threadIdx.x) >= kEpiPChunks)
        cp_async16(&b.Wcr[dst], Wt + (2 * un.Rb * kTB) * n2 + un.Cb * kTB + src);
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
    constexpr int n = 32, n2 = n * n, GLD = n + 1, KLD = kTB + 1;
    constexpr int n3 = n * n * n;
    extern __shared__ __align__(16) unsigned char smp[];
    double2 *Gs = reinterpret_cast<double2 *>(smp);  // n x GLD
    double2 *Ks = Gs + n * GLD;                       // [c_l][r_l] K of a diagonal pair, rows of KLD
    EpiPBuf *buf = reinterpret_cast<EpiPBuf *>(Ks + kTB * KLD);
    float2 *KF = reinterpret_cast<float2 *>(buf + 2);  // [c_l][r_l] next-stage input (FP32), rows of KLD
    __shared__ int site[n];
    __shared__ double wtab[n];  // pair weight by site distance m: U (m = 0), V_m (m <= nv), 0
    __shared__ EpiPUnit units[kEpiPMaxUnits];
    __shared__ __align__(8) uint64_t bar[2];  // one per input buffer
    const int tid = threadIdx.x;
    const int nu = (2 * s.npairs - int(blockIdx.x) + G - 1) / G;
    if (nu <= 0) return;
    if (nu > kEpiPMaxUnits) {
        // grid too small for the unit table (the host sizes it): report, skip the stage
        if (tid == 0) atomicExch(s.err, 90);
        return;
    }
    // step scalars (k_step_begin finished before k_prep started)
    const StageP st = d.cur->st[k];
    const double U = st.U;
    if (tid < nu) {
        const int u = int(blockIdx.x) + tid * G, t = u >= s.npairs ? 1 : 0;
        const int2 rc = s.pairs[u - t * s.npairs];
        units[tid] = EpiPUnit{rc.x, rc.y, t, u};
    }
    if (tid < n) {
        site[tid] = tid % d.Ns;
        // the reference's weights U (same site) and V_m (|i - j| = m <= nv): U * double(si == sj) + V
        wtab[tid] = tid == 0 ? U : (tid <= d.nv ? U * d.law[tid - 1] : 0.0);
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    const double2 *G1 = (k & 1) ? d.G1t1 : d.G1t0;
#pragma unroll
    for (int q = 0; q < n * n / kEpiPThreads; ++q) {
        const int x = tid + q * kEpiPThreads;
        Gs[(x / n) * GLD + x % n] = G1[x];
    }
    // Per-thread constants.  Copies: chunk cq of W tile row crho, 16-byte chunks
    // of a row swizzled: element (row rho, column c) at rho * 32 + ((((c >> 2) ^
    // (rho >> 1)) & 7) << 2) + (c & 3).  Reads: element (r_l, c_l) = (lane, w + kEpiPWarps j),
    // e = c_l * 32 + r_l; its W offsets in the direct tile (rho = 2 c_l + part,
    // c = r_l) and the transposed tile (rho = 2 r_l + part, c = c_l) do not depend
    // on the pair.
    const int crho = (tid % kEpiPChunks) >> 3, cq = tid & 7;
    const int wdst = crho * kTB + (((cq ^ (crho >> 1)) & 7) << 2), wsrc = crho * n2 + 4 * cq;
    const int rl = tid & 31, w = tid >> 5;
    const int ow1 = 2 * w * kTB + ((((rl >> 2) ^ w) & 7) << 2) + (rl & 3);
    int ow2[kEpiPEJ];
#pragma unroll
    for (int j = 0; j < kEpiPEJ; ++j) ow2[j] = 2 * rl * kTB + (((((w + kEpiPWarps * j) >> 2) ^ rl) & 7) << 2) + (w & 3);
    const int e0 = w * kTB + rl;    // element j = 0 (j: + kEpiPWarps 32 j)
    const int og11 = rl * GLD + w;  // Gs[mu1][c_l] (j: + kEpiPWarps j); also KF / Ks at row r_l, column c_l
    const int ogT = w * GLD + rl;   // Gs[c_l][mu1] (j: + kEpiPWarps GLD j); also KF / Ks at row c_l, column r_l
    const int oo = w * 2 * n + rl;  // output offset inside a tile's rows (j: + kEpiPWarps 2n j)
    const float *Wt0 = s.W, *Wt1 = s.W + 2 * s.n4;
    float *const Out0 = sym_out<float>(s, k), *const Out1 = Out0 + 2 * s.n4;
    const int mu1 = rl;
    __syncthreads();
    const int si = site[mu1];
    int sk[kEpiPEJ];
#pragma unroll
    for (int j = 0; j < kEpiPEJ; ++j) sk[j] = site[w + kEpiPWarps * j];
    // W comes from the GEMM launched just before this kernel: wait for it.  The
    // first pair's state tiles (the previous stage's epilogue) and tables
    // (k_prep) are fetched before that: both kernels have completed by the time
    // any CTA of this one runs, which is on an SM that a finished GEMM CTA left
    // (one 200 KB GEMM CTA per SM; each waited for k_prep before it finished).
    // G1 was complete before k_prep started.
    if ((tid & 31) == 0 && tid < 96) epip_issue_bulk(s, k, units[0], buf[0], &bar[0]);
    grid_dep_wait();
    {
        const EpiPUnit un = units[0];
        epip_issue_w(un.t ? Wt1 : Wt0, un, buf[0], wdst, wsrc);
        cp_async_commit();
    }
    for (int i = 0; i < nu; ++i) {
        if (i + 1 < nu) {
            // buffer (i + 1) & 1 was last read by pair i - 1, before the barrier after its K pass
            const EpiPUnit un1 = units[i + 1];
            EpiPBuf &b1 = buf[(i + 1) & 1];
            if ((tid & 31) == 0 && tid < 96) epip_issue_bulk(s, k, un1, b1, &bar[(i + 1) & 1]);
            epip_issue_w(un1.t ? Wt1 : Wt0, un1, b1, wdst, wsrc);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        const bool ok = mbar_wait(&bar[i & 1], (i >> 1) & 1);
        if (!__syncthreads_and(ok)) {
            // copies did not arrive in time: report, let the ones in flight land, return
            cp_async_wait<0>();
            if (tid == 0) {
                atomicExch(s.err, 91);
                if (i + 1 < nu) mbar_wait(&bar[(i + 1) & 1], ((i + 1) >> 1) & 1);
            }
            return;
        }
        const EpiPBuf &b = buf[i & 1];
        const EpiPUnit un = units[i];
        const int t = un.t;
        const int mu2 = un.Rb, nu2 = un.Cb;  // n = 32: one mu2 per row block, one nu2 per column block
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
        double2 C[kEpiPEJ], g11[kEpiPEJ], gT[kEpiPEJ], zd[kEpiPEJ], acs[kEpiPEJ], ycs[kEpiPEJ];
        double wb[kEpiPEJ];
        double2 rb[kEpiPEJ], qb[kEpiPEJ];
#pragma unroll
        for (int j = 0; j < kEpiPEJ; ++j) {
            const int e = e0 + j * kEpiPWarps * kTB;
            const float w1x = b.Wrc[ow1 + j * 2 * kEpiPWarps * kTB], w1y = b.Wrc[ow1 + j * 2 * kEpiPWarps * kTB + kTB];
            const float w2x = b.Wcr[ow2[j]], w2y = b.Wcr[ow2[j] + kTB];
            C[j] = make_double2(double(w1x) - double(w2x), double(w1y) + double(w2y));
            g11[j] = Gs[og11 + kEpiPWarps * j];
            gT[j] = Gs[ogT + kEpiPWarps * GLD * j];
            zd[j] = diag ? make_double2(0.0, 0.0) : c_sub(b.Zm[e], b.Zn[e]);
            acs[j] = b.Ac[e];
            ycs[j] = b.Yc[e];
            wb[j] = wtab[abs(sk[j] - sl)];
            rb[j] = b.Rt[sk[j]];
            qb[j] = b.Qr[w + kEpiPWarps * j];
        }
        double2 Kv[kEpiPEJ];
#pragma unroll
        for (int j = 0; j < kEpiPEJ; ++j) {
            const int nu1 = w + kEpiPWarps * j;
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
        double2 *Ycg = s.Yc + (long long)un.u * (kTB * kTB), *Acg = s.Ac + (long long)un.u * (kTB * kTB);
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
            for (int j = 0; j < kEpiPEJ; ++j) {
                const double2 v = rk4(Kv[j], acs[j], ycs[j], e0 + j * kEpiPWarps * kTB);
                KF[ogT + kEpiPWarps * KLD * j] = make_float2(float(v.x), float(v.y));
            }
            __syncthreads();
        } else {
            // keep the diagonal block exactly Hermitian: K <- (K + K^H) / 2, then the
            // bookkeeping and the particle-2 diagonal D (mu2 == nu2 on these pairs)
#pragma unroll
            for (int j = 0; j < kEpiPEJ; ++j) Ks[ogT + kEpiPWarps * KLD * j] = Kv[j];
            __syncthreads();
            double2 sym[kEpiPEJ];
#pragma unroll
            for (int j = 0; j < kEpiPEJ; ++j) {
                const double2 a = Ks[ogT + kEpiPWarps * KLD * j], bb = c_conj(Ks[og11 + kEpiPWarps * j]);
                sym[j] = make_double2(0.5 * (a.x + bb.x), 0.5 * (a.y + bb.y));
            }
            __syncthreads();
            double2 *Dt = d.D + t * n3;
#pragma unroll
            for (int j = 0; j < kEpiPEJ; ++j) {
                const double2 v = rk4(sym[j], acs[j], ycs[j], e0 + j * kEpiPWarps * kTB);
                KF[ogT + kEpiPWarps * KLD * j] = make_float2(float(v.x), float(v.y));
                Dt[(mu1 * n + w + kEpiPWarps * j) * n + mu2] = v;
            }
            __syncthreads();
        }
        // tile (R, C): tmp_index(n, r_l, mu2, nu2 * 32 + c_l, part), fastest index mu1 = r_l;
        // tile (C, R): element (c, r) = conj(v) at tmp_index(n, c_l, nu2, mu2 * 32 + r_l, part),
        // fastest index nu1 = c_l (the lane), read transposed from the staging tile
        float *Ot = t ? Out1 : Out0;
        float *Orc = Ot + (mu2 * n2 + nu2 * kTB) * 2 * n + oo;
        float *Ocr = Ot + (nu2 * n2 + mu2 * kTB) * 2 * n + oo;
#pragma unroll
        for (int j = 0; j < kEpiPEJ; ++j) {
            const float2 v = KF[ogT + kEpiPWarps * KLD * j];
            Orc[j * kEpiPWarps * 2 * n] = v.x;
            Orc[j * kEpiPWarps * 2 * n + n] = v.y;
        }
        if (!diag) {
#pragma unroll
            for (int j = 0; j < kEpiPEJ; ++j) {
                const float2 v = KF[og11 + kEpiPWarps * j];
                Ocr[j * kEpiPWarps * 2 * n] = v.x;
                Ocr[j * kEpiPWarps * 2 * n + n] = -v.y;
            }
        }
    }
}

}  // namespace g12
