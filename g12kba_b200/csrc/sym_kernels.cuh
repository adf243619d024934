// Mixed-precision ("symmetric") engine kernels.
//
// Physical states of the reference's propagation obey two exact symmetries of
// G2[mu1 mu2; nu1 nu2] (they hold to round-off in the reference's own output,
// starting from G2 = 0):
//   exchange  e:  G2[mu2 mu1; nu2 nu1] = G2[mu1 mu2; nu1 nu2]
//   Hermitian Pe: G2[nu1 nu2; mu1 mu2] = conj(G2[mu1 mu2; nu1 nu2])
// i.e. M = G2 as an n^2 x n^2 matrix (rows r = mu1 + n*mu2, columns
// c = nu1 + n*nu2) is Hermitian and exchange-symmetric, and h is Hermitian.
// Then the two-body commutator of commutators.h:53-99 needs one contraction:
//   T1 = (h (x) 1) M,   W = H2 M = T1 + e(T1),   C = H2 M - M H2 = W - W^H.
// k_sym_gemm* computes W per tile of rows {all mu2} x {c, cbar} (closed under
// e), k_sym_epi forms C = W - W^H on pairs of 32 x 32 tiles (R, C) / (C, R) and
// fuses the rest of the stage (Psi, Pi, K2, RK4 bookkeeping) like k_apply<true>.
//
// Storage (per tensor t = xx, xy; TT = FP32 in the mixed modes, FP64 in FP64SYM):
//   TMP  (TT, GEMM input):    ((mu2*n^2 + c)*2 + part)*n + mu1
//   W    (TT):                (c*2 + part)*n^2 + r
//   Yc, Ac (FP64 complex):    Hermitian-compressed state and RK4 sum: for each
//                             tile pair p = (Rb <= Cb) of 32 x 32 blocks,
//                             [p][c_local*32 + r_local].
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fp64_kernels.cuh"

namespace g12 {

constexpr int kTB = 32;  // epilogue tile edge (rows r and columns c of M)

struct SymDev {
    Dev d;                  // G1 side, tables (Q, Rt, D), schedule, snapshot ring
    int n, cpt;             // cpt: c values per GEMM tile (= 128 / n)
    int gemm_tiles;         // GEMM tiles per tensor
    int nblk, npairs;       // epilogue blocks per edge, tile pairs per tensor
    long long n4;
    float *TMPa, *TMPb;     // 2 tensors each
    float *W;               // 2 tensors
    double2 *Yc, *Ac;       // 2 tensors x npairs x kTB^2
    double2 *Qt, *Rtt;      // transposed copies of Q ([r][b][a]) and Rt ([s][b][a])
    const int *gemm_c;      // [gemm_tiles][cpt] c values
    const int *gemm_partner;// [gemm_tiles][cpt] slot of cbar in the same tile
    const int2 *pairs;      // [npairs] (Rb, Cb), Rb <= Cb
    int *err;               // device error word (bounded waits)
    int g1x;                // k_sym_epi blocks past the tile pairs (blockIdx.y = 0) that run
                            // the stage's G1 side (g1_body); 0: k_g1 is launched on its own
};

// bulk prefetch of a contiguous range into L2 (16-byte aligned, size a multiple of 16)
__device__ __forceinline__ void l2_prefetch_bulk(const void *p, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// stage k reads TMPb (k even) or TMPa (k odd) and writes the other one.  TT is
// the storage type of TMP and W: float (mixed modes) or double (FP64SYM).
template <typename TT = float>
__device__ __forceinline__ const TT *sym_in(const SymDev &s, int k)
{
    return reinterpret_cast<const TT *>((k & 1) ? s.TMPa : s.TMPb);
}
template <typename TT = float>
__device__ __forceinline__ TT *sym_out(const SymDev &s, int k)
{
    return reinterpret_cast<TT *>((k & 1) ? s.TMPb : s.TMPa);
}

// complex pair of the storage type
template <typename TT> struct Cx2;
template <> struct Cx2<float> { using T = float2; };
template <> struct Cx2<double> { using T = double2; };
template <typename TT>
__device__ __forceinline__ typename Cx2<TT>::T mk2(TT a, TT b)
{
    typename Cx2<TT>::T v;
    v.x = a;
    v.y = b;
    return v;
}

__device__ __forceinline__ long long tmp_index(int n, int mu1, int mu2, int c, int part)
{
    return (((long long)mu2 * n * n + c) * 2 + part) * n + mu1;
}

// SIMT version of the W contraction in the storage type TT (FP32: the checker
// of the tensor-core kernels; FP64: the FP64SYM engine), same tiles as the
// tensor-core kernel: T1[mu1][mu2][c] = sum_rho h[mu1][rho] X[rho][mu2][c].
template <typename TT>
__global__ void __launch_bounds__(256) k_sym_gemm_simt(SymDev s, int k)
{
    if (!*s.d.active) return;
    using T2 = typename Cx2<TT>::T;
    const int n = s.n, cpt = s.cpt, rows = cpt * n;
    extern __shared__ double smsimt[];
    TT *X = reinterpret_cast<TT *>(smsimt);  // [rows][2n]
    TT *S = X + rows * 2 * n;                // [rows][2n + 1] (T1 staging)
    T2 *H = reinterpret_cast<T2 *>(S + rows * (2 * n + 1));  // [n][n] (rows = 128: 16-byte aligned)
    const int t = blockIdx.x / s.gemm_tiles, g = blockIdx.x % s.gemm_tiles;
    const TT *Xg = sym_in<TT>(s, k) + t * 2 * s.n4;
    for (int x = threadIdx.x; x < n * n; x += blockDim.x)
        H[x] = mk2<TT>(TT(s.d.h[x].x), TT(s.d.h[x].y));
    for (int e = threadIdx.x; e < rows * 2 * n; e += blockDim.x) {
        const int row = e / (2 * n), kk = e % (2 * n);
        const int slot = row / n, mu2 = row % n;
        const int c = s.gemm_c[g * cpt + slot];
        X[e] = Xg[((long long)mu2 * n * n + c) * 2 * n + kk];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < rows * n; e += blockDim.x) {
        const int row = e / n, mu1 = e % n;
        TT re = 0, im = 0;
        const TT *xr = X + row * 2 * n;
        for (int r = 0; r < n; ++r) {
            const T2 hv = H[mu1 * n + r];
            const TT gr = xr[r], gi = xr[n + r];
            re = fma(hv.x, gr, re);
            re = fma(-hv.y, gi, re);
            im = fma(hv.x, gi, im);
            im = fma(hv.y, gr, im);
        }
        S[row * (2 * n + 1) + mu1] = re;
        S[row * (2 * n + 1) + n + mu1] = im;
    }
    __syncthreads();
    // W[mu1][mu2][c] = T1[mu1][mu2][c] + T1[mu2][mu1][cbar]
    TT *Wg = reinterpret_cast<TT *>(s.W) + t * 2 * s.n4;
    const long long n2 = (long long)n * n;
    for (int e = threadIdx.x; e < cpt * 2 * n * n; e += blockDim.x) {
        const int r = e % (n * n), part = (e / (n * n)) % 2, slot = e / (2 * n * n);
        const int mu1 = r % n, mu2 = r / n;
        const int ps = s.gemm_partner[g * cpt + slot];
        const TT v = S[(slot * n + mu2) * (2 * n + 1) + part * n + mu1] +
                        S[(ps * n + mu1) * (2 * n + 1) + part * n + mu2];
        const int c = s.gemm_c[g * cpt + slot];
        Wg[((long long)c * 2 + part) * n2 + r] = v;
    }
}

// Stage epilogue on a tile pair (R, C) / (C, R): C = W - W^H, Psi, Pi, K2,
// RK4 bookkeeping on the compressed state, next-stage input (both tiles, in
// the storage type TT), particle-2 diagonal D (FP64).
template <int NN, typename TT = float>
__global__ void __launch_bounds__(256, 4) k_sym_epi(SymDev s, int k)
{
    using T2 = typename Cx2<TT>::T;
    if (!*s.d.active) return;
    const Dev &d = s.d;
    if (blockIdx.x >= s.npairs) {
        // the stage's G1 side, folded into this launch (h and Ix come from k_prep)
        if (blockIdx.y == 0 && blockIdx.x - s.npairs < s.g1x) {
            grid_dep_wait();
            g1_body(d, k, blockIdx.x - s.npairs);
        }
        return;
    }
    if (threadIdx.x == 0) {
        // the block's FP64 state tiles (16 KB each, contiguous) do not depend on
        // the GEMM: start them towards L2 before anything else
        const long long tile = ((long long)blockIdx.y * s.npairs + blockIdx.x) * kTB * kTB;
        l2_prefetch_bulk(s.Yc + tile, kTB * kTB * sizeof(double2));
        if (k > 0) l2_prefetch_bulk(s.Ac + tile, kTB * kTB * sizeof(double2));
    }
    constexpr int n = NN;
    constexpr int GLD = NN + 1;   // padded G1 rows (bank-conflict-free column reads)
    constexpr int KLD = kTB + 1;  // padded K rows
    const int Ns = d.Ns;
    const long long n2 = (long long)n * n, n3 = n2 * n;
    const int t = blockIdx.y;
    const int p = blockIdx.x;
    const int2 rc = s.pairs[p];
    const int R0 = rc.x * kTB, C0 = rc.y * kTB;
    const bool diag = rc.x == rc.y;
    extern __shared__ double2 smd[];
    double2 *Gs = smd;                                 // n x GLD
    T2 *Wrc = reinterpret_cast<T2 *>(Gs + n * GLD);    // [c_l][r_l] = W[R0+r_l][C0+c_l]
    T2 *Wcr = Wrc + kTB * (kTB + 1);                   // [r_l][c_l] = W[C0+c_l][R0+r_l]
    double2 *Ks = reinterpret_cast<double2 *>(Wcr + kTB * (kTB + 1));  // [c_l][r_l] tmp_next (or K), rows of KLD
    __shared__ int site[NN];
    const TT *Wg = reinterpret_cast<const TT *>(s.W) + t * 2 * s.n4;
    const double2 *G1 = (k & 1) ? d.G1t1 : d.G1t0;
    if (threadIdx.x < NN) site[threadIdx.x] = threadIdx.x % Ns;
#pragma unroll 4
    for (int x = threadIdx.x; x < n * n; x += blockDim.x) Gs[(x / n) * GLD + x % n] = G1[x];
    // W comes from the GEMM launched just before this kernel (G1 and the tables
    // of k_prep were complete before it started)
    grid_dep_wait();
#pragma unroll
    for (int e = threadIdx.x; e < kTB * kTB; e += blockDim.x) {
        const int rl = e % kTB, cl = e / kTB;
        // W[R0+rl][C0+cl] at (c*2+part)*n2 + r: contiguous in rl
        const long long b1 = (long long)(C0 + cl) * 2 * n2 + R0 + rl;
        Wrc[cl * (kTB + 1) + rl] = mk2<TT>(Wg[b1], Wg[b1 + n2]);
        // W[C0+rl'][R0+cl'] with rl' = rl as the row offset inside block C
        const long long b2 = (long long)(R0 + cl) * 2 * n2 + C0 + rl;
        Wcr[cl * (kTB + 1) + rl] = mk2<TT>(Wg[b2], Wg[b2 + n2]);
    }
    __syncthreads();

    const StageP st = d.cur->st[k];
    const double U = st.U;
    const double2 *__restrict__ Qo = d.Q + t * n3;
    const double2 *__restrict__ Qt = s.Qt + t * n3;
    const double2 *__restrict__ Rtt = s.Rtt;
    double2 *Yc = s.Yc + ((long long)t * s.npairs + p) * kTB * kTB;
    double2 *Ac = s.Ac + ((long long)t * s.npairs + p) * kTB * kTB;
    auto vdist = [&](int s1, int s2) -> double {
        const int m = abs(s1 - s2);
        return (m >= 1 && m <= d.nv) ? U * d.law[m - 1] : 0.0;
    };
    bool fused = false;  // RK bookkeeping done inside the K loop
    if constexpr (NN >= kTB) {
        // n >= 32: every 32 x 32 tile has one mu2 (rows) and one nu2 (columns),
        // so the site weights, Rt, the Pi factor Q and (for xx) the three-G1
        // products of Psi are 32-entry vectors of mu1 or nu1.  A thread keeps
        // one row rl = lane (e = threadIdx.x + 256 j), so the mu1 vectors live
        // in its registers and the nu1 vectors are warp-uniform shared reads.
        __shared__ double wb[kTB];
        __shared__ double2 rb[kTB], qb[kTB], y1[kTB], y2[kTB], hb[kTB];
        const int mu2 = R0 / n, m0 = R0 % n, nu2 = C0 / n, c0 = C0 % n;
        const int sj = site[mu2], sl = site[nu2];
        const double2 *Rt2 = d.Rt + ((long long)mu2 * n + nu2) * Ns;
        const long long q2 = ((long long)nu2 * n + mu2) * n;
        if (threadIdx.x < kTB) {
            const int l = threadIdx.x, nu1 = c0 + l;
            const int sk = site[nu1];
            wb[l] = U * double(sk == sl) + vdist(sk, sl);
            rb[l] = Rt2[sk];
            qb[l] = Qo[q2 + nu1];
            if (t == 0) {
                y1[l] = Gs[mu2 * GLD + nu1];
                y2[l] = Gs[nu2 * GLD + nu1];
                hb[l] = c_mul(Gs[mu2 * GLD + nu1], Gs[nu1 * GLD + nu2]);
            }
        }
        const int rl = threadIdx.x & (kTB - 1);
        const int mu1 = m0 + rl, si = site[mu1];
        const double wa = U * double(si == sj) + vdist(si, sj);
        const double2 ra = Rt2[si], qa = Qo[q2 + mu1];
        double2 x1 = make_double2(0.0, 0.0), x2 = x1, fa = x1;
        if (t == 0) {
            x1 = Gs[mu1 * GLD + mu2];
            x2 = Gs[mu1 * GLD + nu2];
            fa = c_mul(Gs[mu2 * GLD + mu1], Gs[mu1 * GLD + nu2]);
        }
        __syncthreads();
        const double2 g22 = Gs[mu2 * GLD + nu2];
        fused = !diag && !d.debug;
        double2 *Dt = d.D + t * n3;
        const double2 *RttJ = Rtt + (long long)sj * n * n, *RttL = Rtt + (long long)sl * n * n;
        const double2 *QtM = Qt + (long long)mu2 * n * n, *QtN = Qt + (long long)nu2 * n * n;
#pragma unroll 4
        for (int j = 0; j < kTB * kTB / 256; ++j) {
            const int cl = (threadIdx.x >> 5) + 8 * j;
            const int e = cl * kTB + rl;  // = threadIdx.x + 256 j
            const int nu1 = c0 + cl;
            const T2 w1 = Wrc[cl * (kTB + 1) + rl];
            const T2 w2 = Wcr[rl * (kTB + 1) + cl];
            const double2 C = make_double2(double(w1.x) - double(w2.x), double(w1.y) + double(w2.y));
            const double2 g11 = Gs[mu1 * GLD + nu1];
            const double2 g1122 = c_mul(g11, g22);
            const double wd = wa - wb[cl];
            double2 psi = c_scale(g1122, wd);
            psi = c_add(psi, c_i(c_mul(g22, c_sub(RttJ[nu1 * n + mu1], RttL[nu1 * n + mu1]))));
            psi = c_add(psi, c_i(c_mul(g11, c_sub(ra, rb[cl]))));
            if (t == 0) {
                psi = c_sub(psi, c_scale(g1122, U * (double(mu1 == mu2) - double(nu1 == nu2))));
                const double2 e1 = c_sub(c_mul(x1, y1[cl]), c_mul(x2, y2[cl]));
                const double2 e2 = c_sub(fa, hb[cl]);
                psi = c_add(psi, c_scale(c_mi(c_add(c_mul(g22, e1), c_mul(g11, e2))), U));
            }
            const double2 pi = c_mul(g22, c_sub(QtM[nu1 * n + mu1], QtN[nu1 * n + mu1]));
            const double2 piP = c_mul(Gs[nu1 * GLD + mu1], c_sub(qb[cl], qa));
            const double2 K = c_mi(c_sub(c_add(c_add(C, psi), pi), c_conj(piP)));
            if (fused) {
                // RK4 bookkeeping of this element right away (off-diagonal tile pairs)
                const double2 rk = c_add(k == 0 ? make_double2(0.0, 0.0) : Ac[e], c_scale(K, st.w));
                double2 v;
                if (k < 3) {
                    Ac[e] = rk;
                    v = c_add(Yc[e], c_scale(K, st.c_next));
                } else {
                    v = c_add(Yc[e], c_scale(c_scale(rk, st.dt), 1.0 / 6.0));
                    Yc[e] = v;
                }
                Ks[cl * KLD + rl] = v;
                if (mu2 == nu2) {
                    Dt[((long long)mu1 * n + nu1) * n + mu2] = v;
                    Dt[((long long)nu1 * n + mu1) * n + nu2] = c_conj(v);
                }
            } else {
                Ks[cl * KLD + rl] = K;
            }
        }
    } else {
#pragma unroll 4
    for (int e = threadIdx.x; e < kTB * kTB; e += blockDim.x) {
        const int rl = e % kTB, cl = e / kTB;
        const int r = R0 + rl, c = C0 + cl;
        const int mu1 = r % n, mu2 = r / n, nu1 = c % n, nu2 = c / n;
        const T2 w1 = Wrc[cl * (kTB + 1) + rl];
        // W[c][r] = Wcr at (row offset cl in block C -> index rl' = cl, col r -> cl' = rl)
        const T2 w2 = Wcr[rl * (kTB + 1) + cl];
        const double2 C = make_double2(double(w1.x) - double(w2.x), double(w1.y) + double(w2.y));
        const int si = site[mu1], sj = site[mu2], sk = site[nu1], sl = site[nu2];
        const double2 g11 = Gs[mu1 * GLD + nu1], g22 = Gs[mu2 * GLD + nu2];
        const double wd = (U * double(si == sj) + vdist(si, sj)) - (U * double(sk == sl) + vdist(sk, sl));
        double2 psi = c_scale(c_mul(g11, g22), wd);
        psi = c_add(psi, c_i(c_mul(g22, c_sub(Rtt[((long long)sj * n + nu1) * n + mu1], Rtt[((long long)sl * n + nu1) * n + mu1]))));
        const double2 *Rt2 = d.Rt + ((long long)mu2 * n + nu2) * Ns;
        psi = c_add(psi, c_i(c_mul(g11, c_sub(Rt2[si], Rt2[sk]))));
        if (t == 0) {
            psi = c_sub(psi, c_scale(c_mul(g11, g22), U * (double(mu1 == mu2) - double(nu1 == nu2))));
            const double2 e1 = c_sub(c_mul(Gs[mu1 * GLD + mu2], Gs[mu2 * GLD + nu1]), c_mul(Gs[mu1 * GLD + nu2], Gs[nu2 * GLD + nu1]));
            const double2 e2 = c_sub(c_mul(Gs[mu2 * GLD + mu1], Gs[mu1 * GLD + nu2]), c_mul(Gs[mu2 * GLD + nu1], Gs[nu1 * GLD + nu2]));
            psi = c_add(psi, c_scale(c_mi(c_add(c_mul(g22, e1), c_mul(g11, e2))), U));
        }
        // Pi[x] = G1[mu2][nu2] (Q[mu1][nu1][mu2] - Q[mu1][nu1][nu2]); Qt[r][b][a] = Q[a][b][r]
        const double2 pi = c_mul(g22, c_sub(Qt[((long long)mu2 * n + nu1) * n + mu1], Qt[((long long)nu2 * n + nu1) * n + mu1]));
        const long long q2 = ((long long)nu2 * n + mu2) * n;
        const double2 piP = c_mul(Gs[nu1 * GLD + mu1], c_sub(Qo[q2 + nu1], Qo[q2 + mu1]));
        const double2 K = c_mi(c_sub(c_add(c_add(C, psi), pi), c_conj(piP)));
        Ks[cl * KLD + rl] = K;
    }
    }
    __syncthreads();
    if (diag) {
        // keep the diagonal block exactly Hermitian: K <- (K + K^H) / 2
        double2 sym[4];
        int cnt = 0;
        for (int e = threadIdx.x; e < kTB * kTB; e += blockDim.x) {
            const int rl = e % kTB, cl = e / kTB;
            const double2 a = Ks[cl * KLD + rl], b = c_conj(Ks[rl * KLD + cl]);
            sym[cnt++] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
        }
        __syncthreads();
        cnt = 0;
        for (int e = threadIdx.x; e < kTB * kTB; e += blockDim.x) {
            const int rl = e % kTB, cl = e / kTB;
            Ks[cl * KLD + rl] = sym[cnt++];
        }
        __syncthreads();
    }
    if (d.debug) {
        // K of both tiles into d.Y2 in the device orbital layout x = c + n^2 r
        double2 *Kd = d.Y2 + t * n2 * n2;
        for (int e = threadIdx.x; e < kTB * kTB; e += blockDim.x) {
            const int rl = e % kTB, cl = e / kTB;
            const double2 K = Ks[cl * KLD + rl];
            Kd[(long long)(R0 + rl) * n2 + C0 + cl] = K;
            Kd[(long long)(C0 + cl) * n2 + R0 + rl] = c_conj(K);
        }
        return;
    }
    // RK4 bookkeeping on the compressed state; next-stage input value in Ks
    double2 *Dt = d.D + t * n3;
    for (int e = threadIdx.x; e < kTB * kTB && !fused; e += blockDim.x) {
        const int rl = e % kTB, cl = e / kTB;
        const double2 K = Ks[cl * KLD + rl];
        const double2 rk = c_add(k == 0 ? make_double2(0.0, 0.0) : Ac[e], c_scale(K, st.w));
        double2 v;
        if (k < 3) {
            Ac[e] = rk;
            v = c_add(Yc[e], c_scale(K, st.c_next));
        } else {
            v = c_add(Yc[e], c_scale(c_scale(rk, st.dt), 1.0 / 6.0));
            Yc[e] = v;
        }
        Ks[cl * KLD + rl] = v;
        const int r = R0 + rl, c = C0 + cl;
        const int mu1 = r % n, mu2 = r / n, nu1 = c % n, nu2 = c / n;
        if (mu2 == nu2) {
            Dt[((long long)mu1 * n + nu1) * n + mu2] = v;
            // the mirrored element (nu1, nu2; mu1, mu2) holds conj(v)
            if (!diag) Dt[((long long)nu1 * n + mu1) * n + nu2] = c_conj(v);
        }
    }
    __syncthreads();
    TT *Out = sym_out<TT>(s, k) + t * 2 * s.n4;
    // tile (R, C): fastest index mu1 = r % n follows rl
    for (int e = threadIdx.x; e < kTB * kTB; e += blockDim.x) {
        const int rl = e % kTB, cl = e / kTB;
        const int r = R0 + rl, c = C0 + cl;
        const double2 v = Ks[cl * KLD + rl];
        const long long o = tmp_index(n, r % n, r / n, c, 0);
        Out[o] = TT(v.x);
        Out[o + n] = TT(v.y);
    }
    if (!diag) {
        // tile (C, R): element (c, r) = conj(v); fastest index nu1 = c % n follows cl
        for (int e = threadIdx.x; e < kTB * kTB; e += blockDim.x) {
            const int cl = e % kTB, rl = e / kTB;
            const int r = R0 + rl, c = C0 + cl;
            const double2 v = Ks[cl * KLD + rl];
            const long long o = tmp_index(n, c % n, c / n, r, 0);
            Out[o] = TT(v.x);
            Out[o + n] = TT(-v.y);
        }
    }
}

// Full FP64 state (device orbital layout, Y2 of the general engine) -> Yc,
// TMPb (stage-0 input, storage type TT) and D.  One block per tile pair and tensor.
template <typename TT>
__global__ void k_sym_pack(SymDev s, const double2 *Yfull)
{
    const int n = s.n;
    const long long n2 = (long long)n * n, n3 = n2 * n;
    const int t = blockIdx.y, p = blockIdx.x;
    const int2 rc = s.pairs[p];
    const int R0 = rc.x * kTB, C0 = rc.y * kTB;
    const double2 *Y = Yfull + t * s.n4;
    double2 *Yc = s.Yc + ((long long)t * s.npairs + p) * kTB * kTB;
    TT *Out = reinterpret_cast<TT *>(s.TMPb) + t * 2 * s.n4;
    double2 *Dt = s.d.D + t * n3;
    for (int e = threadIdx.x; e < kTB * kTB; e += blockDim.x) {
        const int rl = e % kTB, cl = e / kTB;
        const int r = R0 + rl, c = C0 + cl;
        const int mu1 = r % n, mu2 = r / n, nu1 = c % n, nu2 = c / n;
        // device orbital layout: x = nu1 + n*nu2 + n^2*mu1 + n^3*mu2
        const double2 v = Y[(long long)c + n2 * mu1 + n3 * mu2];
        Yc[e] = v;
        long long o = tmp_index(n, mu1, mu2, c, 0);
        Out[o] = TT(v.x);
        Out[o + n] = TT(v.y);
        if (mu2 == nu2) Dt[((long long)mu1 * n + nu1) * n + mu2] = v;
        if (rc.x != rc.y) {
            o = tmp_index(n, nu1, nu2, r, 0);
            Out[o] = TT(v.x);
            Out[o + n] = TT(-v.y);
            if (nu2 == mu2) Dt[((long long)nu1 * n + mu1) * n + nu2] = c_conj(v);
        }
    }
}

// Yc -> full FP64 state in the device orbital layout (Hermitian expansion).
__global__ void k_sym_unpack(SymDev s, double2 *Yfull)
{
    const int n = s.n;
    const long long n2 = (long long)n * n, n3 = n2 * n;
    const int t = blockIdx.y, p = blockIdx.x;
    const int2 rc = s.pairs[p];
    const int R0 = rc.x * kTB, C0 = rc.y * kTB;
    double2 *Y = Yfull + t * s.n4;
    const double2 *Yc = s.Yc + ((long long)t * s.npairs + p) * kTB * kTB;
    for (int e = threadIdx.x; e < kTB * kTB; e += blockDim.x) {
        const int rl = e % kTB, cl = e / kTB;
        const int r = R0 + rl, c = C0 + cl;
        const int mu1 = r % n, mu2 = r / n, nu1 = c % n, nu2 = c / n;
        const double2 v = Yc[e];
        Y[(long long)c + n2 * mu1 + n3 * mu2] = v;
        if (rc.x != rc.y) Y[(long long)r + n2 * nu1 + n3 * nu2] = c_conj(v);
    }
}

}  // namespace g12
