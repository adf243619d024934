// FP64 device kernels of one RK4 stage of the HF-GKBA G1-G2 equations
// (reference: G12KBA-GW/src/headers/{HF,commutators,psi,pi,collision_integral,
// G1_G2_t_step,RK_solver,AS}.h).
//
// Device layout (per system, n = Ns*Nb, orbital mu = site + band*Ns):
//   G1-like arrays: n x n row-major, element [mu][nu] at nu + n*mu.
//   G2 tensors:     x = nu1 + n*nu2 + n^2*mu1 + n^3*mu2 for G2[mu1 mu2; nu1 nu2]
//                   (the reference's IDX_8D with sites and bands regrouped into
//                   orbitals; identical to it for Nb = 1).  Tensor 0 is G2xxxx,
//                   tensor 1 is G2xyxy, stored back to back.
//   D[t][a][b][r] = G2_t[a, r; b, r]   (n^3, the particle-2 diagonal)
//   Q[t][a][b][r]                        (n^3, Pi factor, see k_prep)
//   Rt[a][b][s]                          (n^2*Ns, Psi factor, see k_prep)
//
// Factorisation used here (derived from the reference loops, not copied):
//   Pi(psi.h/pi.h notation) = G1[mu2][nu2] * (Q[mu1][nu1][mu2] - Q[mu1][nu1][nu2])
//   Q_t[a][b][(s,r)] = -i*U*(S[a][b][s] - D_t'[a][b][(s,r)]) - i*Vp[a][b][s]
//       S[s] = sum_r (Dxx + Dxy)[(s,r)],  Vp[s] = sum_m V_m (S[s+m] + S[s-m]),
//       t' = xx for Pi_xx (pi.h called with G2xy, G2xx) and xy for Pi_xy.
//   collision_int I[mu][nu] = Q_xx[mu][nu][mu].
//   Psi_xy = g11 g22 (W(i,j) - W(k,l)) + i g22 (Rt[mu1][nu1][j] - Rt[mu1][nu1][l])
//                                      + i g11 (Rt[mu2][nu2][i] - Rt[mu2][nu2][k])
//       W(s,s') = U [s=s'] + V_|s-s'|,  Rt[a][b][s] = U R[s] + sum_m V_m (R[s+m] + R[s-m]),
//       R[a][b][s] = sum_r G1[a][(s,r)] G1[(s,r)][b].
//   Psi_xx = Psi_xy - U g11 g22 ([mu1=mu2] - [nu1=nu2])
//            - i U g22 (G1[mu1][mu2]G1[mu2][nu1] - G1[mu1][nu2]G1[nu2][nu1])
//            - i U g11 (G1[mu2][mu1]G1[mu1][nu2] - G1[mu2][nu1]G1[nu1][nu2]).
//   Two-body commutator C = H2 M - M H2 with M = G2 as an n^2 x n^2 matrix and
//   H2 = h (x) 1 + 1 (x) h: k_apply<false> (rows: particle indices mu1, mu2) and
//   k_apply<true> (columns nu1, nu2); each is Y = L X + X R on a batch of n x n
//   matrices X, with (L, R) = (h, h^T) or (h^T, h).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "internal.h"

namespace g12 {

constexpr int kMaxN = 64;

struct Dev {
    int Ns, Nb, n, nv, gate, debug;
    long long n2, n3, n4;
    double t1, t2;
    double law[kMaxN];  // V_m = U_eff * law[m-1], m = 1..nv
    double2 *Y1, *G1t0, *G1t1, *RK1, *h, *Ix, *comm_dbg, *K1_dbg;
    double2 *Y2, *RK2, *TMP0, *TMP1, *TAB, *D, *Q, *Rt;
    double2 *Qt, *Rtt;  // transposed table copies (symmetric engine), or null
    double2 *Zt;        // combined table i Rtt[site(r)] + Qt[t][r] (persistent epilogue at n = 32), or null
    unsigned char *ozb; // bf16 digit tiles of h for the tcgen05 digit GEMM (symmetric engine), or null
    double2 *traj;
    double *dip;
    long long traj_cap;
    long long dip_cap;
    const StepP *sched;
    long long *counter, *limit;
    int *status, *active;
    StepP *cur;
};

// programmatic dependent launch: wait until the preceding kernel of the stream
// has completed and its writes are visible (no effect without such a launch),
// and let the next kernel of the stream start its prologue
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ double2 c_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 c_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 c_mul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 c_scale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 c_conj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 c_i(double2 a) { return make_double2(-a.y, a.x); }    // i*a
__device__ __forceinline__ double2 c_mi(double2 a) { return make_double2(a.y, -a.x); }   // -i*a
__device__ __forceinline__ double2 c_mac(double2 acc, double2 a, double2 b)
{
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
    return acc;
}

__device__ __forceinline__ const double2 *g1_stage(const Dev &d, int k) { return (k & 1) ? d.G1t1 : d.G1t0; }
__device__ __forceinline__ double2 *g1_next(const Dev &d, int k) { return (k & 1) ? d.G1t0 : d.G1t1; }
// stage k reads Y (k = 0) or TMP[(k+1)&1]; stage k < 3 writes TMP[k&1]
__device__ __forceinline__ const double2 *g2_stage(const Dev &d, int k)
{
    return k == 0 ? d.Y2 : (((k + 1) & 1) ? d.TMP1 : d.TMP0);
}
__device__ __forceinline__ double2 *g2_next(const Dev &d, int k) { return (k & 1) ? d.TMP1 : d.TMP0; }

// ---------------------------------------------------------------------------
// Step head (RK_solver.h:98-110): copy this step's scalars, record the
// snapshot and dipole, apply the site-0 density guard, stage-0 G1 input.
__device__ __forceinline__ void step_begin_body(const Dev &d)
{
    __shared__ long long s_step;
    __shared__ int s_act, s_rec;
    const int tid = threadIdx.x;
    const int n = d.n;
    // this thread's first entries of G1, loaded while thread 0 reads the step
    // counter and the schedule (they do not depend on them)
    constexpr int kPre = 4;
    double2 pre[kPre];
#pragma unroll
    for (int q = 0; q < kPre; ++q) {
        const int x = tid + q * int(blockDim.x);
        pre[q] = x < n * n ? d.Y1[x] : make_double2(0.0, 0.0);
    }
    if (tid == 0) {
        const long long s = *d.counter;
        const int act = (*d.status == 0) && (s < *d.limit);
        s_step = s;
        s_act = act;
        s_rec = act ? d.sched[s].record : 0;
    }
    __syncthreads();
    if (!s_act) {
        if (tid == 0) *d.active = 0;
        return;
    }
    const long long s = s_step;
    {
        // this step's scalars, one word per thread
        const uint32_t *src = reinterpret_cast<const uint32_t *>(d.sched + s);
        uint32_t *dst = reinterpret_cast<uint32_t *>(d.cur);
        for (int w = tid; w < int(sizeof(StepP) / 4); w += blockDim.x) dst[w] = src[w];
    }
    double2 *tr = d.traj + (s % d.traj_cap) * d.n2;
#pragma unroll
    for (int q = 0; q < kPre; ++q) {
        const int x = tid + q * int(blockDim.x);
        if (x < n * n) {
            d.G1t0[x] = pre[q];
            if (s_rec) tr[x] = pre[q];
        }
    }
#pragma unroll 4
    for (int x = tid + kPre * int(blockDim.x); x < n * n; x += blockDim.x) {
        const double2 v = d.Y1[x];
        d.G1t0[x] = v;
        if (s_rec) tr[x] = v;
    }
    if (s_rec && tid < 32) {
        // dipole.h:25-32, warp-shuffle reduction over the mirrored diagonal
        const double sq = double(n);
        double acc = 0.0;
        for (int i = tid; i < n / 2; i += 32)
            acc += 2 * (sq / 2 - i - .5) * (d.Y1[i * (n + 1)].y - d.Y1[n * n - i * (n + 1) - 1].y) / sq;
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (tid == 0) {
            d.dip[s % d.dip_cap] = acc;
            int act = 1;
            const double nd = 2 * d.Y1[0].y;
            if (fabs(nd) > 3 || isnan(nd)) {
                *d.status = int(s + 1);
                act = 0;
            }
            *d.active = act;
            *d.counter = s + 1;
        }
    } else if (tid == 0) {
        *d.active = 1;
        *d.counter = s + 1;
    }
}

static __global__ void __launch_bounds__(256) k_step_begin(Dev d) { step_begin_body(d); }

// HF.h:57-104, entry by entry.
// gd: the diagonal G[p][p] of the stage's G1 (staged in shared memory by the
// caller; the diagonal entries of h sum up to 4 Nv of them)
__device__ __forceinline__ double2 h_entry(const Dev &d, const double2 *G, const double2 *gd, int mu, int nu,
                                           const StageP &st)
{
    const int Ns = d.Ns, n = d.n;
    const int i = mu % Ns, a = mu / Ns, j = nu % Ns, b = nu / Ns;
    const double U = st.U;
    double2 v = make_double2(0.0, 0.0);
    if (mu == nu) {
        if (i < st.nq) v.x += st.wq;
        v = c_add(v, c_scale(c_mi(gd[mu]), U));
        for (int g = 0; g < d.Nb; ++g)
            if (g != a) {
                int ig = i + g * Ns;
                v = c_add(v, c_scale(c_mi(gd[ig]), 2.0 * U));
            }
        for (int m = 1; m <= d.nv; ++m) {
            const double Vm = U * d.law[m - 1];
            for (int dd = 0; dd < d.Nb; ++dd) {
                if (i + m < Ns) {
                    int p = (i + m) + dd * Ns;
                    v = c_add(v, c_scale(c_mi(gd[p]), 2.0 * Vm));
                }
                if (i - m >= 0) {
                    int q = (i - m) + dd * Ns;
                    v = c_add(v, c_scale(c_mi(gd[q]), 2.0 * Vm));
                }
            }
        }
    } else {
        if (a == b && abs(i - j) == 1) v.x += -d.t1;
        if (i == j && abs(a - b) == 1) v.x += -d.t2;
        if (i == j) v = c_add(v, c_scale(c_i(G[nu * n + mu]), U));
        const int m = abs(i - j);
        if (m >= 1 && m <= d.nv) v = c_add(v, c_scale(c_i(G[mu * n + nu]), U * d.law[m - 1]));
    }
    return v;
}

// Per (alpha, beta) pair, one warp: Psi factor Rt, Pi factors Q_xx / Q_xy and
// the collision integral; blocks past the pair blocks build h, one entry per
// thread.  With d.Qt set (symmetric engine) the transposed copies
// Qt[t][r][b][a] = Q[t][a][b][r] and Rtt[s][b][a] = Rt[a][b][s] are written too;
// with d.Zt set, their combination Zt[t][r][b][a] = i Rt[a][b][r % Ns] + Q[t][a][b][r]
// (the Psi and Pi factors that the epilogue multiplies by the same G1 entry).
constexpr int kPrepWarps = 4;
// k_prep_wide (the mixed engine at n = 32): the same work in 16-warp blocks,
// 66 of them, which leave 82 SMs free for the digit GEMM's first CTAs
constexpr int kPrepWarpsWide = 16;

template <int W = kPrepWarps>
__host__ __device__ inline int prep_pair_blocks(long long n2)
{
    return int((n2 + W - 1) / W);
}
template <int W = kPrepWarps>
inline int prep_blocks(long long n2)
{
    return prep_pair_blocks<W>(n2) + int((n2 + W * 32 - 1) / (W * 32));
}
template <int W = kPrepWarps>
inline size_t prep_smem()
{
    return size_t(W) * 4 * kMaxN * sizeof(double2);
}

// Exact bf16 digits of the real form of h^T for the tcgen05 digit GEMM of the
// symmetric engine (sym_oz.cuh, k_sym_gemm_oz2), written once per stage by the
// threads that compute h (n = 16 or 32: each 128-thread block holds whole rows of h).
// B row j = po*n + mu1, column kk = pi*n + rho:
//   (po, pi) = (0, 0): Re h, (0, 1): -Im h, (1, 0): Im h, (1, 1): Re h  at h[mu1][rho];
// each row is scaled by 2^(30 - e), e = exponent of its largest |entry|, and
// split by successive round-to-nearest into 4 digits (|d| <= 128).
// Layout: 4 tiles of 2n rows x 128 bytes (128-byte swizzle, K-major), then
// the 2n row scales 2^(e - 6) as floats.
__device__ __forceinline__ void h_digits(const Dev &d, double2 hv, int x)
{
    const int n = d.n;
    const int mu1 = x / n, rho = x % n;
    double m = fmax(fabs(hv.x), fabs(hv.y));
    for (int o = n / 2; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    const int e = (m > 0.0) ? ilogb(m) : 0;
    const int tile = 2 * n * 128;
    const double vals[4] = {hv.x, -hv.y, hv.y, hv.x};
#pragma unroll
    for (int idx = 0; idx < 4; ++idx) {
        const int j = (idx >> 1) * n + mu1, kk = (idx & 1) * n + rho;
        double r = ldexp(vals[idx], 30 - e);
        double dg[4];
        dg[0] = rint(r * 0x1p-24);
        r -= dg[0] * 0x1p24;
        dg[1] = rint(r * 0x1p-16);
        r -= dg[1] * 0x1p16;
        dg[2] = rint(r * 0x1p-8);
        r -= dg[2] * 0x1p8;
        dg[3] = rint(r);
        const int byte = j * 128 + ((((kk >> 3) ^ (j & 7)) << 4) | ((kk & 7) << 1));
#pragma unroll
        for (int q = 0; q < 4; ++q)
            *reinterpret_cast<__nv_bfloat16 *>(d.ozb + q * tile + byte) = __float2bfloat16_rn(float(dg[q]));
    }
    if (rho == 0) {
        float *sc = reinterpret_cast<float *>(d.ozb + 4 * tile);
        sc[mu1] = sc[n + mu1] = float(ldexp(1.0, e - 6));
    }
}

// h (HF.h:57-104), one entry per thread, and its digits for the tensor cores;
// hb: block index among the h blocks
__device__ __forceinline__ void prep_h_part(const Dev &d, int k, int hb)
{
    if (!*d.active) return;
    const StageP st = d.cur->st[k];
    const int n = d.n;
    const long long n2 = (long long)n * n;
    const double2 *__restrict__ G = g1_stage(d, k);
    extern __shared__ double2 sm_h[];
    for (int p = threadIdx.x; p < n; p += blockDim.x) sm_h[p] = G[(long long)p * n + p];
    __syncthreads();
    const long long x = (long long)hb * blockDim.x + threadIdx.x;
    double2 hv = make_double2(0.0, 0.0);
    if (x < n2) {
        hv = h_entry(d, G, sm_h, int(x / n), int(x % n), st);
        d.h[x] = hv;
    }
    if (d.ozb && x < n2) h_digits(d, hv, int(x));  // whole warps (n2 is a multiple of 32 with digits)
}

template <int W>
__device__ __forceinline__ void prep_pair_part(const Dev &d, int k, int bx);

template <int W = kPrepWarps>
__device__ __forceinline__ void prep_body(const Dev &d, int k, int bx)
{
    const int pair_blocks = prep_pair_blocks<W>(d.n2);
    if (bx >= pair_blocks) prep_h_part(d, k, bx - pair_blocks);
    else prep_pair_part<W>(d, k, bx);
}

// the Psi, Pi and collision tables: one (alpha, beta) pair per warp, W warps per block
template <int W>
__device__ __forceinline__ void prep_pair_part(const Dev &d, int k, int bx)
{
    if (!*d.active) return;
    const StageP st = d.cur->st[k];
    const int n = d.n, Ns = d.Ns, Nb = d.Nb, nv = d.nv;
    const long long n2 = (long long)n * n;
    const double2 *__restrict__ G = g1_stage(d, k);
    extern __shared__ double2 sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double2 *wE = sm + warp * (4 * kMaxN);   // n entries
    double2 *wDx = wE + kMaxN;               // n
    double2 *wDy = wDx + kMaxN;              // n
    double2 *wS = wDy + kMaxN;               // R / S, Ns entries
    const long long pair = (long long)bx * W + warp;
    if (pair >= n2) return;
    const int alpha = int(pair / n), beta = int(pair % n);
    const double U = st.U;
    if (!d.gate) {
        if (lane == 0) d.Ix[pair] = make_double2(0.0, 0.0);
        return;
    }
    // issue all global loads of this pair first: G rows/columns and the diagonals D
    double2 ga[2], gb[2], dx[2], dy[2];
    const double2 *Dx = d.D + pair * n, *Dy = d.D + d.n3 + pair * n;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int r = lane + 32 * q;
        if (r < n) {
            ga[q] = G[alpha * n + r];
            gb[q] = G[r * n + beta];
            dx[q] = Dx[r];
            dy[q] = Dy[r];
        }
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int r = lane + 32 * q;
        if (r < n) {
            wE[r] = c_mul(ga[q], gb[q]);  // G1[alpha][(s,b)] G1[(s,b)][beta]
            wDx[r] = dx[q];
            wDy[r] = dy[q];
        }
    }
    __syncwarp();
    // R[s] = sum_b E[(s,b)],  S[s] = sum_b (Dxx + Dxy)[(s,b)]
    double2 Rv[2], Sv[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int sidx = lane + 32 * q;
        double2 r = make_double2(0.0, 0.0), sacc = make_double2(0.0, 0.0);
        if (sidx < Ns)
            for (int b = 0; b < Nb; ++b) {
                r = c_add(r, wE[sidx + b * Ns]);
                sacc = c_add(sacc, c_add(wDx[sidx + b * Ns], wDy[sidx + b * Ns]));
            }
        Rv[q] = r;
        Sv[q] = sacc;
    }
    __syncwarp();
    double2 *wR = wE;  // R over E (E no longer needed)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int sidx = lane + 32 * q;
        if (sidx < Ns) {
            wR[sidx] = Rv[q];
            wS[sidx] = Sv[q];
        }
    }
    __syncwarp();
    // Rt[s] = U R[s] + sum_m V_m (R[s+m] + R[s-m]);  Vp[s] = sum_m V_m (S[s+m] + S[s-m])
    double2 Vpv[2], Rtv[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int sidx = lane + 32 * q;
        Vpv[q] = make_double2(0.0, 0.0);
        Rtv[q] = Vpv[q];
        if (sidx >= Ns) continue;
        double2 acc = c_scale(wR[sidx], U), vp = make_double2(0.0, 0.0);
        for (int m = 1; m <= nv; ++m) {
            const double Vm = U * d.law[m - 1];
            double2 tr = make_double2(0.0, 0.0), ts = make_double2(0.0, 0.0);
            if (sidx + m < Ns) {
                tr = c_add(tr, wR[sidx + m]);
                ts = c_add(ts, wS[sidx + m]);
            }
            if (sidx - m >= 0) {
                tr = c_add(tr, wR[sidx - m]);
                ts = c_add(ts, wS[sidx - m]);
            }
            acc = c_add(acc, c_scale(tr, Vm));
            vp = c_add(vp, c_scale(ts, Vm));
        }
        d.Rt[pair * Ns + sidx] = acc;
        if (d.Rtt) d.Rtt[((long long)sidx * n + beta) * n + alpha] = acc;
        Vpv[q] = vp;
        Rtv[q] = acc;
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int sidx = lane + 32 * q;
        if (sidx < Ns) wE[kMaxN - 1 - sidx] = Vpv[q];  // Vp stored from the top of wE (R no longer read)
    }
    __syncwarp();
    double2 *Qx = d.Q + pair * n, *Qy = d.Q + d.n3 + pair * n;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int r = lane + 32 * q;
        double2 rt = make_double2(0.0, 0.0);
        if (d.Zt) {
            // Rt[pair][r % Ns], held by lane (r % Ns) % 32 in Rtv[(r % Ns) / 32]
            const int src = r < n ? r % Ns : 0;
            double2 a0, a1;
            a0.x = __shfl_sync(0xffffffffu, Rtv[0].x, src & 31);
            a0.y = __shfl_sync(0xffffffffu, Rtv[0].y, src & 31);
            a1.x = __shfl_sync(0xffffffffu, Rtv[1].x, src & 31);
            a1.y = __shfl_sync(0xffffffffu, Rtv[1].y, src & 31);
            rt = (src >> 5) ? a1 : a0;
        }
        if (r >= n) continue;
        const int sidx = r % Ns;
        const double2 S = wS[sidx], vp = wE[kMaxN - 1 - sidx];
        const double2 qx = c_mi(c_add(c_scale(c_sub(S, wDx[r]), U), vp));
        const double2 qy = c_mi(c_add(c_scale(c_sub(S, wDy[r]), U), vp));
        Qx[r] = qx;
        Qy[r] = qy;
        if (d.Qt) {
            d.Qt[((long long)r * n + beta) * n + alpha] = qx;
            d.Qt[d.n3 + ((long long)r * n + beta) * n + alpha] = qy;
        }
        if (d.Zt) {
            d.Zt[((long long)r * n + beta) * n + alpha] = c_add(c_i(rt), qx);
            d.Zt[d.n3 + ((long long)r * n + beta) * n + alpha] = c_add(c_i(rt), qy);
        }
        if (r == alpha) d.Ix[pair] = qx;
    }
}

static __global__ void __launch_bounds__(kPrepWarps * 32) k_prep(Dev d, int k)
{
    grid_dep_launch();  // the symmetric engine's GEMM may start its prologue
    prep_body(d, k, blockIdx.x);
}

static __global__ void __launch_bounds__(kPrepWarpsWide * 32) k_prep_wide(Dev d, int k)
{
    grid_dep_launch();
    prep_body<kPrepWarpsWide>(d, k, blockIdx.x);
}

// G1 side of a stage (commutators.h:28-51, G1_G2_t_step.h:24-47) and the
// G1 RK bookkeeping (RK_solver.h:134-135, 204-208).  One output per thread,
// blocks of 128; each block stages h and G1 in shared memory.
constexpr int kG1Threads = 128;
inline int g1_blocks(long long n2) { return int((n2 + kG1Threads - 1) / kG1Threads); }
inline size_t g1_smem(long long n2) { return size_t(2) * n2 * sizeof(double2); }

__device__ __forceinline__ void g1_body(const Dev &d, int k, int bx)
{
    if (!*d.active) return;
    const StageP st = d.cur->st[k];
    const int n = d.n;
    const int n2 = n * n;
    extern __shared__ double2 sm[];
    double2 *sH = sm, *sG = sm + n2;
    const double2 *G1 = g1_stage(d, k);
#pragma unroll 4
    for (int x = threadIdx.x; x < n2; x += blockDim.x) {
        sH[x] = d.h[x];
        sG[x] = G1[x];
    }
    __syncthreads();
    const int x = bx * blockDim.x + threadIdx.x;
    if (x >= n2) return;
    double2 *G1n = g1_next(d, k);
    const int mu = x / n, nu = x % n;
    double2 hg = make_double2(0.0, 0.0), gh = make_double2(0.0, 0.0);
    for (int r = 0; r < n; ++r) {
        hg = c_mac(hg, sH[mu * n + r], sG[r * n + nu]);
        gh = c_mac(gh, sG[mu * n + r], sH[r * n + nu]);
    }
    const double2 comm = c_sub(hg, gh);
    const double2 K = c_mi(c_add(c_add(comm, d.Ix[x]), c_conj(d.Ix[nu * n + mu])));
    if (d.debug) {
        d.comm_dbg[x] = comm;
        d.K1_dbg[x] = K;
        return;
    }
    const double2 rk = c_add(k == 0 ? make_double2(0.0, 0.0) : d.RK1[x], c_scale(K, st.w));
    if (k < 3) {
        d.RK1[x] = rk;
        G1n[x] = c_add(d.Y1[x], c_scale(K, st.c_next));
    } else {
        d.Y1[x] = c_add(d.Y1[x], c_scale(c_scale(rk, st.dt), 1.0 / 6.0));
    }
}

static __global__ void __launch_bounds__(kG1Threads) k_g1(Dev d, int k) { g1_body(d, k, blockIdx.x); }

// Two-body commutator halves as Y = L X + X R on a batch of n x n matrices
// held in shared memory ("natural" layout: row = slower index).
//   CD = false: rows of M (particle indices), X_c[mu2][mu1] = G2[mu1 mu2; c],
//               (L, R) = (h, h^T), result T = (H2 M) written to TAB.
//   CD = true:  columns of M, X_r[nu2][nu1] = G2[r; nu1 nu2], (L, R) = (h^T, h),
//               C = TAB - (M H2) then the fused epilogue: Psi, Pi, K2
//               (G1_G2_t_step.h:55-86) and the RK4 bookkeeping
//               (RK_solver.h:137-139, 209-213).
// Each thread owns a 4 x 4 register tile with stride S = NP/4 in both
// directions (conflict-free shared-memory rows).
struct ApplyCfg {
    int NP, LD, S, NB;
};

// Fused epilogue of one element G2[r; nu1 nu2] (r = mu1 + n mu2) of the
// column half: C = TAB - Y (Y = (M H2) at that element), Psi, Pi, K2
// (G1_G2_t_step.h:55-86) and the RK4 bookkeeping (RK_solver.h:137-139,
// 209-213).  Gs: the stage's G1, n x n row-major, rows gld apart (shared memory).
struct ApplyEpi {
    long long r;
    StageP st;
    int mu1, mu2, si, sj;
    double U, wij;
    __device__ __forceinline__ ApplyEpi(const Dev &d, const StageP &st_, long long r_) : r(r_), st(st_)
    {
        const int n = d.n, Ns = d.Ns;
        U = st.U;
        const int ri = int(r_);  // a row of M: r < n^2
        mu1 = ri % n;
        mu2 = ri / n;
        si = mu1 % Ns;
        sj = mu2 % Ns;
        wij = U * double(si == sj) + vdist(d, si, sj);
    }
    __device__ __forceinline__ double vdist(const Dev &d, int s1, int s2) const
    {
        const int m = abs(s1 - s2);
        return (m >= 1 && m <= d.nv) ? U * d.law[m - 1] : 0.0;
    }
    // Gs rows are gld apart (n, or n + 1 where consecutive threads read columns)
    __device__ __forceinline__ void element(const Dev &d, int k, int t, int nu1, int nu2, double2 y,
                                            const double2 *Gs, int gld) const
    {
        const int n = d.n, Ns = d.Ns;
        const long long n2 = d.n2, n4 = d.n4;
        const int sk = nu1 % Ns, sl = nu2 % Ns;
        const double2 *Rt1 = d.Rt + ((long long)mu1 * n) * Ns;  // + nu1*Ns + s
        const double2 *Rt2 = d.Rt + ((long long)mu2 * n) * Ns;  // + nu2*Ns + s
        const double2 *Qt = d.Q + t * d.n3;
        const long long x = r * n2 + nu1 + (long long)n * nu2;
        const double2 C = c_sub(d.TAB[t * n4 + x], y);
        const double2 g11 = Gs[mu1 * gld + nu1], g22 = Gs[mu2 * gld + nu2];
        const double wd = wij - (U * double(sk == sl) + vdist(d, sk, sl));
        double2 psi = c_scale(c_mul(g11, g22), wd);
        psi = c_add(psi, c_i(c_mul(g22, c_sub(Rt1[nu1 * Ns + sj], Rt1[nu1 * Ns + sl]))));
        psi = c_add(psi, c_i(c_mul(g11, c_sub(Rt2[nu2 * Ns + si], Rt2[nu2 * Ns + sk]))));
        if (t == 0) {
            psi = c_sub(psi, c_scale(c_mul(g11, g22), U * (double(mu1 == mu2) - double(nu1 == nu2))));
            const double2 e1 = c_sub(c_mul(Gs[mu1 * gld + mu2], Gs[mu2 * gld + nu1]),
                                     c_mul(Gs[mu1 * gld + nu2], Gs[nu2 * gld + nu1]));
            const double2 e2 = c_sub(c_mul(Gs[mu2 * gld + mu1], Gs[mu1 * gld + nu2]),
                                     c_mul(Gs[mu2 * gld + nu1], Gs[nu1 * gld + nu2]));
            psi = c_add(psi, c_scale(c_mi(c_add(c_mul(g22, e1), c_mul(g11, e2))), U));
        }
        const long long q1 = ((long long)mu1 * n + nu1) * n, q2 = ((long long)nu2 * n + mu2) * n;
        const double2 pi = c_mul(g22, c_sub(Qt[q1 + mu2], Qt[q1 + nu2]));
        const double2 piP = c_mul(Gs[nu1 * gld + mu1], c_sub(Qt[q2 + nu1], Qt[q2 + mu1]));
        const double2 K = c_mi(c_sub(c_add(c_add(C, psi), pi), c_conj(piP)));
        if (d.debug) {
            d.TMP0[t * n4 + x] = K;
            return;
        }
        double2 *RKt = d.RK2 + t * n4;
        double2 *Yt = d.Y2 + t * n4;
        double2 *Dt = d.D + t * d.n3;
        const double2 rk = c_add(k == 0 ? make_double2(0.0, 0.0) : RKt[x], c_scale(K, st.w));
        if (k < 3) {
            RKt[x] = rk;
            const double2 tn = c_add(Yt[x], c_scale(K, st.c_next));
            g2_next(d, k)[t * n4 + x] = tn;
            if (mu2 == nu2) Dt[((long long)mu1 * n + nu1) * n + mu2] = tn;
        } else {
            const double2 yn = c_add(Yt[x], c_scale(c_scale(rk, st.dt), 1.0 / 6.0));
            Yt[x] = yn;
            if (mu2 == nu2) Dt[((long long)mu1 * n + nu1) * n + mu2] = yn;
        }
    }
};

template <bool CD>
__device__ __forceinline__ void apply_body(const Dev &d, int k, const ApplyCfg &cfg, int bx, int t)
{
    if (!*d.active) return;
    const int n = d.n, NP = cfg.NP, LD = cfg.LD, S = cfg.S, NB = cfg.NB;
    const long long n2 = d.n2, n4 = d.n4;
    const long long m0 = (long long)bx * NB;
    const int nm = int(min((long long)NB, n2 - m0));
    extern __shared__ double2 sm[];
    double2 *Hs = sm, *HTs = sm + NP * LD, *Xs = sm + 2 * NP * LD;
    double2 *Gs = Xs + (size_t)NB * NP * LD;  // CD only: n*n
    const double2 *X = g2_stage(d, k) + t * n4;

    for (int x = threadIdx.x; x < NP * NP; x += blockDim.x) {
        const int r = x / NP, c = x % NP;
        double2 v = (r < n && c < n) ? d.h[r * n + c] : make_double2(0.0, 0.0);
        Hs[r * LD + c] = v;
        HTs[c * LD + r] = v;
    }
    if (NP != n)
        for (int x = threadIdx.x; x < NB * NP * LD; x += blockDim.x) Xs[x] = make_double2(0.0, 0.0);
    if (CD) {
        const double2 *G1 = g1_stage(d, k);
        for (int x = threadIdx.x; x < n * n; x += blockDim.x) Gs[x] = G1[x];
    }
    __syncthreads();
    if (!CD) {
        // (mu2, mu1, cb) with cb fastest: NB contiguous entries per row of M
        for (long long e = threadIdx.x; e < n2 * NB; e += blockDim.x) {
            const int cb = int(e % NB);
            const long long p = e / NB;  // mu1 + n*mu2
            const int mu1 = int(p % n), mu2 = int(p / n);
            if (cb < nm) Xs[(size_t)cb * NP * LD + mu2 * LD + mu1] = X[p * n2 + m0 + cb];
        }
    } else {
        for (long long e = threadIdx.x; e < (long long)nm * n2; e += blockDim.x) {
            const int rb = int(e / n2);
            const int c = int(e % n2);
            const int nu1 = c % n, nu2 = c / n;
            Xs[(size_t)rb * NP * LD + nu2 * LD + nu1] = X[(m0 + rb) * n2 + c];
        }
    }
    __syncthreads();

    const int mat = threadIdx.x / (S * S), tt = threadIdx.x % (S * S);
    const int ti = tt / S, tj = tt % S;
    const bool live = mat < nm;
    double2 acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = make_double2(0.0, 0.0);
    if (live) {
        const double2 *L = CD ? HTs : Hs;
        const double2 *R = CD ? Hs : HTs;
        const double2 *Xm = Xs + (size_t)mat * NP * LD;
        for (int r = 0; r < n; ++r) {
            double2 l[4], xr[4], xc[4], rr[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                l[q] = L[(ti + S * q) * LD + r];
                xc[q] = Xm[(ti + S * q) * LD + r];
                xr[q] = Xm[r * LD + tj + S * q];
                rr[q] = R[r * LD + tj + S * q];
            }
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    acc[a][b] = c_mac(acc[a][b], l[a], xr[b]);
                    acc[a][b] = c_mac(acc[a][b], xc[a], rr[b]);
                }
        }
    }

    if (!CD) {
        // stage through shared memory so the global stores run along cb
        __syncthreads();
        if (live) {
            double2 *Ym = Xs + (size_t)mat * NP * LD;
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) Ym[(ti + S * a) * LD + tj + S * b] = acc[a][b];
        }
        __syncthreads();
        double2 *T = d.TAB + t * n4;
        for (long long e = threadIdx.x; e < n2 * NB; e += blockDim.x) {
            const int cb = int(e % NB);
            const long long p = e / NB;
            const int mu1 = int(p % n), mu2 = int(p / n);
            if (cb < nm) T[p * n2 + m0 + cb] = Xs[(size_t)cb * NP * LD + mu2 * LD + mu1];
        }
        return;
    }

    // ---- fused epilogue (CD): Y through shared memory, then one element per
    // thread with consecutive threads on consecutive elements (nu1 fastest), so
    // the element's global reads and writes run along rows of M
    __syncthreads();
    if (live) {
        double2 *Ym = Xs + (size_t)mat * NP * LD;
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) Ym[(ti + S * a) * LD + tj + S * b] = acc[a][b];
    }
    __syncthreads();
    const StageP st = d.cur->st[k];
    const int n2i = n * n;
    for (int e = threadIdx.x; e < nm * n2i; e += blockDim.x) {
        const int rb = e / n2i, c = e - rb * n2i;
        const int nu1 = c % n, nu2 = c / n;
        const ApplyEpi ep(d, st, m0 + rb);
        ep.element(d, k, t, nu1, nu2, Xs[(size_t)rb * NP * LD + nu2 * LD + nu1], Gs, n);
    }
}

template <bool CD>
static __global__ void __launch_bounds__(256) k_apply(Dev d, int k, ApplyCfg cfg)
{
    apply_body<CD>(d, k, cfg, blockIdx.x, blockIdx.y);
}

// FP64 tensor-core version of the two halves (n = 16 .. 48): mma.sync
// m8n8k4 f64 (DMMA).  Each warp computes an 8 BI x 8 BJ complex block of
// Y = L X + X R for one matrix (BI x BJ tiles of 8 x 8, real and imaginary
// parts, 4 real products per complex product, accumulated in FP64 like the FMA
// path): kind B = 3 is NP = 24 with 1 x 3 tiles per warp (three warps per
// matrix, for 16 < n <= 24), kind B = 2 is NP = n rounded up to 16 with 2 x 2
// tiles (zero padding either way).  Operands live in shared memory
// as separate real and imaginary planes of NP x LDD doubles, LDD = 12 mod 16,
// so the fragment loads of the row-major A and column-major B operands touch
// each 8-byte bank at most twice per warp.  Results return through the
// X planes; the column half then runs the same per-element epilogue
// (ApplyEpi) as the FMA path, with consecutive threads on consecutive nu1.
struct ApplyTcCfg {
    int NP, LDD, NB, threads, B;
};

// warps per matrix: (NP / 8 BI) x (NP / 8 BJ); kind 3: BI = 1, BJ = 3, kind 2: BI = BJ = 2
__host__ __device__ inline int apply_tc_tpm(const ApplyTcCfg &c)
{
    return c.B == 3 ? (c.NP / 8) * (c.NP / 24) : (c.NP / 16) * (c.NP / 16);
}

inline bool apply_tc_ok(int n) { return n >= 16 && n <= 48; }

// doubles per plane: NP x LDD plus 2, so that the planes of consecutive
// matrices start 4 banks apart (the rows half stages NB matrices with the
// matrix index fastest)
__host__ __device__ inline int apply_tc_plane(int NP, int LDD) { return NP * LDD + 2; }

inline ApplyTcCfg make_apply_tc_cfg(int n, size_t *smem_ab, size_t *smem_cd)
{
    ApplyTcCfg c;
    const bool b3 = n > 16 && n <= 24;
    c.B = b3 ? 3 : 2;
    c.NP = b3 ? 24 : (n + 15) / 16 * 16;
    c.LDD = b3 ? 28 : c.NP + 12;
    const int tpm = apply_tc_tpm(c);
    const size_t plane = size_t(apply_tc_plane(c.NP, c.LDD)) * sizeof(double);
    c.NB = std::max(1, std::min(n * n, (c.B == 3 ? 15 : 8) / tpm));  // 2 matrices per block at n = 32 (6% faster than 4)
    while (c.NB > 1 && (4 + 2 * size_t(c.NB)) * plane + size_t(n) * (n + 1) * sizeof(double2) > 200 * 1024) c.NB--;
    c.threads = c.NB * tpm * 32;
    *smem_ab = (4 + 2 * size_t(c.NB)) * plane;
    *smem_cd = *smem_ab + size_t(n) * (n + 1) * sizeof(double2);
    return c;
}

__device__ __forceinline__ void dmma_f64(double &c0, double &c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

template <bool CD, int BI, int BJ>
__device__ __forceinline__ void apply_tc_body_b(const Dev &d, int k, const ApplyTcCfg &cfg, int bx, int t)
{
    if (!*d.active) return;
    const int n = d.n, NP = cfg.NP, LDD = cfg.LDD, NB = cfg.NB;
    const long long n2 = d.n2, n4 = d.n4;
    const long long m0 = (long long)bx * NB;
    const int nm = int(min((long long)NB, n2 - m0));
    const int PL = apply_tc_plane(NP, LDD);
    extern __shared__ double smtc[];
    double *Lr = smtc, *Li = Lr + PL, *Rr = Li + PL, *Ri = Rr + PL;
    double *Xp = Ri + PL;  // NB x (real, imaginary) planes
    double2 *Gs = reinterpret_cast<double2 *>(Xp + 2 * NB * PL);  // CD only: n x (n + 1)
    const double2 *X = g2_stage(d, k) + t * n4;

    // (L, R) = (h, h^T) for the rows, (h^T, h) for the columns
    for (int x = threadIdx.x; x < NP * NP; x += blockDim.x) {
        const int r = x / NP, c = x % NP;
        const double2 v = (r < n && c < n) ? d.h[r * n + c] : make_double2(0.0, 0.0);
        const int lo = CD ? c * LDD + r : r * LDD + c, ro = CD ? r * LDD + c : c * LDD + r;
        Lr[lo] = v.x;
        Li[lo] = v.y;
        Rr[ro] = v.x;
        Ri[ro] = v.y;
    }
    if (NP != n)
        for (int x = threadIdx.x; x < 2 * NB * PL; x += blockDim.x) Xp[x] = 0.0;
    if (CD) {
        // rows n + 1 apart: the epilogue's threads read G1 along columns too
        const double2 *G1 = g1_stage(d, k);
        for (int x = threadIdx.x; x < n * n; x += blockDim.x) Gs[(x / n) * (n + 1) + x % n] = G1[x];
    }
    __syncthreads();
    if (!CD) {
        // (mu2, mu1, cb) with cb fastest: NB contiguous entries per row of M
        for (long long e = threadIdx.x; e < n2 * NB; e += blockDim.x) {
            const int cb = int(e % NB);
            const long long p = e / NB;  // mu1 + n*mu2
            const int mu1 = int(p % n), mu2 = int(p / n);
            if (cb < nm) {
                const double2 v = X[p * n2 + m0 + cb];
                double *P = Xp + 2 * cb * PL;
                P[mu2 * LDD + mu1] = v.x;
                P[PL + mu2 * LDD + mu1] = v.y;
            }
        }
    } else {
        for (long long e = threadIdx.x; e < (long long)nm * n2; e += blockDim.x) {
            const int rb = int(e / n2), c = int(e % n2);
            const int nu1 = c % n, nu2 = c / n;
            const double2 v = X[(m0 + rb) * n2 + c];
            double *P = Xp + 2 * rb * PL;
            P[nu2 * LDD + nu1] = v.x;
            P[PL + nu2 * LDD + nu1] = v.y;
        }
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const int TWI = NP / (8 * BI), TWJ = NP / (8 * BJ), tpm = TWI * TWJ;
    const int mat = warp / tpm, wt = warp % tpm;
    const int row0 = (wt / TWJ) * 8 * BI, col0 = (wt % TWJ) * 8 * BJ;
    const bool live = mat < nm;
    double yr[BI][BJ][2], yi[BI][BJ][2];
#pragma unroll
    for (int i = 0; i < BI; ++i)
#pragma unroll
        for (int j = 0; j < BJ; ++j)
#pragma unroll
            for (int q = 0; q < 2; ++q) yr[i][j][q] = yi[i][j][q] = 0.0;
    if (live) {
        const double *Xr = Xp + 2 * mat * PL, *Xi = Xr + PL;
        auto step = [&](const double *Ar, const double *Ai, const double *Br, const double *Bi, int k0) {
            double ar[BI], ai[BI], br[BJ], bi[BJ];
#pragma unroll
            for (int i = 0; i < BI; ++i) {
                const int o = (row0 + 8 * i + gid) * LDD + k0 + tig;
                ar[i] = Ar[o];
                ai[i] = Ai[o];
            }
#pragma unroll
            for (int j = 0; j < BJ; ++j) {
                const int o = (k0 + tig) * LDD + col0 + 8 * j + gid;
                br[j] = Br[o];
                bi[j] = Bi[o];
            }
#pragma unroll
            for (int i = 0; i < BI; ++i)
#pragma unroll
                for (int j = 0; j < BJ; ++j) {
                    dmma_f64(yr[i][j][0], yr[i][j][1], ar[i], br[j]);
                    dmma_f64(yr[i][j][0], yr[i][j][1], -ai[i], bi[j]);
                    dmma_f64(yi[i][j][0], yi[i][j][1], ar[i], bi[j]);
                    dmma_f64(yi[i][j][0], yi[i][j][1], ai[i], br[j]);
                }
        };
        // the contraction index runs over n rounded up to 4 (the rest is padding)
        const int KN = (n + 3) & ~3;
        for (int k0 = 0; k0 < KN; k0 += 4) step(Lr, Li, Xr, Xi, k0);  // L X
        for (int k0 = 0; k0 < KN; k0 += 4) step(Xr, Xi, Rr, Ri, k0);  // X R
    }
    __syncthreads();  // every warp has read the X planes
    if (live) {
        double *Yr = Xp + 2 * mat * PL, *Yi = Yr + PL;
#pragma unroll
        for (int i = 0; i < BI; ++i)
#pragma unroll
            for (int j = 0; j < BJ; ++j)
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int o = (row0 + 8 * i + gid) * LDD + col0 + 8 * j + 2 * tig + q;
                    Yr[o] = yr[i][j][q];
                    Yi[o] = yi[i][j][q];
                }
    }
    __syncthreads();
    if (!CD) {
        double2 *T = d.TAB + t * n4;
        for (long long e = threadIdx.x; e < n2 * NB; e += blockDim.x) {
            const int cb = int(e % NB);
            const long long p = e / NB;
            const int mu1 = int(p % n), mu2 = int(p / n);
            if (cb < nm) {
                const double *P = Xp + 2 * cb * PL;
                T[p * n2 + m0 + cb] = make_double2(P[mu2 * LDD + mu1], P[PL + mu2 * LDD + mu1]);
            }
        }
        return;
    }
    const StageP st = d.cur->st[k];
    for (long long e = threadIdx.x; e < (long long)nm * n2; e += blockDim.x) {
        const int rb = int(e / n2), c = int(e % n2);
        const int nu1 = c % n, nu2 = c / n;
        const double *P = Xp + 2 * rb * PL;
        const ApplyEpi ep(d, st, m0 + rb);
        ep.element(d, k, t, nu1, nu2, make_double2(P[nu2 * LDD + nu1], P[PL + nu2 * LDD + nu1]), Gs, n + 1);
    }
}

// the body for the configuration's B (uniform branch; the batch kernel serves
// systems of both kinds)
template <bool CD>
__device__ __forceinline__ void apply_tc_body(const Dev &d, int k, const ApplyTcCfg &cfg, int bx, int t)
{
    if (cfg.B == 3) apply_tc_body_b<CD, 1, 3>(d, k, cfg, bx, t);
    else apply_tc_body_b<CD, 2, 2>(d, k, cfg, bx, t);
}

template <bool CD, int B>
static __global__ void __launch_bounds__(512) k_apply_tc(Dev d, int k, ApplyTcCfg cfg)
{
    apply_tc_body_b<CD, B == 3 ? 1 : 2, B == 3 ? 3 : 2>(d, k, cfg, blockIdx.x, blockIdx.y);
}

// launch of the DMMA half CD with the kernel instance of cfg.B
template <bool CD>
inline void launch_apply_tc(dim3 grid, size_t smem, cudaStream_t s, const Dev &d, int k, const ApplyTcCfg &cfg)
{
    if (cfg.B == 3) k_apply_tc<CD, 3><<<grid, cfg.threads, smem, s>>>(d, k, cfg);
    else k_apply_tc<CD, 2><<<grid, cfg.threads, smem, s>>>(d, k, cfg);
}

template <bool CD>
inline cudaError_t apply_tc_smem_attr(const ApplyTcCfg &cfg, size_t smem)
{
    return cfg.B == 3 ? cudaFuncSetAttribute(k_apply_tc<CD, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))
                      : cudaFuncSetAttribute(k_apply_tc<CD, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
}

// D[t][a][b][r] = Y2_t[a, r; b, r]
static __global__ void k_init_D(Dev d)
{
    const long long total = 2 * d.n3;
    const int n = d.n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int t = int(e / d.n3);
        const long long q = e % d.n3;
        const int r = int(q % n), b = int((q / n) % n), a = int(q / d.n2);
        d.D[e] = d.Y2[t * d.n4 + (long long)b + (long long)n * r + d.n2 * a + d.n2 * n * r];
    }
}

// Total energy of the current state.  The reference computes none; this is
// the energy that the G1-G2 equations conserve while h0 and U are constant:
//   E1 = 2 Tr[h0 rho] + Tr[(h - h0) rho],  rho = -i G1 (one spin projection;
//        h from HF.h:57-104 at U_eff, h0 = h at U = 0),
//   Ec = -Re sum_{p,q} (w_xx(p,q) G2xx[p q; p q] + w_xy(p,q) G2xy[p q; p q])
// with the pair weights of the collision integral (collision_integral.h:41-62):
// on one site w_xy = U and w_xx = U for different bands (0 for p = q); between
// sites m apart w = V_m = U law[m-1].  G2_t[p q; p q] = D[t][(p n + p) n + q].
// One block: out = {E1 + Ec, 2 Tr[h0 rho], Tr[(h - h0) rho], Ec}.
constexpr int kEnergyThreads = 256;
static __global__ void __launch_bounds__(kEnergyThreads) k_energy(Dev d, StageP st, double *out)
{
    __shared__ double2 gd[kMaxN];
    __shared__ double red[3][kEnergyThreads];
    const int n = d.n, Ns = d.Ns;
    const double2 *G = d.Y1;
    for (int p = threadIdx.x; p < n; p += blockDim.x) gd[p] = G[p * (n + 1)];
    __syncthreads();
    StageP st0 = st;
    st0.U = 0.0;
    double e0 = 0.0, eh = 0.0, ec = 0.0;
    for (int x = threadIdx.x; x < n * n; x += blockDim.x) {
        const int mu = x / n, nu = x % n;
        const double2 rho = c_mi(G[nu * n + mu]);  // rho[nu][mu]
        const double2 h = h_entry(d, G, gd, mu, nu, st);
        const double2 h0 = h_entry(d, G, gd, mu, nu, st0);
        e0 += 2.0 * (h0.x * rho.x - h0.y * rho.y);
        eh += (h.x - h0.x) * rho.x - (h.y - h0.y) * rho.y;
        const int i = mu % Ns, a = mu / Ns, j = nu % Ns, b = nu / Ns;
        const int m = abs(i - j);
        double wxx = 0.0, wxy = 0.0;
        if (m == 0) {
            wxy = st.U;
            wxx = (a != b) ? st.U : 0.0;
        } else if (m <= d.nv) {
            wxx = wxy = st.U * d.law[m - 1];
        }
        const long long q = ((long long)mu * n + mu) * n + nu;
        ec -= wxx * d.D[q].x + wxy * d.D[d.n3 + q].x;
    }
    red[0][threadIdx.x] = e0;
    red[1][threadIdx.x] = eh;
    red[2][threadIdx.x] = ec;
    __syncthreads();
    for (int w = kEnergyThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int c = 0; c < 3; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = red[0][0] + red[1][0] + red[2][0];
        out[1] = red[0][0];
        out[2] = red[1][0];
        out[3] = red[2][0];
    }
}

// reference IDX_8D layout <-> device orbital layout
__device__ __forceinline__ long long ref_index(int Ns, int Nb, long long x, int n)
{
    const int nu1 = int(x % n), nu2 = int((x / n) % n), mu1 = int((x / ((long long)n * n)) % n),
              mu2 = int(x / ((long long)n * n * n));
    const long long Ns2 = (long long)Ns * Ns, Nb2 = (long long)Nb * Nb;
    const int k = nu1 % Ns, g = nu1 / Ns, l = nu2 % Ns, dd = nu2 / Ns;
    const int i = mu1 % Ns, a = mu1 / Ns, j = mu2 % Ns, b = mu2 / Ns;
    return (k + (long long)l * Ns) + (g + (long long)dd * Nb) * Ns2 + (i + (long long)j * Ns) * Ns2 * Nb2 +
           (a + (long long)b * Nb) * Ns2 * Ns2 * Nb2;
}

static __global__ void k_from_ref(const double2 *__restrict__ src, double2 *__restrict__ dst, int Ns, int Nb, long long n4)
{
    const int n = Ns * Nb;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < n4; x += (long long)gridDim.x * blockDim.x)
        dst[x] = src[ref_index(Ns, Nb, x, n)];
}

static __global__ void k_to_ref(const double2 *__restrict__ src, double2 *__restrict__ dst, int Ns, int Nb, long long n4)
{
    const int n = Ns * Nb;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < n4; x += (long long)gridDim.x * blockDim.x)
        dst[ref_index(Ns, Nb, x, n)] = src[x];
}

}  // namespace g12
