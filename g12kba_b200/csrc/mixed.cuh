// Mixed-precision engine wiring for engine.cu: buffers, tile tables, TMA
// descriptors and the per-stage launch sequence of the symmetric engine
// (sym_kernels.cuh, sym_tc.cuh).  The G1 side, the Pi/Psi/collision tables,
// the schedule and the snapshot ring are shared with the FP64 engine.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <string>
#include <utility>
#include <vector>

#include "fp64_kernels.cuh"
#include "sym_kernels.cuh"
#include "sym_tc.cuh"
#include "sym_oz.cuh"
#include "sym_epi_p.cuh"

namespace g12 {

struct MixedState {
    int ready = 0;
    int prec = 0;
    bool tc = false;  // tensor-core contraction (else FP32 SIMT)
    int pieces = 2;   // tf32 pieces per operand (2: 3 products, 3: 6 products)
    bool oz = false;  // exact integer-digit bf16 products
    bool dbl = false; // FP64SYM: FP64 stage input and W, FP64 SIMT contraction
    SymDev s{};
    CUtensorMap map_a{}, map_b{};  // TMA views of TMPa / TMPb
    unsigned char *ozb = nullptr;  // h digit tiles (written by k_prep, read by k_sym_gemm_oz2)
    int oz2 = 0;  // bf16 digit GEMM (k_sym_gemm_oz2)
    bool epip = false;       // persistent epilogue k_sym_epi_p (digit GEMM at n = 32)
    double2 *Zt = nullptr;   // its combined Psi/Pi table (written by k_prep)
    int sms = 148;
    size_t epi_smem = 0, simt_smem = 0, tc_smem = 0;
    int tc_grid = 0;
    std::vector<void *> allocs;
};

inline bool mixed_supported(int n, int prec, std::string *why)
{
    if (prec == 1 || prec == 2 || prec == 4) {  // TF32X3, BF16 exact digits, TF32X6
        if (n == 16 || n == 32) return true;
        if (why) *why = "tensor-core mixed precision needs n = Ns*Nb in {16, 32}";
        return false;
    }
    if (prec == 3) {
        if (n == 8 || n == 16 || n == 32 || n == 64) return true;
        if (why) *why = "the FP32 symmetric engine needs n = Ns*Nb in {8, 16, 32, 64}";
        return false;
    }
    if (prec == 5) {
        if (n == 8 || n == 16 || n == 32) return true;
        if (why) *why = "the FP64 symmetric engine needs n = Ns*Nb in {8, 16, 32}";
        return false;
    }
    return false;
}

template <typename T>
inline bool mixed_alloc(MixedState &m, T **p, size_t count)
{
    void *q = nullptr;
    if (cudaMalloc(&q, count * sizeof(T)) != cudaSuccess) return false;
    cudaMemset(q, 0, count * sizeof(T));
    m.allocs.push_back(q);
    *p = static_cast<T *>(q);
    return true;
}

inline bool encode_tmp_map(CUtensorMap *map, float *base, int n, std::string *err)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            if (err) *err = "cuTensorMapEncodeTiled not available";
            return false;
        }
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    // dims (innermost first): (part, rho) 2n floats; c: n^2; mu2: n; tensor: 2
    const cuuint64_t dims[4] = {cuuint64_t(2 * n), cuuint64_t(n) * n, cuuint64_t(n), 2};
    const cuuint64_t strides[3] = {cuuint64_t(2 * n) * 4, cuuint64_t(n) * n * 2 * n * 4,
                                   cuuint64_t(n) * n * n * n * 2 * 4};
    const cuuint32_t box[4] = {32, 1, cuuint32_t(n), 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        if (err) *err = "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")";
        return false;
    }
    return true;
}

// prec: 1 = TF32X3, 4 = TF32X6, 2 = BF16 exact digits (tcgen05), 3 = FP32 SIMT,
// 5 = FP64 SIMT (FP64 stage input and W).
inline int mixed_init(MixedState &m, const Dev &d, int prec, std::string *err)
{
    const int n = d.n;
    if (!mixed_supported(n, prec, err)) return -1;
    m.prec = prec;
    m.tc = (prec == 1 || prec == 2 || prec == 4);
    m.oz = (prec == 2);
    m.dbl = (prec == 5);
    const size_t ts = m.dbl ? 2 : 1;  // floats per stored TMP / W value
    m.pieces = (prec == 4) ? 3 : 2;
    SymDev &s = m.s;
    s.d = d;
    s.n = n;
    s.cpt = 128 / n;
    const long long n2 = (long long)n * n, n3 = n2 * n, n4 = n2 * n2;
    s.n4 = n4;
    s.gemm_tiles = int(n3 / 128);
    s.nblk = int(n2 / kTB);
    s.npairs = s.nblk * (s.nblk + 1) / 2;
    // GEMM tiles: exchange pairs (c, cbar) first, then self-paired diagonal c
    std::vector<int> cs, partner;
    for (int nu2 = 0; nu2 < n; ++nu2)
        for (int nu1 = 0; nu1 < nu2; ++nu1) {
            const int c = nu1 + n * nu2, cb = nu2 + n * nu1;
            const int base = int(cs.size());
            cs.push_back(c);
            cs.push_back(cb);
            partner.push_back(base + 1);
            partner.push_back(base);
        }
    for (int nu = 0; nu < n; ++nu) {
        partner.push_back(int(cs.size()));
        cs.push_back(nu + n * nu);
    }
    std::vector<int> slot_partner(cs.size());
    for (size_t i = 0; i < cs.size(); ++i) slot_partner[i] = partner[i] % s.cpt;
    std::vector<int2> pairs;
    for (int a = 0; a < s.nblk; ++a)
        for (int b = a; b < s.nblk; ++b) pairs.push_back(make_int2(a, b));
    int *gc = nullptr, *gp = nullptr;
    int2 *pp = nullptr;
    bool ok = mixed_alloc(m, &s.TMPa, ts * size_t(2 * 2 * n4)) && mixed_alloc(m, &s.TMPb, ts * size_t(2 * 2 * n4)) &&
              mixed_alloc(m, &s.W, ts * size_t(2 * 2 * n4)) && mixed_alloc(m, &s.Yc, size_t(2) * s.npairs * kTB * kTB) &&
              mixed_alloc(m, &s.Ac, size_t(2) * s.npairs * kTB * kTB) && mixed_alloc(m, &s.Qt, size_t(2 * n3)) &&
              mixed_alloc(m, &s.Rtt, size_t(n2 * d.Ns)) && mixed_alloc(m, &gc, cs.size()) &&
              mixed_alloc(m, &gp, cs.size()) && mixed_alloc(m, &pp, pairs.size()) && mixed_alloc(m, &s.err, 1);
    if (!ok) {
        if (err) *err = "out of device memory (mixed engine)";
        return -3;
    }
    cudaMemcpy(gc, cs.data(), cs.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(gp, slot_partner.data(), cs.size() * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(pp, pairs.data(), pairs.size() * sizeof(int2), cudaMemcpyHostToDevice);
    s.gemm_c = gc;
    s.gemm_partner = gp;
    s.pairs = pp;
    m.epi_smem = size_t(n) * (n + 1) * sizeof(double2) + 2 * kTB * (kTB + 1) * ts * sizeof(float2) +
                 kTB * (kTB + 1) * sizeof(double2);
    m.epi_smem = std::max(m.epi_smem, g1_smem(n2));  // G1-side blocks of k_sym_epi
    m.simt_smem = ts * ((size_t(128) * 2 * n + size_t(128) * (2 * n + 1)) * sizeof(float) + size_t(n2) * sizeof(float2));
    if (m.dbl) {
        cudaFuncSetAttribute(k_sym_epi<8, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(m.epi_smem));
        cudaFuncSetAttribute(k_sym_epi<16, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(m.epi_smem));
        cudaFuncSetAttribute(k_sym_epi<32, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(m.epi_smem));
        cudaFuncSetAttribute(k_sym_gemm_simt<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(m.simt_smem));
    } else {
        cudaFuncSetAttribute(k_sym_epi<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(m.epi_smem));
        cudaFuncSetAttribute(k_sym_epi<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(m.epi_smem));
        cudaFuncSetAttribute(k_sym_epi<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(m.epi_smem));
        cudaFuncSetAttribute(k_sym_epi<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(m.epi_smem));
        cudaFuncSetAttribute(k_sym_gemm_simt<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(m.simt_smem));
    }
    if (m.tc) {
        if (!encode_tmp_map(&m.map_a, s.TMPa, n, err) || !encode_tmp_map(&m.map_b, s.TMPb, n, err)) return -2;
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
        m.oz2 = m.oz;
        if (m.oz2 && n == 32) {
            m.tc_smem = Oz2Shape<32>::SMEM;
            cudaFuncSetAttribute(k_sym_gemm_oz2<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(m.tc_smem));
        } else if (m.oz2) {
            m.tc_smem = Oz2Shape<16>::SMEM;
            cudaFuncSetAttribute(k_sym_gemm_oz2<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(m.tc_smem));
        } else if (n == 32 && m.pieces == 2) {
            m.tc_smem = TcShape<32, 2>::SMEM;
            cudaFuncSetAttribute(k_sym_gemm_tc<32, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(m.tc_smem));
        } else if (n == 32) {
            m.tc_smem = TcShape<32, 3>::SMEM;
            cudaFuncSetAttribute(k_sym_gemm_tc<32, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(m.tc_smem));
        } else if (m.pieces == 2) {
            m.tc_smem = TcShape<16, 2>::SMEM;
            cudaFuncSetAttribute(k_sym_gemm_tc<16, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(m.tc_smem));
        } else {
            m.tc_smem = TcShape<16, 3>::SMEM;
            cudaFuncSetAttribute(k_sym_gemm_tc<16, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(m.tc_smem));
        }
        if (m.oz2 && !mixed_alloc(m, &m.ozb, size_t(kOz2Digits) * Oz2Shape<32>::B_BYTES + 4 * 64)) {
            if (err) *err = "out of device memory (mixed engine)";
            return -3;
        }
        m.tc_grid = m.oz2 ? std::min(2 * s.gemm_tiles, sms) : std::min(2 * s.gemm_tiles, 2 * sms);  // oz2: persistent
        m.sms = sms;
        if (m.oz2 && n == 32) {
            if (!mixed_alloc(m, &m.Zt, size_t(2 * n3))) {
                if (err) *err = "out of device memory (mixed engine)";
                return -3;
            }
            cudaFuncSetAttribute(k_sym_epi_p, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kEpiPSmem));
            m.epip = true;
        }
    }
    if (cudaGetLastError() != cudaSuccess) {
        if (err) *err = "mixed engine set-up failed";
        return -2;
    }
    m.ready = 1;
    return 0;
}

inline void mixed_free(MixedState &m)
{
    for (void *p : m.allocs) cudaFree(p);
    m.allocs.clear();
    m.ready = 0;
}

// the full FP64 state in d.Y2 (device orbital layout) -> compressed state
inline int mixed_on_state(MixedState &m, const Dev &d, cudaStream_t st)
{
    m.s.d = d;
    if (m.dbl) k_sym_pack<double><<<dim3(m.s.npairs, 2), 256, 0, st>>>(m.s, d.Y2);
    else k_sym_pack<float><<<dim3(m.s.npairs, 2), 256, 0, st>>>(m.s, d.Y2);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// compressed state -> full FP64 state in d.Y2
inline int mixed_to_full(MixedState &m, const Dev &d, cudaStream_t st)
{
    m.s.d = d;
    k_sym_unpack<<<dim3(m.s.npairs, 2), 256, 0, st>>>(m.s, d.Y2);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

inline int mixed_kernel_kinds(const MixedState &) { return 2; }

inline const char *mixed_kernel_name(const MixedState &m, int q)
{
    if (q == 0) return m.oz2 ? "k_sym_gemm_oz2" : (m.tc ? "k_sym_gemm_tc" : (m.dbl ? "k_sym_gemm_simt<f64>" : "k_sym_gemm_simt"));
    if (q == 1) return "k_sym_epi";
    return "";
}

// launch with programmatic stream serialisation: the kernel may start while its
// predecessor finishes and waits for it inside (griddepcontrol.wait)
template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

// whether k_sym_epi runs the stage's G1 side itself (the digit-GEMM path)
inline bool mixed_fuses_g1(const MixedState &m) { return m.tc && m.oz2; }

// q = 0: the W contraction, q = 1: the stage epilogue; fuse_g1 (digit-GEMM
// path only) adds the G1-side blocks to the epilogue launch
inline void mixed_enqueue_kind(MixedState &m, const Dev &d, int k, int, int q, cudaStream_t st, bool fuse_g1 = false)
{
    m.s.d = d;
    m.s.g1x = 0;
    const SymDev &s = m.s;
    if (q == 0) {
        if (m.tc) {
            const CUtensorMap &map = (k & 1) ? m.map_a : m.map_b;
            if (m.oz2 && s.n == 32)
                launch_pdl(k_sym_gemm_oz2<32>, dim3(m.tc_grid), dim3(Oz2Shape<32>::THREADS), m.tc_smem, st, s, k, map);
            else if (m.oz2)
                launch_pdl(k_sym_gemm_oz2<16>, dim3(m.tc_grid), dim3(Oz2Shape<16>::THREADS), m.tc_smem, st, s, k, map);
            else if (s.n == 32 && m.pieces == 2) k_sym_gemm_tc<32, 2><<<m.tc_grid, 128, m.tc_smem, st>>>(s, k, map);
            else if (s.n == 32) k_sym_gemm_tc<32, 3><<<m.tc_grid, 128, m.tc_smem, st>>>(s, k, map);
            else if (m.pieces == 2) k_sym_gemm_tc<16, 2><<<m.tc_grid, 128, m.tc_smem, st>>>(s, k, map);
            else k_sym_gemm_tc<16, 3><<<m.tc_grid, 128, m.tc_smem, st>>>(s, k, map);
        } else if (m.dbl) {
            k_sym_gemm_simt<double><<<2 * s.gemm_tiles, 256, m.simt_smem, st>>>(s, k);
        } else {
            k_sym_gemm_simt<float><<<2 * s.gemm_tiles, 256, m.simt_smem, st>>>(s, k);
        }
    } else {
        const dim3 g(s.npairs, 2);
        if (m.oz2 && m.tc && m.epip && !d.debug && d.Zt) {
            // persistent epilogue: one CTA per SM (pair CTAs, then the G1-side CTAs)
            SymDev sf = s;
            sf.g1x = fuse_g1 ? int((s.d.n2 + kEpiPThreads - 1) / kEpiPThreads) : 0;
            const int units = 2 * s.npairs;
            int G = std::max(m.sms - sf.g1x, (units + kEpiPMaxUnits - 1) / kEpiPMaxUnits);
            G = std::min(G, units);
            launch_pdl(k_sym_epi_p, dim3(G + sf.g1x), dim3(kEpiPThreads), kEpiPSmem, st, sf, k);
            return;
        }
        if (m.oz2 && m.tc) {
            SymDev sf = s;
            sf.g1x = fuse_g1 ? int((s.d.n2 + 255) / 256) : 0;
            const dim3 gf(s.npairs + sf.g1x, 2);
            if (s.n == 32) launch_pdl(k_sym_epi<32>, gf, dim3(256), m.epi_smem, st, sf, k);
            else launch_pdl(k_sym_epi<16>, gf, dim3(256), m.epi_smem, st, sf, k);
            return;
        }
        if (m.dbl) {
            if (s.n == 32) k_sym_epi<32, double><<<g, 256, m.epi_smem, st>>>(s, k);
            else if (s.n == 16) k_sym_epi<16, double><<<g, 256, m.epi_smem, st>>>(s, k);
            else k_sym_epi<8, double><<<g, 256, m.epi_smem, st>>>(s, k);
            return;
        }
        if (s.n == 32 && m.oz2) launch_pdl(k_sym_epi<32>, g, dim3(256), m.epi_smem, st, s, k);
        else if (s.n == 16 && m.oz2) launch_pdl(k_sym_epi<16>, g, dim3(256), m.epi_smem, st, s, k);
        else if (s.n == 32) k_sym_epi<32><<<g, 256, m.epi_smem, st>>>(s, k);
        else if (s.n == 16) k_sym_epi<16><<<g, 256, m.epi_smem, st>>>(s, k);
        else if (s.n == 8) k_sym_epi<8><<<g, 256, m.epi_smem, st>>>(s, k);
        else k_sym_epi<64><<<g, 256, m.epi_smem, st>>>(s, k);
    }
}

inline void mixed_enqueue_stage(MixedState &m, const Dev &d, int k, int prec, cudaStream_t st)
{
    for (int q = 0; q < 2; ++q) mixed_enqueue_kind(m, d, k, prec, q, st);
}

inline int mixed_launches_per_stage(const MixedState &) { return 2; }

// device error word of the bounded waits (0: none)
inline int mixed_error(MixedState &m)
{
    int e = 0;
    if (m.s.err) cudaMemcpy(&e, m.s.err, sizeof(int), cudaMemcpyDeviceToHost);
    return e;
}

}  // namespace g12
