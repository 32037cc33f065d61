// Host side of the tensor-core path: weight tables, tensor maps and launches
// of the persistent kernels in tensor_kernels.cuh for one plan's products.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/polymul.h"
#include "pm_device.cuh"
#include "pm_internal.h"
#include "tc_ptx.cuh"
#include "tensor_kernels.cuh"
#include "convert_tile.cuh"
#include "crt_quartic.cuh"

namespace pm {



// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {
// Conversion weights for all kPMax primes: 4 groups of 64 rows x 128 bytes,
// each group's image already in the swizzled shared-memory layout.
std::vector<uint8_t> conversion_image(const std::vector<uint32_t>& primes) {
    const int groups = (kPMax + tc::kConvGroup - 1) / tc::kConvGroup;
    std::vector<uint8_t> img(size_t(groups) * 8192, 0);
    for (size_t i = 0; i < primes.size(); ++i) {
        const uint32_t p = primes[i];
        const int g = int(i) / tc::kConvGroup, jrow = int(i % tc::kConvGroup) * 4;
        uint32_t w = 1;  // 2^(8k) mod p
        for (int k = 0; k < 128; ++k) {
            for (int a = 0; a < 4; ++a)
                img[size_t(g) * 8192 + tc::sw128_offset(jrow + a, k)] = uint8_t(w >> (8 * a));
            w = uint32_t(uint64_t(w) * 256 % p);
        }
    }
    return img;
}
}  // namespace

void tensor_init(PlanCore& s) {
    if (uint32_t(s.P) * 4 > uint32_t(tc::kCrtK)) throw Failure(PM_ERR_UNSUPPORTED, "prime basis too large for the CRT tile");
    if (4 * s.W + 16 > uint32_t(tc::kCrtN)) throw Failure(PM_ERR_UNSUPPORTED, "q too wide for the CRT tile");
    if (s.stride % 4) throw Failure(PM_ERR_UNSUPPORTED, "tensor path needs an even coef_limbs (16-byte coefficient rows)");
    DeviceBasis& B = *s.basis;
    {
        static std::mutex m;
        std::lock_guard<std::mutex> lock(m);
        if (!B.d_conv_weights) {
            const auto img = conversion_image(B.primes);
            cuda_check(cudaMalloc(&B.d_conv_weights, img.size()), "allocate conversion weights");
            cuda_check(cudaMemcpy(B.d_conv_weights, img.data(), img.size(), cudaMemcpyHostToDevice),
                       "upload conversion weights");
        }
    }
    // CRT weights: [2 K-atoms][128 rows][128 B].  Row (i, a) holds the bytes of
    // w_ia = ((P/p_i) mod q) 2^(8a) mod q: digit byte a of t_i times it sums, over a, to
    // t_i (P/p_i) mod q, and the contraction V = sum byte_a(t_i) w_ia stays below 4P 255 q.
    // Columns: 4W value bytes, then 8 bytes of floor(2^64 / p_i) 2^(8a) (the nearest
    // quotient k of sum t_i / p_i), then 8 bytes of floor(2^64 w_ia / q) (V / q to 2^-40).
    const uint32_t NV = 4 * s.W;
    Words total{1};
    for (unsigned i = 0; i < s.P; ++i) total = multiply_small(total, B.primes[i]);
    std::vector<uint8_t> img(32768, 0);
    for (unsigned i = 0; i < s.P; ++i) {
        Words m = total;
        divide_small(m, B.primes[i]);
        const Words mq = mod(m, s.q);
        const uint64_t recip = uint64_t(((unsigned __int128)1 << 64) / B.primes[i]);
        for (int a = 0; a < 4; ++a) {
            const Words w = mod(shift_left(mq, 8 * a), s.q);
            Words f;
            divmod(shift_left(w, 64), s.q, &f, nullptr);
            const Words f64 = padded(f, 2);
            const unsigned __int128 rs = (unsigned __int128)recip << (8 * a);
            const uint32_t k = 4 * i + a, ka = k >> 7, kk = k & 127;
            for (uint32_t J = 0; J < NV; ++J) {
                const uint32_t word = J / 4 < w.size() ? w[J / 4] : 0;
                img[ka * 16384 + tc::sw128_offset(J, kk)] = uint8_t(word >> (8 * (J % 4)));
            }
            for (uint32_t J = 0; J < 8; ++J) {
                img[ka * 16384 + tc::sw128_offset(NV + J, kk)] = uint8_t(rs >> (8 * J));
                img[ka * 16384 + tc::sw128_offset(NV + 8 + J, kk)] = uint8_t(f64[J / 4] >> (8 * (J % 4)));
            }
        }
    }
    cuda_check(cudaMalloc(&s.d_crt_weights, img.size()), "allocate CRT weights");
    cuda_check(cudaMemcpy(s.d_crt_weights, img.data(), img.size(), cudaMemcpyHostToDevice), "upload CRT weights");
    // floor(2^64 (row k of the k table) / q), which joins the estimate of V / q
    const Words pmod = mod(total, s.q);
    const Words pneg = compare(pmod, Words{}) == 0 ? Words{} : subtract(s.q, pmod);
    std::vector<uint64_t> kfrac(2 * size_t(s.P) + 1, 0);
    for (unsigned k = 1; k <= 2 * s.P; ++k) {
        Words f;
        divmod(shift_left(mod(multiply_small(pneg, k), s.q), 64), s.q, &f, nullptr);
        const Words f64 = padded(f, 2);
        kfrac[k] = uint64_t(f64[0]) | (uint64_t(f64[1]) << 32);
    }
    cuda_check(cudaMalloc(&s.d_kfrac, kfrac.size() * 8), "allocate CRT fractions");
    cuda_check(cudaMemcpy(s.d_kfrac, kfrac.data(), kfrac.size() * 8, cudaMemcpyHostToDevice), "upload CRT fractions");
}

void tensor_release(PlanCore& s) {
    cudaFree(s.d_crt_weights);
    s.d_crt_weights = nullptr;
    cudaFree(s.d_kfrac);
    s.d_kfrac = nullptr;
}

namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        cuda_check(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q),
                   "look up cuTensorMapEncodeTiled");
        if (!p || q != cudaDriverEntryPointSuccess) throw Failure(PM_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 4-D map with packed (nested) strides; dims[0] contiguous.
CUtensorMap make_map(CUtensorMapDataType type, const void* base, const cuuint64_t dims[4],
                     const cuuint64_t strides_bytes[3], const cuuint32_t box[4], CUtensorMapSwizzle swizzle) {
    CUtensorMap map;
    const cuuint32_t estride[4] = {1, 1, 1, 1};
    const CUresult r = encode_fn()(&map, type, 4, const_cast<void*>(base), dims, strides_bytes, box, estride,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Failure(PM_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
    return map;
}

// coefficient bytes of `count` products: dims (byte, column, row, product)
CUtensorMap coefficient_map(const PlanCore& s, const void* base, uint32_t count) {
    const uint32_t C = 1u << s.logC, R = 1u << s.logR, Gc = C < 8 ? C : 8;
    const cuuint64_t sb = s.stride * 4ull;
    const cuuint64_t dims[4] = {sb, C, R, count};
    const cuuint64_t strides[3] = {sb, sb * C, sb * C * R};
    const cuuint32_t box[4] = {128, Gc, R, 1};
    return make_map(CU_TENSOR_MAP_DATA_TYPE_UINT8, base, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_128B);
}

// the product planes (plane 0..P-1) of `count` workspaces: dims (column, prime, row, product),
// so a box lands in shared memory as [row][prime][column]
// Residue planes as (column, prime, row, product); a box of box_primes primes lands as
// [row][box_primes][column] (primes past P read as zero).
CUtensorMap residue_map(const PlanCore& s, const void* work, uint32_t count, uint32_t box_primes) {
    const uint32_t C = 1u << s.logC, R = 1u << s.logR, Gc = C < 8 ? C : 8;
    const cuuint64_t dims[4] = {C, s.P, R, count};
    const cuuint64_t strides[3] = {C * R * 4ull, C * 4ull, s.workspace_bytes};
    const cuuint32_t box[4] = {Gc, box_primes, R, 1};
    return make_map(CU_TENSOR_MAP_DATA_TYPE_UINT32, work, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_NONE);
}

template <int LOGR>
void launch_k1t(const PlanCore& s, const uint32_t* a, const uint32_t* b, uint32_t* work, uint32_t count,
                cudaStream_t st) {
    const int C = 1 << s.logC, Gc = C < 8 ? C : 8;
    const int pgs = int((s.P + tc::kConvGroup - 1) / tc::kConvGroup);
    const int items = pgs * int(count) * 2 * (C / Gc);
    int ctas = s.sms * s.tune.conv_ctas_per_sm;
    if (ctas > items) ctas = items;
    if (ctas >= pgs) ctas -= ctas % pgs;  // equal numbers of CTAs per prime group (PlanConvWork::range)
    if (ctas < 1) ctas = 1;
    const size_t smem = k1t_smem_bytes();
    cuda_check(cudaFuncSetAttribute(k1t_convert<LOGR, PlanConvWork>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(smem)),
               "K1T shared memory");
    PlanConvWork w;
    w.map_a = coefficient_map(s, a, count);
    w.map_b = coefficient_map(s, b, count);
    w.work = work;
    w.ws_bstride = s.workspace_bytes / 4;
    w.n = int(s.n);
    w.logC = int(s.logC);
    w.P = int(s.P);
    w.count = int(count);
    w.pgs = pgs;
    k1t_convert<LOGR, PlanConvWork><<<ctas, tc::kConvThreads, smem, st>>>(w, s.plane_pc(), s.conv_weights(),
                                                                           s.plane_fwd(), s.d_err);
}

// the whole basis per tile: two CTAs per SM, contiguous runs of items
template <int LOGR>
void launch_k1w(const PlanCore& s, const uint32_t* a, const uint32_t* b, uint32_t* work, uint32_t count,
                cudaStream_t st, int poly_only = -1) {
    const int C = 1 << s.logC, Gc = C < 8 ? C : 8;
    const int items = int(count) * (poly_only < 0 ? 2 : 1) * (C / Gc);
    int ctas = s.sms * 2;
    if (ctas > items) ctas = items;
    const size_t smem = k1w_smem_bytes();
    // rows of 1024, 2048 or 4096 values (n = 16384 .. 65536): a kernel with that row length built in
    auto kernel = k1w_convert<LOGR, PlanTileWork>;
    if (LOGR == 4 && s.logC == 10) kernel = k1w_convert<LOGR, PlanTileWork, 10>;
    if (LOGR == 4 && s.logC == 11) kernel = k1w_convert<LOGR, PlanTileWork, 11>;
    if (LOGR == 4 && s.logC == 12) kernel = k1w_convert<LOGR, PlanTileWork, 12>;
    cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
               "K1W shared memory");
    PlanTileWork w;
    w.poly_only = poly_only;
    w.map_a = coefficient_map(s, poly_only == 1 ? b : a, count);
    w.map_b = poly_only == 0 ? w.map_a : coefficient_map(s, b, count);
    w.work = work;
    w.ws_bstride = s.workspace_bytes / 4;
    w.n = int(s.n);
    w.logC = int(s.logC);
    w.P = int(s.P);
    w.count = int(count);
    ByteFix fix{};
    if (s.quartic) {
        fix.count = s.quartic->fix_count;
        for (int t = 0; t < 3; ++t) {
            fix.byte[t] = s.quartic->fix_byte[t];
            fix.shift[t] = s.quartic->fix_shift[t];
        }
    }
    kernel<<<ctas, tc::kWideThreads, smem, st>>>(w, s.plane_pc(), s.conv_weights(), s.plane_fwd(), s.d_err, fix);
}

template <int LOGR>
void launch_conversion(const PlanCore& s, const uint32_t* a, const uint32_t* b, uint32_t* work, uint32_t count,
                       cudaStream_t st) {
    if (s.tune.conv_whole_basis)
        launch_k1w<LOGR>(s, a, b, work, count, st);
    else
        launch_k1t<LOGR>(s, a, b, work, count, st);
}

template <int LOGR, int W>
void launch_k3t(const PlanCore& s, const uint32_t* work, uint32_t* c, uint32_t count, cudaStream_t st) {
    const int C = 1 << s.logC, Gc = C < 8 ? C : 8;
    const int items = int(count) * (C / Gc);
    int ctas = s.sms * s.tune.crt_ctas_per_sm;
    if (ctas > items) ctas = items;
    const size_t smem = k3t_smem_bytes<LOGR>();
    // the reduction mod q is a table row: the same kernel for a special-form q; rows of 1024,
    // 2048 or 4096 values (n = 16384 .. 65536) take a kernel with that row length built in
    auto kernel = k3t_crt<LOGR, W, PlanCrtWork>;
    if (LOGR == 4 && s.logC == 10) kernel = k3t_crt<LOGR, W, PlanCrtWork, 10>;
    if (LOGR == 4 && s.logC == 11) kernel = k3t_crt<LOGR, W, PlanCrtWork, 11>;
    if (LOGR == 4 && s.logC == 12) kernel = k3t_crt<LOGR, W, PlanCrtWork, 12>;
    cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
               "K3T shared memory");
    PlanCrtWork w;
    std::memset(&w.map_res, 0, sizeof w.map_res);
    w.use_tma = (C * 4) % 16 == 0;  // rows of fewer than 4 columns cannot be described by a tensor map
    if (w.use_tma) w.map_res = residue_map(s, work, count, tc::kMaxPrimes);  // a constant row stride in the box
    w.work = work;
    w.out = c;
    w.ws_bstride = s.workspace_bytes / 4;
    w.io_bstride = size_t(s.n) * s.stride;
    w.scale = s.d_scale;
    w.consts = s.d_consts;
    w.ktab = s.d_ktab;
    w.crt_w = s.d_crt_weights;
    w.kfrac = s.d_kfrac;
    w.mu_q = s.mu_q;
    w.sbits = int(s.qbits);
    w.delta = s.delta;
    w.n = int(s.n);
    w.logC = int(s.logC);
    w.P = int(s.P);
    w.stride = int(s.stride);
    w.count = int(count);
    kernel<<<ctas, tc::kCrtThreads, smem, st>>>(w, s.plane_pc(), s.plane_inv(), s.d_err);
}

template <int LOGR>
void launch_k3t_w(const PlanCore& s, const uint32_t* work, uint32_t* c, uint32_t count, cudaStream_t st) {
    switch (s.W) {
        case 4: return launch_k3t<LOGR, 4>(s, work, c, count, st);
        case 8: return launch_k3t<LOGR, 8>(s, work, c, count, st);
        case 12: return launch_k3t<LOGR, 12>(s, work, c, count, st);
        case 16: return launch_k3t<LOGR, 16>(s, work, c, count, st);
        case 20: return launch_k3t<LOGR, 20>(s, work, c, count, st);
        case 24: return launch_k3t<LOGR, 24>(s, work, c, count, st);
        case 28: return launch_k3t<LOGR, 28>(s, work, c, count, st);
        default: throw Failure(PM_ERR_UNSUPPORTED, "unsupported width");
    }
}
}  // namespace

namespace {
template <int LOGR, int W>
void launch_k3q(const PlanCore& s, const uint32_t* work, uint32_t* c, uint32_t count, cudaStream_t st) {
    const QuarticTables& Q = *s.quartic;
    const int C = 1 << s.logC, Gc = C < 8 ? C : 8;
    if ((C * 4) % 16) throw Failure(PM_ERR_UNSUPPORTED, "quartic plans need n >= 64");
    const int items = int(count) * (C / Gc);
    int ctas = s.sms * 2;
    if (ctas > items) ctas = items;
    const size_t smem = k3q_smem_bytes<LOGR>();
    auto kernel = s.delta ? k3q_crt<LOGR, W, kReduceSpecial> : k3q_crt<LOGR, W, kReduceGeneral>;
    cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
               "K3Q shared memory");
    QuarticCrtWork w;
    w.map_res = residue_map(s, work, count, s.P);
    w.out = c;
    w.io_bstride = size_t(s.n) * s.stride;
    w.consts = s.d_consts;
    w.ktab = Q.d_ktab;
    w.crt_w = Q.d_crt;
    w.mix = Q.d_mix;
    w.mu_q = s.mu_q;
    w.sbits = int(s.qbits);
    w.delta = s.delta;
    w.n = int(s.n);
    w.logC = int(s.logC);
    w.stride = int(s.stride);
    w.count = int(count);
    kernel<<<ctas, tc::kCrtThreads, smem, st>>>(w, s.plane_pc(), s.plane_inv(), s.d_err);
}
}  // namespace

// The quartic factorization: K1W with the plan's channel-evaluating weights, the row
// kernel over its 64 planes, and K3Q.
void launch_quartic(const PlanCore& s, const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* work,
                    uint32_t count, cudaStream_t st) {
    {
        ProfileScope prof("k1t_convert_cols", st);
        switch (s.logR) {
            case 4: launch_k1w<4>(s, a, b, work, count, st); break;
            case 3: launch_k1w<3>(s, a, b, work, count, st); break;
            case 2: launch_k1w<2>(s, a, b, work, count, st); break;
            default: throw Failure(PM_ERR_UNSUPPORTED, "quartic plans need n >= 64");
        }
    }
    {
        ProfileScope prof("k2_rows", st);
        launch_rows(s, work, count, st);
    }
    {
        ProfileScope prof("k3t_cols_crt", st);
        if (s.W != 28) throw Failure(PM_ERR_UNSUPPORTED, "quartic plans take q of 865..896 bits");
        switch (s.logR) {
            case 4: launch_k3q<4, 28>(s, work, c, count, st); break;
            case 3: launch_k3q<3, 28>(s, work, c, count, st); break;
            default: launch_k3q<2, 28>(s, work, c, count, st); break;
        }
    }
    cuda_check(cudaGetLastError(), "launch quartic product kernels");
    count_launches(3);
}

bool conversion_splits(const PlanCore& s) {
    return (s.flags & PM_CONVERT_TENSOR) && !s.quartic && !s.wide && s.tune.conv_whole_basis;
}

void launch_tensor_convert_poly(const PlanCore& s, const uint32_t* x, int poly, uint32_t* work, cudaStream_t st) {
    if (!conversion_splits(s)) throw Failure(PM_ERR_INVALID, "this plan converts both polynomials in one launch");
    ProfileScope prof("k1t_convert_cols", st);
    const uint32_t* a = poly == 0 ? x : nullptr;
    const uint32_t* b = poly == 1 ? x : nullptr;
    switch (s.logR) {
        case 0: launch_k1w<0>(s, a, b, work, 1, st, poly); break;
        case 1: launch_k1w<1>(s, a, b, work, 1, st, poly); break;
        case 2: launch_k1w<2>(s, a, b, work, 1, st, poly); break;
        case 3: launch_k1w<3>(s, a, b, work, 1, st, poly); break;
        default: launch_k1w<4>(s, a, b, work, 1, st, poly); break;
    }
    cuda_check(cudaGetLastError(), "launch conversion");
    count_launches(1);
}

void launch_tensor_after_conversion(const PlanCore& s, uint32_t* c, uint32_t* work, uint32_t count,
                                    cudaStream_t st) {
    {
        ProfileScope prof("k2_rows", st);
        launch_rows(s, work, count, st);
    }
    {
        ProfileScope prof("k3t_cols_crt", st);
        switch (s.logR) {
            case 0: launch_k3t_w<0>(s, work, c, count, st); break;
            case 1: launch_k3t_w<1>(s, work, c, count, st); break;
            case 2: launch_k3t_w<2>(s, work, c, count, st); break;
            case 3: launch_k3t_w<3>(s, work, c, count, st); break;
            default: launch_k3t_w<4>(s, work, c, count, st); break;
        }
    }
    cuda_check(cudaGetLastError(), "launch tensor product kernels");
    count_launches(2);
}

void launch_tensor(const PlanCore& s, const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* work,
                   uint32_t count, cudaStream_t st) {
    {
        ProfileScope prof("k1t_convert_cols", st);
        switch (s.logR) {
            case 0: launch_conversion<0>(s, a, b, work, count, st); break;
            case 1: launch_conversion<1>(s, a, b, work, count, st); break;
            case 2: launch_conversion<2>(s, a, b, work, count, st); break;
            case 3: launch_conversion<3>(s, a, b, work, count, st); break;
            default: launch_conversion<4>(s, a, b, work, count, st); break;
        }
    }
    {
        ProfileScope prof("k2_rows", st);
        launch_rows(s, work, count, st);
    }
    {
        ProfileScope prof("k3t_cols_crt", st);
        switch (s.logR) {
            case 0: launch_k3t_w<0>(s, work, c, count, st); break;
            case 1: launch_k3t_w<1>(s, work, c, count, st); break;
            case 2: launch_k3t_w<2>(s, work, c, count, st); break;
            case 3: launch_k3t_w<3>(s, work, c, count, st); break;
            default: launch_k3t_w<4>(s, work, c, count, st); break;
        }
    }
    cuda_check(cudaGetLastError(), "launch tensor product kernels");
    count_launches(3);
}

}  // namespace pm
