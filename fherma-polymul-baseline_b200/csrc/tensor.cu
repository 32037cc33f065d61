// Exact residue conversion and CRT reconstruction as INT8 contractions on the
// fifth-generation tensor cores (tcgen05.mma kind::i8, u8 x u8 -> s32 in TMEM).
//
// Conversion (reference: rns/tensor_prepare.h:20-101 does the same contraction
// with WMMA s8 or cuBLAS, centred by -128; unsigned operands need no centring):
//   D[m][4i+a] = sum_k x_k(m) * byte_a(2^(8k) mod p_i)      k < 128 coefficient bytes
//   r_i(m)     = sum_a D[m][4i+a] * 2^(8a)  mod p_i           (< 2^48 before the reduction)
// every D entry is at most 128*255^2 < 2^23, so the s32 accumulation is exact.
//
// CRT (the reference accumulates sum t_i (P/p_i mod q) in a 928-bit cuPQC
// integer, rns/solve.cu:336-420):
//   A[m][4i+a] = byte_a(t_i(m)),  B[J][4i+a] = byte_J((P/p_i mod q) << 8a)  J < NV
//                                 B[NV+J][4i+a] = byte_J(floor(2^64/p_i) << 8a)  J < 8
//   sum_J D[m][J] 2^(8J) = sum_i t_i (P/p_i mod q),  sum_J D[m][NV+J] 2^(8J) = sum_i t_i floor(2^64/p_i)
// every D entry is at most 256*255^2 < 2^24.
//
// Both kernels also run the NTT stages whose butterflies span the 16 rows of
// the 16 x C view of a plane (forward in K1T, inverse in K3T), in registers
// after a shared-memory transpose.  Operands are staged by the threads into
// the canonical K-major 128-byte-swizzled layout; one thread issues the MMAs;
// completion is signalled through an mbarrier with a bounded wait.
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

namespace pm {

namespace tc {
constexpr int kTileM = 128;          // coefficients per tile = 8 columns x 16 rows
constexpr int kConvGroup = 16;       // primes per conversion MMA (N = 64)
constexpr int kConvN = 4 * kConvGroup;
constexpr int kCrtN = 128;           // value bytes + 8 quotient bytes (+ pad)
constexpr int kCrtK = 256;           // 4 bytes per prime, 64 primes
constexpr uint64_t kWaitNs = 1000000000ull;  // bounded mbarrier wait: 1 s

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Bounded wait on an mbarrier phase; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint64_t start = global_ns();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        if (global_ns() - start > kWaitNs) return false;
    }
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// make this thread's generic-proxy shared-memory writes visible to the tensor core
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// K-major operand in the 128-byte swizzle: rows of 128 bytes, 8-row groups
// 1024 bytes apart, 16-byte chunk c of row m stored at chunk c ^ (m % 8).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = uint64_t((saddr >> 4) & 0x3FFF);
    d |= uint64_t(1) << 16;            // leading byte offset (unused by this layout) = 16 B
    d |= uint64_t(1024 >> 4) << 32;    // stride byte offset between 8-row groups
    d |= uint64_t(1) << 46;            // descriptor version for tcgen05
    d |= uint64_t(2) << 61;            // SWIZZLE_128B
    return d;
}

__host__ __device__ constexpr uint32_t idesc_u8(int M, int N) {
    return (2u << 4)                      // D in s32
           | (0u << 7) | (0u << 10)       // A and B unsigned 8-bit, both K-major
           | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mma_u8(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// 4-D tiled TMA load into shared memory, completion counted on `bar` (no multicast)
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

// byte offset of (row m, byte k < 128) inside one 128-byte-swizzled atom column
__host__ __device__ __forceinline__ uint32_t sw128_offset(uint32_t m, uint32_t k) {
    return (m >> 3) * 1024 + (m & 7) * 128 + ((((k >> 4) ^ (m & 7)) & 7) << 4) + (k & 15);
}

}  // namespace tc

// ---------------------------------------------------------------------------
// K1T: tensor-core conversion + forward column stages.
// grid (ctas, prime groups); block 128.  CTA (x, pg) converts the tiles
// x, x + ctas, ... for the 16 primes of group pg.  Tile index -> (product z,
// polynomial, column group cg); the tile holds coefficient r*C + Gc*cg + c in
// row m = r*Gc + c.  A tiles arrive by TMA (box: 128 bytes x Gc columns x R
// rows, 128-byte swizzle, bytes past the coefficient width zero-filled),
// double-buffered so the next tile loads while this one is converted.
// Dynamic shared memory (1024-aligned): A 2 x 16 KB, B 8 KB, transpose 16x128 words.
// ---------------------------------------------------------------------------
template <int LOGR>
__global__ void __launch_bounds__(128) k1t_convert_cols(const __grid_constant__ CUtensorMap map_a,
                                                        const __grid_constant__ CUtensorMap map_b,
                                                        uint32_t* __restrict__ res,
                                                        const PrimeConst* __restrict__ pcs,
                                                        const uint8_t* __restrict__ conv_w,
                                                        const uint2* __restrict__ tw_fwd, int n, int logC, int P,
                                                        int count, size_t ws_bstride, uint32_t* __restrict__ err) {
    constexpr int R = 1 << LOGR;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sbase = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = sbase;                        // 2 x (128 x 128 B)
    uint8_t* sB = sbase + 32768;                // 64 x 128 B
    uint32_t* sT = reinterpret_cast<uint32_t*>(sbase + 32768 + 8192);  // [16][128] residues
    __shared__ uint64_t tma_bar[2], mma_bar;
    __shared__ uint32_t tmem_base;
    __shared__ PrimeConst spc[tc::kConvGroup];

    const int tid = threadIdx.x, warp = tid >> 5;
    const int pg = blockIdx.y;
    const int C = 1 << logC;
    const int Gc = C < 8 ? C : 8;          // columns per tile
    const int groups_per_poly = C / Gc;
    const int tiles = count * 2 * groups_per_poly;
    const int np = min(tc::kConvGroup, P - pg * tc::kConvGroup);  // primes in this group

    // B: this group's pre-swizzled weight image.  A: zero once -- rows past
    // R*Gc (small rings) are never written by the TMA and must stay zero.
    {
        const uint4* src = reinterpret_cast<const uint4*>(conv_w + size_t(pg) * 8192);
        for (int k = tid; k < 512; k += 128) reinterpret_cast<uint4*>(sB)[k] = __ldg(src + k);
        for (int k = tid; k < 2048; k += 128) reinterpret_cast<uint4*>(sA)[k] = make_uint4(0, 0, 0, 0);
        if (tid < tc::kConvGroup) spc[tid] = pcs[min(pg * tc::kConvGroup + tid, P - 1)];
    }
    if (warp == 0) tc::tmem_alloc(&tmem_base, 64);
    if (tid == 0) {
        tc::mbar_init(&tma_bar[0], 1);
        tc::mbar_init(&tma_bar[1], 1);
        tc::mbar_init(&mma_bar, 1);
    }
    tc::fence_smem_async();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tbase = tmem_base;
    const uint32_t taddr = tbase + (uint32_t(32 * (warp & 3)) << 16);
    const uint32_t tile_bytes = 128u * uint32_t(Gc) * uint32_t(R);

    auto issue = [&](int tile, int buf) {
        const int cg = tile % groups_per_poly;
        const int poly = (tile / groups_per_poly) & 1;
        const int z = tile / (2 * groups_per_poly);
        tc::mbar_expect_tx(&tma_bar[buf], tile_bytes);
        tc::tma_load_4d(sA + buf * 16384, poly ? &map_b : &map_a, 0, cg * Gc, 0, z, &tma_bar[buf]);
    };
    if (tid == 0 && int(blockIdx.x) < tiles) issue(blockIdx.x, 0);

    // column-stage role: prime j of the group, column c of the tile
    const int cj = tid / 8, cc = tid % 8;
    const bool col_active = cj < np && cc < Gc;
    const int ci = pg * tc::kConvGroup + (cj < np ? cj : 0);
    uint2 twr[R > 1 ? R - 1 : 1];
#pragma unroll
    for (int k = 1; k < R; ++k) twr[k - 1] = __ldg(tw_fwd + size_t(ci) * kNMax + k);
    const PrimeConst cpc = pcs[ci];

    uint32_t tma_phases = 0, mma_phase = 0;  // bit b: parity of buffer b's next TMA completion
    bool ok = true;
    int k = 0;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++k) {
        const int buf = k & 1;
        const int cg = tile % groups_per_poly;
        const int poly = (tile / groups_per_poly) & 1;
        const int z = tile / (2 * groups_per_poly);
        if (tid == 0) {
            ok = tc::mbar_wait(&tma_bar[buf], (tma_phases >> buf) & 1u) && ok;
            tc::fence_after();
            const uint32_t a0 = tc::smem_u32(sA + buf * 16384), b0 = tc::smem_u32(sB);
            constexpr uint32_t idesc = tc::idesc_u8(tc::kTileM, tc::kConvN);
#pragma unroll
            for (int ks = 0; ks < 4; ++ks)
                tc::mma_u8(tbase, tc::sw128_desc(a0 + 32 * ks), tc::sw128_desc(b0 + 32 * ks), idesc, ks > 0);
            tc::mma_commit(&mma_bar);
            // the other buffer's last reader was the previous tile's MMA, already complete
            if (tile + int(gridDim.x) < tiles) issue(tile + gridDim.x, buf ^ 1);
        }
        tma_phases ^= 1u << buf;
        ok = tc::mbar_wait(&mma_bar, mma_phase) && ok;
        mma_phase ^= 1;
        tc::fence_after();
        // --- residues of row m = tid for the group's 16 primes ---
#pragma unroll
        for (int q4 = 0; q4 < 4; ++q4) {
            uint32_t d[16];
            tc::tmem_ld16(taddr + 16 * q4, d);
            tc::tmem_wait_ld();
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int j = 4 * q4 + u;
                const uint64_t v = uint64_t(d[4 * u]) + (uint64_t(d[4 * u + 1]) << 8) +
                                   (uint64_t(d[4 * u + 2]) << 16) + (uint64_t(d[4 * u + 3]) << 24);
                sT[j * 128 + tid] = reduce60(v, spc[j].p, spc[j].mu);
            }
        }
        tc::fence_before();
        __syncthreads();
        // --- forward column stages in registers, then store ---
        if (col_active) {
            uint32_t v[R];
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = sT[cj * 128 + r * Gc + cc];
#pragma unroll
            for (int s = 0; s < LOGR; ++s) {
                const int t = R >> (s + 1);
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (!(r & t)) ct_bfly(v[r], v[r + t], twr[(1 << s) + (r >> (LOGR - s)) - 1], cpc.p, cpc.two_p);
            }
            uint32_t* dst = res + size_t(z) * ws_bstride + (size_t(poly) * P + ci) * n + size_t(cg) * Gc + cc;
#pragma unroll
            for (int r = 0; r < R; ++r) dst[size_t(r) << logC] = v[r];
        }
        __syncthreads();  // sT is rewritten by the next tile
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after();
        tc::tmem_dealloc(tbase, 64);
    }
    if (!ok && tid == 0) atomicOr(err, 1u);
}

// ---------------------------------------------------------------------------
// K3T: inverse column stages + CRT on the tensor cores.
// grid (ctas); block 128.  Tile index -> (product z, column group cg).  The
// tile's residues for every prime arrive by TMA (box: Gc columns x R rows x P
// primes of u32); the next tile's box is requested as soon as this one has
// been turned into CRT digits, so it loads during the MMA and the epilogue.
// Dynamic shared memory (1024-aligned): A 2 x 16 KB (K = 256), B 2 x 16 KB,
// residue box P*R*Gc words, inverse column twiddles P*(R-1) uint2.
// ---------------------------------------------------------------------------
template <int LOGR, int W>
__global__ void __launch_bounds__(128) k3t_cols_crt(const __grid_constant__ CUtensorMap map_res,
                                                    uint32_t* __restrict__ out, const PrimeConst* __restrict__ pcs,
                                                    const uint2* __restrict__ tw_inv,
                                                    const uint2* __restrict__ scale,
                                                    const uint8_t* __restrict__ crt_w,
                                                    const uint32_t* __restrict__ consts, uint64_t mu_q, int sbits,
                                                    int n, int logC, int P, int stride, int count,
                                                    size_t io_bstride, const uint32_t* __restrict__ work,
                                                    size_t ws_bstride, int use_tma, uint32_t* __restrict__ err) {
    constexpr int R = 1 << LOGR;
    constexpr int NV = 4 * W + 4;  // value byte columns
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sbase = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = sbase;          // [2][128][128 B]
    uint8_t* sB = sbase + 32768;  // [2][128][128 B]
    uint32_t* sR = reinterpret_cast<uint32_t*>(sbase + 65536);  // [P][R][Gc]
    __shared__ uint64_t tma_bar, mma_bar;
    __shared__ uint32_t tmem_base;
    __shared__ uint32_t s_q[2 * W];

    const int tid = threadIdx.x, warp = tid >> 5;
    const int C = 1 << logC;
    const int Gc = C < 8 ? C : 8;
    const int groups = C / Gc;
    const int tiles = count * groups;
    const int box_words = P * R * Gc;
    uint2* sTw = reinterpret_cast<uint2*>(sR + ((box_words + 3) & ~3));  // [P][R-1]
    {
        const uint4* src = reinterpret_cast<const uint4*>(crt_w);
        for (int k = tid; k < 2048; k += 128) reinterpret_cast<uint4*>(sB)[k] = __ldg(src + k);
        for (int k = tid; k < 2048; k += 128) reinterpret_cast<uint4*>(sA)[k] = make_uint4(0, 0, 0, 0);
        for (int k = tid; k < 2 * W; k += 128) s_q[k] = consts[k];
        constexpr int RT = R > 1 ? R - 1 : 1;
        if (R > 1)
            for (int k = tid; k < P * RT; k += 128) sTw[k] = __ldg(tw_inv + size_t(k / RT) * kNMax + 1 + k % RT);
    }
    if (warp == 0) tc::tmem_alloc(&tmem_base, 128);
    if (tid == 0) {
        tc::mbar_init(&tma_bar, 1);
        tc::mbar_init(&mma_bar, 1);
    }
    tc::fence_smem_async();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tbase = tmem_base;
    const uint32_t taddr = tbase + (uint32_t(32 * (warp & 3)) << 16);
    const int pairs = P * Gc;
    // rings with fewer than 4 columns (n < 64) have rows too short for a tensor
    // map; their single-tile box is read by the threads instead
    auto issue = [&](int tile) {
        if (!use_tma) return;
        tc::mbar_expect_tx(&tma_bar, uint32_t(box_words) * 4u);
        tc::tma_load_4d(sR, &map_res, (tile % groups) * Gc, 0, 0, tile / groups, &tma_bar);
    };
    if (tid == 0 && int(blockIdx.x) < tiles) issue(blockIdx.x);

    uint32_t tma_phase = 0, mma_phase = 0;
    bool ok = true;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int cg = tile % groups, z = tile / groups;
        if (use_tma) {
            ok = tc::mbar_wait(&tma_bar, tma_phase) && ok;
            tma_phase ^= 1;
        } else {
            const uint32_t* plane = work + size_t(z) * ws_bstride;
            for (int k = tid; k < box_words; k += 128) {
                const int c = k % Gc, r = (k / Gc) % R, i = k / (Gc * R);
                sR[k] = plane[size_t(i) * n + (size_t(r) << logC) + size_t(cg) * Gc + c];
            }
            __syncthreads();
        }
        // --- inverse column stages and CRT digits into A ---
        for (int pr = tid; pr < pairs; pr += 128) {
            const int i = pr / Gc, c = pr - i * Gc;
            const PrimeConst pc = pcs[i];
            uint32_t v[R];
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = sR[(i * R + r) * Gc + c];
            const uint2* tw = sTw + i * (R - 1) - 1;  // tw[k] = Psi_inv_rev[k], k >= 1
#pragma unroll
            for (int s = LOGR - 1; s >= 0; --s) {
                const int t = R >> (s + 1);
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (!(r & t)) gs_bfly(v[r], v[r + t], tw[(1 << s) + (r >> (LOGR - s))], pc.p, pc.two_p);
            }
            const uint2 sc = __ldg(scale + i);
            const uint32_t ka = uint32_t(i) >> 5, kb = (4u * i) & 127u;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t t = csub(shoup_mul(v[r], sc, pc.p), pc.p);
                *reinterpret_cast<uint32_t*>(sA + ka * 16384 + tc::sw128_offset(c * R + r, kb)) = t;
            }
        }
        tc::fence_smem_async();
        tc::fence_before();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after();
            // the residue box is free again: fetch the next tile's during the MMA and epilogue
            if (tile + int(gridDim.x) < tiles) issue(tile + gridDim.x);
            const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
            constexpr uint32_t idesc = tc::idesc_u8(tc::kTileM, tc::kCrtN);
#pragma unroll
            for (int ks = 0; ks < 8; ++ks) {
                const uint32_t off = (ks >> 2) * 16384 + 32 * (ks & 3);
                tc::mma_u8(tbase, tc::sw128_desc(a0 + off), tc::sw128_desc(b0 + off), idesc, ks > 0);
            }
            tc::mma_commit(&mma_bar);
        }
        ok = tc::mbar_wait(&mma_bar, mma_phase) && ok;
        mma_phase ^= 1;
        tc::fence_after();
        // --- carry-propagate the byte columns of row m = tid ---
        // value: NV/4 = W+1 words plus the carry-out; quotient estimate: 8 columns
        uint32_t acc[W + 2];
        uint64_t carry = 0;
        uint64_t fsum0 = 0, fsum1 = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            uint32_t d[16];
            tc::tmem_ld16(taddr + 16 * q, d);
            tc::tmem_wait_ld();
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int J = 16 * q + 4 * u;  // first byte column of this 32-bit word
                const uint64_t s = uint64_t(d[4 * u]) + (uint64_t(d[4 * u + 1]) << 8) +
                                   (uint64_t(d[4 * u + 2]) << 16) + (uint64_t(d[4 * u + 3]) << 24);
                if (J < NV) {
                    const uint64_t x = s + carry;
                    acc[J / 4] = uint32_t(x);
                    carry = x >> 32;
                } else if (J == NV) {
                    fsum0 = s;
                } else if (J == NV + 4) {
                    fsum1 = s;
                }
            }
        }
        acc[W + 1] = uint32_t(carry);
        const uint64_t f1 = fsum1 + (fsum0 >> 32);
        // nearest integer of sum t_i / p_i: (f1 * 2^32 + low) / 2^64 rounded
        const uint32_t nearest = uint32_t(f1 >> 32) + (uint32_t(f1) >> 31);
        const int cc = tid / R, rr = tid % R;
        if (cc < Gc) {
            const size_t J = (size_t(rr) << logC) + size_t(cg) * Gc + cc;
            crt_finish<W>(acc, nearest, s_q, mu_q, sbits, out + size_t(z) * io_bstride + J * stride, stride);
        }
        tc::fence_before();
        __syncthreads();
    }
    if (warp == 0) {
        tc::fence_after();
        tc::tmem_dealloc(tbase, 128);
    }
    if (!ok && tid == 0) atomicOr(err, 1u);
}

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
    if (4 * s.W + 4 + 8 > uint32_t(tc::kCrtN)) throw Failure(PM_ERR_UNSUPPORTED, "q too wide for the CRT tile");
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
    // CRT weights: [2 K-atoms][128 rows][128 B]
    const uint32_t NV = 4 * s.W + 4;
    Words total{1};
    for (unsigned i = 0; i < s.P; ++i) total = multiply_small(total, B.primes[i]);
    std::vector<uint8_t> img(32768, 0);
    for (unsigned i = 0; i < s.P; ++i) {
        Words m = total;
        divide_small(m, B.primes[i]);
        const Words mq = mod(m, s.q);
        const uint64_t recip = uint64_t(((unsigned __int128)1 << 64) / B.primes[i]);
        for (int a = 0; a < 4; ++a) {
            const Words shifted = shift_left(mq, 8 * a);
            const unsigned __int128 rs = (unsigned __int128)recip << (8 * a);
            const uint32_t k = 4 * i + a, ka = k >> 7, kk = k & 127;
            for (uint32_t J = 0; J < NV; ++J) {
                const uint32_t word = J / 4 < shifted.size() ? shifted[J / 4] : 0;
                img[ka * 16384 + tc::sw128_offset(J, kk)] = uint8_t(word >> (8 * (J % 4)));
            }
            for (uint32_t J = 0; J < 8; ++J) img[ka * 16384 + tc::sw128_offset(NV + J, kk)] = uint8_t(rs >> (8 * J));
        }
    }
    cuda_check(cudaMalloc(&s.d_crt_weights, img.size()), "allocate CRT weights");
    cuda_check(cudaMemcpy(s.d_crt_weights, img.data(), img.size(), cudaMemcpyHostToDevice), "upload CRT weights");
    cuda_check(cudaMalloc(&s.d_err, sizeof(uint32_t)), "allocate error word");
    cuda_check(cudaMemset(s.d_err, 0, sizeof(uint32_t)), "clear error word");
}

void tensor_release(PlanCore& s) {
    cudaFree(s.d_crt_weights);
    cudaFree(s.d_err);
    s.d_crt_weights = nullptr;
    s.d_err = nullptr;
}

namespace {
int sm_count() {
    static int count = 0;
    if (!count) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        if (!count) count = 148;
    }
    return count;
}

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

// the product planes (plane 0..P-1) of `count` workspaces: dims (column, row, prime, product)
CUtensorMap residue_map(const PlanCore& s, const void* work, uint32_t count) {
    const uint32_t C = 1u << s.logC, R = 1u << s.logR, Gc = C < 8 ? C : 8;
    const cuuint64_t dims[4] = {C, R, s.P, count};
    const cuuint64_t strides[3] = {C * 4ull, C * R * 4ull, s.workspace_bytes};
    const cuuint32_t box[4] = {Gc, R, s.P, 1};
    return make_map(CU_TENSOR_MAP_DATA_TYPE_UINT32, work, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_NONE);
}

template <int LOGR>
void launch_k1t(const PlanCore& s, const uint32_t* a, const uint32_t* b, uint32_t* work, uint32_t count,
                cudaStream_t st) {
    const int C = 1 << s.logC, Gc = C < 8 ? C : 8;
    const int groups = int((s.P + tc::kConvGroup - 1) / tc::kConvGroup);
    const int tiles = int(count) * 2 * (C / Gc);
    int ctas = sm_count() * 4 / groups;
    if (ctas > tiles) ctas = tiles;
    if (ctas < 1) ctas = 1;
    const size_t smem = 1024 + 32768 + 8192 + 16 * 128 * 4;
    cuda_check(cudaFuncSetAttribute(k1t_convert_cols<LOGR>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
               "K1T shared memory");
    const CUtensorMap ma = coefficient_map(s, a, count), mb = coefficient_map(s, b, count);
    dim3 grid(ctas, groups);
    k1t_convert_cols<LOGR><<<grid, 128, smem, st>>>(ma, mb, work, s.basis->d_pc, s.basis->d_conv_weights,
                                                    s.basis->d_tw_fwd, int(s.n), int(s.logC), int(s.P), int(count),
                                                    s.workspace_bytes / 4, s.d_err);
}

template <int LOGR, int W>
void launch_k3t(const PlanCore& s, const uint32_t* work, uint32_t* c, uint32_t count, cudaStream_t st) {
    const int C = 1 << s.logC, Gc = C < 8 ? C : 8, R = 1 << s.logR;
    const int tiles = int(count) * (C / Gc);
    int ctas = sm_count() * 2;
    if (ctas > tiles) ctas = tiles;
    const size_t box_words = size_t(s.P) * R * Gc;
    const size_t smem = 1024 + 65536 + ((box_words + 3) & ~size_t(3)) * 4 + size_t(s.P) * (R > 1 ? R - 1 : 1) * 8;
    cuda_check(cudaFuncSetAttribute(k3t_cols_crt<LOGR, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)),
               "K3T shared memory");
    const bool use_tma = (C * 4) % 16 == 0;
    CUtensorMap mr;
    std::memset(&mr, 0, sizeof mr);
    if (use_tma) mr = residue_map(s, work, count);
    k3t_cols_crt<LOGR, W><<<ctas, 128, smem, st>>>(mr, c, s.basis->d_pc, s.basis->d_tw_inv, s.d_scale,
                                                    s.d_crt_weights, s.d_consts, s.mu_q, int(s.qbits), int(s.n),
                                                    int(s.logC), int(s.P), int(s.stride), int(count),
                                                    size_t(s.n) * s.stride, work, s.workspace_bytes / 4,
                                                    use_tma ? 1 : 0, s.d_err);
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

void launch_tensor(const PlanCore& s, const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* work,
                   uint32_t count, cudaStream_t st) {
    {
        ProfileScope prof("k1t_convert_cols", st);
        switch (s.logR) {
            case 0: launch_k1t<0>(s, a, b, work, count, st); break;
            case 1: launch_k1t<1>(s, a, b, work, count, st); break;
            case 2: launch_k1t<2>(s, a, b, work, count, st); break;
            case 3: launch_k1t<3>(s, a, b, work, count, st); break;
            default: launch_k1t<4>(s, a, b, work, count, st); break;
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
