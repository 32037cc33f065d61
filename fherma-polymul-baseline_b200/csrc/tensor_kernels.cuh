// The tensor-core passes as persistent kernels over an abstract work source.
//
// K1T (conversion + forward column stages) and K3T (inverse column stages +
// CRT) loop over work items; a Work type says how many items there are, what
// each one is and where its product's data lives:
//   PlanConvWork / PlanCrtWork   `count` products of one plan, items computed
//                                from the index (maps are kernel parameters);
//   TableConvWork / TableCrtWork products of different n and q (an uneven
//                                batch), items and per-product descriptors read
//                                from device tables (maps in global memory).
// Each CTA takes a contiguous chunk of items, so the operand tables it keeps in
// shared memory (prime-group weights, a product's CRT weights) change rarely.
//
// Conversion (reference: rns/tensor_prepare.h:20-101 does the same contraction
// with WMMA s8 or cuBLAS, centred by -128; unsigned operands need no centring):
//   D[m][4i+a] = sum_k x_k(m) * byte_a(2^(8k) mod p_i)      k < 128 coefficient bytes
//   r_i(m)     = sum_a D[m][4i+a] * 2^(8a)  mod p_i          (< 2^48 before the reduction)
// every D entry is at most 128*255^2 < 2^23, so the s32 accumulation is exact.
// CRT (the reference accumulates sum t_i (P/p_i mod q) in a 928-bit cuPQC
// integer, rns/solve.cu:336-420):
//   A[m][4i+a] = byte_a(t_i(m)),  B[J][4i+a] = byte_J((P/p_i mod q) << 8a)  J < NV
//                                 B[NV+J][4i+a] = byte_J(floor(2^64/p_i) << 8a)  J < 8
// every D entry is at most 256*255^2 < 2^24.
#pragma once

#include <cuda.h>

#include <cstdint>
#include <type_traits>

#include "pm_device.cuh"
#include "tc_ptx.cuh"

namespace pm {

namespace tc {
constexpr int kTileM = 128;     // coefficients per tile = 8 columns x 16 rows
constexpr int kConvGroup = 16;  // primes per conversion MMA (N = 64)
constexpr int kConvN = 4 * kConvGroup;
constexpr int kCrtN = 128;      // value bytes + 8 quotient bytes (+ pad)
constexpr int kCrtK = 256;      // 4 bytes per prime, 64 primes
constexpr int kMaxPrimes = 64;
constexpr int kCrtThreads = 256;  // K3T: 8 warps for the digit phase, warps 0-3 for the epilogue
}  // namespace tc

struct ConvItem {
    int z, pg, poly, cg;
};
struct ConvTarget {
    const CUtensorMap* map;  // coefficient bytes (dims: byte, column, row, product)
    int mz;                  // product coordinate inside that map
    uint32_t* res;           // this product's residue planes
    int n, logC, P;
};
struct CrtTarget {
    const CUtensorMap* map;  // residue planes (dims: column, row, prime, product)
    int mz;
    const uint32_t* work;    // the same planes, for rings too small for a tensor map
    uint32_t* out;           // this product's output coefficients
    const uint2* scale;
    const uint32_t* consts;  // q[W], (-P mod q)[W]
    const uint32_t* ktab;    // [2P+1][W] k (-P mod q) mod q
    const uint8_t* crt_w;    // [2][128][128] pre-swizzled CRT weights
    const uint64_t* kfrac;   // [2P+1] floor(2^64 (row k of ktab) / q)
    uint64_t mu_q;
    int sbits, n, logC, P, stride, use_tma;
    uint32_t delta;          // special-form q = 2^sbits - delta, or 0
};

// Per-product descriptor of an uneven batch (device table).
struct BatchProduct {
    int n, logC, P, W, sbits, stride;
    uint32_t delta;  // special-form q = 2^sbits - delta, or 0
    uint64_t mu_q;
    uint64_t io_off;  // u32 words from the batch's a (b, c) base to this product
    uint64_t ws_off;  // u32 words from the batch's workspace base to its planes
    const uint2* scale;
    const uint32_t* consts;
    const uint32_t* ktab;
    const uint8_t* crt_w;
    const uint64_t* kfrac;
};

struct PlanConvWork {
    CUtensorMap map_a, map_b;
    uint32_t* work;
    size_t ws_bstride;
    int n, logC, P, count, pgs;
    // column groups per row: C / min(C, 8) = 2^lg, lg = logC - min(logC, 3)
    __device__ int lg() const { return logC - min(logC, 3); }
    __device__ int total() const { return pgs * (count << (lg() + 1)); }
    __device__ ConvItem item(int k) const {
        const int g = lg();
        const int per_pg = count << (g + 1);
        const int pg = k / per_pg, rest = k - pg * per_pg;
        return ConvItem{rest >> (g + 1), pg, (rest >> g) & 1, rest & ((1 << g) - 1)};
    }
    __device__ ConvTarget target(int z, int poly) const {
        return ConvTarget{poly ? &map_b : &map_a, z, work + z * ws_bstride, n, logC, P};
    }
    // CTA b of `grid` (a multiple of pgs): prime group b / m, m = grid / pgs, and the
    // (b % m)-th of m equal runs of that group's tiles.  The CTAs of different prime groups
    // with the same run read the same coefficient tiles at about the same time, so three of
    // every four TMA loads of a tile hit L2 instead of streaming the inputs once per group.
    __device__ int2 range(int b, int grid) const {
        const int per_pg = count << (lg() + 1);
        const int m = grid / pgs;
        if (m == 0) {  // fewer CTAs than prime groups: contiguous runs of everything
            const int all = total(), chunk = (all + grid - 1) / grid;
            return make_int2(min(all, b * chunk), min(all, (b + 1) * chunk));
        }
        const int pg = b / m, j = b - pg * m;
        if (pg >= pgs) return make_int2(0, 0);
        const int chunk = (per_pg + m - 1) / m;
        return make_int2(pg * per_pg + min(j * chunk, per_pg), pg * per_pg + min((j + 1) * chunk, per_pg));
    }
};

struct TableConvWork {
    const uint4* items;  // (z, pg, poly, cg)
    int nitems;
    const BatchProduct* prod;
    const CUtensorMap* maps;  // [3 * products]: a, b, residues
    uint32_t* work;
    __device__ int total() const { return nitems; }
    __device__ ConvItem item(int k) const {
        const uint4 v = items[k];
        return ConvItem{int(v.x), int(v.y), int(v.z), int(v.w)};
    }
    __device__ ConvTarget target(int z, int poly) const {
        const BatchProduct& d = prod[z];
        return ConvTarget{maps + 3 * z + poly, 0, work + d.ws_off, d.n, d.logC, d.P};
    }
    __device__ int2 range(int b, int grid) const {  // contiguous runs of the table
        const int chunk = (nitems + grid - 1) / grid;
        return make_int2(min(nitems, b * chunk), min(nitems, (b + 1) * chunk));
    }
};

struct PlanCrtWork {
    CUtensorMap map_res;
    const uint32_t* work;
    uint32_t* out;
    size_t ws_bstride, io_bstride;
    const uint2* scale;
    const uint32_t* consts;
    const uint32_t* ktab;
    const uint8_t* crt_w;
    const uint64_t* kfrac;
    uint64_t mu_q;
    int sbits, n, logC, P, stride, count, use_tma;
    uint32_t delta;
    __device__ int lg() const { return logC - min(logC, 3); }  // column groups per row = 2^lg
    __device__ int total() const { return count << lg(); }
    __device__ int2 item(int k) const { return make_int2(k >> lg(), k & ((1 << lg()) - 1)); }
    __device__ CrtTarget target(int z) const {
        return CrtTarget{&map_res, z, work + z * ws_bstride, out + z * io_bstride, scale, consts, ktab, crt_w,
                         kfrac, mu_q, sbits, n, logC, P, stride, use_tma, delta};
    }
};

struct TableCrtWork {
    const uint2* items;  // (z, cg)
    int nitems;
    const BatchProduct* prod;
    const CUtensorMap* maps;
    const uint32_t* work;
    uint32_t* out;
    __device__ int total() const { return nitems; }
    __device__ int2 item(int k) const {
        const uint2 v = items[k];
        return make_int2(int(v.x), int(v.y));
    }
    __device__ CrtTarget target(int z) const {
        const BatchProduct& d = prod[z];
        return CrtTarget{maps + 3 * z + 2, 0, work + d.ws_off, out + d.io_off, d.scale, d.consts, d.ktab, d.crt_w,
                         d.kfrac, d.mu_q, d.sbits, d.n, d.logC, d.P, d.stride, 1, d.delta};
    }
};

// ---------------------------------------------------------------------------
// K1T: tensor-core conversion + forward column stages, persistent and warp
// specialised.  Block kConvThreads = 160: warps 0-3 are the workers (epilogue
// and column stages, one coefficient row per thread), warp 4 the producer.
// A tile holds coefficient r*C + Gc*cg + c of one polynomial in row m = r*Gc + c
// and arrives by TMA (box: 128 bytes x Gc columns x R rows, 128-byte swizzle,
// bytes past the coefficient width zero-filled).  Items are ordered prime group
// first.
// Producer (one lane issues): B (the group's pre-swizzled weights, 8 KB) by bulk
// copy when the group changes; per item: wait for its A tile, wait until the
// workers have drained the accumulator it reuses, four tcgen05.mma (M=128,
// N=64, K=32) into that accumulator, commit; once the MMA is complete its A tile
// takes the TMA of the item two ahead.
// Workers: wait for the item's MMA, tcgen05.ld -> two 32-bit partial sums ->
// lazy Barrett (the group's primes and factors held in registers, the column
// twiddles in shared memory: 96 registers a thread, so four CTAs fit per SM) ->
// padded transpose, release the accumulator (mbarrier arrival), then 4 forward
// column stages in registers -> residue planes.  Only the workers meet at (named) barriers, so the producer's
// waits never hold them.
// Barriers: tma_full[2], mma_full[2], tmem_empty[2] (128 arrivals), b_full.
// Dynamic shared memory (1024-aligned): A 2 x 16 KB, B 8 KB, transpose
// 16 x kTS words (kTS = 136: the four primes a warp reads per row sit 8 banks
// apart).  TMEM: 2 x 64 columns.
// ---------------------------------------------------------------------------
constexpr int kTS = 136;
namespace tc {
constexpr int kConvThreads = 160;
}

template <int LOGR, class Work>
__global__ void __launch_bounds__(tc::kConvThreads, 4) k1t_convert(const __grid_constant__ Work w,
                                                                const PrimeConst* __restrict__ pcs,
                                                                const uint8_t* __restrict__ conv_w,
                                                                const uint2* __restrict__ tw_fwd,
                                                                uint32_t* __restrict__ err) {
    constexpr int R = 1 << LOGR;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sbase = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = sbase;                        // 2 x (128 x 128 B)
    uint8_t* sB = sbase + 32768;                // 64 x 128 B
    uint32_t* sT = reinterpret_cast<uint32_t*>(sbase + 32768 + 8192);  // [16][kTS] residues
    __shared__ uint64_t tma_full[2], mma_full[2], tmem_empty[2], b_full;
    __shared__ uint32_t tmem_base;
    __shared__ volatile uint32_t s_abort;
    __shared__ uint2 spm[tc::kConvGroup];  // the group's primes and floor(2^48 / p)
    __shared__ uint2 stw[tc::kConvGroup][R > 1 ? R - 1 : 1];  // the group's forward column twiddles

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int2 range = w.range(int(blockIdx.x), int(gridDim.x));
    const int begin = range.x, end = range.y;

    for (int k = tid; k < 2048; k += tc::kConvThreads) reinterpret_cast<uint4*>(sA)[k] = make_uint4(0, 0, 0, 0);
    if (warp == 0) tc::tmem_alloc(&tmem_base, 128);
    if (tid == 0) {
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(&tma_full[b], 1);
            tc::mbar_init(&mma_full[b], 1);
            tc::mbar_init(&tmem_empty[b], 128);
        }
        tc::mbar_init(&b_full, 1);
        s_abort = 0;
    }
    tc::fence_smem_async();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tbase = tmem_base;
    bool ok = true;

    if (warp == 4) {
        // ------------------------------ producer ------------------------------
        // every lane runs the loop (uniform control flow); lane 0 issues
        auto issue = [&](int k, int buf) {
            const ConvItem it = w.item(k);
            const ConvTarget t = w.target(it.z, it.poly);
            const int C = 1 << t.logC, Gc = C < 8 ? C : 8;
            tc::mbar_expect_tx(&tma_full[buf], 128u * uint32_t(Gc) * uint32_t(R));
            tc::tma_load_4d(sA + buf * 16384, t.map, 0, it.cg * Gc, 0, t.mz, &tma_full[buf]);
        };
        auto wait = [&](uint64_t* bar, uint32_t parity) {
            const bool done = __all_sync(0xffffffffu, tc::mbar_wait(bar, parity));
            ok = ok && done;
            return done;
        };
        uint32_t ph_tma = 0, ph_mma = 0, ph_empty = 0, ph_b = 0, pending = 0;  // bit b: buffer b
        bool b_pending = false;
        if (lane == 0) {
            if (begin < end) issue(begin, 0);
            if (begin + 1 < end) issue(begin + 1, 1);
        }
        pending = (begin < end ? 1u : 0u) | (begin + 1 < end ? 2u : 0u);
        int loaded_pg = -1, kk = 0;
        for (int k = begin; k < end; ++k, ++kk) {
            if (__any_sync(0xffffffffu, s_abort != 0)) break;  // a worker gave up a wait
            const int buf = kk & 1;
            const int pg = w.item(k).pg;
            if (pg != loaded_pg) {  // every earlier MMA was waited for: B may be rewritten
                if (lane == 0) {
                    tc::mbar_expect_tx(&b_full, 8192u);
                    tc::bulk_load(sB, conv_w + size_t(pg) * 8192, 8192u, &b_full);
                }
                b_pending = true;
                if (!wait(&b_full, ph_b)) break;
                ph_b ^= 1u;
                b_pending = false;
                loaded_pg = pg;
            }
            if (!wait(&tma_full[buf], (ph_tma >> buf) & 1u)) break;
            ph_tma ^= 1u << buf;
            pending &= ~(1u << buf);
            if (kk >= 2) {
                if (!wait(&tmem_empty[buf], (ph_empty >> buf) & 1u)) break;
                ph_empty ^= 1u << buf;
            }
            tc::fence_after();
            if (lane == 0) {
                const uint32_t a0 = tc::smem_u32(sA + buf * 16384), b0 = tc::smem_u32(sB);
                constexpr uint32_t idesc = tc::idesc_u8(tc::kTileM, tc::kConvN);
#pragma unroll
                for (int ks = 0; ks < 4; ++ks)
                    tc::mma_u8(tbase + 64 * buf, tc::sw128_desc(a0 + 32 * ks), tc::sw128_desc(b0 + 32 * ks), idesc,
                               ks > 0);
                tc::mma_commit(&mma_full[buf]);
            }
            __syncwarp();
            // the MMA has read its A tile (and B): the tile takes the item two ahead
            if (!wait(&mma_full[buf], (ph_mma >> buf) & 1u)) break;
            ph_mma ^= 1u << buf;
            if (k + 2 < end) {
                if (lane == 0) issue(k + 2, buf);
                pending |= 1u << buf;
            }
        }
        if (!ok) s_abort = 1;
        // copies requested but not consumed land before the CTA's shared memory goes away
        for (int b = 0; b < 2; ++b)
            if (pending & (1u << b)) tc::mbar_wait(&tma_full[b], (ph_tma >> b) & 1u);
        if (b_pending) tc::mbar_wait(&b_full, ph_b);
    } else {
        // ------------------------------ workers -------------------------------
        const uint32_t taddr = tbase + (uint32_t(32 * warp) << 16);
        // column-stage role: prime j of the group, column c of the tile
        const int cj = tid / 8, cc = tid % 8;
        uint2 rpm[tc::kConvGroup];  // the group's primes and floor(2^48 / p)
        PrimeConst cpc{};
        int cur_pg = -1;
        uint32_t ph_mma = 0;
        int kk = 0;
        for (int k = begin; k < end; ++k, ++kk) {
            const ConvItem it = w.item(k);
            const ConvTarget t = w.target(it.z, it.poly);
            const int C = 1 << t.logC, Gc = C < 8 ? C : 8;
            const int buf = kk & 1;
            if (it.pg != cur_pg) {  // the previous item's closing barrier ended every read of spm
                if (tid < tc::kConvGroup) {
                    const PrimeConst g = pcs[it.pg * tc::kConvGroup + tid];
                    spm[tid] = make_uint2(g.p, g.mu >> 13);  // floor(floor(2^61 / p) / 2^13)
                }
                const int ci = it.pg * tc::kConvGroup + cj;
                constexpr int RT = R > 1 ? R - 1 : 1;
                if (R > 1)
                    for (int q = tid; q < tc::kConvGroup * RT; q += 128)
                        stw[q / RT][q % RT] = __ldg(tw_fwd + size_t(it.pg * tc::kConvGroup + q / RT) * kNMax + 1 + q % RT);
                cpc = pcs[ci];
                cur_pg = it.pg;
                tc::bar_sync(1, 128);
#pragma unroll
                for (int j = 0; j < tc::kConvGroup; ++j) rpm[j] = spm[j];
            }
            const int np = min(tc::kConvGroup, t.P - it.pg * tc::kConvGroup);
            ok = tc::mbar_wait(&mma_full[buf], (ph_mma >> buf) & 1u) && ok;
            ph_mma ^= 1u << buf;
            tc::fence_after();
            // --- residues of row m = tid for the group's 16 primes ---
            // byte-plane sums d_a <= 128 * 255^2 < 2^23, so lo = d0 + 2^8 d1 and hi = d2 + 2^8 d3
            // are below 2^31.01 and the residue input is hi 2^16 + lo
#pragma unroll
            for (int q4 = 0; q4 < 4; ++q4) {
                uint32_t d[16];
                tc::tmem_ld16(taddr + 64 * buf + 16 * q4, d);
                tc::tmem_wait_ld();
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int j = 4 * q4 + u;
                    const uint32_t lo = d[4 * u] + (d[4 * u + 1] << 8);
                    const uint32_t hi = d[4 * u + 2] + (d[4 * u + 3] << 8);
                    sT[j * kTS + tid] = reduce48_lazy(lo, hi, rpm[j].x, rpm[j].y);  // [0, 3p): butterfly input
                }
            }
            tc::fence_before();
            tc::mbar_arrive(&tmem_empty[buf]);  // this thread's accumulator reads are complete
            tc::bar_sync(1, 128);
            // --- forward column stages in registers, then store ---
            if (cj < np && cc < Gc) {
                const int ci = it.pg * tc::kConvGroup + cj;
                uint32_t v[R];
                const uint32_t* col = sT + cj * kTS + cc;
                if (Gc == 8) {  // every ring of 128 coefficients or more: constant offsets
#pragma unroll
                    for (int r = 0; r < R; ++r) v[r] = col[r * 8];
                } else {
#pragma unroll
                    for (int r = 0; r < R; ++r) v[r] = col[r * Gc];
                }
#pragma unroll
                for (int s = 0; s < LOGR; ++s) {
                    const int h = R >> (s + 1);
#pragma unroll
                    for (int r = 0; r < R; ++r)
                        if (!(r & h))
                            ct_bfly(v[r], v[r + h], stw[cj][(1 << s) + (r >> (LOGR - s)) - 1], cpc.p, cpc.two_p);
                }
                uint32_t* dst = t.res + (size_t(it.poly) * t.P + ci) * t.n + size_t(it.cg) * Gc + cc;
                const size_t row = size_t(1) << t.logC;
#pragma unroll
                for (int r = 0; r < R; ++r, dst += row) *dst = v[r];
            }
            // sT is rewritten by the next item; a failed wait (or the producer's) ends the loop for all workers
            if (tc::bar_sync_or(1, 128, !ok || s_abort)) break;
        }
        if (!ok) s_abort = 1;
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after();
        tc::tmem_dealloc(tbase, 128);
    }
    if (!ok) atomicOr(err, 1u);
}

// a[0..3] += b[0..3] + cy, cy in {0, 1} in and out (one add-with-carry chain;
// adding 2^32 - 1 to cy sets the carry flag exactly when cy is 1)
__device__ __forceinline__ void add4_carry(uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t& a3,
                                           const uint32_t (&b)[4], uint32_t& cy) {
    asm("add.cc.u32 %4, %4, 0xFFFFFFFF;\n\t"
        "addc.cc.u32 %0, %0, %5;\n\t"
        "addc.cc.u32 %1, %1, %6;\n\t"
        "addc.cc.u32 %2, %2, %7;\n\t"
        "addc.cc.u32 %3, %3, %8;\n\t"
        "addc.u32 %4, 0, 0;"
        : "+r"(a0), "+r"(a1), "+r"(a2), "+r"(a3), "+r"(cy)
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]));
}
__device__ __forceinline__ void add1_carry(uint32_t& a, uint32_t b, uint32_t& cy) {
    asm("add.cc.u32 %1, %1, 0xFFFFFFFF;\n\t"
        "addc.cc.u32 %0, %0, %2;\n\t"
        "addc.u32 %1, 0, 0;"
        : "+r"(a), "+r"(cy)
        : "r"(b));
}

// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// K3T: inverse column stages + CRT on the tensor cores, persistent.  Block of
// kCrtThreads = 256: all eight warps run the digit phase (the column stages of
// the tile's (prime, column) pairs), warps 0-3 (the owners of the 128 TMEM
// lanes) the per-coefficient epilogue.
// An item's residues for every prime arrive by TMA (box: Gc columns x 64 primes x
// R rows of u32, the primes past P zero-filled, landing as [row][prime][column]:
// a constant row stride, and the 4 primes x 8 columns a warp reads per row fall
// in 32 distinct banks); the next item's box is
// requested as soon as this one has been turned into CRT digits, so it loads
// during the MMA and the epilogue.  A-tile row m = r*Gc + c holds the digits of
// coefficient (row r, column c): a warp's digit stores (8 columns x 4 primes)
// then also hit 32 distinct banks of the 128-byte swizzle.
// The CRT weights, q constants and column twiddles of the current product stay
// in shared memory until an item of another product needs its own.
// Dynamic shared memory (1024-aligned): A 2 x 16 KB (K = 256), B 2 x 16 KB,
// residue box 64*R*8 words, inverse column twiddles 64*(R-1) uint2.
// ---------------------------------------------------------------------------
// LOGC > 0: every item's rows hold 2^LOGC values (a plan's launch at a common ring size), so
// the tile's column count and the output offsets are constants; 0: read from the item.
template <int LOGR, int W, class Work, int LOGC = 0>
__global__ void __launch_bounds__(tc::kCrtThreads, 2) k3t_crt(const __grid_constant__ Work w, const PrimeConst* __restrict__ pcs,
                                               const uint2* __restrict__ tw_inv, uint32_t* __restrict__ err) {
    constexpr int R = 1 << LOGR;
    constexpr int RT = R > 1 ? R - 1 : 1;
    constexpr int NV = 4 * W;  // value byte columns, then 8 + 8 quotient-estimate columns
    static_assert(NV + 16 <= tc::kCrtN, "value and estimate columns fill at most the 128 TMEM columns");
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sbase = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = sbase;                                        // [2][128][128 B]
    uint8_t* sB = sbase + 32768;                                // [2][128][128 B]
    uint32_t* sR = reinterpret_cast<uint32_t*>(sbase + 65536);  // [R][P][Gc]
    uint2* sTw = reinterpret_cast<uint2*>(sR + tc::kMaxPrimes * R * 8);  // [P][R-1]
    __shared__ uint64_t tma_bar, mma_bar;
    __shared__ uint32_t tmem_base;
    __shared__ __align__(16) uint32_t s_q[2 * W];
    __shared__ uint32_t s_p[tc::kMaxPrimes];                // the product's primes
    __shared__ uint2 s_sc[2 * tc::kMaxPrimes];              // its CRT scales s_i, then s_i psi_i^-brev(1)
    __shared__ uint64_t s_kf[2 * tc::kMaxPrimes + 1];       // floor(2^64 (row k of its k table) / q)

    const int tid = threadIdx.x, warp = tid >> 5;
    const int total = w.total();
    const int chunk = (total + int(gridDim.x) - 1) / int(gridDim.x);
    const int begin = int(blockIdx.x) * chunk;
    const int end = min(total, begin + chunk);

    for (int k = tid; k < 2048; k += tc::kCrtThreads) reinterpret_cast<uint4*>(sA)[k] = make_uint4(0, 0, 0, 0);
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

    auto issue = [&](int k) {
        const int2 it = w.item(k);
        const CrtTarget t = w.target(it.x);
        if (!t.use_tma) return;
        const int C = 1 << (LOGC ? LOGC : t.logC), Gc = C < 8 ? C : 8;
        tc::mbar_expect_tx(&tma_bar, uint32_t(tc::kMaxPrimes * R * Gc) * 4u);  // the whole box, absent primes zero-filled
        tc::tma_load_4d(sR, t.map, it.y * Gc, 0, 0, t.mz, &tma_bar);
    };
    if (tid == 0 && begin < end) issue(begin);

    const uint8_t* cur_w = nullptr;  // the product whose tables are in shared memory
    int cur_P = 0;
    uint32_t tma_phase = 0, mma_phase = 0;
    bool ok = true;
    for (int k = begin; k < end; ++k) {
        const int2 it = w.item(k);
        const CrtTarget t = w.target(it.x);
        const int logC = LOGC ? LOGC : t.logC;
        const int C = 1 << logC, Gc = C < 8 ? C : 8;
        const int cg = it.y;
        if (t.crt_w != cur_w || t.P != cur_P) {  // the previous item's MMA is complete: B may be rewritten
            const uint4* src = reinterpret_cast<const uint4*>(t.crt_w);
            for (int q = tid; q < 2048; q += tc::kCrtThreads) reinterpret_cast<uint4*>(sB)[q] = __ldg(src + q);
            for (int q = tid; q < 2 * W; q += tc::kCrtThreads) s_q[q] = t.consts[q];
            for (int q = tid; q <= 2 * t.P; q += tc::kCrtThreads) s_kf[q] = __ldg(t.kfrac + q);
            for (int q = tid; q < t.P; q += tc::kCrtThreads) {
                s_p[q] = __ldg(&pcs[q].p);
                s_sc[q] = __ldg(t.scale + q);
                s_sc[tc::kMaxPrimes + q] = __ldg(t.scale + t.P + q);
            }
            if (R > 1)
                for (int q = tid; q < t.P * RT; q += tc::kCrtThreads)
                    sTw[q] = __ldg(tw_inv + size_t(q / RT) * kNMax + 1 + q % RT);
            if (t.P != cur_P)  // K columns of absent primes must read as zero
                for (int q = tid; q < 2048; q += tc::kCrtThreads) reinterpret_cast<uint4*>(sA)[q] = make_uint4(0, 0, 0, 0);
            cur_w = t.crt_w;
            cur_P = t.P;
            tc::fence_smem_async();
            __syncthreads();
        }
        if (t.use_tma) {
            ok = tc::mbar_wait(&tma_bar, tma_phase) && ok;
            tma_phase ^= 1;
        } else {
            const int box = t.P * R * Gc;
            for (int q = tid; q < box; q += tc::kCrtThreads) {
                const int c = q % Gc, i = (q / Gc) % t.P, r = q / (Gc * t.P);
                sR[(r * tc::kMaxPrimes + i) * Gc + c] = t.work[size_t(i) * t.n + (size_t(r) << t.logC) + size_t(cg) * Gc + c];
            }
            __syncthreads();
        }
        // --- inverse column stages and CRT digits into A ---
        const int pairs = t.P * Gc;
        // one (prime, column) pair; G is the tile's column count when known at compile time
        auto digits = [&](auto gconst, int pr) {
            constexpr int G = decltype(gconst)::value;
            const int gc = G ? G : Gc;
            const int i = G ? pr / G : pr / Gc, c = pr - i * gc;
            const uint32_t p = s_p[i], two_p = 2 * p;
            uint32_t v[R];
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = sR[(r * tc::kMaxPrimes + i) * gc + c];
            const uint2* tw = sTw + i * RT - 1;  // tw[k] = Psi_inv_rev[k], k >= 1
#pragma unroll
            for (int s = LOGR - 1; s >= 1; --s) {
                const int h = R >> (s + 1);
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (!(r & h)) gs_bfly(v[r], v[r + h], tw[(1 << s) + (r >> (LOGR - s))], p, two_p);
            }
            // last stage (one twiddle per prime) with the CRT scale s_i folded in:
            // x' = s_i (x + y), y' = s_i w (x - y); digits t_i in [0, 2p) (an extra p_i
            // adds P to the CRT sum and 1 to its nearest quotient, which cancel)
            const uint2 sc = s_sc[i];
            if constexpr (LOGR > 0) {
                const uint2 sw = s_sc[tc::kMaxPrimes + i];
#pragma unroll
                for (int r = 0; r < R / 2; ++r) {
                    const uint32_t x = v[r], y = v[r + R / 2];
                    v[r] = shoup_mul(x + y, sc, p);
                    v[r + R / 2] = shoup_mul(x - y + two_p, sw, p);
                }
            } else {
                v[0] = shoup_mul(v[0], sc, p);
            }
            const uint32_t ka = uint32_t(i) >> 5, kb = (4u * i) & 127u;
#pragma unroll
            for (int r = 0; r < R; ++r)
                *reinterpret_cast<uint32_t*>(sA + ka * 16384 + tc::sw128_offset(r * gc + c, kb)) = v[r];
        };
        if (Gc == 8) {
            for (int pr = tid; pr < pairs; pr += tc::kCrtThreads) digits(std::integral_constant<int, 8>{}, pr);
        } else {
            for (int pr = tid; pr < pairs; pr += tc::kCrtThreads) digits(std::integral_constant<int, 0>{}, pr);
        }
        tc::fence_smem_async();
        tc::fence_before();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after();
            // the residue box is free again: fetch the next item's during the MMA and epilogue
            if (k + 1 < end) issue(k + 1);
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
        // --- the CRT value of row m = tid (warps 0-3, the TMEM lane owners) ---
        if (warp < 4) {
            // The 16 estimate columns first.  Columns NV..NV+7 give sum t_i floor(2^64/p_i),
            // whose nearest integer over 2^64 is the CRT's k; columns NV+8..NV+15 give
            // sum byte_a(t_i) floor(2^64 w_ia / q), 2^64 V/q less under 2^-40 of a unit.
            // With G_k = floor(2^64 (row k) / q) added, the integer part Q is the quotient
            // of V + row k by q, or one less: V + row k - Q q lies in [0, 2q).
            uint32_t e[16];
            tc::tmem_ld16(taddr + NV, e);
            tc::tmem_wait_ld();
            uint64_t fs[4];  // four-column sums, below 2^48
#pragma unroll
            for (int u = 0; u < 4; ++u)
                fs[u] = uint64_t(e[4 * u] + (e[4 * u + 1] << 8)) + (uint64_t(e[4 * u + 2] + (e[4 * u + 3] << 8)) << 16);
            const uint64_t fk = fs[1] + (fs[0] >> 32);
            const uint32_t k = min(uint32_t(fk >> 32) + (uint32_t(fk) >> 31), uint32_t(2 * t.P));
            const uint64_t gk = s_kf[k];
            const uint64_t low = (fs[2] & 0xffffffffull) + (gk & 0xffffffffull);
            const uint32_t Q = uint32_t((fs[3] + (fs[2] >> 32) + (gk >> 32) + (low >> 32)) >> 32);
            const uint4* krow = reinterpret_cast<const uint4*>(t.ktab + size_t(k) * W);
            // Word j of the value columns gives lo_j = d_4j + 2^8 d_4j+1 and hi_j = d_4j+2 +
            // 2^8 d_4j+3 (column sums d <= 256 * 255^2, so both are below 2^32), and V is
            // sum_j lo_j 2^(32j) + sum_j hi_j 2^(32j+16).  Word j of the second sum is the
            // funnel shift of hi_j and hi_j-1, so V is one add-with-carry chain, run four
            // words per TMEM load.
            uint32_t acc[W + 2];
            uint32_t cy = 0, prev_hi = 0;
#pragma unroll
            for (int q2 = 0; q2 < (NV + 31) / 32; ++q2) {
                uint32_t d[2][16];
                tc::tmem_ld16(taddr + 32 * q2, d[0]);
                if (32 * q2 + 16 < NV) tc::tmem_ld16(taddr + 32 * q2 + 16, d[1]);
                tc::tmem_wait_ld();
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int j0 = 8 * q2 + 4 * h;  // first word of this load
                    if (j0 >= W) break;
                    uint32_t b[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const uint32_t lo = d[h][4 * u] + (d[h][4 * u + 1] << 8);
                        const uint32_t hi = d[h][4 * u + 2] + (d[h][4 * u + 3] << 8);
                        b[u] = __funnelshift_l(prev_hi, hi, 16);
                        acc[j0 + u] = lo;
                        prev_hi = hi;
                    }
                    add4_carry(acc[j0], acc[j0 + 1], acc[j0 + 2], acc[j0 + 3], b, cy);
                }
            }
            acc[W] = cy + (prev_hi >> 16);
            acc[W + 1] = 0;
            uint32_t row[W + 2];
#pragma unroll
            for (int u = 0; u < W / 4; ++u) {
                const uint4 x = __ldg(krow + u);
                row[4 * u] = x.x;
                row[4 * u + 1] = x.y;
                row[4 * u + 2] = x.z;
                row[4 * u + 3] = x.w;
            }
            row[W] = row[W + 1] = 0;
            mp_add<W + 2>(acc, row);
            // minus Q q: one W-word multiply-accumulate (Q < 2^16)
            uint32_t qw[W];
#pragma unroll
            for (int u = 0; u < W / 4; ++u) {
                const uint4 x = reinterpret_cast<const uint4*>(s_q)[u];
                qw[4 * u] = x.x;
                qw[4 * u + 1] = x.y;
                qw[4 * u + 2] = x.z;
                qw[4 * u + 3] = x.w;
            }
#pragma unroll
            for (int u = 0; u < W + 2; ++u) row[u] = 0;
            crt_mac<W>(row, Q, qw);
            mp_sub<W + 2>(acc, row);
            final_sub_q<W>(acc, s_q);
            const int rr = tid / Gc, cc = tid % Gc;
            if (rr < R) {
                const size_t J = (size_t(rr) << logC) + size_t(cg) * Gc + cc;
                store_coef<W>(acc, t.out + J * t.stride, t.stride);
            }
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

// shared-memory bytes the kernels above ask for
constexpr size_t k1t_smem_bytes() { return 1024 + 32768 + 8192 + 16 * kTS * 4; }
template <int LOGR>
constexpr size_t k3t_smem_bytes() {
    return 1024 + 65536 + size_t(tc::kMaxPrimes) * (1 << LOGR) * 8 * 4 +
           size_t(tc::kMaxPrimes) * ((1 << LOGR) > 1 ? (1 << LOGR) - 1 : 1) * 8;
}

}  // namespace pm
