// K1W: tensor-core conversion + forward column stages, one coefficient tile
// through the whole prime basis at once.
//
// K1T (tensor_kernels.cuh) runs a tile once per group of 16 primes: its
// coefficient bytes stream in four times (L2 catches part of it) and each CTA
// keeps four worker warps.  Here a CTA keeps the conversion weights of all 64
// basis primes resident (B: 256 rows x 128 bytes, the four group images back
// to back, loaded once per launch), takes each A tile (128 coefficients x 128
// bytes) once, and issues four tcgen05.mma.cta_group::1.kind::i8 of M=128,
// N=256, K=32 into one 256-column TMEM accumulator:
//   D[m][4i+a] = sum_k x_k(m) * byte_a(2^(8k) mod p_i)   every entry < 128*255^2 < 2^23.
// Eight worker warps split the epilogue: warps w and w+4 share TMEM lanes
// 32(w%4).. and take primes 0-31 and 32-63 of those rows (tcgen05.ld of 16
// columns = 4 primes at a time -> lazy Barrett on hi 2^16 + lo -> residue in
// [0, 3p) -> transposed into shared memory), release the accumulator, then
// all 256 take (prime, column) pairs through the R forward column stages and
// store them to the residue planes.  The release lets the next tile's MMA run
// while the column stages of this one do.  A producer warp (warp 8) issues
// the TMA loads (two A buffers, 128-byte swizzle, no multicast) and the MMAs.
// Two CTAs fit on an SM (about 110 KB of shared memory and 256 TMEM columns
// each), so one CTA's MMA and loads overlap the other's epilogue as well.
//
// Work: items (product z, polynomial, column group cg); a tile holds
// coefficient r*C + Gc*cg + c in row m = r*Gc + c (Gc = min(C, 8)), as in K1T.
// Barriers: tma_full[2], mma_full, tmem_empty (256 arrivals), b_full.  Every
// wait is bounded; a wait that gives up stops the CTA, lets its copies land,
// frees the TMEM and sets the plan's error word.
#pragma once

#include "tensor_kernels.cuh"

namespace pm {

namespace tc {
constexpr int kWideThreads = 288;  // 8 worker warps + 1 producer warp
constexpr int kWideN = 256;        // accumulator columns: 64 primes x 4 bytes
}  // namespace tc

struct TileItem {
    int z, poly, cg;
};

// `count` products of one plan: items (z, poly, cg) numbered product-major; with
// poly_only = 0 or 1, the items of that polynomial alone (its conversion can start
// while the other polynomial is still arriving).
struct PlanTileWork {
    CUtensorMap map_a, map_b;
    uint32_t* work;
    size_t ws_bstride;
    int n, logC, P, count;
    int poly_only;  // -1: both polynomials
    __device__ int lg() const { return logC - min(logC, 3); }  // column groups per row = 2^lg
    __device__ int total() const { return count << (lg() + (poly_only < 0 ? 1 : 0)); }
    __device__ TileItem item(int k) const {
        const int g = lg();
        if (poly_only >= 0) return TileItem{k >> g, poly_only, k & ((1 << g) - 1)};
        return TileItem{k >> (g + 1), (k >> g) & 1, k & ((1 << g) - 1)};
    }
    __device__ ConvTarget target(int z, int poly) const {
        return ConvTarget{poly ? &map_b : &map_a, z, work + z * ws_bstride, n, logC, P};
    }
};

// Bytes a plan adds to each A row before the MMA (the quartic factorization's part
// boundaries inside a byte): column 112 + t takes byte[byte[t]] >> shift[t].
struct ByteFix {
    int count;
    int byte[3], shift[3];
};

constexpr int kTW = 136;  // transpose row stride (words): 4 primes of a warp's pairs 8 banks apart
constexpr size_t k1w_smem_bytes() { return 1024 + 32768 + 32768 + size_t(tc::kMaxPrimes) * kTW * 4; }

// LOGC > 0: every item's rows hold 2^LOGC values (a plan's launch at a common ring size),
// so row strides and plane offsets are constants; 0: read from the item.
template <int LOGR, class Work, int LOGC = 0>
__global__ void __launch_bounds__(tc::kWideThreads, 2) k1w_convert(const __grid_constant__ Work w,
                                                                    const PrimeConst* __restrict__ pcs,
                                                                    const uint8_t* __restrict__ conv_w,
                                                                    const uint2* __restrict__ tw_fwd,
                                                                    uint32_t* __restrict__ err, const ByteFix fix) {
    constexpr int R = 1 << LOGR;
    constexpr int RT = R > 1 ? R - 1 : 1;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sbase = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = sbase;                                             // 2 x (128 x 128 B)
    uint8_t* sB = sbase + 32768;                                     // 256 x 128 B
    uint32_t* sT = reinterpret_cast<uint32_t*>(sbase + 65536);      // [64][kTW] residues
    __shared__ uint64_t tma_full[2], mma_full, tmem_empty, b_full;
    __shared__ uint32_t tmem_base;
    __shared__ volatile uint32_t s_abort;
    __shared__ uint2 spm[tc::kMaxPrimes];          // p, floor(2^48 / p)
    __shared__ uint2 stw[tc::kMaxPrimes][RT];      // forward column twiddles of every prime

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int total = w.total();
    const int chunk = (total + int(gridDim.x) - 1) / int(gridDim.x);
    const int begin = min(total, int(blockIdx.x) * chunk);
    const int end = min(total, begin + chunk);
    const int P = w.P;

    for (int k = tid; k < 2048; k += tc::kWideThreads) reinterpret_cast<uint4*>(sA)[k] = make_uint4(0, 0, 0, 0);
    for (int i = tid; i < tc::kMaxPrimes; i += tc::kWideThreads) {
        const PrimeConst g = pcs[i];
        spm[i] = make_uint2(g.p, g.mu >> 13);  // floor(floor(2^61 / p) / 2^13) = floor(2^48 / p)
    }
    if (R > 1)
        for (int q = tid; q < P * RT; q += tc::kWideThreads)
            stw[q / RT][q % RT] = __ldg(tw_fwd + size_t(q / RT) * kNMax + 1 + q % RT);
    if (warp == 0) tc::tmem_alloc(&tmem_base, tc::kWideN);
    if (tid == 0) {
        for (int b = 0; b < 2; ++b) tc::mbar_init(&tma_full[b], 1);
        tc::mbar_init(&mma_full, 1);
        tc::mbar_init(&tmem_empty, 256);
        tc::mbar_init(&b_full, 1);
        s_abort = 0;
    }
    tc::fence_smem_async();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tbase = tmem_base;
    bool ok = true;

    if (warp == 8) {
        // ------------------------------ producer ------------------------------
        auto issue = [&](int k, int buf) {
            const TileItem it = w.item(k);
            const ConvTarget t = w.target(it.z, it.poly);
            const int C = 1 << (LOGC ? LOGC : t.logC), Gc = C < 8 ? C : 8;
            tc::mbar_expect_tx(&tma_full[buf], 128u * uint32_t(Gc) * uint32_t(R));
            tc::tma_load_4d(sA + buf * 16384, t.map, 0, it.cg * Gc, 0, t.mz, &tma_full[buf]);
        };
        auto wait = [&](uint64_t* bar, uint32_t parity) {
            const bool done = __all_sync(0xffffffffu, tc::mbar_wait(bar, parity));
            ok = ok && done;
            return done;
        };
        uint32_t ph_tma = 0, ph_mma = 0, ph_empty = 0, pending = 0;  // bit b: buffer b
        bool b_pending = false;
        if (lane == 0 && begin < end) {
            tc::mbar_expect_tx(&b_full, 32768u);
            tc::bulk_load(sB, conv_w, 32768u, &b_full);
            issue(begin, 0);
            if (begin + 1 < end) issue(begin + 1, 1);
        }
        if (begin < end) {
            b_pending = true;
            pending = 1u | (begin + 1 < end ? 2u : 0u);
            if (wait(&b_full, 0)) b_pending = false;
        }
        int kk = 0;
        for (int k = begin; k < end && ok; ++k, ++kk) {
            if (__any_sync(0xffffffffu, s_abort != 0)) break;  // a worker gave up a wait
            const int buf = kk & 1;
            if (!wait(&tma_full[buf], (ph_tma >> buf) & 1u)) break;
            ph_tma ^= 1u << buf;
            pending &= ~(1u << buf);
            if (kk >= 1) {  // the workers have read the previous tile's accumulator
                if (!wait(&tmem_empty, ph_empty)) break;
                ph_empty ^= 1u;
            }
            if (fix.count) {  // the plan's extra bytes, written by this warp, seen by the MMA
                uint8_t* tile = sA + buf * 16384;
                for (int m = lane; m < tc::kTileM; m += 32)
#pragma unroll
                    for (int t = 0; t < 3; ++t)  // constant indices: the parameter stays out of local memory
                        if (t < fix.count)
                            tile[tc::sw128_offset(m, 112 + t)] =
                                uint8_t(tile[tc::sw128_offset(m, fix.byte[t])] >> fix.shift[t]);
                tc::fence_smem_async();
                __syncwarp();
            }
            tc::fence_after();
            if (lane == 0) {
                const uint32_t a0 = tc::smem_u32(sA + buf * 16384), b0 = tc::smem_u32(sB);
                constexpr uint32_t idesc = tc::idesc_u8(tc::kTileM, tc::kWideN);
#pragma unroll
                for (int ks = 0; ks < 4; ++ks)
                    tc::mma_u8(tbase, tc::sw128_desc(a0 + 32 * ks), tc::sw128_desc(b0 + 32 * ks), idesc, ks > 0);
                tc::mma_commit(&mma_full);
            }
            __syncwarp();
            // the MMA has read its A tile: the buffer takes the item two ahead
            if (!wait(&mma_full, ph_mma)) break;
            ph_mma ^= 1u;
            if (k + 2 < end) {
                if (lane == 0) issue(k + 2, buf);
                pending |= 1u << buf;
            }
        }
        if (!ok) s_abort = 1;
        // copies requested but not consumed land before the CTA's shared memory goes away
        for (int b = 0; b < 2; ++b)
            if (pending & (1u << b)) tc::mbar_wait(&tma_full[b], (ph_tma >> b) & 1u);
        if (b_pending) tc::mbar_wait(&b_full, 0);
    } else {
        // ------------------------------ workers -------------------------------
        const int half = warp >> 2;  // primes 32*half .. 32*half + 31 of TMEM lanes 32(warp%4)..
        const int row = tid & 127;   // tile row m = this thread's TMEM lane
        const uint32_t taddr = tbase + (uint32_t(32 * (warp & 3)) << 16) + uint32_t(128 * half);
        const int ilo = 32 * half;
        uint32_t ph_mma = 0;
        for (int k = begin; k < end; ++k) {
            const TileItem it = w.item(k);
            const ConvTarget t = w.target(it.z, it.poly);
            const int logC = LOGC ? LOGC : t.logC;
            const int C = 1 << logC, Gc = C < 8 ? C : 8;
            const size_t n = LOGC ? size_t(1) << (LOGR + LOGC) : size_t(t.n);
            const int tP = t.P;  // this item's basis (at most the launch's P)
            const int ihi = min(tP, ilo + 32);
            ok = tc::mbar_wait(&mma_full, ph_mma) && ok;
            ph_mma ^= 1u;
            tc::fence_after();
            // --- residues of row m for this half's primes: hi 2^16 + lo, hi and lo below 2^31.01 ---
            // eight primes per wait: two 16-column loads in flight, their primes' constants
            // read from shared memory before the wait (the wait orders every memory access)
#pragma unroll
            for (int q8 = 0; q8 < 4; ++q8) {
                if (ilo + 8 * q8 >= ihi) break;  // warp-uniform
                uint2 pm[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) pm[u] = spm[ilo + 8 * q8 + u];
                uint32_t d[2][16];
                tc::tmem_ld16(taddr + 32 * q8, d[0]);
                tc::tmem_ld16(taddr + 32 * q8 + 16, d[1]);
                tc::tmem_wait_ld();
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int i = ilo + 8 * q8 + u;
                    const uint32_t* e = d[u >> 2] + 4 * (u & 3);
                    const uint32_t lo = e[0] + (e[1] << 8);
                    const uint32_t hi = e[2] + (e[3] << 8);
                    sT[i * kTW + row] = reduce48_lazy(lo, hi, pm[u].x, pm[u].y);  // [0, 3p): butterfly input
                }
            }
            tc::fence_before();
            tc::mbar_arrive(&tmem_empty);  // this thread's accumulator reads are complete
            tc::bar_sync(1, 256);
            // --- forward column stages of (prime, column) pairs, then the residue planes ---
            const int pairs = tP * Gc;
            for (int pr = tid; pr < pairs; pr += 256) {
                const int i = Gc == 8 ? pr >> 3 : pr / Gc, c = pr - i * Gc;
                const uint32_t p = spm[i].x, two_p = 2 * p;
                uint32_t v[R];
                const uint32_t* col = sT + i * kTW + c;
                if (Gc == 8) {
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
                        if (!(r & h)) ct_bfly(v[r], v[r + h], stw[i][(1 << s) + (r >> (LOGR - s)) - 1], p, two_p);
                }
                uint32_t* dst = t.res + (size_t(it.poly) * tP + i) * n + size_t(it.cg) * Gc + c;
                const size_t rowstride = size_t(1) << logC;
#pragma unroll
                for (int r = 0; r < R; ++r, dst += rowstride) *dst = v[r];
            }
            // sT is rewritten by the next item; a failed wait (or the producer's) ends the loop for all workers
            if (tc::bar_sync_or(1, 256, !ok || s_abort)) break;
        }
        if (!ok) s_abort = 1;
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after();
        tc::tmem_dealloc(tbase, tc::kWideN);
    }
    if (!ok) atomicOr(err, 1u);
}

}  // namespace pm
