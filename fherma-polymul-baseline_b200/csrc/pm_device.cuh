// The three fused passes of a negacyclic product, batched over products.
//
//   K1 convert_cols : wide coefficients -> residues mod every prime, then the
//                     first log2(R) forward NTT stages ("column" stages, whose
//                     butterflies span the R rows of an R x C view) done across
//                     the lanes of a warp.
//   K2 rows         : per (product, prime, row): the remaining forward stages of
//                     a and b in registers + shared memory, the pointwise
//                     product, and the first inverse stages -- one read of a, b
//                     and one write of the product per row.
//   K3 cols_crt     : the last inverse stages across warp lanes, the CRT digit
//                     t_i = r_i * N^-1 * (P/p_i)^-1, exact CRT accumulation,
//                     fixed-point nearest quotient and the reduction mod q.
//
// The reference runs the same algebra as nine kernels per product
// (rns/solve.cu:128-420: transpose_inputs, prepare_rns, reverse_rns,
// small_rns x2, fused_tail_rns x2, product_rns, reconstruct_rns).  Its
// psi-twist tables are replaced by psi-merged twiddles (research/
// negacyclic_order.py ordering), which need no twist pass and let one
// bit-reversed twiddle table per prime serve every N <= 65536 as a prefix.
//
// Lazy ranges (Harvey): forward values stay in [0, 4p), inverse values in
// [0, 2p); primes are below 2^30 so 4p fits a 32-bit word.
//
// Batch layout: product z reads a, b at io + z*io_bstride words, writes c
// there too, and owns the residue planes at work + z*ws_bstride words
// ([2][P][n] u32: plane 0 = a, then the product; plane 1 = b).
#pragma once

#include <cstdint>

#include "crt_mac.cuh"
#include "pm_common.cuh"

namespace pm {

// ---------------------------------------------------------------------------
// K1: conversion + forward column stages (plain SIMT conversion).
// grid (C/G, 2*count, prime groups), block R*G threads; thread (g, r) owns
// coefficient r*C + col0 + g.  Dynamic shared memory: ppc*W uint2 limb powers.
// ---------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(256) k1_convert_cols(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                                                       uint32_t* __restrict__ res, const PrimeConst* __restrict__ pcs,
                                                       const uint2* __restrict__ conv_pow,
                                                       const uint2* __restrict__ tw_fwd, int n, int logR, int logC,
                                                       int P, int stride, int ppc, size_t io_bstride,
                                                       size_t ws_bstride) {
    extern __shared__ uint2 s_pow[];
    __shared__ uint32_t tile[256];
    const int z = blockIdx.y >> 1, poly = blockIdx.y & 1;
    const int i0 = blockIdx.z * ppc;
    const int i1 = min(P, i0 + ppc);
    for (int k = threadIdx.x; k < (i1 - i0) * W; k += blockDim.x)
        s_pow[k] = __ldg(conv_pow + size_t(i0 + k / W) * kPowWords + k % W);
    const int R = 1 << logR;
    const int G = blockDim.x >> logR;
    const int r = threadIdx.x & (R - 1), g = threadIdx.x >> logR;
    const int col0 = blockIdx.x * G;
    const size_t J = (size_t(r) << logC) + col0 + g;
    const uint32_t* src = (poly ? b : a) + z * io_bstride + J * stride;
    uint32_t x[W];
#pragma unroll
    for (int k = 0; k < W; k += 2) {
        uint2 v = make_uint2(0, 0);
        if (k < stride) v = __ldg(reinterpret_cast<const uint2*>(src + k));
        x[k] = v.x;
        x[k + 1] = v.y;
    }
    const unsigned mask = blockDim.x >= 32 ? 0xffffffffu : ((1u << blockDim.x) - 1);
    uint32_t* dst = res + z * ws_bstride + size_t(poly) * P * n;
    const int t = threadIdx.x, tr = t / G, tg = t % G;
    __syncthreads();
    for (int i = i0; i < i1; ++i) {
        const PrimeConst pc = pcs[i];
        const uint2* cp = s_pow + (i - i0) * W;
        uint64_t acc = 0;
#pragma unroll
        for (int k = 0; k < W; ++k) acc += shoup_mul(x[k], cp[k], pc.p);
        uint32_t v = reduce60_lazy(acc, pc.p, pc.mu);  // [0, 3p): the column stages take [0, 4p)
        const uint2* tw = tw_fwd + size_t(i) * kNMax;
        for (int s = 0; s < logR; ++s) {
            const int bit = logR - 1 - s;
            const bool upper = (r >> bit) & 1;
            const uint2 w = __ldg(tw + (1 << s) + (r >> (logR - s)));
            const uint32_t send = upper ? shoup_mul(v, w, pc.p) : csub(v, pc.two_p);
            const uint32_t recv = __shfl_xor_sync(mask, send, 1 << bit);
            v = upper ? recv - send + pc.two_p : send + recv;
        }
        __syncthreads();
        tile[r * G + g] = v;
        __syncthreads();
        dst[size_t(i) * n + (size_t(tr) << logC) + col0 + tg] = tile[t];
    }
}

// ---------------------------------------------------------------------------
// K2: row stages.  Element mapping of a pass over stages s0..s0+K-1 of a row
// of C = 2^LOGC values, V = 2^LV values per thread (LV = 3, or 4 for the
// radix-16 passes of the persistent row kernel), T = C/V threads per row:
//   d = C >> (s0+K); for group m < V>>K: gid = pass_gid(tid, m), blk = gid / d,
//   o = gid % d; value l of the group sits at blk*(d<<K) + o + l*d.
// Twiddle of row stage s = s0+u for the value pair starting at l: the row-local
// table entry 2^s + blk*2^u + (l >> (K-u)), which holds
//   Psi_rev[(R + r) * 2^s + blk * 2^u + (l >> (K-u))].
//
// Warp-local exchanges (WL: passes of K = LV stages, T >= 32).  In such a pass
// (one group, gid = tid) with d <= 32, warp w's values are exactly the words
// [32V w, 32V (w + 1)) (the swizzle keeps bits 5 and up).  The closing pass of
// K < LV stages (d = 1) gets the same property by numbering its V>>K groups
// so that warp w owns gids [w 2^(LV+5-K), (w+1) 2^(LV+5-K)).  An exchange
// between two such passes is then a warp's own business: __syncwarp instead
// of a CTA barrier.
// ---------------------------------------------------------------------------
template <int K, bool WL, int LV = 3>
__device__ __forceinline__ int pass_gid(int tid, int T, int m) {
    if constexpr (WL && K < LV)
        return ((tid >> 5) << (LV + 5 - K)) + (m << 5) + (tid & 31);
    else
        return tid + T * m;
}

// true when a pass of K stages at stride d = 2^logd keeps each warp inside its 32V words
template <int K, bool WL, int LV = 3>
__host__ __device__ constexpr bool pass_warp_local(int logd) {
    return WL && (K == LV ? logd <= 5 : logd == 0);
}

template <int K, bool WL = false, int LV = 3>
__device__ __forceinline__ int pass_index(int tid, int T, int m, int l, int logd) {
    const int gid = pass_gid<K, WL, LV>(tid, T, m);
    const int blk = gid >> logd;
    const int o = gid & ((1 << logd) - 1);
    return (blk << (logd + K)) + o + (l << logd);
}

// A pass index is a disjoint OR of thread bits (blk, o) and element bits (l),
// and swz is linear over GF(2), so swz(idx) = swz(thread part) ^ swz(l << logd):
// one XOR with a constant per access.
template <int K, bool WL, int LV>
__device__ __forceinline__ int pass_thread_base(int tid, int T, int m, int logd) {
    const int gid = pass_gid<K, WL, LV>(tid, T, m);
    const int blk = gid >> logd;
    const int o = gid & ((1 << logd) - 1);
    return swz((blk << (logd + K)) | o);
}

template <int K, bool WL, int LV = 3>
__device__ __forceinline__ void pass_store(const uint32_t (&v)[1 << LV], uint32_t* s, int tid, int T, int logd) {
#pragma unroll
    for (int m = 0; m < ((1 << LV) >> K); ++m) {
        const int tb = pass_thread_base<K, WL, LV>(tid, T, m, logd);
#pragma unroll
        for (int l = 0; l < (1 << K); ++l) s[tb ^ swz(l << logd)] = v[(m << K) + l];
    }
}

template <int K, bool WL, int LV = 3>
__device__ __forceinline__ void pass_load(uint32_t (&v)[1 << LV], const uint32_t* s, int tid, int T, int logd) {
#pragma unroll
    for (int m = 0; m < ((1 << LV) >> K); ++m) {
        const int tb = pass_thread_base<K, WL, LV>(tid, T, m, logd);
#pragma unroll
        for (int l = 0; l < (1 << K); ++l) v[(m << K) + l] = s[tb ^ swz(l << logd)];
    }
}

template <int K, bool WL, int LV = 3>
__device__ __forceinline__ void pass_forward(uint32_t (&va)[1 << LV], uint32_t (&vb)[1 << LV], int tid, int T, int s0,
                                             int logd, const uint2* tw, uint32_t p, uint32_t two_p) {
#pragma unroll
    for (int m = 0; m < ((1 << LV) >> K); ++m) {
        const int blk = pass_gid<K, WL, LV>(tid, T, m) >> logd;
#pragma unroll
        for (int u = 0; u < K; ++u) {
            const int h = 1 << (K - 1 - u);
            const uint2* tws = tw + ((1 << (s0 + u)) + (blk << u));
#pragma unroll
            for (int l = 0; l < (1 << K); ++l) {
                if (l & h) continue;
                const uint2 w = tws[l >> (K - u)];
                ct_bfly(va[(m << K) + l], va[(m << K) + l + h], w, p, two_p);
                ct_bfly(vb[(m << K) + l], vb[(m << K) + l + h], w, p, two_p);
            }
        }
    }
}

template <int K, bool WL, int LV = 3>
__device__ __forceinline__ void pass_inverse(uint32_t (&v)[1 << LV], int tid, int T, int s0, int logd, const uint2* tw,
                                             uint32_t p, uint32_t two_p) {
#pragma unroll
    for (int m = 0; m < ((1 << LV) >> K); ++m) {
        const int blk = pass_gid<K, WL, LV>(tid, T, m) >> logd;
#pragma unroll
        for (int u = K - 1; u >= 0; --u) {
            const int h = 1 << (K - 1 - u);
            const uint2* tws = tw + ((1 << (s0 + u)) + (blk << u));
#pragma unroll
            for (int l = 0; l < (1 << K); ++l) {
                if (l & h) continue;
                gs_bfly(v[(m << K) + l], v[(m << K) + l + h], tws[l >> (K - u)], p, two_p);
            }
        }
    }
}

// The barrier after an exchange store: only the warp when both layouts keep it in its 32V words.
__device__ __forceinline__ void exchange_sync(bool warp_local) {
    if (warp_local)
        __syncwarp();
    else
        __syncthreads();
}

// The forward row stages of a and b, the pointwise product and the inverse row
// stages of one row, starting from the values a thread holds for the first pass
// (pass_index<KP, false, LV> with s0 = 0) and ending with the product in the
// same places.  sa, sb: 2C words of exchange space; stf, sti: the row's twiddles.
// Every exchange stores a thread's values back to the very words that thread
// loaded in the pass (so no barrier is needed before the store), then meets the
// others before the next pass loads its own layout.  after_last_load() runs on
// every thread once the last pass has loaded its values (sa and sb are not
// read again).
struct NoHook {
    __device__ void operator()() const {}
};

template <int LOGC, int KP, class Hook = NoHook, int LV = 3>
__device__ __forceinline__ void row_transform(uint32_t (&va)[1 << LV], uint32_t (&vb)[1 << LV], uint32_t* sa,
                                              uint32_t* sb, const uint2* stf, const uint2* sti, int tid,
                                              const PrimeConst& pc, Hook after_last_load = Hook{}) {
    constexpr int C = 1 << LOGC;
    constexpr int T = C >> LV;
    constexpr int NP = LOGC / KP;   // full passes
    constexpr int REM = LOGC % KP;  // stages of the closing pass
    constexpr bool WL = KP == LV && T >= 32;
    constexpr int KR = REM > 0 ? REM : KP;  // closing pass radix (unused when REM = 0)
    static_assert(KP <= LV, "a pass holds at most V values per group");
#pragma unroll
    for (int q = 0; q < NP; ++q) {
        const int s0 = KP * q, logd = LOGC - s0 - KP;
        if (q > 0) {
            pass_load<KP, WL, LV>(va, sa, tid, T, logd);
            pass_load<KP, WL, LV>(vb, sb, tid, T, logd);
        }
        pass_forward<KP, WL, LV>(va, vb, tid, T, s0, logd, stf, pc.p, pc.two_p);
        if (q + 1 < NP || REM) {
            pass_store<KP, WL, LV>(va, sa, tid, T, logd);
            pass_store<KP, WL, LV>(vb, sb, tid, T, logd);
            const bool next_local =
                q + 1 < NP ? pass_warp_local<KP, WL, LV>(logd - KP) : pass_warp_local<KR, WL, LV>(0);
            exchange_sync(pass_warp_local<KP, WL, LV>(logd) && next_local);
        }
    }
    if constexpr (REM > 0) {
        const int s0 = KP * NP, logd = 0;
        pass_load<REM, WL, LV>(va, sa, tid, T, logd);
        pass_load<REM, WL, LV>(vb, sb, tid, T, logd);
        pass_forward<REM, WL, LV>(va, vb, tid, T, s0, logd, stf, pc.p, pc.two_p);
    }
    // pointwise product in Montgomery form (a factor 2^-32 the CRT scale removes), in [0, 2p)
#pragma unroll
    for (int l = 0; l < (1 << LV); ++l)
        va[l] = mont_mul(csub(va[l], pc.two_p), csub(vb[l], pc.two_p), pc.p, pc.pinv);
    if constexpr (REM > 0) {
        const int s0 = KP * NP, logd = 0;
        pass_inverse<REM, WL, LV>(va, tid, T, s0, logd, sti, pc.p, pc.two_p);
        pass_store<REM, WL, LV>(va, sa, tid, T, logd);
        exchange_sync(pass_warp_local<REM, WL, LV>(0) && pass_warp_local<KP, WL, LV>(LOGC - KP * NP));
    }
#pragma unroll
    for (int q = NP - 1; q >= 0; --q) {
        const int s0 = KP * q, logd = LOGC - s0 - KP;
        if (q + 1 < NP || REM) pass_load<KP, WL, LV>(va, sa, tid, T, logd);
        if (q == 0) after_last_load();
        pass_inverse<KP, WL, LV>(va, tid, T, s0, logd, sti, pc.p, pc.two_p);
        if (q > 0) {
            pass_store<KP, WL, LV>(va, sa, tid, T, logd);
            exchange_sync(pass_warp_local<KP, WL, LV>(logd) && pass_warp_local<KP, WL, LV>(logd + KP));
        }
    }
}

constexpr int k2_threads(int logc) { return logc >= 12 ? 512 : (logc >= 11 ? 256 : 128); }
constexpr int k2_min_blocks(int logc) { return logc >= 12 ? 1 : (logc >= 11 ? 3 : 7); }

// Rows of C = 2^LOGC >= 8, passes of KP stages (radix 2^KP, KP = 2 or 3; the
// last forward pass takes the remaining LOGC % KP stages).  grid
// (R / rows_per_cta, P, count), block rows_per_cta * C/8.  Dynamic shared
// memory per row: C uint2 forward and C uint2 inverse twiddles, then 2C words
// of data.  The product overwrites the a plane in place.
// One row r of prime i of the residue planes at `res` ([2][P][n]); the calling
// CTA gives each row T = C/8 threads (sub = row slot in the CTA, tid = thread in
// the row) and 24*C bytes of dynamic shared memory per row slot.
template <int LOGC, int KP>
__device__ __forceinline__ void k2_row_body(uint32_t* __restrict__ res, const PrimeConst& pc,
                                            const uint2* __restrict__ tw_fwd, const uint2* __restrict__ tw_inv,
                                            int n, int logR, int P, int i, int r, int sub, int tid,
                                            int rows_per_cta) {
    constexpr int C = 1 << LOGC;
    constexpr int T = C / 8;
    static_assert(KP == 2 || KP == 3, "pass radix");
    extern __shared__ __align__(16) uint2 smem2[];
    const int R = 1 << logR;
    uint2* stf = smem2 + sub * 2 * C;
    uint2* sti = stf + C;
    uint32_t* sa = reinterpret_cast<uint32_t*>(smem2 + rows_per_cta * 2 * C) + sub * 2 * C;
    uint32_t* sb = sa + C;
    uint32_t* ga = res + size_t(i) * n + size_t(r) * C;
    const uint32_t* gb = res + size_t(P + i) * n + size_t(r) * C;
    constexpr int logd0 = LOGC - KP;  // first pass: s0 = 0

    uint32_t va[8], vb[8];
#pragma unroll
    for (int m = 0; m < (8 >> KP); ++m)
#pragma unroll
        for (int l = 0; l < (1 << KP); ++l) {
            const int idx = pass_index<KP>(tid, T, m, l, logd0);
            va[(m << KP) + l] = ga[idx];
            vb[(m << KP) + l] = gb[idx];
        }
    // this row's twiddles: local entry j = 2^s + i' holds Psi_rev[(R + r) 2^s + i']
    {
        const uint2* gf = tw_fwd + size_t(i) * kNMax;
        const uint2* gi = tw_inv + size_t(i) * kNMax;
        for (int j = tid; j < C; j += T) {
            if (j == 0) continue;
            const int s = 31 - __clz(j);
            const int gidx = ((R + r) << s) + (j - (1 << s));
            stf[j] = __ldg(gf + gidx);
            sti[j] = __ldg(gi + gidx);
        }
    }
    __syncthreads();
    row_transform<LOGC, KP>(va, vb, sa, sb, stf, sti, tid, pc);
#pragma unroll
    for (int m = 0; m < (8 >> KP); ++m)
#pragma unroll
        for (int l = 0; l < (1 << KP); ++l) ga[pass_index<KP>(tid, T, m, l, logd0)] = va[(m << KP) + l];
}

template <int LOGC, int KP>
__global__ void __launch_bounds__(k2_threads(LOGC), k2_min_blocks(LOGC))
    k2_rows(uint32_t* __restrict__ res, const PrimeConst* __restrict__ pcs, const uint2* __restrict__ tw_fwd,
            const uint2* __restrict__ tw_inv, int n, int logR, int P, size_t ws_bstride) {
    constexpr int T = (1 << LOGC) / 8;
    const int sub = threadIdx.x / T, tid = threadIdx.x % T;
    const int rows_per_cta = blockDim.x / T;
    const int i = blockIdx.y;
    k2_row_body<LOGC, KP>(res + blockIdx.z * ws_bstride, pcs[i], tw_fwd, tw_inv, n, logR, P, i,
                          blockIdx.x * rows_per_cta + sub, sub, tid, rows_per_cta);
}

// Rows of C <= 4 (N <= 128): one thread per row, everything in registers.
// grid ((R+31)/32, P, count).
static __global__ void k2_rows_small(uint32_t* __restrict__ res, const PrimeConst* __restrict__ pcs,
                              const uint2* __restrict__ tw_fwd, const uint2* __restrict__ tw_inv, int n, int logR,
                              int logC, int P, size_t ws_bstride) {
    const int R = 1 << logR, C = 1 << logC;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (r >= R) return;
    const PrimeConst pc = pcs[i];
    res += blockIdx.z * ws_bstride;
    uint32_t* ga = res + size_t(i) * n + size_t(r) * C;
    const uint32_t* gb = res + size_t(P + i) * n + size_t(r) * C;
    const uint2* twf = tw_fwd + size_t(i) * kNMax;
    const uint2* twi = tw_inv + size_t(i) * kNMax;
    uint32_t va[4], vb[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        va[j] = j < C ? ga[j] : 0;
        vb[j] = j < C ? gb[j] : 0;
    }
    for (int s = 0; s < logC; ++s) {
        const int t = C >> (s + 1);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (j < C && !(j & t)) {
                const uint2 w = twf[((R + r) << s) + (j >> (logC - s))];
                // register indices must be compile-time; select the partner explicitly
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (k == j + t) {
                        ct_bfly(va[j], va[k], w, pc.p, pc.two_p);
                        ct_bfly(vb[j], vb[k], w, pc.p, pc.two_p);
                    }
            }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) va[j] = mont_mul(csub(va[j], pc.two_p), csub(vb[j], pc.two_p), pc.p, pc.pinv);
    for (int s = logC - 1; s >= 0; --s) {
        const int t = C >> (s + 1);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (j < C && !(j & t)) {
                const uint2 w = twi[((R + r) << s) + (j >> (logC - s))];
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (k == j + t) gs_bfly(va[j], va[k], w, pc.p, pc.two_p);
            }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (j < C) ga[j] = va[j];
}

// ---------------------------------------------------------------------------
// Multiprecision tail of the CRT, per coefficient, all in registers, with the
// carry-chain helpers of crt_mac.cuh.
// v (W+2 words) mod q, v < 2^(sbits+37); q has sbits bits and at most W words
// (W is its word count rounded up to a multiple of 4, so sbits > 32(W-4));
// mu_q = floor(2^(sbits+62) / q).  Leaves the canonical residue in v[0..W).
// ---------------------------------------------------------------------------
template <int W>
__device__ __forceinline__ void reduce_mod_q(uint32_t (&v)[W + 2], const uint32_t* __restrict__ q, uint64_t mu_q,
                                             int sbits) {
    // X = floor(v / 2^(sbits-26)) < 2^63; only words W-5 .. W+1 can hold it
    const int sh = sbits - 26;
    uint64_t X = 0;
#pragma unroll
    for (int k = (W >= 5 ? W - 5 : 0); k < W + 2; ++k) {
        const int pos = 32 * k - sh;  // bit position of word k inside X
        if (pos > -32 && pos < 64) X |= pos >= 0 ? uint64_t(v[k]) << pos : uint64_t(v[k]) >> (-pos);
    }
    // Q = floor(X mu_q / 2^88) <= v / q, and v/q - X mu_q / 2^88 is below
    // 2^(sbits+62) / q / 2^88 (the floor in X; q > 2^(sbits-1)) + X / 2^88 (the
    // floor in mu_q), each under 2^-25: Q is at most 1 below floor(v / q)
    const uint64_t Q = __umul64hi(X, mu_q) >> 24;
    uint32_t qw[W];
#pragma unroll
    for (int k = 0; k < W; ++k) qw[k] = q[k];
    uint32_t t[W + 2], u[W + 2];
#pragma unroll
    for (int k = 0; k < W + 2; ++k) t[k] = u[k] = 0;
    crt_mac<W>(t, uint32_t(Q), qw);        // low 32 bits of Q times q
    crt_mac<W>(u, uint32_t(Q >> 32), qw);  // high bits (< 2^6) times q, subtracted one word up
    mp_sub<W + 2>(v, t);
    mp_sub_hi<W>(v, u);
    // [0, 2q) -> [0, q)
    uint32_t qq[W + 2];
#pragma unroll
    for (int k = 0; k < W + 2; ++k) qq[k] = k < W ? qw[k] : 0u;
    uint32_t d[W + 2];
#pragma unroll
    for (int k = 0; k < W + 2; ++k) d[k] = v[k];
    const uint32_t borrowed = mp_sub<W + 2>(d, qq);
#pragma unroll
    for (int k = 0; k < W + 2; ++k) v[k] = borrowed ? v[k] : d[k];
}

// v mod q for a special-form q = 2^k - delta (k = sbits >= 80, delta < 2^32;
// the reference's FHERMA modulus 2^868 - 11993087 is one): with v = hi 2^k + lo,
// v = lo + hi * delta (mod q), and lo + hi * delta < 2^k + 2^70 < 2q, so one
// conditional subtraction finishes.  Same contract as reduce_mod_q otherwise.
template <int W>
__device__ __forceinline__ void reduce_special(uint32_t (&v)[W + 2], const uint32_t* __restrict__ q, int k,
                                               uint32_t delta) {
    // hi = floor(v / 2^k) < 2^38 from words W-4 .. W+1; those words keep v mod 2^k
    uint64_t hi = 0;
#pragma unroll
    for (int j = (W >= 4 ? W - 4 : 0); j < W + 2; ++j) {
        const int pos = 32 * j - k;  // bit position of word j inside hi
        if (pos > -32 && pos < 64) hi |= pos >= 0 ? uint64_t(v[j]) << pos : uint64_t(v[j]) >> (-pos);
        if (32 * j >= k)
            v[j] = 0;
        else if (32 * j + 32 > k)
            v[j] &= (1u << (k - 32 * j)) - 1u;
    }
    const uint64_t p0 = uint64_t(uint32_t(hi)) * delta, p1 = (hi >> 32) * delta;
    const uint64_t mid = (p0 >> 32) + uint32_t(p1);
    mp_add3<W + 2>(v, uint32_t(p0), uint32_t(mid), uint32_t(p1 >> 32) + uint32_t(mid >> 32));
    uint32_t qq[W + 2], d[W + 2];
#pragma unroll
    for (int j = 0; j < W + 2; ++j) {
        qq[j] = j < W ? q[j] : 0u;
        d[j] = v[j];
    }
    const uint32_t borrowed = mp_sub<W + 2>(d, qq);
#pragma unroll
    for (int j = 0; j < W + 2; ++j) v[j] = borrowed ? v[j] : d[j];
}

// Reduction of the final CRT step: the general one, the special-form one, or
// the one delta selects at run time (kernels whose products may be either).
enum CrtReduction { kReduceGeneral = 0, kReduceSpecial = 1, kReduceEither = 2 };

// One output coefficient: v[0..W) and zero words up to its stride.
template <int W>
__device__ __forceinline__ void store_coef(const uint32_t (&v)[W + 2], uint32_t* dst, int stride) {
    if ((stride & 3) == 0 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
#pragma unroll
        for (int k = 0; k < W; k += 4)
            if (k < stride) *reinterpret_cast<uint4*>(dst + k) = make_uint4(v[k], v[k + 1], v[k + 2], v[k + 3]);
        for (int k = W; k < stride; k += 4) *reinterpret_cast<uint4*>(dst + k) = make_uint4(0, 0, 0, 0);
        return;
    }
#pragma unroll
    for (int k = 0; k < W; k += 2)
        if (k < stride) *reinterpret_cast<uint2*>(dst + k) = make_uint2(v[k], v[k + 1]);
    for (int k = W; k < stride; ++k) dst[k] = 0;
}

// v in [0, 2q) -> [0, q).  v >= q needs a non-zero word W or W+1, or top four words
// (W-4 .. W-1, which hold q's top non-zero word) at least q's: a four-word compare
// decides, and the full subtraction runs only then -- rarely, when the quotient
// estimate was one low.
template <int W>
__device__ __forceinline__ void final_sub_q(uint32_t (&v)[W + 2], const uint32_t* __restrict__ q) {
    static_assert(W >= 4 && W % 4 == 0, "q words come in fours");
    uint32_t borrow = 0;
    asm("sub.cc.u32 %0, %1, %5;\n\t"
        "subc.cc.u32 %0, %2, %6;\n\t"
        "subc.cc.u32 %0, %3, %7;\n\t"
        "subc.cc.u32 %0, %4, %8;\n\t"
        "subc.u32 %0, 0, 0;"
        : "+r"(borrow)
        : "r"(v[W - 4]), "r"(v[W - 3]), "r"(v[W - 2]), "r"(v[W - 1]), "r"(q[W - 4]), "r"(q[W - 3]), "r"(q[W - 2]),
          "r"(q[W - 1]));
    if ((v[W] | v[W + 1]) == 0 && borrow != 0) return;
    uint32_t qq[W + 2], d[W + 2];
#pragma unroll
    for (int k = 0; k < W + 2; ++k) {
        qq[k] = k < W ? q[k] : 0u;
        d[k] = v[k];
    }
    const uint32_t borrowed = mp_sub<W + 2>(d, qq);
#pragma unroll
    for (int k = 0; k < W + 2; ++k) v[k] = borrowed ? v[k] : d[k];
}

// Final CRT step shared by the SIMT and tensor paths: v += nearest *
// (-P mod q), reduce mod q, store one coefficient (stride words).  With ktab
// (rows k = 0 .. 2P of k (-P mod q) mod q, W words each, 16-byte aligned) the
// correction is one table row added instead of a W-word multiply-accumulate:
// the same value mod q, and below v + q, inside reduce_mod_q's range.
template <int W, int RED = kReduceEither>
__device__ __forceinline__ void crt_finish(uint32_t (&v)[W + 2], uint32_t nearest, const uint32_t* s_q,
                                           uint64_t mu_q, int sbits, uint32_t delta, uint32_t* dst, int stride,
                                           const uint32_t* __restrict__ ktab = nullptr) {
    if (ktab) {
        uint32_t row[W + 2];
        const uint4* r4 = reinterpret_cast<const uint4*>(ktab + size_t(nearest) * W);
#pragma unroll
        for (int k = 0; k < W / 4; ++k) {
            const uint4 x = __ldg(r4 + k);
            row[4 * k] = x.x;
            row[4 * k + 1] = x.y;
            row[4 * k + 2] = x.z;
            row[4 * k + 3] = x.w;
        }
        row[W] = row[W + 1] = 0;
        mp_add<W + 2>(v, row);
    } else {
        uint32_t pneg[W];
#pragma unroll
        for (int k = 0; k < W; ++k) pneg[k] = s_q[W + k];
        crt_mac<W>(v, nearest, pneg);
    }
    if constexpr (RED == kReduceSpecial) {
        reduce_special<W>(v, s_q, sbits, delta);
    } else if constexpr (RED == kReduceGeneral) {
        reduce_mod_q<W>(v, s_q, mu_q, sbits);
    } else {
        if (delta)
            reduce_special<W>(v, s_q, sbits, delta);
        else
            reduce_mod_q<W>(v, s_q, mu_q, sbits);
    }
    store_coef<W>(v, dst, stride);
}

// ---------------------------------------------------------------------------
// K3: inverse column stages + CRT (plain SIMT accumulation).
// grid (C/G, count), block R*G.  Dynamic shared memory: P*W words of
// (P/p_i) mod q rows, then P*R*G words holding every prime's residue tile,
// loaded up front so all loads are in flight at once.
// consts = q[W] followed by (-P mod q)[W].
// ---------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(256) k3_cols_crt(const uint32_t* __restrict__ res, uint32_t* __restrict__ out,
                                                   const PrimeConst* __restrict__ pcs,
                                                   const uint2* __restrict__ tw_inv, const uint2* __restrict__ scale,
                                                   const uint32_t* __restrict__ mq,
                                                   const uint32_t* __restrict__ consts,
                                                   const uint32_t* __restrict__ ktab, uint64_t mu_q, int sbits,
                                                   uint32_t delta, int n, int logR, int logC, int P, int stride,
                                                   size_t io_bstride,
                                                   size_t ws_bstride) {
    extern __shared__ uint32_t sm3[];
    __shared__ uint32_t s_q[2 * W];
    const int RG = blockDim.x;
    uint32_t* s_mq = sm3;
    uint32_t* tiles = sm3 + P * W;
    const int R = 1 << logR;
    const int G = blockDim.x >> logR;
    const int r = threadIdx.x & (R - 1), g = threadIdx.x >> logR;
    const int col0 = blockIdx.x * G;
    const int t = threadIdx.x, tr = t / G, tg = t % G;
    res += blockIdx.y * ws_bstride;
    out += blockIdx.y * io_bstride;
    for (int k = threadIdx.x; k < P * W; k += blockDim.x) s_mq[k] = mq[k];
    for (int k = threadIdx.x; k < 2 * W; k += blockDim.x) s_q[k] = consts[k];
    for (int i = 0; i < P; ++i) tiles[i * RG + t] = res[size_t(i) * n + (size_t(tr) << logC) + col0 + tg];
    __syncthreads();
    const unsigned mask = blockDim.x >= 32 ? 0xffffffffu : ((1u << blockDim.x) - 1);
    uint32_t acc[W + 2];
#pragma unroll
    for (int k = 0; k < W + 2; ++k) acc[k] = 0;
    uint64_t f0 = 0, f1 = 0;
    for (int i = 0; i < P; ++i) {
        uint32_t v = tiles[i * RG + r * G + g];
        const PrimeConst pc = pcs[i];
        const uint2* tw = tw_inv + size_t(i) * kNMax;
        for (int s = logR - 1; s >= 0; --s) {
            const int bit = logR - 1 - s;
            const bool upper = (r >> bit) & 1;
            const uint32_t other = __shfl_xor_sync(mask, v, 1 << bit);
            if (!upper) {
                v = csub(v + other, pc.two_p);
            } else {
                const uint2 w = __ldg(tw + (1 << s) + (r >> (logR - s)));
                v = shoup_mul(other - v + pc.two_p, w, pc.p);
            }
        }
        const uint32_t ti = csub(shoup_mul(v, __ldg(scale + i), pc.p), pc.p);
        uint32_t m[W];
#pragma unroll
        for (int k = 0; k < W; ++k) m[k] = s_mq[i * W + k];
        crt_mac<W>(acc, ti, m);
        f0 += uint64_t(ti) * uint32_t(pc.recip);
        f1 += uint64_t(ti) * uint32_t(pc.recip >> 32);
        if ((i & 3) == 3) {
            f1 += f0 >> 32;
            f0 &= 0xffffffffull;
        }
    }
    f1 += f0 >> 32;
    // nearest integer of sum t_i / p_i (the fraction is f1:f0 / 2^64)
    const uint32_t nearest = uint32_t((f1 + (1ull << 31)) >> 32);
    const size_t J = (size_t(r) << logC) + col0 + g;
    crt_finish<W>(acc, nearest, s_q, mu_q, sbits, delta, out + J * stride, stride, ktab);
}

}  // namespace pm
