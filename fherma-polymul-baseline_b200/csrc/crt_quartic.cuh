// K3Q: inverse column stages, the quartic channel interpolation and the CRT on
// the tensor cores, for the quartic factorization (q = B^4 - delta).
//
// The residue planes hold, for each of 16 primes p_i, four channels j: the
// product evaluated at Y = rho_ij = r_i iota_i^j (r_i^4 = delta, iota_i^2 = -1
// mod p_i).  Per coefficient and prime the four channels interpolate back to
// the four components c_m of the product in Z[X, Y] / (X^n + 1, Y^4 - delta)
// (quartic/solve.cu reconstructs them the same way before its CRT512):
//   c_m = (1/4) r_i^-m sum_j iota_i^-jm C_ij   (mod p_i),
// a 4-point inverse DFT (one butterfly level across thread pairs by warp
// shuffle, one in registers) and a scale that also carries the CRT factor
// s_i = 2^32 n^-1 (P/p_i)^-1.  One INT8 contraction then gives
//   c = sum_m 2^(bbits m) (sum_i t_mi (P/p_i) - k_m P)  mod q,
// with K = 4 components x 16 primes x 4 bytes = 256 and N = 160 columns: the
// value bytes of sum t_mi ((P/p_i) 2^(bbits m) mod q) (4W + 4 of them) and, per
// component, eight bytes of sum_i t_mi floor(2^64/p_i) for its nearest quotient
// k_m; the four corrections k_m (-P 2^(bbits m) mod q) come from tables.
//
// Block of 256 threads (as K3T): all eight warps run the digit phase, thread
// pair (2t, 2t+1) taking prime i and column c, channels (0, 1) and (2, 3);
// warps 0-3 (the TMEM lane owners) run the per-coefficient epilogue.
#pragma once

#include "tensor_kernels.cuh"

namespace pm {

namespace tc {
constexpr int kQuarticCrtN = 160;
constexpr int kQuarticBAtom = kQuarticCrtN * 128;  // bytes of one 128-byte K atom of B
}  // namespace tc

struct QuarticCrtWork {
    CUtensorMap map_res;       // the 64 planes of `count` workspaces (residue_map)
    uint32_t* out;
    size_t io_bstride;
    const uint32_t* consts;    // q[W], (-P mod q)[W]
    const uint32_t* ktab;      // [4][33][W]
    const uint8_t* crt_w;      // [2][160 rows][128 B]
    const uint2* mix;          // [16] iota^-1, then [4][16] component scales
    uint64_t mu_q;
    int sbits, n, logC, stride, count;
    uint32_t delta;
    __device__ int lg() const { return logC - min(logC, 3); }
    __device__ int total() const { return count << lg(); }
};

template <int LOGR>
constexpr size_t k3q_smem_bytes() {
    return 1024 + 32768 + 2 * tc::kQuarticBAtom + size_t(64) * (1 << LOGR) * 8 * 4 +
           size_t(16) * ((1 << LOGR) > 1 ? (1 << LOGR) - 1 : 1) * 8 + 80 * 8;
}

template <int LOGR, int W, int RED>
__global__ void __launch_bounds__(tc::kCrtThreads, 2) k3q_crt(const __grid_constant__ QuarticCrtWork w,
                                                               const PrimeConst* __restrict__ pcs,
                                                               const uint2* __restrict__ tw_inv,
                                                               uint32_t* __restrict__ err) {
    constexpr int R = 1 << LOGR;
    constexpr int RT = R > 1 ? R - 1 : 1;
    constexpr int NV = 4 * W + 4;  // value byte columns
    static_assert(NV + 32 <= tc::kQuarticCrtN, "value and quotient columns fit N");
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sbase = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = sbase;                                                        // [2][128][128 B]
    uint8_t* sB = sbase + 32768;                                                // [2][160][128 B]
    uint32_t* sR = reinterpret_cast<uint32_t*>(sB + 2 * tc::kQuarticBAtom);     // [R][64][Gc]
    uint2* sTw = reinterpret_cast<uint2*>(sR + 64 * R * 8);                     // [16][R-1]
    uint2* sMix = sTw + 16 * RT;                                                // [16] + [4][16]
    __shared__ uint64_t tma_bar, mma_bar;
    __shared__ uint32_t tmem_base;
    __shared__ uint32_t s_q[2 * W];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int total = w.total();
    const int chunk = (total + int(gridDim.x) - 1) / int(gridDim.x);
    const int begin = int(blockIdx.x) * chunk;
    const int end = min(total, begin + chunk);
    const int C = 1 << w.logC, Gc = C < 8 ? C : 8, lg = w.lg();

    for (int k = tid; k < 2048; k += tc::kCrtThreads) reinterpret_cast<uint4*>(sA)[k] = make_uint4(0, 0, 0, 0);
    for (int q = tid; q < 2 * tc::kQuarticBAtom / 16; q += tc::kCrtThreads)
        reinterpret_cast<uint4*>(sB)[q] = __ldg(reinterpret_cast<const uint4*>(w.crt_w) + q);
    for (int q = tid; q < 2 * W; q += tc::kCrtThreads) s_q[q] = w.consts[q];
    if (R > 1)
        for (int q = tid; q < 16 * RT; q += tc::kCrtThreads)
            sTw[q] = __ldg(tw_inv + size_t(4 * (q / RT)) * kNMax + 1 + q % RT);
    for (int q = tid; q < 80; q += tc::kCrtThreads) sMix[q] = __ldg(w.mix + q);
    if (warp == 0) tc::tmem_alloc(&tmem_base, 256);
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
        tc::mbar_expect_tx(&tma_bar, uint32_t(64 * R * Gc) * 4u);
        tc::tma_load_4d(sR, &w.map_res, (k & ((1 << lg) - 1)) * Gc, 0, 0, k >> lg, &tma_bar);
    };
    if (tid == 0 && begin < end) issue(begin);

    uint32_t tma_phase = 0, mma_phase = 0;
    bool ok = true;
    for (int k = begin; k < end; ++k) {
        const int z = k >> lg, cg = k & ((1 << lg) - 1);
        ok = tc::mbar_wait(&tma_bar, tma_phase) && ok;
        tma_phase ^= 1;
        // --- inverse column stages of channels (2 half, 2 half + 1), interpolation, digits ---
        const int tasks = 32 * Gc;  // (prime, column, half): whole warps
        for (int pr = tid; pr < tasks; pr += tc::kCrtThreads) {
            const int half = pr & 1, pc_ = pr >> 1;
            const int i = pc_ / Gc, c = pc_ - i * Gc;
            const uint32_t p = __ldg(&pcs[4 * i].p), two_p = 2 * p;
            const uint2* tw = sTw + i * RT - 1;  // tw[k] = Psi_inv_rev[k], k >= 1
            uint32_t v[2][R];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int plane = 4 * i + 2 * half + h;
#pragma unroll
                for (int r = 0; r < R; ++r) v[h][r] = sR[(r * 64 + plane) * Gc + c];
#pragma unroll
                for (int s = LOGR - 1; s >= 0; --s) {
                    const int hh = R >> (s + 1);
#pragma unroll
                    for (int r = 0; r < R; ++r)
                        if (!(r & hh)) gs_bfly(v[h][r], v[h][r + hh], tw[(1 << s) + (r >> (LOGR - s))], p, two_p);
                }
            }
            // channels in [0, 2p): half 0 holds C0, C1; half 1 holds C2, C3
            const uint2 iinv = sMix[i];
            const uint2 sa = sMix[16 + (half) * 16 + i], sb = sMix[16 + (half + 2) * 16 + i];
            const uint32_t ka = uint32_t(64 * half + 4 * i) >> 7, kba = uint32_t(64 * half + 4 * i) & 127u;
            const uint32_t kb2 = uint32_t(64 * (half + 2) + 4 * i) >> 7, kbb = uint32_t(64 * (half + 2) + 4 * i) & 127u;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                // first level: (C0, C2) -> E0, E1 on half 0; (C1, C3) -> O0, O1 on half 1
                const uint32_t mine = v[0][r], send = half ? v[0][r] : v[1][r];
                const uint32_t other = __shfl_xor_sync(0xffffffffu, send, 1);
                // half 0: x = C0, y = C2; half 1: x = C1 (other), y = C3 (own v[1])
                const uint32_t x = half ? other : mine, y = half ? v[1][r] : other;
                uint32_t e0 = csub(x + y, two_p);         // E0 or O0
                uint32_t e1 = x - y + two_p;              // in (0, 4p)
                e1 = half ? shoup_mul(e1, iinv, p) : csub(e1, two_p);  // O1 = iota^-1 (C1 - C3), or E1
                // second level: half 0 needs O0, half 1 needs E1
                const uint32_t got = __shfl_xor_sync(0xffffffffu, half ? e0 : e1, 1);
                // half 0: t0 = E0 + O0, t2 = E0 - O0; half 1: t1 = E1 + O1, t3 = E1 - O1
                const uint32_t u = half ? got : e0, wv = half ? e1 : got;
                const uint32_t ta = u + wv, tb = u - wv + two_p;  // [0, 4p)
                const uint32_t da = shoup_mul(ta, sa, p), db = shoup_mul(tb, sb, p);  // digits in [0, 2p)
                const uint32_t row = uint32_t(r * Gc + c);
                *reinterpret_cast<uint32_t*>(sA + ka * 16384 + tc::sw128_offset(row, kba)) = da;
                *reinterpret_cast<uint32_t*>(sA + kb2 * 16384 + tc::sw128_offset(row, kbb)) = db;
            }
        }
        tc::fence_smem_async();
        tc::fence_before();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after();
            if (k + 1 < end) issue(k + 1);  // the residue box is free again
            const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
            constexpr uint32_t idesc = tc::idesc_u8(tc::kTileM, tc::kQuarticCrtN);
#pragma unroll
            for (int ks = 0; ks < 8; ++ks) {
                const uint32_t ao = (ks >> 2) * 16384 + 32 * (ks & 3), bo = (ks >> 2) * tc::kQuarticBAtom + 32 * (ks & 3);
                tc::mma_u8(tbase, tc::sw128_desc(a0 + ao), tc::sw128_desc(b0 + bo), idesc, ks > 0);
            }
            tc::mma_commit(&mma_bar);
        }
        ok = tc::mbar_wait(&mma_bar, mma_phase) && ok;
        mma_phase ^= 1;
        tc::fence_after();
        if (warp < 4) {
            uint32_t acc[W + 2];
            uint64_t carry = 0;
            uint64_t fs[4][2] = {};
#pragma unroll
            for (int q = 0; q < tc::kQuarticCrtN / 16; ++q) {
                uint32_t d[16];
                tc::tmem_ld16(taddr + 16 * q, d);
                tc::tmem_wait_ld();
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int J = 16 * q + 4 * u;
                    const uint32_t lo = d[4 * u] + (d[4 * u + 1] << 8), hi = d[4 * u + 2] + (d[4 * u + 3] << 8);
                    const uint64_t s = uint64_t(lo) + (uint64_t(hi) << 16);
                    if (J < NV) {
                        const uint64_t x = s + carry;
                        acc[J / 4] = uint32_t(x);
                        carry = x >> 32;
                    } else if (J < NV + 32) {
                        fs[(J - NV) / 8][((J - NV) / 4) & 1] = s;
                    }
                }
            }
            acc[W + 1] = uint32_t(carry);
            uint32_t nearest[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const uint64_t f1 = fs[m][1] + (fs[m][0] >> 32);
                // digits below 2 p_i: the sum of t / p_i is below 32 (the clamp only guards the table)
                nearest[m] = min(uint32_t(f1 >> 32) + (uint32_t(f1) >> 31), 32u);
            }
            // three of the four corrections here, the fourth inside crt_finish
#pragma unroll
            for (int m = 1; m < 4; ++m) {
                uint32_t row[W + 2];
                const uint4* r4 = reinterpret_cast<const uint4*>(w.ktab + (size_t(m) * 33 + nearest[m]) * W);
#pragma unroll
                for (int q = 0; q < W / 4; ++q) {
                    const uint4 x = __ldg(r4 + q);
                    row[4 * q] = x.x;
                    row[4 * q + 1] = x.y;
                    row[4 * q + 2] = x.z;
                    row[4 * q + 3] = x.w;
                }
                row[W] = row[W + 1] = 0;
                mp_add<W + 2>(acc, row);
            }
            const int rr = tid / Gc, cc = tid % Gc;
            if (rr < R) {
                const size_t J = (size_t(rr) << w.logC) + size_t(cg) * Gc + cc;
                crt_finish<W, RED>(acc, nearest[0], s_q, w.mu_q, w.sbits, w.delta,
                                   w.out + size_t(z) * w.io_bstride + J * w.stride, w.stride, w.ktab);
            }
        }
        (void)lane;
        tc::fence_before();
        __syncthreads();
    }
    if (warp == 0) {
        tc::fence_after();
        tc::tmem_dealloc(tbase, 256);
    }
    if (!ok && tid == 0) atomicOr(err, 1u);
}

}  // namespace pm
