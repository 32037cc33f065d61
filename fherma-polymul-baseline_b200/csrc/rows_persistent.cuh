// K2P: the row stages of K2 as a persistent kernel.
//
// Work items are (prime i, row r, product z), numbered pair-major (all
// products of a (prime, row) pair in a row), so the items a CTA takes in a row
// share their twiddles.  A work source says how many items there are and
// where each one's rows live: PlanRowWork computes them for `count` products
// of one plan (pair = i * R + r, item = pair * count + z); a batch of products
// of one row size but different q reads them from a table.  Each CTA owns a contiguous range of
// items and, for each of them:
//   - stages the pair's 2C forward/inverse row twiddles with bulk copies, only
//     when the pair changes (once per pair instead of once per product);
//   - has the item's two rows (a and b, 4C bytes each) in shared memory already:
//     they were requested by bulk copy while the previous item was finishing;
//   - runs the same register/shared-memory passes as K2 (row_transform) on
//     them, using the data buffer itself as the exchange space; as soon as
//     every thread holds the values of the last pass, the buffer is free and
//     the next item's rows are requested into it, landing while this item's
//     last stages run and its product row is stored.
// One data buffer instead of two keeps a CTA at 48 KB (C = 2048), so four CTAs
// share an SM; at C = 4096, 96 KB and two.  One row per CTA, C >= 1024, with
// T = C/16 threads of 16 values (radix-16 passes, the default: two exchanges
// per direction instead of three, up to 128 registers a thread) or T = C/8
// threads of 8 values (radix 4 or 8, at most 64 registers).  Bulk copies need
// 16-byte aligned rows: the host launches this kernel only on 16-byte aligned
// workspaces.
//
// Dynamic shared memory: C uint2 forward and C uint2 inverse twiddles, one data
// buffer of 2C words, two mbarriers (data, twiddles): 24C + 16 B.
#pragma once

#include <cstdint>

#include "pm_device.cuh"
#include "tc_ptx.cuh"

namespace pm {

// One row item: prime i, row r, the row of a (C words) and the distance to b's.
struct RowItem {
    int i, r;
    uint32_t* a;
    size_t b_off;
};

struct PlanRowWork {
    uint32_t* res;  // residue planes of product 0; product z at res + z * ws_bstride
    size_t ws_bstride;
    int n, logR, logC, P, count;
    __device__ int total() const { return (P << logR) * count; }
    __device__ RowItem item(int k) const {
        const int pair = k / count, z = k - pair * count;
        const int i = pair >> logR, r = pair & ((1 << logR) - 1);
        return RowItem{i, r, res + size_t(z) * ws_bstride + size_t(i) * n + (size_t(r) << logC), size_t(P) * n};
    }
};

constexpr int k2p_min_blocks(int logc) { return logc >= 12 ? 2 : (logc >= 11 ? 4 : 8); }
// values a thread: 16 for radix-16 passes (KP = 4), else 8
constexpr int k2p_lv(int kp) { return kp == 4 ? 4 : 3; }
constexpr int k2p_threads(int logc, int kp) { return (1 << logc) >> k2p_lv(kp); }
constexpr size_t k2p_smem_bytes(int logc) { return (size_t(24) << logc) + 2 * sizeof(uint64_t); }

template <int LOGC, int KP, class Work>
__global__ void __launch_bounds__(k2p_threads(LOGC, KP), k2p_min_blocks(LOGC))
    k2p_rows(const __grid_constant__ Work w, const PrimeConst* __restrict__ pcs, const uint2* __restrict__ tw_fwd,
             const uint2* __restrict__ tw_inv, int logR, uint32_t* __restrict__ err) {
    constexpr int LV = k2p_lv(KP), V = 1 << LV;
    constexpr int C = 1 << LOGC, T = C >> LV;
    constexpr int logd0 = LOGC - KP;  // first pass: s0 = 0
    static_assert(LOGC >= 10, "one row per CTA needs C >= 1024");
    extern __shared__ __align__(16) uint2 smem2[];
    uint2* stf = smem2;
    uint2* sti = smem2 + C;
    uint32_t* sd = reinterpret_cast<uint32_t*>(smem2 + 2 * C);  // [2C] words
    uint64_t* bars = reinterpret_cast<uint64_t*>(sd + 2 * C);   // data, twiddles

    const int tid = threadIdx.x;
    const int R = 1 << logR;
    const int total = w.total();
    const int begin = int(int64_t(blockIdx.x) * total / gridDim.x);
    const int end = int(int64_t(blockIdx.x + 1) * total / gridDim.x);
    if (tid == 0) {
        tc::mbar_init(&bars[0], 1);
        tc::mbar_init(&bars[1], 1);
    }
    tc::fence_smem_async();
    __syncthreads();

    auto issue_rows = [&](int k) {
        const RowItem it = w.item(k);
        tc::mbar_expect_tx(&bars[0], 8u * C);
        tc::bulk_load(sd, it.a, 4u * C, &bars[0]);
        tc::bulk_load(sd + C, it.a + it.b_off, 4u * C, &bars[0]);
    };
    // every thread tracks the copies: bit b of `phases` is the parity of barrier
    // b's next completion, bit b of `pending` marks a copy not yet seen complete
    uint32_t phases = 0, pending = 0;
    bool ok = true;
    auto wait = [&](int b) {
        const bool done = tc::mbar_wait(&bars[b], (phases >> b) & 1u);
        if (done) {
            phases ^= 1u << b;
            pending &= ~(1u << b);
        }
        ok = ok && done;
    };
    if (begin < end) {
        if (tid == 0) issue_rows(begin);
        pending |= 1u;
    }
    int cur_pair = -1;
    PrimeConst pc{};
    for (int k = begin; k < end; ++k) {
        const RowItem it = w.item(k);
        const int i = it.i, r = it.r, pair = i * R + r;
        if (pair != cur_pair) {
            if (cur_pair >= 0) __syncthreads();  // every thread is done with the previous pair's twiddles
            if (tid == 0) {
                const uint2* gf = tw_fwd + size_t(i) * kNMax;
                const uint2* gi = tw_inv + size_t(i) * kNMax;
                // local entry j = 2^s + i' holds Psi_rev[(R + r) 2^s + i']; stage s > 0 is one
                // contiguous, 16-byte aligned run of 2^s entries, stage 0 a single entry
                tc::mbar_expect_tx(&bars[1], 16u * uint32_t(C - 2));
                for (int s = 1; s < LOGC; ++s) {
                    tc::bulk_load(stf + (1 << s), gf + (size_t(R + r) << s), 8u << s, &bars[1]);
                    tc::bulk_load(sti + (1 << s), gi + (size_t(R + r) << s), 8u << s, &bars[1]);
                }
                stf[1] = __ldg(gf + R + r);
                sti[1] = __ldg(gi + R + r);
            }
            pending |= 2u;
            pc = pcs[i];
            wait(1);
            __syncthreads();  // entry 1, written by thread 0
            cur_pair = pair;
        }
        wait(0);

        uint32_t* sa = sd;
        uint32_t* sb = sa + C;
        uint32_t va[V], vb[V];
#pragma unroll
        for (int m = 0; m < (V >> KP); ++m)
#pragma unroll
            for (int l = 0; l < (1 << KP); ++l) {
                const int idx = pass_index<KP, false, LV>(tid, T, m, l, logd0);
                va[(m << KP) + l] = sa[idx];
                vb[(m << KP) + l] = sb[idx];
            }
        // the rows arrived unswizzled and the exchanges store swizzled: every thread
        // has its values before any exchange store lands in this buffer (and a wait
        // that gave up on any thread stops them all here)
        if (__syncthreads_or(!ok)) break;
        // once every thread holds the last pass's values, the buffer takes the next item's rows
        auto hook = [&]() {
            tc::fence_smem_async();
            __syncthreads();
            if (k + 1 < end) {
                if (tid == 0) issue_rows(k + 1);
                pending |= 1u;
            }
        };
        row_transform<LOGC, KP, decltype(hook), LV>(va, vb, sa, sb, stf, sti, tid, pc, hook);
        uint32_t* ga = it.a;
#pragma unroll
        for (int m = 0; m < (V >> KP); ++m)
#pragma unroll
            for (int l = 0; l < (1 << KP); ++l) ga[pass_index<KP, false, LV>(tid, T, m, l, logd0)] = va[(m << KP) + l];
    }
    // after a wait gave up (and the loop stopped): copies already requested land
    // before the CTA's shared memory goes away; no new copies were requested
    if (tid == 0) {
        for (int b = 0; b < 2; ++b)
            if (pending & (1u << b)) tc::mbar_wait(&bars[b], (phases >> b) & 1u);
        if (!ok) atomicOr(err, 1u);
    }
}

}  // namespace pm
