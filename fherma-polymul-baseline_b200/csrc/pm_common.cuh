// Constants and modular arithmetic shared by the device kernels and the host
// code that prepares their tables.
#pragma once

#include <cstdint>

namespace pm {

constexpr int kLogNMax = 16;
constexpr int kNMax = 1 << kLogNMax;  // largest ring dimension; twiddle tables are this long
constexpr int kPMax = 64;             // largest prime basis
constexpr int kWMax = 28;             // largest q in 32-bit words (896 bits)
constexpr int kPowWords = 32;         // rows of 2^(32k) mod p kept per prime

struct PrimeConst {
    uint32_t p;
    uint32_t two_p;
    uint32_t mu;    // floor(2^61 / p), p in (2^29, 2^30)
    uint32_t pinv;  // p^-1 mod 2^32 (Montgomery reduction)
    uint64_t recip; // floor(2^64 / p)
};

// x * w mod p up to one extra p: result in [0, 2p) for any 32-bit x.
// w = (value, floor(value * 2^32 / p)).
__device__ __forceinline__ uint32_t shoup_mul(uint32_t x, uint2 w, uint32_t p) {
    return x * w.x - __umulhi(x, w.y) * p;
}

// [0, 2m) -> [0, m); the unsigned min picks x - m exactly when it did not wrap.
__device__ __forceinline__ uint32_t csub(uint32_t x, uint32_t m) { return min(x, x - m); }

// x mod p up to two extra p, for x < 2^60: Barrett with mu = floor(2^61/p), whose
// quotient estimate is at most 2 below floor(x/p), without the two corrections --
// the result lies in [0, 3p), enough for a forward butterfly input.
__device__ __forceinline__ uint32_t reduce60_lazy(uint64_t x, uint32_t p, uint32_t mu) {
    const uint32_t q = uint32_t((uint64_t(uint32_t(x >> 29)) * mu) >> 32);
    return uint32_t(x) - q * p;
}

// (hi 2^16 + lo) mod p up to two extra p, for hi < 2^32 - 2^16, any 32-bit lo
// and m = floor(2^48 / p), without forming the 48-bit value: u = hi + (lo >> 16)
// is its top part, u 2^16 <= v < u 2^16 + 2^16, and q = floor(u m / 2^32)
// satisfies v/p - 2 - 2^16/p < q <= v/p, so v - q p lies in [0, 3p) and is
// exact in 32-bit arithmetic.
__device__ __forceinline__ uint32_t reduce48_lazy(uint32_t lo, uint32_t hi, uint32_t p, uint32_t m) {
    const uint32_t q = __umulhi(hi + (lo >> 16), m);
    return lo + (hi << 16) - q * p;
}

// x * y * 2^-32 mod p up to one extra p, for x, y in [0, 2p): result in (0, 2p).
// Montgomery reduction with m = lo(xy) p^-1: xy - m p is a multiple of 2^32 and,
// as xy < 4p^2 < p 2^32, (xy - m p) / 2^32 lies in (-p, p).
__device__ __forceinline__ uint32_t mont_mul(uint32_t x, uint32_t y, uint32_t p, uint32_t pinv) {
    const uint64_t t = uint64_t(x) * y;
    const uint32_t m = uint32_t(t) * pinv;
    return uint32_t(t >> 32) - __umulhi(m, p) + p;
}

// Forward Cooley-Tukey butterfly, Harvey lazy: x, y in [0, 4p) -> [0, 4p).
__device__ __forceinline__ void ct_bfly(uint32_t& x, uint32_t& y, uint2 w, uint32_t p, uint32_t two_p) {
    uint32_t xr = csub(x, two_p);
    uint32_t t = shoup_mul(y, w, p);
    x = xr + t;
    y = xr - t + two_p;
}

// Inverse Gentleman-Sande butterfly, Harvey lazy: x, y in [0, 2p) -> [0, 2p).
__device__ __forceinline__ void gs_bfly(uint32_t& x, uint32_t& y, uint2 w, uint32_t p, uint32_t two_p) {
    uint32_t s = x + y;
    uint32_t d = x - y + two_p;
    x = csub(s, two_p);
    y = shoup_mul(d, w, p);
}

// Shared-memory swizzle: index bits 5, 6, 7 and 8 flip the bank bits {0, 2},
// {1, 3}, {0, 1, 4} and {0, 2, 3, 4}.  Only bits 0..4 change, as a function of
// bits that do not, so it maps every aligned power-of-two range onto itself and
// is linear over GF(2).  With it the 32 lanes of a warp reach 32 distinct banks
// in every pass layout of the row kernels at C = 1024..4096, with 8 or 16
// values a thread (passes at stride 2^logd, and the closing pass at stride 1,
// whose per-access element bits sit in the low bits and need lane bits XORed
// into them).
__device__ __forceinline__ int swz(int idx) {
    const int x = (idx >> 5) & 3;
    return idx ^ x ^ (x << 2) ^ (((idx >> 7) & 1) * 19) ^ (((idx >> 8) & 1) * 29);
}

}  // namespace pm
