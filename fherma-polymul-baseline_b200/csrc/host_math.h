// Host-side integer arithmetic for plan set-up (untimed): 32-bit modular
// helpers and little-endian multiprecision numbers of 32-bit words.
//
// Plays the role of the reference's wide_host.h and the helpers at the top of
// rns/host_setup.h:11-56, written for general odd moduli rather than the
// special form 2^868 - c.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace pm {

using Words = std::vector<uint32_t>;

inline uint32_t mulmod(uint32_t a, uint32_t b, uint32_t p) { return uint32_t(uint64_t(a) * b % p); }

inline uint32_t powmod(uint32_t a, uint64_t e, uint32_t p) {
    uint32_t r = 1 % p;
    while (e) {
        if (e & 1) r = mulmod(r, a, p);
        a = mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}

// Deterministic Miller-Rabin; bases 2, 3, 5, 7 are exact below 3.2e9.
inline bool is_prime32(uint32_t n) {
    if (n < 2) return false;
    for (uint32_t s : {2u, 3u, 5u, 7u, 11u, 13u}) {
        if (n == s) return true;
        if (n % s == 0) return false;
    }
    uint32_t d = n - 1;
    unsigned r = 0;
    while (!(d & 1)) {
        d >>= 1;
        ++r;
    }
    for (uint32_t base : {2u, 3u, 5u, 7u}) {
        uint32_t x = powmod(base, d, n);
        if (x == 1 || x == n - 1) continue;
        bool composite = true;
        for (unsigned i = 1; i < r && composite; ++i) {
            x = mulmod(x, x, n);
            if (x == n - 1) composite = false;
        }
        if (composite) return false;
    }
    return true;
}

inline uint32_t bit_reverse(uint32_t x, unsigned bits) {
    uint32_t r = 0;
    for (unsigned i = 0; i < bits; ++i) {
        r = (r << 1) | (x & 1);
        x >>= 1;
    }
    return r;
}

// Shoup companion floor(w * 2^32 / p) of a constant multiplier w < p.
inline uint32_t shoup_of(uint32_t w, uint32_t p) { return uint32_t((uint64_t(w) << 32) / p); }

inline unsigned bit_length(const Words& a) {
    for (size_t i = a.size(); i--;)
        if (a[i]) return unsigned(i * 32 + 32 - __builtin_clz(a[i]));
    return 0;
}

inline void trim(Words& a) {
    while (!a.empty() && a.back() == 0) a.pop_back();
}

inline int compare(const Words& a, const Words& b) {
    size_t n = a.size() > b.size() ? a.size() : b.size();
    for (size_t i = n; i--;) {
        uint32_t x = i < a.size() ? a[i] : 0, y = i < b.size() ? b[i] : 0;
        if (x != y) return x < y ? -1 : 1;
    }
    return 0;
}

// a - b, requires a >= b
inline Words subtract(const Words& a, const Words& b) {
    Words r(a.size());
    int64_t borrow = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        int64_t v = int64_t(a[i]) - (i < b.size() ? int64_t(b[i]) : 0) - borrow;
        borrow = v < 0;
        r[i] = uint32_t(v + (borrow << 32));
    }
    if (borrow) throw std::logic_error("multiprecision subtract underflow");
    return r;
}

inline Words multiply_small(const Words& a, uint32_t s) {
    Words r(a.size() + 1);
    uint64_t carry = 0;
    for (size_t i = 0; i < a.size(); ++i) {
        uint64_t v = uint64_t(a[i]) * s + carry;
        r[i] = uint32_t(v);
        carry = v >> 32;
    }
    r[a.size()] = uint32_t(carry);
    trim(r);
    return r;
}

inline uint32_t divide_small(Words& a, uint32_t d) {
    uint64_t rem = 0;
    for (size_t i = a.size(); i--;) {
        uint64_t v = (rem << 32) | a[i];
        a[i] = uint32_t(v / d);
        rem = v % d;
    }
    trim(a);
    return uint32_t(rem);
}

inline uint32_t mod_small(const Words& a, uint32_t p) {
    uint64_t rem = 0;
    for (size_t i = a.size(); i--;) rem = ((rem << 32) | a[i]) % p;
    return uint32_t(rem);
}

inline Words shift_left(const Words& a, unsigned bits) {
    Words r(a.size() + bits / 32 + 1, 0);
    unsigned w = bits / 32, b = bits % 32;
    for (size_t i = 0; i < a.size(); ++i) {
        r[i + w] |= a[i] << b;
        if (b) r[i + w + 1] |= a[i] >> (32 - b);
    }
    trim(r);
    return r;
}

// floor(x / q) and x mod q by binary long division (set-up only).
inline void divmod(const Words& x, const Words& q, Words* quotient, Words* remainder) {
    unsigned xb = bit_length(x);
    Words rem;
    Words quo((xb + 31) / 32 + 1, 0);
    for (unsigned bit = xb; bit--;) {
        rem = shift_left(rem, 1);
        if ((x[bit / 32] >> (bit % 32)) & 1) {
            if (rem.empty()) rem.push_back(0);
            rem[0] |= 1;
        }
        if (compare(rem, q) >= 0) {
            rem = subtract(rem, q);
            trim(rem);
            quo[bit / 32] |= 1u << (bit % 32);
        }
    }
    trim(quo);
    trim(rem);
    if (quotient) *quotient = quo;
    if (remainder) *remainder = rem;
}

inline Words mod(const Words& x, const Words& q) {
    Words r;
    divmod(x, q, nullptr, &r);
    return r;
}

inline Words padded(Words a, size_t n) {
    if (a.size() > n) throw std::logic_error("value wider than its slot");
    a.resize(n, 0);
    return a;
}

}  // namespace pm
