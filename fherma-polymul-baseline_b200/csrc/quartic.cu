// The quartic factorization of the reference's best backend, for
// q = B^4 - delta, B = 2^bbits (quartic/host_setup.h:41-110 finds its basis and
// roots the same way; quartic/solve.cu evaluates, multiplies, interpolates and
// recombines).  With Y = B, a coefficient x = sum_m x_m Y^m (four parts of bbits
// bits) is a polynomial in Y, and a product mod (X^n + 1, q) is the product in
// Z[X, Y] / (X^n + 1, Y^4 - delta) evaluated at Y = B mod q.  Its four components
// c_m have |c_m| < n (1 + 3 delta) (B - 1)^2, so 16 primes p_i with delta a
// fourth power mod p_i carry them (P > 4 x that bound): modulo p_i, Y^4 - delta
// splits at Y = rho_ij = r_i iota_i^j (r_i^4 = delta, iota_i^2 = -1), giving
// four independent negacyclic products per prime -- 64 residue planes for the
// same kernels as the RNS method:
//   - conversion (K1W): x -> sum_m x_m rho_ij^m mod p_i in one contraction,
//     weights 2^s rho_ij^m for the byte at bit 8k = bbits m + s; a byte that
//     straddles a part boundary keeps its low bits in part m - 1 and its high
//     bits (copied into a spare column by the producer warp) move to part m;
//   - rows (K2P) unchanged, over 64 planes;
//   - K3Q interpolates the channels per prime and runs one CRT contraction over
//     (component, prime) with weights (P/p_i) 2^(bbits m) mod q.
#include <cuda_runtime.h>

#include <vector>

#include "../../include/polymul.h"
#include "pm_internal.h"
#include "tc_ptx.cuh"

namespace pm {

QuarticTables::~QuarticTables() {
    cudaFree(d_pc);
    cudaFree(d_tw_fwd);
    cudaFree(d_tw_inv);
    cudaFree(d_conv);
    cudaFree(d_crt);
    cudaFree(d_mix);
    cudaFree(d_ktab);
}

namespace {

constexpr size_t kQuarticBAtomBytes = 160 * 128;  // one 128-byte K atom of the K3Q weights (N = 160)

// a square root of a quadratic residue mod an odd prime (Tonelli-Shanks)
uint32_t sqrt_mod(uint32_t a, uint32_t p) {
    a %= p;
    if (a == 0) return 0;
    if (powmod(a, (p - 1) / 2, p) != 1) throw Failure(PM_ERR_UNSUPPORTED, "quartic: no square root");
    uint32_t odd = p - 1;
    unsigned order = 0;
    while (!(odd & 1)) {
        odd >>= 1;
        ++order;
    }
    uint32_t z = 2;
    while (powmod(z, (p - 1) / 2, p) != p - 1) ++z;
    uint32_t c = powmod(z, odd, p), x = powmod(a, (odd + 1) / 2, p), t = powmod(a, odd, p);
    while (t != 1) {
        unsigned i = 0;
        uint32_t u = t;
        while (u != 1) {
            u = mulmod(u, u, p);
            if (++i >= order) throw Failure(PM_ERR_UNSUPPORTED, "quartic: square root failed");
        }
        const uint32_t b = powmod(c, uint64_t(1) << (order - i - 1), p);
        x = mulmod(x, b, p);
        c = mulmod(b, b, p);
        t = mulmod(t, c, p);
        order = i;
    }
    return x;
}

Words small_words(uint64_t v) {
    Words w{uint32_t(v), uint32_t(v >> 32)};
    trim(w);
    return w;
}

Words pow2_words(unsigned e) {
    Words w(e / 32 + 1, 0);
    w[e / 32] = 1u << (e % 32);
    return w;
}

Words mul_words(const Words& a, const Words& b) {
    Words r(a.size() + b.size() + 1, 0);
    for (size_t i = 0; i < a.size(); ++i) {
        uint64_t carry = 0;
        for (size_t j = 0; j < b.size(); ++j) {
            const uint64_t t = uint64_t(a[i]) * b[j] + r[i + j] + carry;
            r[i + j] = uint32_t(t);
            carry = t >> 32;
        }
        for (size_t k = i + b.size(); carry; ++k) {
            const uint64_t t = uint64_t(r[k]) + carry;
            r[k] = uint32_t(t);
            carry = t >> 32;
        }
    }
    trim(r);
    return r;
}

template <class T>
T* upload_vec(const std::vector<T>& v, const char* what) {
    T* d = nullptr;
    cuda_check(cudaMalloc(&d, v.size() * sizeof(T)), what);
    cuda_check(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), what);
    return d;
}

}  // namespace

void quartic_init(PlanCore& s) {
    if (!(s.flags & PM_CONVERT_TENSOR)) throw Failure(PM_ERR_INVALID, "PM_QUARTIC runs on the tensor path only");
    if (s.coef_limbs != 14) throw Failure(PM_ERR_UNSUPPORTED, "PM_QUARTIC takes 14-limb coefficients");
    if (s.n < 64) throw Failure(PM_ERR_UNSUPPORTED, "PM_QUARTIC needs n >= 64");
    const unsigned k = s.qbits;
    if (s.W != 28 || k % 4) throw Failure(PM_ERR_UNSUPPORTED, "PM_QUARTIC needs q of 772..896 bits, a multiple of 4");
    const Words top = pow2_words(k);
    if (compare(s.q, top) >= 0) throw Failure(PM_ERR_UNSUPPORTED, "PM_QUARTIC: q above 2^bits");
    Words dw = subtract(top, s.q);
    trim(dw);
    if (dw.empty() || bit_length(dw) > 28) throw Failure(PM_ERR_UNSUPPORTED, "PM_QUARTIC needs q = 2^k - delta, 0 < delta < 2^28");
    const uint32_t delta = dw[0];
    auto Q = std::make_unique<QuarticTables>();
    Q->bbits = k / 4;
    const unsigned bbits = Q->bbits;

    // 16 primes p = 1 mod 2^17 below 2^30 with delta a fourth power mod p (quartic/host_setup.h:55-68)
    unsigned found = 0;
    Words P{1};
    for (uint64_t cand = (uint64_t(1) << 30) - (uint64_t(1) << 17) + 1; found < 16; cand -= uint64_t(1) << 17) {
        if (cand <= (uint64_t(1) << 29)) throw Failure(PM_ERR_UNSUPPORTED, "quartic prime search ran below 2^29");
        const uint32_t p = uint32_t(cand);
        if (is_prime32(p) && powmod(delta % p, (p - 1) / 4, p) == 1) {
            Q->primes[found++] = p;
            P = multiply_small(P, p);
        }
    }
    // P > 4 n (1 + 3 delta) (B - 1)^2: the components' magnitude with room for the nearest quotient
    {
        Words bm1 = subtract(pow2_words(bbits), Words{1});
        trim(bm1);
        Words bound = mul_words(bm1, bm1);
        bound = multiply_small(bound, s.n);
        bound = mul_words(bound, small_words(1 + 3ull * delta));
        bound = multiply_small(bound, 4);
        if (compare(P, bound) <= 0)
            throw Failure(PM_ERR_UNSUPPORTED, "PM_QUARTIC: 16 primes below 2^30 do not cover n (1 + 3 delta) B^2");
    }

    const int W = int(s.W);
    std::vector<PrimeConst> pc(64);
    std::vector<uint2> fwd(size_t(64) * kNMax), inv(size_t(64) * kNMax);
    std::vector<uint8_t> conv(4 * 8192, 0);
    std::vector<uint8_t> crt(2 * kQuarticBAtomBytes, 0);
    std::vector<uint2> mix(80);
    std::vector<uint32_t> ktab(size_t(4) * 33 * W, 0);
    // the straddling bytes: boundary bbits m inside byte b / 8 moves that byte's high bits
    Q->fix_count = 0;
    for (unsigned m = 1; m < 4; ++m) {
        const unsigned b = bbits * m;
        if (b % 8 == 0) continue;
        Q->fix_byte[Q->fix_count] = int(b / 8);
        Q->fix_shift[Q->fix_count] = int(b % 8);
        ++Q->fix_count;
    }
    for (int i = 0; i < 16; ++i) {
        const uint32_t p = Q->primes[i];
        const uint32_t r = sqrt_mod(sqrt_mod(delta, p), p);
        if (powmod(r, 4, p) != delta % p) throw Failure(PM_ERR_UNSUPPORTED, "quartic fourth root");
        const uint32_t iota = sqrt_mod(p - 1, p);
        twiddle_tables(p, fwd.data() + size_t(4 * i) * kNMax, inv.data() + size_t(4 * i) * kNMax);
        for (int j = 1; j < 4; ++j) {
            std::copy(fwd.begin() + size_t(4 * i) * kNMax, fwd.begin() + size_t(4 * i + 1) * kNMax,
                      fwd.begin() + size_t(4 * i + j) * kNMax);
            std::copy(inv.begin() + size_t(4 * i) * kNMax, inv.begin() + size_t(4 * i + 1) * kNMax,
                      inv.begin() + size_t(4 * i + j) * kNMax);
        }
        const uint32_t two_b = powmod(2, bbits, p);
        for (int j = 0; j < 4; ++j) {
            const int plane = 4 * i + j;
            pc[plane] = prime_const(p);
            const uint32_t rho = mulmod(r, powmod(iota, uint64_t(j), p), p);
            uint32_t rho_m[4] = {1, rho, mulmod(rho, rho, p), 0};
            rho_m[3] = mulmod(rho_m[2], rho, p);
            // conversion weights of plane (prime i, channel j): group plane / 16, rows 4 (plane % 16) + a
            auto put = [&](unsigned col, uint32_t wv) {
                for (int a = 0; a < 4; ++a)
                    conv[size_t(plane / 16) * 8192 + tc::sw128_offset(4 * (plane % 16) + a, col)] = uint8_t(wv >> (8 * a));
            };
            for (unsigned kb = 0; kb < 112; ++kb) {
                const unsigned m = 8 * kb / bbits;
                if (m >= 4) continue;  // bytes above the top part are zero in every coefficient below q
                const unsigned sh = 8 * kb - bbits * m;
                put(kb, mulmod(powmod(2, sh, p), rho_m[m], p));
            }
            for (int t = 0; t < Q->fix_count; ++t) {
                const unsigned m = (unsigned(Q->fix_byte[t]) * 8 + unsigned(Q->fix_shift[t])) / bbits;
                // the byte's high part was weighted 2^bbits rho^(m-1) with the byte; it belongs to rho^m
                const uint32_t wrong = mulmod(two_b, rho_m[m - 1], p);
                put(112u + unsigned(t), (rho_m[m] + p - wrong) % p);
            }
        }
        // CRT: s_i = 2^32 n^-1 (P/p_i)^-1, component scales s_i r^-m / 4
        Words Mi = P;
        divide_small(Mi, p);
        const uint32_t minv = powmod(mod_small(Mi, p), p - 2, p);
        const uint32_t ninv = powmod(s.n % p, p - 2, p);
        const uint32_t si = mulmod(mulmod(minv, ninv, p), uint32_t((uint64_t(1) << 32) % p), p);
        const uint32_t rinv = powmod(r, p - 2, p), inv4 = powmod(4, p - 2, p);
        const uint32_t iinv = powmod(iota, p - 2, p);
        mix[i] = make_uint2(iinv, shoup_of(iinv, p));
        uint32_t f = mulmod(si, inv4, p);
        for (int m = 0; m < 4; ++m) {
            mix[16 + 16 * m + i] = make_uint2(f, shoup_of(f, p));
            f = mulmod(f, rinv, p);
        }
        // CRT weight rows: K index 4 (16 m + i) + a; value bytes of ((P/p_i) 2^(bbits m) mod q) << 8a,
        // quotient bytes of floor(2^64 / p_i) << 8a in component m's group
        const uint64_t recip = uint64_t(((unsigned __int128)1 << 64) / p);
        const int NV = 4 * W + 4;
        for (int m = 0; m < 4; ++m) {
            const Words wm = mod(mul_words(Mi, pow2_words(bbits * m)), s.q);
            for (int a = 0; a < 4; ++a) {
                const Words sh = shift_left(wm, 8 * a);
                const unsigned kidx = 4 * (16 * m + i) + a, atom = kidx >> 7, kk = kidx & 127;
                for (int J = 0; J < NV; ++J) {
                    const uint32_t word = size_t(J / 4) < sh.size() ? sh[J / 4] : 0;
                    crt[atom * kQuarticBAtomBytes + tc::sw128_offset(J, kk)] = uint8_t(word >> (8 * (J % 4)));
                }
                const unsigned __int128 rs = (unsigned __int128)recip << (8 * a);
                for (int J = 0; J < 8; ++J)
                    crt[atom * kQuarticBAtomBytes + tc::sw128_offset(NV + 8 * m + J, kk)] = uint8_t(rs >> (8 * J));
            }
        }
    }
    // corrections k (-P 2^(bbits m)) mod q, k <= 32 (digits below 2 p_i, 16 primes)
    for (int m = 0; m < 4; ++m) {
        const Words pm = mod(mul_words(P, pow2_words(bbits * m)), s.q);
        Words neg = compare(pm, Words{}) == 0 ? Words{} : subtract(s.q, pm);
        trim(neg);
        for (unsigned kq = 1; kq <= 32; ++kq) {
            const Words row = padded(mod(multiply_small(neg, kq), s.q), size_t(W));
            std::copy(row.begin(), row.end(), ktab.begin() + (size_t(m) * 33 + kq) * W);
        }
    }
    Q->d_pc = upload_vec(pc, "quartic prime constants");
    Q->d_tw_fwd = upload_vec(fwd, "quartic forward twiddles");
    Q->d_tw_inv = upload_vec(inv, "quartic inverse twiddles");
    Q->d_conv = upload_vec(conv, "quartic conversion weights");
    Q->d_crt = upload_vec(crt, "quartic CRT weights");
    Q->d_mix = upload_vec(mix, "quartic interpolation constants");
    Q->d_ktab = upload_vec(ktab, "quartic CRT correction tables");
    s.quartic = std::move(Q);
    s.P = 64;
    s.delta = delta;  // q = 2^k - delta: the folding reduction mod q
}

}  // namespace pm
