// Direct wide-modulus NTT (PM_WIDE_NTT): the negacyclic product computed with
// the NTT taken modulo q itself, for a prime q = 1 (mod 2n) -- the reference's
// wide backend (solve.cu:357-520, cuPQC 868-bit Montgomery arithmetic), kept for
// comparison with the RNS method: every butterfly is a W-word Montgomery
// multiplication instead of 59 word-sized ones plus conversion and CRT.
//
// Per launch group of `count` products, on a workspace [count][2][n][W] u32:
//   to_mont    a, b -> Montgomery form (x R mod q, R = 2^(32W)), zero-extended to W words
//   ct_stage   log2(n) forward Cooley-Tukey stages on a and b (psi-merged, bit-reversed
//              twiddles Psi_rev[k] = psi^brev(k), the ordering of the RNS kernels)
//   pointwise  a <- a b
//   gs_stage   log2(n) inverse Gentleman-Sande stages on a
//   from_mont  c = a n^-1 (leaving Montgomery form), written with the caller's stride
// One butterfly (or coefficient) per thread; every value stays canonical in [0, q).
#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "../../include/polymul.h"
#include "crt_mac.cuh"
#include "host_math.h"
#include "pm_internal.h"

namespace pm {

// ---------------------------------------------------------------------------
// device arithmetic mod q on W-word values
// ---------------------------------------------------------------------------
namespace {

template <int W>
__device__ __forceinline__ void load_w(uint32_t (&v)[W], const uint32_t* p) {
#pragma unroll
    for (int k = 0; k < W; k += 4) {
        const uint4 t = *reinterpret_cast<const uint4*>(p + k);
        v[k] = t.x;
        v[k + 1] = t.y;
        v[k + 2] = t.z;
        v[k + 3] = t.w;
    }
}

template <int W>
__device__ __forceinline__ void store_w(uint32_t* p, const uint32_t (&v)[W]) {
#pragma unroll
    for (int k = 0; k < W; k += 4) *reinterpret_cast<uint4*>(p + k) = make_uint4(v[k], v[k + 1], v[k + 2], v[k + 3]);
}

// r = a b R^-1 mod q (coarsely integrated operand scanning); a, b < q < R
template <int W>
__device__ __forceinline__ void mont_mul_w(uint32_t (&r)[W], const uint32_t (&a)[W], const uint32_t (&b)[W],
                                           const uint32_t (&q)[W], uint32_t qinv) {
    uint32_t t[W + 2];
#pragma unroll
    for (int j = 0; j < W + 2; ++j) t[j] = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) {
        crt_mac<W>(t, a[i], b);
        const uint32_t m = t[0] * qinv;  // t + m q = 0 (mod 2^32)
        crt_mac<W>(t, m, q);
#pragma unroll
        for (int j = 0; j < W + 1; ++j) t[j] = t[j + 1];
        t[W + 1] = 0;
    }
    // t < 2q: one conditional subtraction
    uint32_t d[W];
#pragma unroll
    for (int j = 0; j < W; ++j) d[j] = t[j];
    const uint32_t borrow = mp_sub<W>(d, q);
    const bool take = t[W] != 0 || !borrow;
#pragma unroll
    for (int j = 0; j < W; ++j) r[j] = take ? d[j] : t[j];
}

template <int W>
__device__ __forceinline__ void add_mod_w(uint32_t (&r)[W], const uint32_t (&x)[W], const uint32_t (&y)[W],
                                          const uint32_t (&q)[W]) {
    uint32_t s[W], d[W];
#pragma unroll
    for (int j = 0; j < W; ++j) s[j] = x[j];
    const uint32_t carry = mp_add<W>(s, y);
#pragma unroll
    for (int j = 0; j < W; ++j) d[j] = s[j];
    const uint32_t borrow = mp_sub<W>(d, q);
    const bool take = carry || !borrow;
#pragma unroll
    for (int j = 0; j < W; ++j) r[j] = take ? d[j] : s[j];
}

template <int W>
__device__ __forceinline__ void sub_mod_w(uint32_t (&r)[W], const uint32_t (&x)[W], const uint32_t (&y)[W],
                                          const uint32_t (&q)[W]) {
    uint32_t d[W], e[W];
#pragma unroll
    for (int j = 0; j < W; ++j) d[j] = x[j];
    const uint32_t borrow = mp_sub<W>(d, y);
#pragma unroll
    for (int j = 0; j < W; ++j) e[j] = d[j];
    mp_add<W>(e, q);
#pragma unroll
    for (int j = 0; j < W; ++j) r[j] = borrow ? e[j] : d[j];
}

struct WideArgs {
    const uint32_t* q;    // [W]
    const uint32_t* r2;   // [W] R^2 mod q
    const uint32_t* ninv; // [W] n^-1 mod q (plain)
    uint32_t qinv;        // -q^-1 mod 2^32
    int n, logn;
};

template <int W>
__device__ __forceinline__ void load_q(uint32_t (&q)[W], const uint32_t* g) {
#pragma unroll
    for (int j = 0; j < W; ++j) q[j] = __ldg(g + j);
}

// grid (n/128, 2 count): z = 2 product + polynomial
template <int W>
__global__ void __launch_bounds__(128) wide_to_mont(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                                                    uint32_t* __restrict__ work, WideArgs w, int stride,
                                                    size_t io_bstride) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w.n) return;
    const int z = blockIdx.y >> 1, poly = blockIdx.y & 1;
    const uint32_t* src = (poly ? b : a) + size_t(z) * io_bstride + size_t(i) * stride;
    uint32_t x[W], q[W], r2[W], y[W];
#pragma unroll
    for (int k = 0; k < W; ++k) x[k] = k < stride ? src[k] : 0u;
    load_q<W>(q, w.q);
    load_q<W>(r2, w.r2);
    mont_mul_w<W>(y, x, r2, q, w.qinv);
    store_w<W>(work + (size_t(blockIdx.y) * w.n + i) * W, y);
}

// stage s of the forward transform on `planes` arrays of n values, grid (n/2/128, planes)
template <int W>
__global__ void __launch_bounds__(128) wide_ct_stage(uint32_t* __restrict__ x, const uint32_t* __restrict__ tw,
                                                     WideArgs w, int s, size_t pstride) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= w.n / 2) return;
    x += size_t(blockIdx.y) * pstride;
    const int lh = w.logn - 1 - s, h = 1 << lh;
    const int blk = j >> lh, off = j & (h - 1);
    const int i0 = (blk << (lh + 1)) + off, i1 = i0 + h;
    uint32_t q[W], u[W], v[W], wt[W], t[W];
    load_q<W>(q, w.q);
    load_w<W>(u, x + size_t(i0) * W);
    load_w<W>(v, x + size_t(i1) * W);
    load_w<W>(wt, tw + size_t((1 << s) + blk) * W);
    mont_mul_w<W>(t, v, wt, q, w.qinv);
    add_mod_w<W>(v, u, t, q);
    store_w<W>(x + size_t(i0) * W, v);
    sub_mod_w<W>(v, u, t, q);
    store_w<W>(x + size_t(i1) * W, v);
}

template <int W>
__global__ void __launch_bounds__(128) wide_gs_stage(uint32_t* __restrict__ x, const uint32_t* __restrict__ tw,
                                                     WideArgs w, int s, size_t pstride) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= w.n / 2) return;
    x += size_t(blockIdx.y) * pstride;
    const int lh = w.logn - 1 - s, h = 1 << lh;
    const int blk = j >> lh, off = j & (h - 1);
    const int i0 = (blk << (lh + 1)) + off, i1 = i0 + h;
    uint32_t q[W], u[W], v[W], wt[W], t[W];
    load_q<W>(q, w.q);
    load_w<W>(u, x + size_t(i0) * W);
    load_w<W>(v, x + size_t(i1) * W);
    load_w<W>(wt, tw + size_t((1 << s) + blk) * W);
    add_mod_w<W>(t, u, v, q);
    store_w<W>(x + size_t(i0) * W, t);
    sub_mod_w<W>(t, u, v, q);
    mont_mul_w<W>(u, t, wt, q, w.qinv);
    store_w<W>(x + size_t(i1) * W, u);
}

// a <- a b for each product (grid (n/128, count), product planes 2n W apart)
template <int W>
__global__ void __launch_bounds__(128) wide_pointwise(uint32_t* __restrict__ work, WideArgs w) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w.n) return;
    uint32_t* pa = work + (size_t(blockIdx.y) * 2 * w.n + i) * W;
    const uint32_t* pb = pa + size_t(w.n) * W;
    uint32_t q[W], x[W], y[W], r[W];
    load_q<W>(q, w.q);
    load_w<W>(x, pa);
    load_w<W>(y, pb);
    mont_mul_w<W>(r, x, y, q, w.qinv);
    store_w<W>(pa, r);
}

// c = a n^-1, out of Montgomery form, written with the caller's stride
template <int W>
__global__ void __launch_bounds__(128) wide_from_mont(const uint32_t* __restrict__ work, uint32_t* __restrict__ c,
                                                      WideArgs w, int stride, size_t io_bstride) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w.n) return;
    const int z = blockIdx.y;
    uint32_t q[W], x[W], ni[W], r[W];
    load_q<W>(q, w.q);
    load_q<W>(ni, w.ninv);
    load_w<W>(x, work + (size_t(z) * 2 * w.n + i) * W);
    mont_mul_w<W>(r, x, ni, q, w.qinv);
    uint32_t* dst = c + size_t(z) * io_bstride + size_t(i) * stride;
#pragma unroll
    for (int k = 0; k < W; ++k)
        if (k < stride) dst[k] = r[k];
    for (int k = W; k < stride; ++k) dst[k] = 0;
}

// ---------------------------------------------------------------------------
// host arithmetic: fixed-width Montgomery multiplication for the set-up
// ---------------------------------------------------------------------------
struct HostMont {
    int W = 0;
    Words q;  // W words
    uint32_t qinv = 0;
    Words r2;    // R^2 mod q
    Words one;   // R mod q (1 in Montgomery form)

    explicit HostMont(const Words& qq, int w) : W(w), q(padded(qq, size_t(w))) {
        uint32_t inv = q[0];
        for (int it = 0; it < 5; ++it) inv *= 2u - q[0] * inv;
        qinv = 0u - inv;
        Words rr(2 * size_t(W) + 1, 0);
        rr[2 * size_t(W)] = 1;
        r2 = padded(mod(rr, qq), size_t(W));
        one = mul(r2, unit());
    }
    Words unit() const {
        Words u(size_t(W), 0);
        u[0] = 1;
        return u;
    }
    Words mul(const Words& a, const Words& b) const {
        std::vector<uint32_t> t(size_t(W) + 2, 0);
        for (int i = 0; i < W; ++i) {
            uint64_t c = 0;
            for (int j = 0; j < W; ++j) {
                const uint64_t x = uint64_t(a[i]) * b[j] + t[j] + c;
                t[j] = uint32_t(x);
                c = x >> 32;
            }
            uint64_t x = uint64_t(t[W]) + c;
            t[W] = uint32_t(x);
            t[W + 1] += uint32_t(x >> 32);
            const uint32_t m = t[0] * qinv;
            c = 0;
            for (int j = 0; j < W; ++j) {
                x = uint64_t(m) * q[j] + t[j] + c;
                t[j] = uint32_t(x);
                c = x >> 32;
            }
            x = uint64_t(t[W]) + c;
            t[W] = uint32_t(x);
            t[W + 1] += uint32_t(x >> 32);
            for (int j = 0; j < W + 1; ++j) t[j] = t[j + 1];
            t[W + 1] = 0;
        }
        Words r(t.begin(), t.begin() + W);
        Words tt(t.begin(), t.begin() + W + 1);
        trim(tt);
        Words qq = q;
        trim(qq);
        if (compare(tt, qq) >= 0) r = padded(subtract(tt, qq), size_t(W));
        return r;
    }
    Words to_mont(const Words& x) const { return mul(padded(x, size_t(W)), r2); }
    Words from_mont(const Words& x) const {
        Words r = mul(x, unit());
        trim(r);
        return r;
    }
    // base^e (plain in, plain out)
    Words pow(const Words& base, const Words& e) const {
        const Words b = to_mont(base);
        Words r = one;
        for (int bit = int(bit_length(e)); bit--;) {
            r = mul(r, r);
            if ((e[bit / 32] >> (bit % 32)) & 1) r = mul(r, b);
        }
        return from_mont(r);
    }
};

Words shift_right(const Words& a, unsigned bits) {
    Words r;
    const unsigned w = bits / 32, b = bits % 32;
    for (size_t i = w; i < a.size(); ++i) {
        uint32_t v = a[i] >> b;
        if (b && i + 1 < a.size()) v |= a[i + 1] << (32 - b);
        r.push_back(v);
    }
    trim(r);
    return r;
}

bool is_one(const Words& x) {
    Words t = x;
    trim(t);
    return t.size() == 1 && t[0] == 1;
}

// Miller-Rabin with the first twelve prime bases (a set-up check, not a proof)
bool probably_prime(const Words& n, const HostMont& M) {
    Words nm1 = subtract(n, Words{1});
    trim(nm1);
    unsigned r = 0;
    while (r < bit_length(nm1) && !((nm1[r / 32] >> (r % 32)) & 1)) ++r;
    const Words d = shift_right(nm1, r);
    for (uint32_t a : {2u, 3u, 5u, 7u, 11u, 13u, 17u, 19u, 23u, 29u, 31u, 37u}) {
        Words x = M.pow(Words{a}, d);
        if (is_one(x) || compare(x, nm1) == 0) continue;
        bool witness = true;
        for (unsigned k = 1; k < r && witness; ++k) {
            x = M.from_mont(M.mul(M.to_mont(x), M.to_mont(x)));
            if (compare(x, nm1) == 0) witness = false;
        }
        if (witness) return false;
    }
    return true;
}

template <int W>
void launch_wide_w(const PlanCore& s, const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* work,
                   uint32_t count, cudaStream_t st) {
    const WideTables& T = *s.wide;
    WideArgs w{T.d_q, T.d_r2, T.d_ninv, T.qinv, int(s.n), int(s.logn)};
    const size_t io = size_t(s.n) * s.stride;
    const size_t plane = size_t(s.n) * W;
    const dim3 blk(128);
    const unsigned nb = (s.n + 127) / 128, hb = (s.n / 2 + 127) / 128;
    wide_to_mont<W><<<dim3(nb, 2 * count), blk, 0, st>>>(a, b, work, w, int(s.stride), io);
    for (uint32_t st_ = 0; st_ < s.logn; ++st_)
        wide_ct_stage<W><<<dim3(hb, 2 * count), blk, 0, st>>>(work, T.d_tw_fwd, w, int(st_), plane);
    wide_pointwise<W><<<dim3(nb, count), blk, 0, st>>>(work, w);
    for (int st_ = int(s.logn) - 1; st_ >= 0; --st_)
        wide_gs_stage<W><<<dim3(hb, count), blk, 0, st>>>(work, T.d_tw_inv, w, st_, 2 * plane);
    wide_from_mont<W><<<dim3(nb, count), blk, 0, st>>>(work, c, w, int(s.stride), io);
    cuda_check(cudaGetLastError(), "wide NTT launches");
    count_launches(3 + 2 * s.logn);
}

}  // namespace

WideTables::~WideTables() {
    cudaFree(d_q);
    cudaFree(d_r2);
    cudaFree(d_ninv);
    cudaFree(d_tw_fwd);
    cudaFree(d_tw_inv);
}

size_t wide_workspace_bytes(const PlanCore& s) { return size_t(2) * s.n * s.W * sizeof(uint32_t); }

void wide_init(PlanCore& s) {
    if (s.n < 2) throw Failure(PM_ERR_UNSUPPORTED, "wide NTT needs n >= 2");
    Words q = s.q;
    trim(q);
    if (q.empty() || !(q[0] & 1)) throw Failure(PM_ERR_UNSUPPORTED, "wide NTT needs an odd prime q");
    const HostMont M(q, int(s.W));
    // 2n | q - 1
    Words qm1 = subtract(q, Words{1});
    trim(qm1);
    for (unsigned bit = 0; bit <= s.logn; ++bit)
        if (bit >= bit_length(qm1) || ((qm1[bit / 32] >> (bit % 32)) & 1))
            throw Failure(PM_ERR_UNSUPPORTED, "wide NTT needs q = 1 (mod 2n)");
    if (!probably_prime(q, M)) throw Failure(PM_ERR_UNSUPPORTED, "wide NTT needs a prime q");
    // psi of order exactly 2n: g^((q-1)/2n) with psi^n = -1
    const Words e = shift_right(qm1, s.logn + 1);
    Words psi;
    for (uint32_t g = 2; g < 1000; ++g) {
        Words cand = M.pow(Words{g}, e);
        Words half = M.pow(cand, Words{s.n});
        if (compare(half, qm1) == 0) {
            psi = cand;
            break;
        }
    }
    if (psi.empty()) throw Failure(PM_ERR_UNSUPPORTED, "no 2n-th root of unity found");
    Words ipsi = M.pow(psi, subtract(Words{2 * s.n}, Words{1}));  // psi^(2n-1) = psi^-1
    // powers in Montgomery form, then the bit-reversed tables
    const size_t W = s.W;
    std::vector<uint32_t> fwd(size_t(s.n) * W), inv(size_t(s.n) * W);
    {
        const Words pm = M.to_mont(psi), ipm = M.to_mont(ipsi);
        Words p = M.one, ip = M.one;
        std::vector<Words> pw(s.n), ipw(s.n);
        for (uint32_t k = 0; k < s.n; ++k) {
            pw[k] = p;
            ipw[k] = ip;
            p = M.mul(p, pm);
            ip = M.mul(ip, ipm);
        }
        for (uint32_t k = 0; k < s.n; ++k) {
            const uint32_t rk = bit_reverse(k, s.logn);
            std::copy(pw[rk].begin(), pw[rk].end(), fwd.begin() + size_t(k) * W);
            std::copy(ipw[rk].begin(), ipw[rk].end(), inv.begin() + size_t(k) * W);
        }
    }
    // n^-1 = q - (q-1)/n
    const Words ninv = padded(subtract(q, shift_right(qm1, s.logn)), W);
    auto T = std::make_unique<WideTables>();
    T->qinv = M.qinv;
    auto up = [](uint32_t** d, const std::vector<uint32_t>& h, const char* what) {
        cuda_check(cudaMalloc(d, h.size() * 4), what);
        cuda_check(cudaMemcpy(*d, h.data(), h.size() * 4, cudaMemcpyHostToDevice), what);
    };
    up(&T->d_q, M.q, "wide NTT modulus");
    up(&T->d_r2, M.r2, "wide NTT R^2");
    up(&T->d_ninv, ninv, "wide NTT n^-1");
    up(&T->d_tw_fwd, fwd, "wide NTT forward twiddles");
    up(&T->d_tw_inv, inv, "wide NTT inverse twiddles");
    s.wide = std::move(T);
}

void launch_wide(const PlanCore& s, const uint32_t* a, const uint32_t* b, uint32_t* c, uint32_t* work,
                 uint32_t count, cudaStream_t st) {
    ProfileScope prof("wide_ntt", st);
    switch (s.W) {
        case 4: return launch_wide_w<4>(s, a, b, c, work, count, st);
        case 8: return launch_wide_w<8>(s, a, b, c, work, count, st);
        case 12: return launch_wide_w<12>(s, a, b, c, work, count, st);
        case 16: return launch_wide_w<16>(s, a, b, c, work, count, st);
        case 20: return launch_wide_w<20>(s, a, b, c, work, count, st);
        case 24: return launch_wide_w<24>(s, a, b, c, work, count, st);
        case 28: return launch_wide_w<28>(s, a, b, c, work, count, st);
        default: throw Failure(PM_ERR_UNSUPPORTED, "unsupported width for the wide NTT");
    }
}

}  // namespace pm
