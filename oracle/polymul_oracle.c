/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle for the negacyclic multiplier.
 *
 * Nothing in the product path links, loads or calls this file.  Only the tests,
 * the smoke check and the CPU-baseline leg of the benchmark use it, and there
 * only as the checker (or as the timed CPU port of the reference method).
 *
 * It restates, in plain C, the reference's RNS method for
 *     c = a * b  mod (X^N + 1, q)
 * from ilyausmanov2015/fherma-polymul-baseline:
 *   - prime basis, roots and CRT constants:   rns/host_setup.h:61-126
 *   - residue of a wide coefficient mod p:    rns/solve.cu:138-157
 *   - negacyclic CT forward / GS inverse with
 *     odd-root (psi-merged) bit-reversed twiddles: research/negacyclic_order.py:7-22
 *   - pointwise product:                      rns/solve.cu:327-333
 *   - CRT with fixed-point nearest quotient:  rns/solve.cu:336-420,
 *                                             research/validate_rns.py:80-89
 * The reference's final fold only works for q = 2^868 - c (rns/solve.cu:360-382);
 * this restatement reduces modulo any odd q instead, which agrees with the
 * fold wherever the fold applies.
 *
 * Two further independent checkers live here: a schoolbook negacyclic product
 * over multiprecision integers (tests/validate.py:39-44 defines it) and a
 * dump of the basis constants so they can be compared with the reference's
 * own rns::setup compiled from its header (oracle/ref_setup_dump.cpp).
 *
 * Coefficients are little-endian 32-bit words, `words` per coefficient (the
 * reference's N x L x u32 tensors, fherma.h:27-42; the same bytes as
 * N x (L/2) x u64).
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAX_PRIMES 96
#define ORC_MAX_WORDS 32 /* up to 1024-bit q */

typedef unsigned __int128 u128;

/* ---------------- small modular helpers ---------------- */
static uint32_t mulmod(uint32_t a, uint32_t b, uint32_t p) { return (uint32_t)((uint64_t)a * b % p); }
static uint32_t powmod(uint32_t a, uint64_t e, uint32_t p) {
    uint32_t r = 1 % p;
    while (e) {
        if (e & 1) r = mulmod(r, a, p);
        a = mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}
/* Deterministic Miller-Rabin for 32-bit n (bases 2,3,5,7 suffice below 3.2e9). */
static int is_prime32(uint32_t n) {
    if (n < 2) return 0;
    static const uint32_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (unsigned i = 0; i < sizeof small / sizeof small[0]; ++i) {
        if (n == small[i]) return 1;
        if (n % small[i] == 0) return 0;
    }
    uint32_t d = n - 1;
    unsigned s = 0;
    while (!(d & 1)) { d >>= 1; ++s; }
    static const uint32_t bases[] = {2, 3, 5, 7};
    for (unsigned i = 0; i < 4; ++i) {
        uint32_t x = powmod(bases[i], d, n);
        if (x == 1 || x == n - 1) continue;
        int composite = 1;
        for (unsigned r = 1; r < s; ++r) {
            x = mulmod(x, x, n);
            if (x == n - 1) { composite = 0; break; }
        }
        if (composite) return 0;
    }
    return 1;
}
static unsigned brev(unsigned x, unsigned bits) {
    unsigned r = 0;
    for (unsigned i = 0; i < bits; ++i) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

/* ---------------- multiprecision (little-endian u32 words) ---------------- */
static unsigned mp_bits(const uint32_t* a, unsigned n) {
    for (unsigned i = n; i--;)
        if (a[i]) return i * 32 + 32 - (unsigned)__builtin_clz(a[i]);
    return 0;
}
static int mp_cmp(const uint32_t* a, const uint32_t* b, unsigned n) {
    for (unsigned i = n; i--;)
        if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    return 0;
}
/* a -= b over n words, returns borrow */
static uint32_t mp_sub(uint32_t* a, const uint32_t* b, unsigned n) {
    uint64_t borrow = 0;
    for (unsigned i = 0; i < n; ++i) {
        uint64_t v = (uint64_t)a[i] - b[i] - borrow;
        a[i] = (uint32_t)v;
        borrow = (v >> 63) & 1;
    }
    return (uint32_t)borrow;
}
/* a += b*s over n words (a has n words; carry out returned) */
static uint32_t mp_addmul(uint32_t* a, const uint32_t* b, unsigned bn, uint32_t s, unsigned n) {
    uint64_t carry = 0;
    unsigned i = 0;
    for (; i < bn; ++i) {
        uint64_t v = (uint64_t)b[i] * s + a[i] + carry;
        a[i] = (uint32_t)v;
        carry = v >> 32;
    }
    for (; i < n && carry; ++i) {
        uint64_t v = (uint64_t)a[i] + carry;
        a[i] = (uint32_t)v;
        carry = v >> 32;
    }
    return (uint32_t)carry;
}
/* x (xn words) mod q (qn words) -> r (qn words).  Shift-subtract, one bit at a time. */
static void mp_mod(const uint32_t* x, unsigned xn, const uint32_t* q, unsigned qn, uint32_t* r) {
    uint32_t acc[ORC_MAX_WORDS + 1];
    memset(acc, 0, sizeof acc);
    uint32_t qq[ORC_MAX_WORDS + 1];
    memset(qq, 0, sizeof qq);
    memcpy(qq, q, qn * 4);
    for (unsigned bit = mp_bits(x, xn); bit--;) {
        /* acc = 2*acc + bit */
        uint32_t carry = (x[bit / 32] >> (bit % 32)) & 1;
        for (unsigned i = 0; i <= qn; ++i) {
            uint32_t next = acc[i] >> 31;
            acc[i] = (acc[i] << 1) | carry;
            carry = next;
        }
        if (mp_cmp(acc, qq, qn + 1) >= 0) mp_sub(acc, qq, qn + 1);
    }
    memcpy(r, acc, qn * 4);
}
static uint32_t mp_mod_small(const uint32_t* x, unsigned n, uint32_t p) {
    uint64_t r = 0;
    for (unsigned i = n; i--;) r = ((r << 32) | x[i]) % p;
    return (uint32_t)r;
}
/* exact division by a small d, returns remainder */
static uint32_t mp_div_small(uint32_t* x, unsigned n, uint32_t d) {
    uint64_t r = 0;
    for (unsigned i = n; i--;) {
        uint64_t v = (r << 32) | x[i];
        x[i] = (uint32_t)(v / d);
        r = v % d;
    }
    return (uint32_t)r;
}

/* ---------------- the prime basis ---------------- */
typedef struct {
    unsigned count;
    uint32_t p[ORC_MAX_PRIMES];
    uint32_t psi[ORC_MAX_PRIMES];        /* primitive 2n-th root */
    uint32_t crt_inv[ORC_MAX_PRIMES];    /* (P/p_i)^-1 mod p_i */
    uint64_t recip[ORC_MAX_PRIMES];      /* floor(2^64 / p_i) */
    uint32_t product[2 * ORC_MAX_PRIMES + 2]; /* P */
    unsigned product_words;
} orc_basis;

/*
 * Primes descend from the largest p < 2^bits with p = 1 mod order, step -order
 * (rns/host_setup.h:67-80 with bits=31, order=65536).  With count == 0 the
 * basis grows until P > 2^(2*qbits + 2 + log2 n), which covers the signed
 * negacyclic range 4*N*(q-1)^2 that rns/host_setup.h:81-83 demands.
 */
static int basis_make(orc_basis* B, unsigned n, unsigned qbits, unsigned bits, uint32_t order, unsigned count) {
    memset(B, 0, sizeof *B);
    B->product_words = 2 * ORC_MAX_PRIMES + 2;
    B->product[0] = 1;
    unsigned logn = 0;
    while ((1u << logn) < n) ++logn;
    unsigned need_bits = 2 * qbits + 2 + logn + 1; /* P >= 2^(need_bits-1) + 1  i.e. > 2^(2w+2+logn) */
    uint64_t cand = ((uint64_t)1 << bits) - order + 1;
    while (1) {
        if (count ? B->count == count : mp_bits(B->product, B->product_words) >= need_bits) break;
        if (B->count == ORC_MAX_PRIMES || cand < order) return -1;
        if (is_prime32((uint32_t)cand)) {
            uint32_t p = (uint32_t)cand;
            B->p[B->count++] = p;
            /* product *= p */
            uint64_t carry = 0;
            for (unsigned i = 0; i < B->product_words; ++i) {
                uint64_t v = (uint64_t)B->product[i] * p + carry;
                B->product[i] = (uint32_t)v;
                carry = v >> 32;
            }
        }
        cand -= order;
    }
    for (unsigned i = 0; i < B->count; ++i) {
        uint32_t p = B->p[i];
        /* psi: the first g = 2,3,... whose (p-1)/(2n) power has order exactly 2n
           (rns/host_setup.h:102-107) */
        B->psi[i] = 0;
        for (uint32_t g = 2; g < 100000; ++g) {
            uint32_t root = powmod(g, (p - 1) / (2 * (uint64_t)n), p);
            if (powmod(root, n, p) == p - 1) { B->psi[i] = root; break; }
        }
        if (!B->psi[i]) return -2;
        uint32_t m[2 * ORC_MAX_PRIMES + 2];
        memcpy(m, B->product, sizeof m);
        if (mp_div_small(m, B->product_words, p)) return -3;
        B->crt_inv[i] = powmod(mp_mod_small(m, B->product_words, p), p - 2, p);
        B->recip[i] = (uint64_t)((((u128)1) << 64) / p);
    }
    return 0;
}

/* ---------------- NTT (psi-merged negacyclic, exact arithmetic) ---------------- */
static void ntt_forward(uint32_t* a, unsigned n, uint32_t psi, uint32_t p) {
    unsigned logn = 0;
    while ((1u << logn) < n) ++logn;
    for (unsigned m = 1, t = n / 2; m < n; m *= 2, t /= 2)
        for (unsigned i = 0; i < m; ++i) {
            uint32_t w = powmod(psi, brev(m + i, logn), p);
            for (unsigned j = 2 * i * t; j < 2 * i * t + t; ++j) {
                uint32_t u = a[j], v = mulmod(a[j + t], w, p);
                a[j] = (uint32_t)(((uint64_t)u + v) % p);
                a[j + t] = (uint32_t)(((uint64_t)u + p - v) % p);
            }
        }
}
static void ntt_inverse(uint32_t* a, unsigned n, uint32_t psi, uint32_t p) {
    unsigned logn = 0;
    while ((1u << logn) < n) ++logn;
    uint32_t ipsi = powmod(psi, p - 2, p);
    for (unsigned m = n / 2, t = 1; m >= 1; m /= 2, t *= 2)
        for (unsigned i = 0; i < m; ++i) {
            uint32_t w = powmod(ipsi, brev(m + i, logn), p);
            for (unsigned j = 2 * i * t; j < 2 * i * t + t; ++j) {
                uint32_t u = a[j], v = a[j + t];
                a[j] = (uint32_t)(((uint64_t)u + v) % p);
                a[j + t] = mulmod((uint32_t)(((uint64_t)u + p - v) % p), w, p);
            }
        }
    uint32_t ninv = powmod(n % p, p - 2, p);
    for (unsigned j = 0; j < n; ++j) a[j] = mulmod(a[j], ninv, p);
}

/* ---------------- threaded per-prime work ---------------- */
typedef struct {
    const orc_basis* B;
    unsigned n, words;
    const uint32_t *a, *b;
    uint32_t* t; /* [count][n] CRT digits */
    unsigned next;
    pthread_mutex_t lock;
} prime_job;

static void* prime_worker(void* arg) {
    prime_job* J = (prime_job*)arg;
    uint32_t* x = (uint32_t*)malloc((size_t)J->n * 4);
    uint32_t* y = (uint32_t*)malloc((size_t)J->n * 4);
    for (;;) {
        pthread_mutex_lock(&J->lock);
        unsigned i = J->next++;
        pthread_mutex_unlock(&J->lock);
        if (i >= J->B->count) break;
        uint32_t p = J->B->p[i];
        for (unsigned k = 0; k < J->n; ++k) {
            x[k] = mp_mod_small(J->a + (size_t)k * J->words, J->words, p);
            y[k] = mp_mod_small(J->b + (size_t)k * J->words, J->words, p);
        }
        ntt_forward(x, J->n, J->B->psi[i], p);
        ntt_forward(y, J->n, J->B->psi[i], p);
        for (unsigned k = 0; k < J->n; ++k) x[k] = mulmod(x[k], y[k], p);
        ntt_inverse(x, J->n, J->B->psi[i], p);
        for (unsigned k = 0; k < J->n; ++k) J->t[(size_t)i * J->n + k] = mulmod(x[k], J->B->crt_inv[i], p);
    }
    free(x);
    free(y);
    return NULL;
}

typedef struct {
    const orc_basis* B;
    unsigned n, words, qw;
    const uint32_t* q;
    const uint32_t* mq;  /* [count][qw] (P/p_i) mod q */
    const uint32_t* pneg; /* (-P) mod q */
    const uint32_t* t;
    uint32_t* c;
    unsigned begin, end;
} crt_job;

static void* crt_worker(void* arg) {
    crt_job* J = (crt_job*)arg;
    unsigned aw = J->qw + 3;
    for (unsigned k = J->begin; k < J->end; ++k) {
        uint32_t acc[ORC_MAX_WORDS + 4];
        memset(acc, 0, sizeof acc);
        u128 frac = 0;
        for (unsigned i = 0; i < J->B->count; ++i) {
            uint32_t ti = J->t[(size_t)i * J->n + k];
            mp_addmul(acc, J->mq + (size_t)i * J->qw, J->qw, ti, aw);
            frac += (u128)ti * J->B->recip[i];
        }
        /* nearest integer of sum t_i / p_i (rns/solve.cu:405-408) */
        uint32_t nearest = (uint32_t)((frac + ((u128)1 << 63)) >> 64);
        mp_addmul(acc, J->pneg, J->qw, nearest, aw);
        uint32_t r[ORC_MAX_WORDS];
        mp_mod(acc, aw, J->q, J->qw, r);
        uint32_t* out = J->c + (size_t)k * J->words;
        memset(out, 0, J->words * 4);
        memcpy(out, r, (J->qw < J->words ? J->qw : J->words) * 4);
    }
    return NULL;
}

/*
 * Public oracle entry: c = a*b mod (X^n+1, q) through the RNS method.
 * q: qw 32-bit words, odd, top word non-zero.  a, b, c: n x words u32.
 * bits/order/count select the prime basis (0,0,0 -> 30-bit primes = 1 mod 2^17,
 * count sized from the bound).  Returns 0 or a negative error code.
 */
int orc_rns_multiply(unsigned n, const uint32_t* q, unsigned qw, const uint32_t* a, const uint32_t* b,
                     uint32_t* c, unsigned words, unsigned threads, unsigned bits, uint32_t order,
                     unsigned count) {
    if (!n || (n & (n - 1)) || qw == 0 || qw > ORC_MAX_WORDS || words < qw) return -10;
    if (!bits) bits = 30;
    if (!order) order = 1u << 17;
    if ((uint64_t)2 * n > order || (order & (order - 1))) return -11;
    if (!threads) threads = 1;
    unsigned qbits = mp_bits(q, qw);
    orc_basis* B = (orc_basis*)malloc(sizeof *B);
    int status = basis_make(B, n, qbits, bits, order, count);
    if (status) { free(B); return status; }
    size_t tn = (size_t)B->count * n;
    uint32_t* t = (uint32_t*)malloc(tn * 4);
    uint32_t* mq = (uint32_t*)calloc((size_t)B->count * qw, 4);
    uint32_t pneg[ORC_MAX_WORDS];
    {
        uint32_t r[ORC_MAX_WORDS];
        mp_mod(B->product, B->product_words, q, qw, r);
        /* pneg = (q - r) mod q */
        memcpy(pneg, q, qw * 4);
        mp_sub(pneg, r, qw);
        if (mp_cmp(pneg, q, qw) == 0) memset(pneg, 0, qw * 4);
    }
    for (unsigned i = 0; i < B->count; ++i) {
        uint32_t m[2 * ORC_MAX_PRIMES + 2];
        memcpy(m, B->product, sizeof m);
        mp_div_small(m, B->product_words, B->p[i]);
        mp_mod(m, B->product_words, q, qw, mq + (size_t)i * qw);
    }
    prime_job pj = {B, n, words, a, b, t, 0, PTHREAD_MUTEX_INITIALIZER};
    pthread_t tid[256];
    unsigned nt = threads > 256 ? 256 : threads;
    for (unsigned i = 0; i < nt; ++i) pthread_create(&tid[i], NULL, prime_worker, &pj);
    for (unsigned i = 0; i < nt; ++i) pthread_join(tid[i], NULL);
    crt_job cj[256];
    for (unsigned i = 0; i < nt; ++i) {
        cj[i] = (crt_job){B, n, words, qw, q, mq, pneg, t, c, (unsigned)((uint64_t)n * i / nt),
                          (unsigned)((uint64_t)n * (i + 1) / nt)};
        pthread_create(&tid[i], NULL, crt_worker, &cj[i]);
    }
    for (unsigned i = 0; i < nt; ++i) pthread_join(tid[i], NULL);
    free(t);
    free(mq);
    free(B);
    return 0;
}

/* Schoolbook negacyclic product (tests/validate.py:39-44), n x words in/out. */
typedef struct {
    unsigned n, words, qw;
    const uint32_t *q, *a, *b;
    uint32_t* c;
    unsigned begin, end;
} school_job;

static void* school_worker(void* arg) {
    school_job* J = (school_job*)arg;
    unsigned sw = 2 * J->qw + 2;
    uint32_t pos[2 * ORC_MAX_WORDS + 2], neg[2 * ORC_MAX_WORDS + 2];
    for (unsigned k = J->begin; k < J->end; ++k) {
        memset(pos, 0, sizeof pos);
        memset(neg, 0, sizeof neg);
        for (unsigned i = 0; i < J->n; ++i) {
            unsigned j = (k + J->n - i) % J->n;
            uint32_t* dst = i + j < J->n ? pos : neg;
            const uint32_t* x = J->a + (size_t)i * J->words;
            const uint32_t* y = J->b + (size_t)j * J->words;
            for (unsigned u = 0; u < J->qw; ++u)
                if (x[u]) mp_addmul(dst + u, y, J->qw, x[u], sw - u);
        }
        uint32_t rp[ORC_MAX_WORDS], rn[ORC_MAX_WORDS];
        mp_mod(pos, sw, J->q, J->qw, rp);
        mp_mod(neg, sw, J->q, J->qw, rn);
        if (mp_sub(rp, rn, J->qw)) {
            /* went negative: add q back */
            uint64_t carry = 0;
            for (unsigned u = 0; u < J->qw; ++u) {
                uint64_t v = (uint64_t)rp[u] + J->q[u] + carry;
                rp[u] = (uint32_t)v;
                carry = v >> 32;
            }
        }
        uint32_t* out = J->c + (size_t)k * J->words;
        memset(out, 0, J->words * 4);
        memcpy(out, rp, J->qw * 4);
    }
    return NULL;
}

int orc_schoolbook(unsigned n, const uint32_t* q, unsigned qw, const uint32_t* a, const uint32_t* b, uint32_t* c,
                   unsigned words, unsigned threads) {
    if (!n || qw == 0 || qw > ORC_MAX_WORDS || words < qw) return -10;
    if (!threads) threads = 1;
    unsigned nt = threads > 256 ? 256 : threads;
    if (nt > n) nt = n;
    pthread_t tid[256];
    school_job sj[256];
    for (unsigned i = 0; i < nt; ++i) {
        sj[i] = (school_job){n, words, qw, q, a, b, c, (unsigned)((uint64_t)n * i / nt),
                             (unsigned)((uint64_t)n * (i + 1) / nt)};
        pthread_create(&tid[i], NULL, school_worker, &sj[i]);
    }
    for (unsigned i = 0; i < nt; ++i) pthread_join(tid[i], NULL);
    return 0;
}

/*
 * Basis constants for comparison with the reference's rns::setup
 * (rns/host_setup.h:61-126): primes, (P/p_i) mod q (29-word rows like
 * bases_mod_q), P mod q, floor(2^64/p_i), and the first twiddle of each
 * prime's forward table (psi^1).  Arrays sized count, count*qw, qw.
 */
int orc_basis_dump(unsigned n, const uint32_t* q, unsigned qw, unsigned bits, uint32_t order, unsigned count,
                   uint32_t* primes, uint32_t* bases_mod_q, uint32_t* product_mod_q, uint64_t* recip,
                   uint32_t* psi, unsigned* count_out) {
    orc_basis* B = (orc_basis*)malloc(sizeof *B);
    int status = basis_make(B, n, mp_bits(q, qw), bits, order, count);
    if (status) { free(B); return status; }
    for (unsigned i = 0; i < B->count; ++i) {
        primes[i] = B->p[i];
        recip[i] = B->recip[i];
        psi[i] = B->psi[i];
        uint32_t m[2 * ORC_MAX_PRIMES + 2];
        memcpy(m, B->product, sizeof m);
        mp_div_small(m, B->product_words, B->p[i]);
        mp_mod(m, B->product_words, q, qw, bases_mod_q + (size_t)i * qw);
    }
    mp_mod(B->product, B->product_words, q, qw, product_mod_q);
    *count_out = B->count;
    free(B);
    return 0;
}
