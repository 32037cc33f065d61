// Test infrastructure only: the small part of GMP's C++ interface (gmpxx.h)
// that the reference's CPU emulation of its kernels uses
// (tests/cuda_emulation.h:87-156: mpz_class arithmetic, mpz_import/export,
// mpz_invert), over the system's runtime libgmp.so.10.  GMP's development
// headers are not installed here, so the few C entry points are declared by
// hand from the GMP manual's documented prototypes (mpz_t is documented as an
// array of one __mpz_struct {int alloc; int size; mp_limb_t* d}).  Eager
// evaluation, no expression templates: enough for the emulation, nothing more.
#pragma once

#include <cstddef>
#include <cstdint>

extern "C" {
typedef unsigned long mp_limb_t;
typedef long mp_size_t;
typedef unsigned long mp_bitcnt_t;
typedef struct {
    int _mp_alloc;
    int _mp_size;
    mp_limb_t* _mp_d;
} __mpz_struct;
typedef __mpz_struct mpz_t[1];
typedef __mpz_struct* mpz_ptr;
typedef const __mpz_struct* mpz_srcptr;

void __gmpz_init(mpz_ptr);
void __gmpz_init_set(mpz_ptr, mpz_srcptr);
void __gmpz_init_set_ui(mpz_ptr, unsigned long);
void __gmpz_init_set_si(mpz_ptr, long);
void __gmpz_clear(mpz_ptr);
void __gmpz_set(mpz_ptr, mpz_srcptr);
void __gmpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mul_ui(mpz_ptr, mpz_srcptr, unsigned long);
void __gmpz_mul_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_fdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_tdiv_r(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_and(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_ior(mpz_ptr, mpz_srcptr, mpz_srcptr);
int __gmpz_cmp(mpz_srcptr, mpz_srcptr);
int __gmpz_invert(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_import(mpz_ptr, size_t, int, size_t, int, size_t, const void*);
void* __gmpz_export(void*, size_t*, int, size_t, int, size_t, mpz_srcptr);
}

inline void mpz_import(mpz_ptr r, size_t count, int order, size_t size, int endian, size_t nails, const void* op) {
    __gmpz_import(r, count, order, size, endian, nails, op);
}
inline void* mpz_export(void* rop, size_t* countp, int order, size_t size, int endian, size_t nails, mpz_srcptr op) {
    return __gmpz_export(rop, countp, order, size, endian, nails, op);
}
inline int mpz_invert(mpz_ptr r, mpz_srcptr a, mpz_srcptr m) { return __gmpz_invert(r, a, m); }

class mpz_class {
    mpz_t v_;

public:
    mpz_class() { __gmpz_init(v_); }
    mpz_class(const mpz_class& o) { __gmpz_init_set(v_, o.v_); }
    mpz_class(mpz_class&& o) noexcept {
        __gmpz_init(v_);
        __mpz_struct t = v_[0];
        v_[0] = o.v_[0];
        o.v_[0] = t;
    }
    mpz_class(unsigned long x) { __gmpz_init_set_ui(v_, x); }
    mpz_class(unsigned int x) { __gmpz_init_set_ui(v_, x); }
    mpz_class(long x) { __gmpz_init_set_si(v_, x); }
    mpz_class(int x) { __gmpz_init_set_si(v_, x); }
    ~mpz_class() { __gmpz_clear(v_); }
    mpz_class& operator=(const mpz_class& o) {
        if (this != &o) __gmpz_set(v_, o.v_);
        return *this;
    }
    mpz_class& operator=(mpz_class&& o) noexcept {
        __mpz_struct t = v_[0];
        v_[0] = o.v_[0];
        o.v_[0] = t;
        return *this;
    }
    mpz_ptr get_mpz_t() { return v_; }
    mpz_srcptr get_mpz_t() const { return v_; }

    friend mpz_class operator+(const mpz_class& a, const mpz_class& b) { mpz_class r; __gmpz_add(r.v_, a.v_, b.v_); return r; }
    friend mpz_class operator-(const mpz_class& a, const mpz_class& b) { mpz_class r; __gmpz_sub(r.v_, a.v_, b.v_); return r; }
    friend mpz_class operator*(const mpz_class& a, const mpz_class& b) { mpz_class r; __gmpz_mul(r.v_, a.v_, b.v_); return r; }
    friend mpz_class operator*(const mpz_class& a, unsigned long b) { mpz_class r; __gmpz_mul_ui(r.v_, a.v_, b); return r; }
    friend mpz_class operator*(const mpz_class& a, unsigned int b) { return a * static_cast<unsigned long>(b); }
    // truncating remainder, as C++ and GMP's operator% define it
    friend mpz_class operator%(const mpz_class& a, const mpz_class& b) { mpz_class r; __gmpz_tdiv_r(r.v_, a.v_, b.v_); return r; }
    // two's-complement bitwise and/or, as GMP defines them for negative operands
    friend mpz_class operator&(const mpz_class& a, const mpz_class& b) { mpz_class r; __gmpz_and(r.v_, a.v_, b.v_); return r; }
    friend mpz_class operator|(const mpz_class& a, const mpz_class& b) { mpz_class r; __gmpz_ior(r.v_, a.v_, b.v_); return r; }
    friend mpz_class operator<<(const mpz_class& a, unsigned long n) { mpz_class r; __gmpz_mul_2exp(r.v_, a.v_, n); return r; }
    friend mpz_class operator>>(const mpz_class& a, unsigned long n) { mpz_class r; __gmpz_fdiv_q_2exp(r.v_, a.v_, n); return r; }
    friend mpz_class operator<<(const mpz_class& a, unsigned int n) { return a << static_cast<unsigned long>(n); }
    friend mpz_class operator>>(const mpz_class& a, unsigned int n) { return a >> static_cast<unsigned long>(n); }
    friend mpz_class operator<<(const mpz_class& a, int n) { return a << static_cast<unsigned long>(n); }
    friend mpz_class operator>>(const mpz_class& a, int n) { return a >> static_cast<unsigned long>(n); }
    mpz_class& operator&=(const mpz_class& b) { __gmpz_and(v_, v_, b.v_); return *this; }
    mpz_class& operator|=(const mpz_class& b) { __gmpz_ior(v_, v_, b.v_); return *this; }
    mpz_class& operator+=(const mpz_class& b) { __gmpz_add(v_, v_, b.v_); return *this; }
    friend bool operator==(const mpz_class& a, const mpz_class& b) { return __gmpz_cmp(a.v_, b.v_) == 0; }
    friend bool operator!=(const mpz_class& a, const mpz_class& b) { return __gmpz_cmp(a.v_, b.v_) != 0; }
    friend bool operator<(const mpz_class& a, const mpz_class& b) { return __gmpz_cmp(a.v_, b.v_) < 0; }
    friend bool operator<=(const mpz_class& a, const mpz_class& b) { return __gmpz_cmp(a.v_, b.v_) <= 0; }
    friend bool operator>(const mpz_class& a, const mpz_class& b) { return __gmpz_cmp(a.v_, b.v_) > 0; }
    friend bool operator>=(const mpz_class& a, const mpz_class& b) { return __gmpz_cmp(a.v_, b.v_) >= 0; }
};
