// Generated by gen_crt_mac.py -- do not edit.
// Multiword arithmetic as PTX carry chains (see the generator for the contracts).
#pragma once
#include <cstdint>
namespace pm {
template <int W> __device__ __forceinline__ void crt_mac(uint32_t (&a)[W + 2], uint32_t t, const uint32_t (&m)[W]);
template <int N> __device__ __forceinline__ uint32_t mp_sub(uint32_t (&a)[N], const uint32_t (&b)[N]);
template <int W> __device__ __forceinline__ void mp_sub_hi(uint32_t (&a)[W + 2], const uint32_t (&b)[W + 2]);
template <int N> __device__ __forceinline__ void mp_add3(uint32_t (&a)[N], uint32_t t0, uint32_t t1, uint32_t t2);
template <int N> __device__ __forceinline__ uint32_t mp_add(uint32_t (&a)[N], const uint32_t (&b)[N]);
template <> __device__ __forceinline__ void crt_mac<4>(uint32_t (&a)[6], uint32_t t, const uint32_t (&m)[4]) {
    asm("mad.lo.cc.u32 %0, %10, %6, %0;\n\tmadc.lo.cc.u32 %1, %10, %7, %1;\n\tmadc.lo.cc.u32 %2, %10, %8, %2;\n\tmadc.lo.cc.u32 %3, %10, %9, %3;\n\taddc.cc.u32 %4, %4, 0;\n\taddc.u32 %5, %5, 0;\n\tmad.hi.cc.u32 %1, %10, %6, %1;\n\tmadc.hi.cc.u32 %2, %10, %7, %2;\n\tmadc.hi.cc.u32 %3, %10, %8, %3;\n\tmadc.hi.cc.u32 %4, %10, %9, %4;\n\taddc.u32 %5, %5, 0;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5])
        : "r"(m[0]), "r"(m[1]), "r"(m[2]), "r"(m[3]), "r"(t));
}
template <> __device__ __forceinline__ uint32_t mp_sub<4>(uint32_t (&a)[4], const uint32_t (&b)[4]) {
    uint32_t mask;
    asm("sub.cc.u32 %1, %1, %5;\n\tsubc.cc.u32 %2, %2, %6;\n\tsubc.cc.u32 %3, %3, %7;\n\tsubc.cc.u32 %4, %4, %8;\n\tsubc.u32 %0, 0, 0;"
        : "=r"(mask), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]));
    return mask;
}
template <> __device__ __forceinline__ uint32_t mp_add<4>(uint32_t (&a)[4], const uint32_t (&b)[4]) {
    uint32_t carry;
    asm("add.cc.u32 %1, %1, %5;\n\taddc.cc.u32 %2, %2, %6;\n\taddc.cc.u32 %3, %3, %7;\n\taddc.cc.u32 %4, %4, %8;\n\taddc.u32 %0, 0, 0;"
        : "=r"(carry), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]));
    return carry;
}
template <> __device__ __forceinline__ uint32_t mp_sub<6>(uint32_t (&a)[6], const uint32_t (&b)[6]) {
    uint32_t mask;
    asm("sub.cc.u32 %1, %1, %7;\n\tsubc.cc.u32 %2, %2, %8;\n\tsubc.cc.u32 %3, %3, %9;\n\tsubc.cc.u32 %4, %4, %10;\n\tsubc.cc.u32 %5, %5, %11;\n\tsubc.cc.u32 %6, %6, %12;\n\tsubc.u32 %0, 0, 0;"
        : "=r"(mask), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]));
    return mask;
}
template <> __device__ __forceinline__ uint32_t mp_add<6>(uint32_t (&a)[6], const uint32_t (&b)[6]) {
    uint32_t carry;
    asm("add.cc.u32 %1, %1, %7;\n\taddc.cc.u32 %2, %2, %8;\n\taddc.cc.u32 %3, %3, %9;\n\taddc.cc.u32 %4, %4, %10;\n\taddc.cc.u32 %5, %5, %11;\n\taddc.cc.u32 %6, %6, %12;\n\taddc.u32 %0, 0, 0;"
        : "=r"(carry), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]));
    return carry;
}
template <> __device__ __forceinline__ void mp_sub_hi<4>(uint32_t (&a)[6], const uint32_t (&b)[6]) {
    asm("sub.cc.u32 %1, %1, %6;\n\tsubc.cc.u32 %2, %2, %7;\n\tsubc.cc.u32 %3, %3, %8;\n\tsubc.cc.u32 %4, %4, %9;\n\tsubc.cc.u32 %5, %5, %10;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]));
}
template <> __device__ __forceinline__ void mp_add3<6>(uint32_t (&a)[6], uint32_t t0, uint32_t t1, uint32_t t2) {
    asm("add.cc.u32 %0, %0, %6;\n\taddc.cc.u32 %1, %1, %7;\n\taddc.cc.u32 %2, %2, %8;\n\taddc.cc.u32 %3, %3, 0;\n\taddc.cc.u32 %4, %4, 0;\n\taddc.u32 %5, %5, 0;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5])
        : "r"(t0), "r"(t1), "r"(t2));
}
template <> __device__ __forceinline__ void crt_mac<8>(uint32_t (&a)[10], uint32_t t, const uint32_t (&m)[8]) {
    asm("mad.lo.cc.u32 %0, %18, %10, %0;\n\tmadc.lo.cc.u32 %1, %18, %11, %1;\n\tmadc.lo.cc.u32 %2, %18, %12, %2;\n\tmadc.lo.cc.u32 %3, %18, %13, %3;\n\tmadc.lo.cc.u32 %4, %18, %14, %4;\n\tmadc.lo.cc.u32 %5, %18, %15, %5;\n\tmadc.lo.cc.u32 %6, %18, %16, %6;\n\tmadc.lo.cc.u32 %7, %18, %17, %7;\n\taddc.cc.u32 %8, %8, 0;\n\taddc.u32 %9, %9, 0;\n\tmad.hi.cc.u32 %1, %18, %10, %1;\n\tmadc.hi.cc.u32 %2, %18, %11, %2;\n\tmadc.hi.cc.u32 %3, %18, %12, %3;\n\tmadc.hi.cc.u32 %4, %18, %13, %4;\n\tmadc.hi.cc.u32 %5, %18, %14, %5;\n\tmadc.hi.cc.u32 %6, %18, %15, %6;\n\tmadc.hi.cc.u32 %7, %18, %16, %7;\n\tmadc.hi.cc.u32 %8, %18, %17, %8;\n\taddc.u32 %9, %9, 0;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9])
        : "r"(m[0]), "r"(m[1]), "r"(m[2]), "r"(m[3]), "r"(m[4]), "r"(m[5]), "r"(m[6]), "r"(m[7]), "r"(t));
}
template <> __device__ __forceinline__ uint32_t mp_sub<8>(uint32_t (&a)[8], const uint32_t (&b)[8]) {
    uint32_t mask;
    asm("sub.cc.u32 %1, %1, %9;\n\tsubc.cc.u32 %2, %2, %10;\n\tsubc.cc.u32 %3, %3, %11;\n\tsubc.cc.u32 %4, %4, %12;\n\tsubc.cc.u32 %5, %5, %13;\n\tsubc.cc.u32 %6, %6, %14;\n\tsubc.cc.u32 %7, %7, %15;\n\tsubc.cc.u32 %8, %8, %16;\n\tsubc.u32 %0, 0, 0;"
        : "=r"(mask), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
    return mask;
}
template <> __device__ __forceinline__ uint32_t mp_add<8>(uint32_t (&a)[8], const uint32_t (&b)[8]) {
    uint32_t carry;
    asm("add.cc.u32 %1, %1, %9;\n\taddc.cc.u32 %2, %2, %10;\n\taddc.cc.u32 %3, %3, %11;\n\taddc.cc.u32 %4, %4, %12;\n\taddc.cc.u32 %5, %5, %13;\n\taddc.cc.u32 %6, %6, %14;\n\taddc.cc.u32 %7, %7, %15;\n\taddc.cc.u32 %8, %8, %16;\n\taddc.u32 %0, 0, 0;"
        : "=r"(carry), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
    return carry;
}
template <> __device__ __forceinline__ uint32_t mp_sub<10>(uint32_t (&a)[10], const uint32_t (&b)[10]) {
    uint32_t mask;
    asm("sub.cc.u32 %1, %1, %11;\n\tsubc.cc.u32 %2, %2, %12;\n\tsubc.cc.u32 %3, %3, %13;\n\tsubc.cc.u32 %4, %4, %14;\n\tsubc.cc.u32 %5, %5, %15;\n\tsubc.cc.u32 %6, %6, %16;\n\tsubc.cc.u32 %7, %7, %17;\n\tsubc.cc.u32 %8, %8, %18;\n\tsubc.cc.u32 %9, %9, %19;\n\tsubc.cc.u32 %10, %10, %20;\n\tsubc.u32 %0, 0, 0;"
        : "=r"(mask), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]));
    return mask;
}
template <> __device__ __forceinline__ uint32_t mp_add<10>(uint32_t (&a)[10], const uint32_t (&b)[10]) {
    uint32_t carry;
    asm("add.cc.u32 %1, %1, %11;\n\taddc.cc.u32 %2, %2, %12;\n\taddc.cc.u32 %3, %3, %13;\n\taddc.cc.u32 %4, %4, %14;\n\taddc.cc.u32 %5, %5, %15;\n\taddc.cc.u32 %6, %6, %16;\n\taddc.cc.u32 %7, %7, %17;\n\taddc.cc.u32 %8, %8, %18;\n\taddc.cc.u32 %9, %9, %19;\n\taddc.cc.u32 %10, %10, %20;\n\taddc.u32 %0, 0, 0;"
        : "=r"(carry), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]));
    return carry;
}
template <> __device__ __forceinline__ void mp_sub_hi<8>(uint32_t (&a)[10], const uint32_t (&b)[10]) {
    asm("sub.cc.u32 %1, %1, %10;\n\tsubc.cc.u32 %2, %2, %11;\n\tsubc.cc.u32 %3, %3, %12;\n\tsubc.cc.u32 %4, %4, %13;\n\tsubc.cc.u32 %5, %5, %14;\n\tsubc.cc.u32 %6, %6, %15;\n\tsubc.cc.u32 %7, %7, %16;\n\tsubc.cc.u32 %8, %8, %17;\n\tsubc.cc.u32 %9, %9, %18;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]));
}
template <> __device__ __forceinline__ void mp_add3<10>(uint32_t (&a)[10], uint32_t t0, uint32_t t1, uint32_t t2) {
    asm("add.cc.u32 %0, %0, %10;\n\taddc.cc.u32 %1, %1, %11;\n\taddc.cc.u32 %2, %2, %12;\n\taddc.cc.u32 %3, %3, 0;\n\taddc.cc.u32 %4, %4, 0;\n\taddc.cc.u32 %5, %5, 0;\n\taddc.cc.u32 %6, %6, 0;\n\taddc.cc.u32 %7, %7, 0;\n\taddc.cc.u32 %8, %8, 0;\n\taddc.u32 %9, %9, 0;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9])
        : "r"(t0), "r"(t1), "r"(t2));
}
template <> __device__ __forceinline__ void crt_mac<12>(uint32_t (&a)[14], uint32_t t, const uint32_t (&m)[12]) {
    asm("mad.lo.cc.u32 %0, %26, %14, %0;\n\tmadc.lo.cc.u32 %1, %26, %15, %1;\n\tmadc.lo.cc.u32 %2, %26, %16, %2;\n\tmadc.lo.cc.u32 %3, %26, %17, %3;\n\tmadc.lo.cc.u32 %4, %26, %18, %4;\n\tmadc.lo.cc.u32 %5, %26, %19, %5;\n\tmadc.lo.cc.u32 %6, %26, %20, %6;\n\tmadc.lo.cc.u32 %7, %26, %21, %7;\n\tmadc.lo.cc.u32 %8, %26, %22, %8;\n\tmadc.lo.cc.u32 %9, %26, %23, %9;\n\tmadc.lo.cc.u32 %10, %26, %24, %10;\n\tmadc.lo.cc.u32 %11, %26, %25, %11;\n\taddc.cc.u32 %12, %12, 0;\n\taddc.u32 %13, %13, 0;\n\tmad.hi.cc.u32 %1, %26, %14, %1;\n\tmadc.hi.cc.u32 %2, %26, %15, %2;\n\tmadc.hi.cc.u32 %3, %26, %16, %3;\n\tmadc.hi.cc.u32 %4, %26, %17, %4;\n\tmadc.hi.cc.u32 %5, %26, %18, %5;\n\tmadc.hi.cc.u32 %6, %26, %19, %6;\n\tmadc.hi.cc.u32 %7, %26, %20, %7;\n\tmadc.hi.cc.u32 %8, %26, %21, %8;\n\tmadc.hi.cc.u32 %9, %26, %22, %9;\n\tmadc.hi.cc.u32 %10, %26, %23, %10;\n\tmadc.hi.cc.u32 %11, %26, %24, %11;\n\tmadc.hi.cc.u32 %12, %26, %25, %12;\n\taddc.u32 %13, %13, 0;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13])
        : "r"(m[0]), "r"(m[1]), "r"(m[2]), "r"(m[3]), "r"(m[4]), "r"(m[5]), "r"(m[6]), "r"(m[7]), "r"(m[8]), "r"(m[9]), "r"(m[10]), "r"(m[11]), "r"(t));
}
template <> __device__ __forceinline__ uint32_t mp_sub<12>(uint32_t (&a)[12], const uint32_t (&b)[12]) {
    uint32_t mask;
    asm("sub.cc.u32 %1, %1, %13;\n\tsubc.cc.u32 %2, %2, %14;\n\tsubc.cc.u32 %3, %3, %15;\n\tsubc.cc.u32 %4, %4, %16;\n\tsubc.cc.u32 %5, %5, %17;\n\tsubc.cc.u32 %6, %6, %18;\n\tsubc.cc.u32 %7, %7, %19;\n\tsubc.cc.u32 %8, %8, %20;\n\tsubc.cc.u32 %9, %9, %21;\n\tsubc.cc.u32 %10, %10, %22;\n\tsubc.cc.u32 %11, %11, %23;\n\tsubc.cc.u32 %12, %12, %24;\n\tsubc.u32 %0, 0, 0;"
        : "=r"(mask), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]));
    return mask;
}
template <> __device__ __forceinline__ uint32_t mp_add<12>(uint32_t (&a)[12], const uint32_t (&b)[12]) {
    uint32_t carry;
    asm("add.cc.u32 %1, %1, %13;\n\taddc.cc.u32 %2, %2, %14;\n\taddc.cc.u32 %3, %3, %15;\n\taddc.cc.u32 %4, %4, %16;\n\taddc.cc.u32 %5, %5, %17;\n\taddc.cc.u32 %6, %6, %18;\n\taddc.cc.u32 %7, %7, %19;\n\taddc.cc.u32 %8, %8, %20;\n\taddc.cc.u32 %9, %9, %21;\n\taddc.cc.u32 %10, %10, %22;\n\taddc.cc.u32 %11, %11, %23;\n\taddc.cc.u32 %12, %12, %24;\n\taddc.u32 %0, 0, 0;"
        : "=r"(carry), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]));
    return carry;
}
template <> __device__ __forceinline__ uint32_t mp_sub<14>(uint32_t (&a)[14], const uint32_t (&b)[14]) {
    uint32_t mask;
    asm("sub.cc.u32 %1, %1, %15;\n\tsubc.cc.u32 %2, %2, %16;\n\tsubc.cc.u32 %3, %3, %17;\n\tsubc.cc.u32 %4, %4, %18;\n\tsubc.cc.u32 %5, %5, %19;\n\tsubc.cc.u32 %6, %6, %20;\n\tsubc.cc.u32 %7, %7, %21;\n\tsubc.cc.u32 %8, %8, %22;\n\tsubc.cc.u32 %9, %9, %23;\n\tsubc.cc.u32 %10, %10, %24;\n\tsubc.cc.u32 %11, %11, %25;\n\tsubc.cc.u32 %12, %12, %26;\n\tsubc.cc.u32 %13, %13, %27;\n\tsubc.cc.u32 %14, %14, %28;\n\tsubc.u32 %0, 0, 0;"
        : "=r"(mask), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]));
    return mask;
}
template <> __device__ __forceinline__ uint32_t mp_add<14>(uint32_t (&a)[14], const uint32_t (&b)[14]) {
    uint32_t carry;
    asm("add.cc.u32 %1, %1, %15;\n\taddc.cc.u32 %2, %2, %16;\n\taddc.cc.u32 %3, %3, %17;\n\taddc.cc.u32 %4, %4, %18;\n\taddc.cc.u32 %5, %5, %19;\n\taddc.cc.u32 %6, %6, %20;\n\taddc.cc.u32 %7, %7, %21;\n\taddc.cc.u32 %8, %8, %22;\n\taddc.cc.u32 %9, %9, %23;\n\taddc.cc.u32 %10, %10, %24;\n\taddc.cc.u32 %11, %11, %25;\n\taddc.cc.u32 %12, %12, %26;\n\taddc.cc.u32 %13, %13, %27;\n\taddc.cc.u32 %14, %14, %28;\n\taddc.u32 %0, 0, 0;"
        : "=r"(carry), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]));
    return carry;
}
template <> __device__ __forceinline__ void mp_sub_hi<12>(uint32_t (&a)[14], const uint32_t (&b)[14]) {
    asm("sub.cc.u32 %1, %1, %14;\n\tsubc.cc.u32 %2, %2, %15;\n\tsubc.cc.u32 %3, %3, %16;\n\tsubc.cc.u32 %4, %4, %17;\n\tsubc.cc.u32 %5, %5, %18;\n\tsubc.cc.u32 %6, %6, %19;\n\tsubc.cc.u32 %7, %7, %20;\n\tsubc.cc.u32 %8, %8, %21;\n\tsubc.cc.u32 %9, %9, %22;\n\tsubc.cc.u32 %10, %10, %23;\n\tsubc.cc.u32 %11, %11, %24;\n\tsubc.cc.u32 %12, %12, %25;\n\tsubc.cc.u32 %13, %13, %26;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]));
}
template <> __device__ __forceinline__ void mp_add3<14>(uint32_t (&a)[14], uint32_t t0, uint32_t t1, uint32_t t2) {
    asm("add.cc.u32 %0, %0, %14;\n\taddc.cc.u32 %1, %1, %15;\n\taddc.cc.u32 %2, %2, %16;\n\taddc.cc.u32 %3, %3, 0;\n\taddc.cc.u32 %4, %4, 0;\n\taddc.cc.u32 %5, %5, 0;\n\taddc.cc.u32 %6, %6, 0;\n\taddc.cc.u32 %7, %7, 0;\n\taddc.cc.u32 %8, %8, 0;\n\taddc.cc.u32 %9, %9, 0;\n\taddc.cc.u32 %10, %10, 0;\n\taddc.cc.u32 %11, %11, 0;\n\taddc.cc.u32 %12, %12, 0;\n\taddc.u32 %13, %13, 0;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13])
        : "r"(t0), "r"(t1), "r"(t2));
}
template <> __device__ __forceinline__ void crt_mac<16>(uint32_t (&a)[18], uint32_t t, const uint32_t (&m)[16]) {
    asm("mad.lo.cc.u32 %0, %34, %18, %0;\n\tmadc.lo.cc.u32 %1, %34, %19, %1;\n\tmadc.lo.cc.u32 %2, %34, %20, %2;\n\tmadc.lo.cc.u32 %3, %34, %21, %3;\n\tmadc.lo.cc.u32 %4, %34, %22, %4;\n\tmadc.lo.cc.u32 %5, %34, %23, %5;\n\tmadc.lo.cc.u32 %6, %34, %24, %6;\n\tmadc.lo.cc.u32 %7, %34, %25, %7;\n\tmadc.lo.cc.u32 %8, %34, %26, %8;\n\tmadc.lo.cc.u32 %9, %34, %27, %9;\n\tmadc.lo.cc.u32 %10, %34, %28, %10;\n\tmadc.lo.cc.u32 %11, %34, %29, %11;\n\tmadc.lo.cc.u32 %12, %34, %30, %12;\n\tmadc.lo.cc.u32 %13, %34, %31, %13;\n\tmadc.lo.cc.u32 %14, %34, %32, %14;\n\tmadc.lo.cc.u32 %15, %34, %33, %15;\n\taddc.cc.u32 %16, %16, 0;\n\taddc.u32 %17, %17, 0;\n\tmad.hi.cc.u32 %1, %34, %18, %1;\n\tmadc.hi.cc.u32 %2, %34, %19, %2;\n\tmadc.hi.cc.u32 %3, %34, %20, %3;\n\tmadc.hi.cc.u32 %4, %34, %21, %4;\n\tmadc.hi.cc.u32 %5, %34, %22, %5;\n\tmadc.hi.cc.u32 %6, %34, %23, %6;\n\tmadc.hi.cc.u32 %7, %34, %24, %7;\n\tmadc.hi.cc.u32 %8, %34, %25, %8;\n\tmadc.hi.cc.u32 %9, %34, %26, %9;\n\tmadc.hi.cc.u32 %10, %34, %27, %10;\n\tmadc.hi.cc.u32 %11, %34, %28, %11;\n\tmadc.hi.cc.u32 %12, %34, %29, %12;\n\tmadc.hi.cc.u32 %13, %34, %30, %13;\n\tmadc.hi.cc.u32 %14, %34, %31, %14;\n\tmadc.hi.cc.u32 %15, %34, %32, %15;\n\tmadc.hi.cc.u32 %16, %34, %33, %16;\n\taddc.u32 %17, %17, 0;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17])
        : "r"(m[0]), "r"(m[1]), "r"(m[2]), "r"(m[3]), "r"(m[4]), "r"(m[5]), "r"(m[6]), "r"(m[7]), "r"(m[8]), "r"(m[9]), "r"(m[10]), "r"(m[11]), "r"(m[12]), "r"(m[13]), "r"(m[14]), "r"(m[15]), "r"(t));
}
template <> __device__ __forceinline__ uint32_t mp_sub<16>(uint32_t (&a)[16], const uint32_t (&b)[16]) {
    uint32_t mask;
    asm("sub.cc.u32 %1, %1, %17;\n\tsubc.cc.u32 %2, %2, %18;\n\tsubc.cc.u32 %3, %3, %19;\n\tsubc.cc.u32 %4, %4, %20;\n\tsubc.cc.u32 %5, %5, %21;\n\tsubc.cc.u32 %6, %6, %22;\n\tsubc.cc.u32 %7, %7, %23;\n\tsubc.cc.u32 %8, %8, %24;\n\tsubc.cc.u32 %9, %9, %25;\n\tsubc.cc.u32 %10, %10, %26;\n\tsubc.cc.u32 %11, %11, %27;\n\tsubc.cc.u32 %12, %12, %28;\n\tsubc.cc.u32 %13, %13, %29;\n\tsubc.cc.u32 %14, %14, %30;\n\tsubc.cc.u32 %15, %15, %31;\n\tsubc.cc.u32 %16, %16, %32;\n\tsubc.u32 %0, 0, 0;"
        : "=r"(mask), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]));
    return mask;
}
template <> __device__ __forceinline__ uint32_t mp_add<16>(uint32_t (&a)[16], const uint32_t (&b)[16]) {
    uint32_t carry;
    asm("add.cc.u32 %1, %1, %17;\n\taddc.cc.u32 %2, %2, %18;\n\taddc.cc.u32 %3, %3, %19;\n\taddc.cc.u32 %4, %4, %20;\n\taddc.cc.u32 %5, %5, %21;\n\taddc.cc.u32 %6, %6, %22;\n\taddc.cc.u32 %7, %7, %23;\n\taddc.cc.u32 %8, %8, %24;\n\taddc.cc.u32 %9, %9, %25;\n\taddc.cc.u32 %10, %10, %26;\n\taddc.cc.u32 %11, %11, %27;\n\taddc.cc.u32 %12, %12, %28;\n\taddc.cc.u32 %13, %13, %29;\n\taddc.cc.u32 %14, %14, %30;\n\taddc.cc.u32 %15, %15, %31;\n\taddc.cc.u32 %16, %16, %32;\n\taddc.u32 %0, 0, 0;"
        : "=r"(carry), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]));
    return carry;
}
template <> __device__ __forceinline__ uint32_t mp_sub<18>(uint32_t (&a)[18], const uint32_t (&b)[18]) {
    uint32_t mask;
    asm("sub.cc.u32 %1, %1, %19;\n\tsubc.cc.u32 %2, %2, %20;\n\tsubc.cc.u32 %3, %3, %21;\n\tsubc.cc.u32 %4, %4, %22;\n\tsubc.cc.u32 %5, %5, %23;\n\tsubc.cc.u32 %6, %6, %24;\n\tsubc.cc.u32 %7, %7, %25;\n\tsubc.cc.u32 %8, %8, %26;\n\tsubc.cc.u32 %9, %9, %27;\n\tsubc.cc.u32 %10, %10, %28;\n\tsubc.cc.u32 %11, %11, %29;\n\tsubc.cc.u32 %12, %12, %30;\n\tsubc.cc.u32 %13, %13, %31;\n\tsubc.cc.u32 %14, %14, %32;\n\tsubc.cc.u32 %15, %15, %33;\n\tsubc.cc.u32 %16, %16, %34;\n\tsubc.cc.u32 %17, %17, %35;\n\tsubc.cc.u32 %18, %18, %36;\n\tsubc.u32 %0, 0, 0;"
        : "=r"(mask), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]));
    return mask;
}
template <> __device__ __forceinline__ uint32_t mp_add<18>(uint32_t (&a)[18], const uint32_t (&b)[18]) {
    uint32_t carry;
    asm("add.cc.u32 %1, %1, %19;\n\taddc.cc.u32 %2, %2, %20;\n\taddc.cc.u32 %3, %3, %21;\n\taddc.cc.u32 %4, %4, %22;\n\taddc.cc.u32 %5, %5, %23;\n\taddc.cc.u32 %6, %6, %24;\n\taddc.cc.u32 %7, %7, %25;\n\taddc.cc.u32 %8, %8, %26;\n\taddc.cc.u32 %9, %9, %27;\n\taddc.cc.u32 %10, %10, %28;\n\taddc.cc.u32 %11, %11, %29;\n\taddc.cc.u32 %12, %12, %30;\n\taddc.cc.u32 %13, %13, %31;\n\taddc.cc.u32 %14, %14, %32;\n\taddc.cc.u32 %15, %15, %33;\n\taddc.cc.u32 %16, %16, %34;\n\taddc.cc.u32 %17, %17, %35;\n\taddc.cc.u32 %18, %18, %36;\n\taddc.u32 %0, 0, 0;"
        : "=r"(carry), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]));
    return carry;
}
template <> __device__ __forceinline__ void mp_sub_hi<16>(uint32_t (&a)[18], const uint32_t (&b)[18]) {
    asm("sub.cc.u32 %1, %1, %18;\n\tsubc.cc.u32 %2, %2, %19;\n\tsubc.cc.u32 %3, %3, %20;\n\tsubc.cc.u32 %4, %4, %21;\n\tsubc.cc.u32 %5, %5, %22;\n\tsubc.cc.u32 %6, %6, %23;\n\tsubc.cc.u32 %7, %7, %24;\n\tsubc.cc.u32 %8, %8, %25;\n\tsubc.cc.u32 %9, %9, %26;\n\tsubc.cc.u32 %10, %10, %27;\n\tsubc.cc.u32 %11, %11, %28;\n\tsubc.cc.u32 %12, %12, %29;\n\tsubc.cc.u32 %13, %13, %30;\n\tsubc.cc.u32 %14, %14, %31;\n\tsubc.cc.u32 %15, %15, %32;\n\tsubc.cc.u32 %16, %16, %33;\n\tsubc.cc.u32 %17, %17, %34;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]));
}
template <> __device__ __forceinline__ void mp_add3<18>(uint32_t (&a)[18], uint32_t t0, uint32_t t1, uint32_t t2) {
    asm("add.cc.u32 %0, %0, %18;\n\taddc.cc.u32 %1, %1, %19;\n\taddc.cc.u32 %2, %2, %20;\n\taddc.cc.u32 %3, %3, 0;\n\taddc.cc.u32 %4, %4, 0;\n\taddc.cc.u32 %5, %5, 0;\n\taddc.cc.u32 %6, %6, 0;\n\taddc.cc.u32 %7, %7, 0;\n\taddc.cc.u32 %8, %8, 0;\n\taddc.cc.u32 %9, %9, 0;\n\taddc.cc.u32 %10, %10, 0;\n\taddc.cc.u32 %11, %11, 0;\n\taddc.cc.u32 %12, %12, 0;\n\taddc.cc.u32 %13, %13, 0;\n\taddc.cc.u32 %14, %14, 0;\n\taddc.cc.u32 %15, %15, 0;\n\taddc.cc.u32 %16, %16, 0;\n\taddc.u32 %17, %17, 0;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17])
        : "r"(t0), "r"(t1), "r"(t2));
}
template <> __device__ __forceinline__ void crt_mac<20>(uint32_t (&a)[22], uint32_t t, const uint32_t (&m)[20]) {
    asm("mad.lo.cc.u32 %0, %42, %22, %0;\n\tmadc.lo.cc.u32 %1, %42, %23, %1;\n\tmadc.lo.cc.u32 %2, %42, %24, %2;\n\tmadc.lo.cc.u32 %3, %42, %25, %3;\n\tmadc.lo.cc.u32 %4, %42, %26, %4;\n\tmadc.lo.cc.u32 %5, %42, %27, %5;\n\tmadc.lo.cc.u32 %6, %42, %28, %6;\n\tmadc.lo.cc.u32 %7, %42, %29, %7;\n\tmadc.lo.cc.u32 %8, %42, %30, %8;\n\tmadc.lo.cc.u32 %9, %42, %31, %9;\n\tmadc.lo.cc.u32 %10, %42, %32, %10;\n\tmadc.lo.cc.u32 %11, %42, %33, %11;\n\tmadc.lo.cc.u32 %12, %42, %34, %12;\n\tmadc.lo.cc.u32 %13, %42, %35, %13;\n\tmadc.lo.cc.u32 %14, %42, %36, %14;\n\tmadc.lo.cc.u32 %15, %42, %37, %15;\n\tmadc.lo.cc.u32 %16, %42, %38, %16;\n\tmadc.lo.cc.u32 %17, %42, %39, %17;\n\tmadc.lo.cc.u32 %18, %42, %40, %18;\n\tmadc.lo.cc.u32 %19, %42, %41, %19;\n\taddc.cc.u32 %20, %20, 0;\n\taddc.u32 %21, %21, 0;\n\tmad.hi.cc.u32 %1, %42, %22, %1;\n\tmadc.hi.cc.u32 %2, %42, %23, %2;\n\tmadc.hi.cc.u32 %3, %42, %24, %3;\n\tmadc.hi.cc.u32 %4, %42, %25, %4;\n\tmadc.hi.cc.u32 %5, %42, %26, %5;\n\tmadc.hi.cc.u32 %6, %42, %27, %6;\n\tmadc.hi.cc.u32 %7, %42, %28, %7;\n\tmadc.hi.cc.u32 %8, %42, %29, %8;\n\tmadc.hi.cc.u32 %9, %42, %30, %9;\n\tmadc.hi.cc.u32 %10, %42, %31, %10;\n\tmadc.hi.cc.u32 %11, %42, %32, %11;\n\tmadc.hi.cc.u32 %12, %42, %33, %12;\n\tmadc.hi.cc.u32 %13, %42, %34, %13;\n\tmadc.hi.cc.u32 %14, %42, %35, %14;\n\tmadc.hi.cc.u32 %15, %42, %36, %15;\n\tmadc.hi.cc.u32 %16, %42, %37, %16;\n\tmadc.hi.cc.u32 %17, %42, %38, %17;\n\tmadc.hi.cc.u32 %18, %42, %39, %18;\n\tmadc.hi.cc.u32 %19, %42, %40, %19;\n\tmadc.hi.cc.u32 %20, %42, %41, %20;\n\taddc.u32 %21, %21, 0;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21])
        : "r"(m[0]), "r"(m[1]), "r"(m[2]), "r"(m[3]), "r"(m[4]), "r"(m[5]), "r"(m[6]), "r"(m[7]), "r"(m[8]), "r"(m[9]), "r"(m[10]), "r"(m[11]), "r"(m[12]), "r"(m[13]), "r"(m[14]), "r"(m[15]), "r"(m[16]), "r"(m[17]), "r"(m[18]), "r"(m[19]), "r"(t));
}
template <> __device__ __forceinline__ uint32_t mp_sub<20>(uint32_t (&a)[20], const uint32_t (&b)[20]) {
    uint32_t mask;
    asm("sub.cc.u32 %1, %1, %21;\n\tsubc.cc.u32 %2, %2, %22;\n\tsubc.cc.u32 %3, %3, %23;\n\tsubc.cc.u32 %4, %4, %24;\n\tsubc.cc.u32 %5, %5, %25;\n\tsubc.cc.u32 %6, %6, %26;\n\tsubc.cc.u32 %7, %7, %27;\n\tsubc.cc.u32 %8, %8, %28;\n\tsubc.cc.u32 %9, %9, %29;\n\tsubc.cc.u32 %10, %10, %30;\n\tsubc.cc.u32 %11, %11, %31;\n\tsubc.cc.u32 %12, %12, %32;\n\tsubc.cc.u32 %13, %13, %33;\n\tsubc.cc.u32 %14, %14, %34;\n\tsubc.cc.u32 %15, %15, %35;\n\tsubc.cc.u32 %16, %16, %36;\n\tsubc.cc.u32 %17, %17, %37;\n\tsubc.cc.u32 %18, %18, %38;\n\tsubc.cc.u32 %19, %19, %39;\n\tsubc.cc.u32 %20, %20, %40;\n\tsubc.u32 %0, 0, 0;"
        : "=r"(mask), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]), "r"(b[18]), "r"(b[19]));
    return mask;
}
template <> __device__ __forceinline__ uint32_t mp_add<20>(uint32_t (&a)[20], const uint32_t (&b)[20]) {
    uint32_t carry;
    asm("add.cc.u32 %1, %1, %21;\n\taddc.cc.u32 %2, %2, %22;\n\taddc.cc.u32 %3, %3, %23;\n\taddc.cc.u32 %4, %4, %24;\n\taddc.cc.u32 %5, %5, %25;\n\taddc.cc.u32 %6, %6, %26;\n\taddc.cc.u32 %7, %7, %27;\n\taddc.cc.u32 %8, %8, %28;\n\taddc.cc.u32 %9, %9, %29;\n\taddc.cc.u32 %10, %10, %30;\n\taddc.cc.u32 %11, %11, %31;\n\taddc.cc.u32 %12, %12, %32;\n\taddc.cc.u32 %13, %13, %33;\n\taddc.cc.u32 %14, %14, %34;\n\taddc.cc.u32 %15, %15, %35;\n\taddc.cc.u32 %16, %16, %36;\n\taddc.cc.u32 %17, %17, %37;\n\taddc.cc.u32 %18, %18, %38;\n\taddc.cc.u32 %19, %19, %39;\n\taddc.cc.u32 %20, %20, %40;\n\taddc.u32 %0, 0, 0;"
        : "=r"(carry), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]), "r"(b[18]), "r"(b[19]));
    return carry;
}
template <> __device__ __forceinline__ uint32_t mp_sub<22>(uint32_t (&a)[22], const uint32_t (&b)[22]) {
    uint32_t mask;
    asm("sub.cc.u32 %1, %1, %23;\n\tsubc.cc.u32 %2, %2, %24;\n\tsubc.cc.u32 %3, %3, %25;\n\tsubc.cc.u32 %4, %4, %26;\n\tsubc.cc.u32 %5, %5, %27;\n\tsubc.cc.u32 %6, %6, %28;\n\tsubc.cc.u32 %7, %7, %29;\n\tsubc.cc.u32 %8, %8, %30;\n\tsubc.cc.u32 %9, %9, %31;\n\tsubc.cc.u32 %10, %10, %32;\n\tsubc.cc.u32 %11, %11, %33;\n\tsubc.cc.u32 %12, %12, %34;\n\tsubc.cc.u32 %13, %13, %35;\n\tsubc.cc.u32 %14, %14, %36;\n\tsubc.cc.u32 %15, %15, %37;\n\tsubc.cc.u32 %16, %16, %38;\n\tsubc.cc.u32 %17, %17, %39;\n\tsubc.cc.u32 %18, %18, %40;\n\tsubc.cc.u32 %19, %19, %41;\n\tsubc.cc.u32 %20, %20, %42;\n\tsubc.cc.u32 %21, %21, %43;\n\tsubc.cc.u32 %22, %22, %44;\n\tsubc.u32 %0, 0, 0;"
        : "=r"(mask), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]), "r"(b[18]), "r"(b[19]), "r"(b[20]), "r"(b[21]));
    return mask;
}
template <> __device__ __forceinline__ uint32_t mp_add<22>(uint32_t (&a)[22], const uint32_t (&b)[22]) {
    uint32_t carry;
    asm("add.cc.u32 %1, %1, %23;\n\taddc.cc.u32 %2, %2, %24;\n\taddc.cc.u32 %3, %3, %25;\n\taddc.cc.u32 %4, %4, %26;\n\taddc.cc.u32 %5, %5, %27;\n\taddc.cc.u32 %6, %6, %28;\n\taddc.cc.u32 %7, %7, %29;\n\taddc.cc.u32 %8, %8, %30;\n\taddc.cc.u32 %9, %9, %31;\n\taddc.cc.u32 %10, %10, %32;\n\taddc.cc.u32 %11, %11, %33;\n\taddc.cc.u32 %12, %12, %34;\n\taddc.cc.u32 %13, %13, %35;\n\taddc.cc.u32 %14, %14, %36;\n\taddc.cc.u32 %15, %15, %37;\n\taddc.cc.u32 %16, %16, %38;\n\taddc.cc.u32 %17, %17, %39;\n\taddc.cc.u32 %18, %18, %40;\n\taddc.cc.u32 %19, %19, %41;\n\taddc.cc.u32 %20, %20, %42;\n\taddc.cc.u32 %21, %21, %43;\n\taddc.cc.u32 %22, %22, %44;\n\taddc.u32 %0, 0, 0;"
        : "=r"(carry), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]), "r"(b[18]), "r"(b[19]), "r"(b[20]), "r"(b[21]));
    return carry;
}
template <> __device__ __forceinline__ void mp_sub_hi<20>(uint32_t (&a)[22], const uint32_t (&b)[22]) {
    asm("sub.cc.u32 %1, %1, %22;\n\tsubc.cc.u32 %2, %2, %23;\n\tsubc.cc.u32 %3, %3, %24;\n\tsubc.cc.u32 %4, %4, %25;\n\tsubc.cc.u32 %5, %5, %26;\n\tsubc.cc.u32 %6, %6, %27;\n\tsubc.cc.u32 %7, %7, %28;\n\tsubc.cc.u32 %8, %8, %29;\n\tsubc.cc.u32 %9, %9, %30;\n\tsubc.cc.u32 %10, %10, %31;\n\tsubc.cc.u32 %11, %11, %32;\n\tsubc.cc.u32 %12, %12, %33;\n\tsubc.cc.u32 %13, %13, %34;\n\tsubc.cc.u32 %14, %14, %35;\n\tsubc.cc.u32 %15, %15, %36;\n\tsubc.cc.u32 %16, %16, %37;\n\tsubc.cc.u32 %17, %17, %38;\n\tsubc.cc.u32 %18, %18, %39;\n\tsubc.cc.u32 %19, %19, %40;\n\tsubc.cc.u32 %20, %20, %41;\n\tsubc.cc.u32 %21, %21, %42;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]), "r"(b[18]), "r"(b[19]), "r"(b[20]));
}
template <> __device__ __forceinline__ void mp_add3<22>(uint32_t (&a)[22], uint32_t t0, uint32_t t1, uint32_t t2) {
    asm("add.cc.u32 %0, %0, %22;\n\taddc.cc.u32 %1, %1, %23;\n\taddc.cc.u32 %2, %2, %24;\n\taddc.cc.u32 %3, %3, 0;\n\taddc.cc.u32 %4, %4, 0;\n\taddc.cc.u32 %5, %5, 0;\n\taddc.cc.u32 %6, %6, 0;\n\taddc.cc.u32 %7, %7, 0;\n\taddc.cc.u32 %8, %8, 0;\n\taddc.cc.u32 %9, %9, 0;\n\taddc.cc.u32 %10, %10, 0;\n\taddc.cc.u32 %11, %11, 0;\n\taddc.cc.u32 %12, %12, 0;\n\taddc.cc.u32 %13, %13, 0;\n\taddc.cc.u32 %14, %14, 0;\n\taddc.cc.u32 %15, %15, 0;\n\taddc.cc.u32 %16, %16, 0;\n\taddc.cc.u32 %17, %17, 0;\n\taddc.cc.u32 %18, %18, 0;\n\taddc.cc.u32 %19, %19, 0;\n\taddc.cc.u32 %20, %20, 0;\n\taddc.u32 %21, %21, 0;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21])
        : "r"(t0), "r"(t1), "r"(t2));
}
template <> __device__ __forceinline__ void crt_mac<24>(uint32_t (&a)[26], uint32_t t, const uint32_t (&m)[24]) {
    asm("mad.lo.cc.u32 %0, %50, %26, %0;\n\tmadc.lo.cc.u32 %1, %50, %27, %1;\n\tmadc.lo.cc.u32 %2, %50, %28, %2;\n\tmadc.lo.cc.u32 %3, %50, %29, %3;\n\tmadc.lo.cc.u32 %4, %50, %30, %4;\n\tmadc.lo.cc.u32 %5, %50, %31, %5;\n\tmadc.lo.cc.u32 %6, %50, %32, %6;\n\tmadc.lo.cc.u32 %7, %50, %33, %7;\n\tmadc.lo.cc.u32 %8, %50, %34, %8;\n\tmadc.lo.cc.u32 %9, %50, %35, %9;\n\tmadc.lo.cc.u32 %10, %50, %36, %10;\n\tmadc.lo.cc.u32 %11, %50, %37, %11;\n\tmadc.lo.cc.u32 %12, %50, %38, %12;\n\tmadc.lo.cc.u32 %13, %50, %39, %13;\n\tmadc.lo.cc.u32 %14, %50, %40, %14;\n\tmadc.lo.cc.u32 %15, %50, %41, %15;\n\tmadc.lo.cc.u32 %16, %50, %42, %16;\n\tmadc.lo.cc.u32 %17, %50, %43, %17;\n\tmadc.lo.cc.u32 %18, %50, %44, %18;\n\tmadc.lo.cc.u32 %19, %50, %45, %19;\n\tmadc.lo.cc.u32 %20, %50, %46, %20;\n\tmadc.lo.cc.u32 %21, %50, %47, %21;\n\tmadc.lo.cc.u32 %22, %50, %48, %22;\n\tmadc.lo.cc.u32 %23, %50, %49, %23;\n\taddc.cc.u32 %24, %24, 0;\n\taddc.u32 %25, %25, 0;\n\tmad.hi.cc.u32 %1, %50, %26, %1;\n\tmadc.hi.cc.u32 %2, %50, %27, %2;\n\tmadc.hi.cc.u32 %3, %50, %28, %3;\n\tmadc.hi.cc.u32 %4, %50, %29, %4;\n\tmadc.hi.cc.u32 %5, %50, %30, %5;\n\tmadc.hi.cc.u32 %6, %50, %31, %6;\n\tmadc.hi.cc.u32 %7, %50, %32, %7;\n\tmadc.hi.cc.u32 %8, %50, %33, %8;\n\tmadc.hi.cc.u32 %9, %50, %34, %9;\n\tmadc.hi.cc.u32 %10, %50, %35, %10;\n\tmadc.hi.cc.u32 %11, %50, %36, %11;\n\tmadc.hi.cc.u32 %12, %50, %37, %12;\n\tmadc.hi.cc.u32 %13, %50, %38, %13;\n\tmadc.hi.cc.u32 %14, %50, %39, %14;\n\tmadc.hi.cc.u32 %15, %50, %40, %15;\n\tmadc.hi.cc.u32 %16, %50, %41, %16;\n\tmadc.hi.cc.u32 %17, %50, %42, %17;\n\tmadc.hi.cc.u32 %18, %50, %43, %18;\n\tmadc.hi.cc.u32 %19, %50, %44, %19;\n\tmadc.hi.cc.u32 %20, %50, %45, %20;\n\tmadc.hi.cc.u32 %21, %50, %46, %21;\n\tmadc.hi.cc.u32 %22, %50, %47, %22;\n\tmadc.hi.cc.u32 %23, %50, %48, %23;\n\tmadc.hi.cc.u32 %24, %50, %49, %24;\n\taddc.u32 %25, %25, 0;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21]), "+r"(a[22]), "+r"(a[23]), "+r"(a[24]), "+r"(a[25])
        : "r"(m[0]), "r"(m[1]), "r"(m[2]), "r"(m[3]), "r"(m[4]), "r"(m[5]), "r"(m[6]), "r"(m[7]), "r"(m[8]), "r"(m[9]), "r"(m[10]), "r"(m[11]), "r"(m[12]), "r"(m[13]), "r"(m[14]), "r"(m[15]), "r"(m[16]), "r"(m[17]), "r"(m[18]), "r"(m[19]), "r"(m[20]), "r"(m[21]), "r"(m[22]), "r"(m[23]), "r"(t));
}
template <> __device__ __forceinline__ uint32_t mp_sub<24>(uint32_t (&a)[24], const uint32_t (&b)[24]) {
    uint32_t mask;
    asm("sub.cc.u32 %1, %1, %25;\n\tsubc.cc.u32 %2, %2, %26;\n\tsubc.cc.u32 %3, %3, %27;\n\tsubc.cc.u32 %4, %4, %28;\n\tsubc.cc.u32 %5, %5, %29;\n\tsubc.cc.u32 %6, %6, %30;\n\tsubc.cc.u32 %7, %7, %31;\n\tsubc.cc.u32 %8, %8, %32;\n\tsubc.cc.u32 %9, %9, %33;\n\tsubc.cc.u32 %10, %10, %34;\n\tsubc.cc.u32 %11, %11, %35;\n\tsubc.cc.u32 %12, %12, %36;\n\tsubc.cc.u32 %13, %13, %37;\n\tsubc.cc.u32 %14, %14, %38;\n\tsubc.cc.u32 %15, %15, %39;\n\tsubc.cc.u32 %16, %16, %40;\n\tsubc.cc.u32 %17, %17, %41;\n\tsubc.cc.u32 %18, %18, %42;\n\tsubc.cc.u32 %19, %19, %43;\n\tsubc.cc.u32 %20, %20, %44;\n\tsubc.cc.u32 %21, %21, %45;\n\tsubc.cc.u32 %22, %22, %46;\n\tsubc.cc.u32 %23, %23, %47;\n\tsubc.cc.u32 %24, %24, %48;\n\tsubc.u32 %0, 0, 0;"
        : "=r"(mask), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21]), "+r"(a[22]), "+r"(a[23])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]), "r"(b[18]), "r"(b[19]), "r"(b[20]), "r"(b[21]), "r"(b[22]), "r"(b[23]));
    return mask;
}
template <> __device__ __forceinline__ uint32_t mp_add<24>(uint32_t (&a)[24], const uint32_t (&b)[24]) {
    uint32_t carry;
    asm("add.cc.u32 %1, %1, %25;\n\taddc.cc.u32 %2, %2, %26;\n\taddc.cc.u32 %3, %3, %27;\n\taddc.cc.u32 %4, %4, %28;\n\taddc.cc.u32 %5, %5, %29;\n\taddc.cc.u32 %6, %6, %30;\n\taddc.cc.u32 %7, %7, %31;\n\taddc.cc.u32 %8, %8, %32;\n\taddc.cc.u32 %9, %9, %33;\n\taddc.cc.u32 %10, %10, %34;\n\taddc.cc.u32 %11, %11, %35;\n\taddc.cc.u32 %12, %12, %36;\n\taddc.cc.u32 %13, %13, %37;\n\taddc.cc.u32 %14, %14, %38;\n\taddc.cc.u32 %15, %15, %39;\n\taddc.cc.u32 %16, %16, %40;\n\taddc.cc.u32 %17, %17, %41;\n\taddc.cc.u32 %18, %18, %42;\n\taddc.cc.u32 %19, %19, %43;\n\taddc.cc.u32 %20, %20, %44;\n\taddc.cc.u32 %21, %21, %45;\n\taddc.cc.u32 %22, %22, %46;\n\taddc.cc.u32 %23, %23, %47;\n\taddc.cc.u32 %24, %24, %48;\n\taddc.u32 %0, 0, 0;"
        : "=r"(carry), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21]), "+r"(a[22]), "+r"(a[23])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]), "r"(b[18]), "r"(b[19]), "r"(b[20]), "r"(b[21]), "r"(b[22]), "r"(b[23]));
    return carry;
}
template <> __device__ __forceinline__ uint32_t mp_sub<26>(uint32_t (&a)[26], const uint32_t (&b)[26]) {
    uint32_t mask;
    asm("sub.cc.u32 %1, %1, %27;\n\tsubc.cc.u32 %2, %2, %28;\n\tsubc.cc.u32 %3, %3, %29;\n\tsubc.cc.u32 %4, %4, %30;\n\tsubc.cc.u32 %5, %5, %31;\n\tsubc.cc.u32 %6, %6, %32;\n\tsubc.cc.u32 %7, %7, %33;\n\tsubc.cc.u32 %8, %8, %34;\n\tsubc.cc.u32 %9, %9, %35;\n\tsubc.cc.u32 %10, %10, %36;\n\tsubc.cc.u32 %11, %11, %37;\n\tsubc.cc.u32 %12, %12, %38;\n\tsubc.cc.u32 %13, %13, %39;\n\tsubc.cc.u32 %14, %14, %40;\n\tsubc.cc.u32 %15, %15, %41;\n\tsubc.cc.u32 %16, %16, %42;\n\tsubc.cc.u32 %17, %17, %43;\n\tsubc.cc.u32 %18, %18, %44;\n\tsubc.cc.u32 %19, %19, %45;\n\tsubc.cc.u32 %20, %20, %46;\n\tsubc.cc.u32 %21, %21, %47;\n\tsubc.cc.u32 %22, %22, %48;\n\tsubc.cc.u32 %23, %23, %49;\n\tsubc.cc.u32 %24, %24, %50;\n\tsubc.cc.u32 %25, %25, %51;\n\tsubc.cc.u32 %26, %26, %52;\n\tsubc.u32 %0, 0, 0;"
        : "=r"(mask), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21]), "+r"(a[22]), "+r"(a[23]), "+r"(a[24]), "+r"(a[25])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]), "r"(b[18]), "r"(b[19]), "r"(b[20]), "r"(b[21]), "r"(b[22]), "r"(b[23]), "r"(b[24]), "r"(b[25]));
    return mask;
}
template <> __device__ __forceinline__ uint32_t mp_add<26>(uint32_t (&a)[26], const uint32_t (&b)[26]) {
    uint32_t carry;
    asm("add.cc.u32 %1, %1, %27;\n\taddc.cc.u32 %2, %2, %28;\n\taddc.cc.u32 %3, %3, %29;\n\taddc.cc.u32 %4, %4, %30;\n\taddc.cc.u32 %5, %5, %31;\n\taddc.cc.u32 %6, %6, %32;\n\taddc.cc.u32 %7, %7, %33;\n\taddc.cc.u32 %8, %8, %34;\n\taddc.cc.u32 %9, %9, %35;\n\taddc.cc.u32 %10, %10, %36;\n\taddc.cc.u32 %11, %11, %37;\n\taddc.cc.u32 %12, %12, %38;\n\taddc.cc.u32 %13, %13, %39;\n\taddc.cc.u32 %14, %14, %40;\n\taddc.cc.u32 %15, %15, %41;\n\taddc.cc.u32 %16, %16, %42;\n\taddc.cc.u32 %17, %17, %43;\n\taddc.cc.u32 %18, %18, %44;\n\taddc.cc.u32 %19, %19, %45;\n\taddc.cc.u32 %20, %20, %46;\n\taddc.cc.u32 %21, %21, %47;\n\taddc.cc.u32 %22, %22, %48;\n\taddc.cc.u32 %23, %23, %49;\n\taddc.cc.u32 %24, %24, %50;\n\taddc.cc.u32 %25, %25, %51;\n\taddc.cc.u32 %26, %26, %52;\n\taddc.u32 %0, 0, 0;"
        : "=r"(carry), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21]), "+r"(a[22]), "+r"(a[23]), "+r"(a[24]), "+r"(a[25])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]), "r"(b[18]), "r"(b[19]), "r"(b[20]), "r"(b[21]), "r"(b[22]), "r"(b[23]), "r"(b[24]), "r"(b[25]));
    return carry;
}
template <> __device__ __forceinline__ void mp_sub_hi<24>(uint32_t (&a)[26], const uint32_t (&b)[26]) {
    asm("sub.cc.u32 %1, %1, %26;\n\tsubc.cc.u32 %2, %2, %27;\n\tsubc.cc.u32 %3, %3, %28;\n\tsubc.cc.u32 %4, %4, %29;\n\tsubc.cc.u32 %5, %5, %30;\n\tsubc.cc.u32 %6, %6, %31;\n\tsubc.cc.u32 %7, %7, %32;\n\tsubc.cc.u32 %8, %8, %33;\n\tsubc.cc.u32 %9, %9, %34;\n\tsubc.cc.u32 %10, %10, %35;\n\tsubc.cc.u32 %11, %11, %36;\n\tsubc.cc.u32 %12, %12, %37;\n\tsubc.cc.u32 %13, %13, %38;\n\tsubc.cc.u32 %14, %14, %39;\n\tsubc.cc.u32 %15, %15, %40;\n\tsubc.cc.u32 %16, %16, %41;\n\tsubc.cc.u32 %17, %17, %42;\n\tsubc.cc.u32 %18, %18, %43;\n\tsubc.cc.u32 %19, %19, %44;\n\tsubc.cc.u32 %20, %20, %45;\n\tsubc.cc.u32 %21, %21, %46;\n\tsubc.cc.u32 %22, %22, %47;\n\tsubc.cc.u32 %23, %23, %48;\n\tsubc.cc.u32 %24, %24, %49;\n\tsubc.cc.u32 %25, %25, %50;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21]), "+r"(a[22]), "+r"(a[23]), "+r"(a[24]), "+r"(a[25])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]), "r"(b[18]), "r"(b[19]), "r"(b[20]), "r"(b[21]), "r"(b[22]), "r"(b[23]), "r"(b[24]));
}
template <> __device__ __forceinline__ void mp_add3<26>(uint32_t (&a)[26], uint32_t t0, uint32_t t1, uint32_t t2) {
    asm("add.cc.u32 %0, %0, %26;\n\taddc.cc.u32 %1, %1, %27;\n\taddc.cc.u32 %2, %2, %28;\n\taddc.cc.u32 %3, %3, 0;\n\taddc.cc.u32 %4, %4, 0;\n\taddc.cc.u32 %5, %5, 0;\n\taddc.cc.u32 %6, %6, 0;\n\taddc.cc.u32 %7, %7, 0;\n\taddc.cc.u32 %8, %8, 0;\n\taddc.cc.u32 %9, %9, 0;\n\taddc.cc.u32 %10, %10, 0;\n\taddc.cc.u32 %11, %11, 0;\n\taddc.cc.u32 %12, %12, 0;\n\taddc.cc.u32 %13, %13, 0;\n\taddc.cc.u32 %14, %14, 0;\n\taddc.cc.u32 %15, %15, 0;\n\taddc.cc.u32 %16, %16, 0;\n\taddc.cc.u32 %17, %17, 0;\n\taddc.cc.u32 %18, %18, 0;\n\taddc.cc.u32 %19, %19, 0;\n\taddc.cc.u32 %20, %20, 0;\n\taddc.cc.u32 %21, %21, 0;\n\taddc.cc.u32 %22, %22, 0;\n\taddc.cc.u32 %23, %23, 0;\n\taddc.cc.u32 %24, %24, 0;\n\taddc.u32 %25, %25, 0;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21]), "+r"(a[22]), "+r"(a[23]), "+r"(a[24]), "+r"(a[25])
        : "r"(t0), "r"(t1), "r"(t2));
}
template <> __device__ __forceinline__ void crt_mac<28>(uint32_t (&a)[30], uint32_t t, const uint32_t (&m)[28]) {
    asm("mad.lo.cc.u32 %0, %58, %30, %0;\n\tmadc.lo.cc.u32 %1, %58, %31, %1;\n\tmadc.lo.cc.u32 %2, %58, %32, %2;\n\tmadc.lo.cc.u32 %3, %58, %33, %3;\n\tmadc.lo.cc.u32 %4, %58, %34, %4;\n\tmadc.lo.cc.u32 %5, %58, %35, %5;\n\tmadc.lo.cc.u32 %6, %58, %36, %6;\n\tmadc.lo.cc.u32 %7, %58, %37, %7;\n\tmadc.lo.cc.u32 %8, %58, %38, %8;\n\tmadc.lo.cc.u32 %9, %58, %39, %9;\n\tmadc.lo.cc.u32 %10, %58, %40, %10;\n\tmadc.lo.cc.u32 %11, %58, %41, %11;\n\tmadc.lo.cc.u32 %12, %58, %42, %12;\n\tmadc.lo.cc.u32 %13, %58, %43, %13;\n\tmadc.lo.cc.u32 %14, %58, %44, %14;\n\tmadc.lo.cc.u32 %15, %58, %45, %15;\n\tmadc.lo.cc.u32 %16, %58, %46, %16;\n\tmadc.lo.cc.u32 %17, %58, %47, %17;\n\tmadc.lo.cc.u32 %18, %58, %48, %18;\n\tmadc.lo.cc.u32 %19, %58, %49, %19;\n\tmadc.lo.cc.u32 %20, %58, %50, %20;\n\tmadc.lo.cc.u32 %21, %58, %51, %21;\n\tmadc.lo.cc.u32 %22, %58, %52, %22;\n\tmadc.lo.cc.u32 %23, %58, %53, %23;\n\tmadc.lo.cc.u32 %24, %58, %54, %24;\n\tmadc.lo.cc.u32 %25, %58, %55, %25;\n\tmadc.lo.cc.u32 %26, %58, %56, %26;\n\tmadc.lo.cc.u32 %27, %58, %57, %27;\n\taddc.cc.u32 %28, %28, 0;\n\taddc.u32 %29, %29, 0;\n\tmad.hi.cc.u32 %1, %58, %30, %1;\n\tmadc.hi.cc.u32 %2, %58, %31, %2;\n\tmadc.hi.cc.u32 %3, %58, %32, %3;\n\tmadc.hi.cc.u32 %4, %58, %33, %4;\n\tmadc.hi.cc.u32 %5, %58, %34, %5;\n\tmadc.hi.cc.u32 %6, %58, %35, %6;\n\tmadc.hi.cc.u32 %7, %58, %36, %7;\n\tmadc.hi.cc.u32 %8, %58, %37, %8;\n\tmadc.hi.cc.u32 %9, %58, %38, %9;\n\tmadc.hi.cc.u32 %10, %58, %39, %10;\n\tmadc.hi.cc.u32 %11, %58, %40, %11;\n\tmadc.hi.cc.u32 %12, %58, %41, %12;\n\tmadc.hi.cc.u32 %13, %58, %42, %13;\n\tmadc.hi.cc.u32 %14, %58, %43, %14;\n\tmadc.hi.cc.u32 %15, %58, %44, %15;\n\tmadc.hi.cc.u32 %16, %58, %45, %16;\n\tmadc.hi.cc.u32 %17, %58, %46, %17;\n\tmadc.hi.cc.u32 %18, %58, %47, %18;\n\tmadc.hi.cc.u32 %19, %58, %48, %19;\n\tmadc.hi.cc.u32 %20, %58, %49, %20;\n\tmadc.hi.cc.u32 %21, %58, %50, %21;\n\tmadc.hi.cc.u32 %22, %58, %51, %22;\n\tmadc.hi.cc.u32 %23, %58, %52, %23;\n\tmadc.hi.cc.u32 %24, %58, %53, %24;\n\tmadc.hi.cc.u32 %25, %58, %54, %25;\n\tmadc.hi.cc.u32 %26, %58, %55, %26;\n\tmadc.hi.cc.u32 %27, %58, %56, %27;\n\tmadc.hi.cc.u32 %28, %58, %57, %28;\n\taddc.u32 %29, %29, 0;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21]), "+r"(a[22]), "+r"(a[23]), "+r"(a[24]), "+r"(a[25]), "+r"(a[26]), "+r"(a[27]), "+r"(a[28]), "+r"(a[29])
        : "r"(m[0]), "r"(m[1]), "r"(m[2]), "r"(m[3]), "r"(m[4]), "r"(m[5]), "r"(m[6]), "r"(m[7]), "r"(m[8]), "r"(m[9]), "r"(m[10]), "r"(m[11]), "r"(m[12]), "r"(m[13]), "r"(m[14]), "r"(m[15]), "r"(m[16]), "r"(m[17]), "r"(m[18]), "r"(m[19]), "r"(m[20]), "r"(m[21]), "r"(m[22]), "r"(m[23]), "r"(m[24]), "r"(m[25]), "r"(m[26]), "r"(m[27]), "r"(t));
}
template <> __device__ __forceinline__ uint32_t mp_sub<28>(uint32_t (&a)[28], const uint32_t (&b)[28]) {
    uint32_t mask;
    asm("sub.cc.u32 %1, %1, %29;\n\tsubc.cc.u32 %2, %2, %30;\n\tsubc.cc.u32 %3, %3, %31;\n\tsubc.cc.u32 %4, %4, %32;\n\tsubc.cc.u32 %5, %5, %33;\n\tsubc.cc.u32 %6, %6, %34;\n\tsubc.cc.u32 %7, %7, %35;\n\tsubc.cc.u32 %8, %8, %36;\n\tsubc.cc.u32 %9, %9, %37;\n\tsubc.cc.u32 %10, %10, %38;\n\tsubc.cc.u32 %11, %11, %39;\n\tsubc.cc.u32 %12, %12, %40;\n\tsubc.cc.u32 %13, %13, %41;\n\tsubc.cc.u32 %14, %14, %42;\n\tsubc.cc.u32 %15, %15, %43;\n\tsubc.cc.u32 %16, %16, %44;\n\tsubc.cc.u32 %17, %17, %45;\n\tsubc.cc.u32 %18, %18, %46;\n\tsubc.cc.u32 %19, %19, %47;\n\tsubc.cc.u32 %20, %20, %48;\n\tsubc.cc.u32 %21, %21, %49;\n\tsubc.cc.u32 %22, %22, %50;\n\tsubc.cc.u32 %23, %23, %51;\n\tsubc.cc.u32 %24, %24, %52;\n\tsubc.cc.u32 %25, %25, %53;\n\tsubc.cc.u32 %26, %26, %54;\n\tsubc.cc.u32 %27, %27, %55;\n\tsubc.cc.u32 %28, %28, %56;\n\tsubc.u32 %0, 0, 0;"
        : "=r"(mask), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21]), "+r"(a[22]), "+r"(a[23]), "+r"(a[24]), "+r"(a[25]), "+r"(a[26]), "+r"(a[27])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]), "r"(b[18]), "r"(b[19]), "r"(b[20]), "r"(b[21]), "r"(b[22]), "r"(b[23]), "r"(b[24]), "r"(b[25]), "r"(b[26]), "r"(b[27]));
    return mask;
}
template <> __device__ __forceinline__ uint32_t mp_add<28>(uint32_t (&a)[28], const uint32_t (&b)[28]) {
    uint32_t carry;
    asm("add.cc.u32 %1, %1, %29;\n\taddc.cc.u32 %2, %2, %30;\n\taddc.cc.u32 %3, %3, %31;\n\taddc.cc.u32 %4, %4, %32;\n\taddc.cc.u32 %5, %5, %33;\n\taddc.cc.u32 %6, %6, %34;\n\taddc.cc.u32 %7, %7, %35;\n\taddc.cc.u32 %8, %8, %36;\n\taddc.cc.u32 %9, %9, %37;\n\taddc.cc.u32 %10, %10, %38;\n\taddc.cc.u32 %11, %11, %39;\n\taddc.cc.u32 %12, %12, %40;\n\taddc.cc.u32 %13, %13, %41;\n\taddc.cc.u32 %14, %14, %42;\n\taddc.cc.u32 %15, %15, %43;\n\taddc.cc.u32 %16, %16, %44;\n\taddc.cc.u32 %17, %17, %45;\n\taddc.cc.u32 %18, %18, %46;\n\taddc.cc.u32 %19, %19, %47;\n\taddc.cc.u32 %20, %20, %48;\n\taddc.cc.u32 %21, %21, %49;\n\taddc.cc.u32 %22, %22, %50;\n\taddc.cc.u32 %23, %23, %51;\n\taddc.cc.u32 %24, %24, %52;\n\taddc.cc.u32 %25, %25, %53;\n\taddc.cc.u32 %26, %26, %54;\n\taddc.cc.u32 %27, %27, %55;\n\taddc.cc.u32 %28, %28, %56;\n\taddc.u32 %0, 0, 0;"
        : "=r"(carry), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21]), "+r"(a[22]), "+r"(a[23]), "+r"(a[24]), "+r"(a[25]), "+r"(a[26]), "+r"(a[27])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]), "r"(b[18]), "r"(b[19]), "r"(b[20]), "r"(b[21]), "r"(b[22]), "r"(b[23]), "r"(b[24]), "r"(b[25]), "r"(b[26]), "r"(b[27]));
    return carry;
}
template <> __device__ __forceinline__ uint32_t mp_sub<30>(uint32_t (&a)[30], const uint32_t (&b)[30]) {
    uint32_t mask;
    asm("sub.cc.u32 %1, %1, %31;\n\tsubc.cc.u32 %2, %2, %32;\n\tsubc.cc.u32 %3, %3, %33;\n\tsubc.cc.u32 %4, %4, %34;\n\tsubc.cc.u32 %5, %5, %35;\n\tsubc.cc.u32 %6, %6, %36;\n\tsubc.cc.u32 %7, %7, %37;\n\tsubc.cc.u32 %8, %8, %38;\n\tsubc.cc.u32 %9, %9, %39;\n\tsubc.cc.u32 %10, %10, %40;\n\tsubc.cc.u32 %11, %11, %41;\n\tsubc.cc.u32 %12, %12, %42;\n\tsubc.cc.u32 %13, %13, %43;\n\tsubc.cc.u32 %14, %14, %44;\n\tsubc.cc.u32 %15, %15, %45;\n\tsubc.cc.u32 %16, %16, %46;\n\tsubc.cc.u32 %17, %17, %47;\n\tsubc.cc.u32 %18, %18, %48;\n\tsubc.cc.u32 %19, %19, %49;\n\tsubc.cc.u32 %20, %20, %50;\n\tsubc.cc.u32 %21, %21, %51;\n\tsubc.cc.u32 %22, %22, %52;\n\tsubc.cc.u32 %23, %23, %53;\n\tsubc.cc.u32 %24, %24, %54;\n\tsubc.cc.u32 %25, %25, %55;\n\tsubc.cc.u32 %26, %26, %56;\n\tsubc.cc.u32 %27, %27, %57;\n\tsubc.cc.u32 %28, %28, %58;\n\tsubc.cc.u32 %29, %29, %59;\n\tsubc.cc.u32 %30, %30, %60;\n\tsubc.u32 %0, 0, 0;"
        : "=r"(mask), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21]), "+r"(a[22]), "+r"(a[23]), "+r"(a[24]), "+r"(a[25]), "+r"(a[26]), "+r"(a[27]), "+r"(a[28]), "+r"(a[29])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]), "r"(b[18]), "r"(b[19]), "r"(b[20]), "r"(b[21]), "r"(b[22]), "r"(b[23]), "r"(b[24]), "r"(b[25]), "r"(b[26]), "r"(b[27]), "r"(b[28]), "r"(b[29]));
    return mask;
}
template <> __device__ __forceinline__ uint32_t mp_add<30>(uint32_t (&a)[30], const uint32_t (&b)[30]) {
    uint32_t carry;
    asm("add.cc.u32 %1, %1, %31;\n\taddc.cc.u32 %2, %2, %32;\n\taddc.cc.u32 %3, %3, %33;\n\taddc.cc.u32 %4, %4, %34;\n\taddc.cc.u32 %5, %5, %35;\n\taddc.cc.u32 %6, %6, %36;\n\taddc.cc.u32 %7, %7, %37;\n\taddc.cc.u32 %8, %8, %38;\n\taddc.cc.u32 %9, %9, %39;\n\taddc.cc.u32 %10, %10, %40;\n\taddc.cc.u32 %11, %11, %41;\n\taddc.cc.u32 %12, %12, %42;\n\taddc.cc.u32 %13, %13, %43;\n\taddc.cc.u32 %14, %14, %44;\n\taddc.cc.u32 %15, %15, %45;\n\taddc.cc.u32 %16, %16, %46;\n\taddc.cc.u32 %17, %17, %47;\n\taddc.cc.u32 %18, %18, %48;\n\taddc.cc.u32 %19, %19, %49;\n\taddc.cc.u32 %20, %20, %50;\n\taddc.cc.u32 %21, %21, %51;\n\taddc.cc.u32 %22, %22, %52;\n\taddc.cc.u32 %23, %23, %53;\n\taddc.cc.u32 %24, %24, %54;\n\taddc.cc.u32 %25, %25, %55;\n\taddc.cc.u32 %26, %26, %56;\n\taddc.cc.u32 %27, %27, %57;\n\taddc.cc.u32 %28, %28, %58;\n\taddc.cc.u32 %29, %29, %59;\n\taddc.cc.u32 %30, %30, %60;\n\taddc.u32 %0, 0, 0;"
        : "=r"(carry), "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21]), "+r"(a[22]), "+r"(a[23]), "+r"(a[24]), "+r"(a[25]), "+r"(a[26]), "+r"(a[27]), "+r"(a[28]), "+r"(a[29])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]), "r"(b[18]), "r"(b[19]), "r"(b[20]), "r"(b[21]), "r"(b[22]), "r"(b[23]), "r"(b[24]), "r"(b[25]), "r"(b[26]), "r"(b[27]), "r"(b[28]), "r"(b[29]));
    return carry;
}
template <> __device__ __forceinline__ void mp_sub_hi<28>(uint32_t (&a)[30], const uint32_t (&b)[30]) {
    asm("sub.cc.u32 %1, %1, %30;\n\tsubc.cc.u32 %2, %2, %31;\n\tsubc.cc.u32 %3, %3, %32;\n\tsubc.cc.u32 %4, %4, %33;\n\tsubc.cc.u32 %5, %5, %34;\n\tsubc.cc.u32 %6, %6, %35;\n\tsubc.cc.u32 %7, %7, %36;\n\tsubc.cc.u32 %8, %8, %37;\n\tsubc.cc.u32 %9, %9, %38;\n\tsubc.cc.u32 %10, %10, %39;\n\tsubc.cc.u32 %11, %11, %40;\n\tsubc.cc.u32 %12, %12, %41;\n\tsubc.cc.u32 %13, %13, %42;\n\tsubc.cc.u32 %14, %14, %43;\n\tsubc.cc.u32 %15, %15, %44;\n\tsubc.cc.u32 %16, %16, %45;\n\tsubc.cc.u32 %17, %17, %46;\n\tsubc.cc.u32 %18, %18, %47;\n\tsubc.cc.u32 %19, %19, %48;\n\tsubc.cc.u32 %20, %20, %49;\n\tsubc.cc.u32 %21, %21, %50;\n\tsubc.cc.u32 %22, %22, %51;\n\tsubc.cc.u32 %23, %23, %52;\n\tsubc.cc.u32 %24, %24, %53;\n\tsubc.cc.u32 %25, %25, %54;\n\tsubc.cc.u32 %26, %26, %55;\n\tsubc.cc.u32 %27, %27, %56;\n\tsubc.cc.u32 %28, %28, %57;\n\tsubc.cc.u32 %29, %29, %58;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21]), "+r"(a[22]), "+r"(a[23]), "+r"(a[24]), "+r"(a[25]), "+r"(a[26]), "+r"(a[27]), "+r"(a[28]), "+r"(a[29])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]), "r"(b[12]), "r"(b[13]), "r"(b[14]), "r"(b[15]), "r"(b[16]), "r"(b[17]), "r"(b[18]), "r"(b[19]), "r"(b[20]), "r"(b[21]), "r"(b[22]), "r"(b[23]), "r"(b[24]), "r"(b[25]), "r"(b[26]), "r"(b[27]), "r"(b[28]));
}
template <> __device__ __forceinline__ void mp_add3<30>(uint32_t (&a)[30], uint32_t t0, uint32_t t1, uint32_t t2) {
    asm("add.cc.u32 %0, %0, %30;\n\taddc.cc.u32 %1, %1, %31;\n\taddc.cc.u32 %2, %2, %32;\n\taddc.cc.u32 %3, %3, 0;\n\taddc.cc.u32 %4, %4, 0;\n\taddc.cc.u32 %5, %5, 0;\n\taddc.cc.u32 %6, %6, 0;\n\taddc.cc.u32 %7, %7, 0;\n\taddc.cc.u32 %8, %8, 0;\n\taddc.cc.u32 %9, %9, 0;\n\taddc.cc.u32 %10, %10, 0;\n\taddc.cc.u32 %11, %11, 0;\n\taddc.cc.u32 %12, %12, 0;\n\taddc.cc.u32 %13, %13, 0;\n\taddc.cc.u32 %14, %14, 0;\n\taddc.cc.u32 %15, %15, 0;\n\taddc.cc.u32 %16, %16, 0;\n\taddc.cc.u32 %17, %17, 0;\n\taddc.cc.u32 %18, %18, 0;\n\taddc.cc.u32 %19, %19, 0;\n\taddc.cc.u32 %20, %20, 0;\n\taddc.cc.u32 %21, %21, 0;\n\taddc.cc.u32 %22, %22, 0;\n\taddc.cc.u32 %23, %23, 0;\n\taddc.cc.u32 %24, %24, 0;\n\taddc.cc.u32 %25, %25, 0;\n\taddc.cc.u32 %26, %26, 0;\n\taddc.cc.u32 %27, %27, 0;\n\taddc.cc.u32 %28, %28, 0;\n\taddc.u32 %29, %29, 0;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]), "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15]), "+r"(a[16]), "+r"(a[17]), "+r"(a[18]), "+r"(a[19]), "+r"(a[20]), "+r"(a[21]), "+r"(a[22]), "+r"(a[23]), "+r"(a[24]), "+r"(a[25]), "+r"(a[26]), "+r"(a[27]), "+r"(a[28]), "+r"(a[29])
        : "r"(t0), "r"(t1), "r"(t2));
}
}  // namespace pm
