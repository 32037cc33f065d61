"""Writes crt_mac.cuh: multiword helpers as single PTX carry chains, one
specialization per width W (python gen_crt_mac.py > crt_mac.cuh):

  crt_mac<W>(a[W+2], t, m[W])       a += t * m           (low halves into a[k], high halves into a[k+1])
  mp_sub<N>(a[N], b[N]) -> mask     a -= b, mask = 0xffffffff if it borrowed out, else 0
  mp_sub_hi<W>(a[W+2], b[W+2])      a -= b * 2^32 (b[W+1] must be 0)
  mp_add3<N>(a[N], t0, t1, t2)      a += t2 * 2^64 + t1 * 2^32 + t0 (carry out of a[N-1] dropped)
  mp_add<N>(a[N], b[N]) -> carry    a += b, carry = 1 if it carried out, else 0
(mp_sub and mp_add for N = W and N = W + 2.)
"""
WIDTHS = [4, 8, 12, 16, 20, 24, 28]


def mac_body(W):
    acc = [f"%{i}" for i in range(W + 2)]
    m = [f"%{W + 2 + i}" for i in range(W)]
    t = f"%{2 * W + 2}"
    lo = [f"mad.lo.cc.u32 {acc[0]}, {t}, {m[0]}, {acc[0]};"]
    lo += [f"madc.lo.cc.u32 {acc[k]}, {t}, {m[k]}, {acc[k]};" for k in range(1, W)]
    lo += [f"addc.cc.u32 {acc[W]}, {acc[W]}, 0;", f"addc.u32 {acc[W + 1]}, {acc[W + 1]}, 0;"]
    hi = [f"mad.hi.cc.u32 {acc[1]}, {t}, {m[0]}, {acc[1]};"]
    hi += [f"madc.hi.cc.u32 {acc[k + 1]}, {t}, {m[k]}, {acc[k + 1]};" for k in range(1, W)]
    hi += [f"addc.u32 {acc[W + 1]}, {acc[W + 1]}, 0;"]
    return "\\n\\t".join(lo + hi)


def sub_body(N):
    a = [f"%{i + 1}" for i in range(N)]
    b = [f"%{N + 1 + i}" for i in range(N)]
    lines = [f"sub.cc.u32 {a[0]}, {a[0]}, {b[0]};"]
    lines += [f"subc.cc.u32 {a[k]}, {a[k]}, {b[k]};" for k in range(1, N)]
    lines += ["subc.u32 %0, 0, 0;"]
    return "\\n\\t".join(lines)


def sub_hi_body(W):
    n = W + 2
    a = [f"%{i}" for i in range(n)]
    b = [f"%{n + i}" for i in range(n - 1)]
    lines = [f"sub.cc.u32 {a[1]}, {a[1]}, {b[0]};"]
    lines += [f"subc.cc.u32 {a[k]}, {a[k]}, {b[k - 1]};" for k in range(2, n)]
    return "\\n\\t".join(lines)


def add_body(N):
    a = [f"%{i + 1}" for i in range(N)]
    b = [f"%{N + 1 + i}" for i in range(N)]
    lines = [f"add.cc.u32 {a[0]}, {a[0]}, {b[0]};"]
    lines += [f"addc.cc.u32 {a[k]}, {a[k]}, {b[k]};" for k in range(1, N)]
    lines += ["addc.u32 %0, 0, 0;"]
    return "\\n\\t".join(lines)


def add3_body(N):
    a = [f"%{i}" for i in range(N)]
    lines = [f"add.cc.u32 {a[0]}, {a[0]}, %{N};", f"addc.cc.u32 {a[1]}, {a[1]}, %{N + 1};",
             f"addc.cc.u32 {a[2]}, {a[2]}, %{N + 2};"]
    lines += [f"addc.cc.u32 {a[k]}, {a[k]}, 0;" for k in range(3, N - 1)]
    lines += [f"addc.u32 {a[N - 1]}, {a[N - 1]}, 0;"]
    return "\\n\\t".join(lines)


def main():
    out = ["// Generated by gen_crt_mac.py -- do not edit.",
           "// Multiword arithmetic as PTX carry chains (see the generator for the contracts).",
           "#pragma once", "#include <cstdint>", "namespace pm {",
           "template <int W> __device__ __forceinline__ void crt_mac(uint32_t (&a)[W + 2], uint32_t t, const uint32_t (&m)[W]);",
           "template <int N> __device__ __forceinline__ uint32_t mp_sub(uint32_t (&a)[N], const uint32_t (&b)[N]);",
           "template <int W> __device__ __forceinline__ void mp_sub_hi(uint32_t (&a)[W + 2], const uint32_t (&b)[W + 2]);",
           "template <int N> __device__ __forceinline__ void mp_add3(uint32_t (&a)[N], uint32_t t0, uint32_t t1, uint32_t t2);",
           "template <int N> __device__ __forceinline__ uint32_t mp_add(uint32_t (&a)[N], const uint32_t (&b)[N]);"]
    for W in WIDTHS:
        outs = ", ".join(f'"+r"(a[{i}])' for i in range(W + 2))
        ins = ", ".join(f'"r"(m[{i}])' for i in range(W)) + ', "r"(t)'
        out.append(f"template <> __device__ __forceinline__ void crt_mac<{W}>(uint32_t (&a)[{W + 2}], uint32_t t, "
                   f"const uint32_t (&m)[{W}]) {{")
        out.append(f'    asm("{mac_body(W)}"\n        : {outs}\n        : {ins});')
        out.append("}")
        for N in (W, W + 2):
            outs = '"=r"(mask), ' + ", ".join(f'"+r"(a[{i}])' for i in range(N))
            ins = ", ".join(f'"r"(b[{i}])' for i in range(N))
            out.append(f"template <> __device__ __forceinline__ uint32_t mp_sub<{N}>(uint32_t (&a)[{N}], "
                       f"const uint32_t (&b)[{N}]) {{")
            out.append("    uint32_t mask;")
            out.append(f'    asm("{sub_body(N)}"\n        : {outs}\n        : {ins});')
            out.append("    return mask;")
            out.append("}")
            outs = '"=r"(carry), ' + ", ".join(f'"+r"(a[{i}])' for i in range(N))
            out.append(f"template <> __device__ __forceinline__ uint32_t mp_add<{N}>(uint32_t (&a)[{N}], "
                       f"const uint32_t (&b)[{N}]) {{")
            out.append("    uint32_t carry;")
            out.append(f'    asm("{add_body(N)}"\n        : {outs}\n        : {ins});')
            out.append("    return carry;")
            out.append("}")
        N = W + 2
        outs = ", ".join(f'"+r"(a[{i}])' for i in range(N))
        ins = ", ".join(f'"r"(b[{i}])' for i in range(N - 1))
        out.append(f"template <> __device__ __forceinline__ void mp_sub_hi<{W}>(uint32_t (&a)[{N}], "
                   f"const uint32_t (&b)[{N}]) {{")
        out.append(f'    asm("{sub_hi_body(W)}"\n        : {outs}\n        : {ins});')
        out.append("}")
        outs = ", ".join(f'"+r"(a[{i}])' for i in range(N))
        out.append(f"template <> __device__ __forceinline__ void mp_add3<{N}>(uint32_t (&a)[{N}], uint32_t t0, "
                   f"uint32_t t1, uint32_t t2) {{")
        out.append(f'    asm("{add3_body(N)}"\n        : {outs}\n        : "r"(t0), "r"(t1), "r"(t2));')
        out.append("}")
    out.append("}  // namespace pm")
    print("\n".join(out))


if __name__ == "__main__":
    main()
