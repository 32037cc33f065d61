"""Writes crt_mac.cuh: acc[0..W+1] += t * m[0..W-1] as one PTX carry chain per
width W (two chains: the low halves of t*m[k] into acc[k], the high halves into
acc[k+1]).  Run: python gen_crt_mac.py > crt_mac.cuh"""
WIDTHS = [4, 8, 12, 16, 20, 24, 28]


def body(W):
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


def main():
    out = ["// Generated by gen_crt_mac.py -- do not edit.",
           "// acc (W+2 words) += t * m (W words), exact, as PTX carry chains.",
           "#pragma once", "#include <cstdint>", "namespace pm {",
           "template <int W> __device__ __forceinline__ void crt_mac(uint32_t (&a)[W + 2], uint32_t t, const uint32_t (&m)[W]);"]
    for W in WIDTHS:
        outs = ", ".join(f'"+r"(a[{i}])' for i in range(W + 2))
        ins = ", ".join(f'"r"(m[{i}])' for i in range(W)) + ', "r"(t)'
        out.append(f"template <> __device__ __forceinline__ void crt_mac<{W}>(uint32_t (&a)[{W + 2}], uint32_t t, "
                   f"const uint32_t (&m)[{W}]) {{")
        out.append(f'    asm("{body(W)}"\n        : {outs}\n        : {ins});')
        out.append("}")
    out.append("}  // namespace pm")
    print("\n".join(out))


if __name__ == "__main__":
    main()
