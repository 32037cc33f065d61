"""Test infrastructure only: build the reference's own RNS kernels as a CPU
program, the way the reference's tests/build_emulation.py does it, into
oracle/_ref/rns_emulated.

The reference's emulation turns every CUDA kernel of rns/solve.cu into a C++20
coroutine that yields at each __syncthreads() (and each warp shuffle), runs the
"threads" of a block one barrier phase at a time, and backs the cuPQC big
integers with GMP (tests/cuda_emulation.h).  Its own driver writes into the
source tree and calls clang++ with macOS paths, so this recipe applies the same
source rewrite here (tests/build_emulation.py:17-41: the include swap, launch
bounds dropped, kernel bodies turned into coroutines, the 20 launch sites into
emulate_launch calls) and compiles with g++ against:
  - oracle/emulation/gmpxx.h: the mpz_class subset over the runtime libgmp;
  - oracle/emulation/cuda_runtime_stubs.h: host-side CUDA runtime calls the
    rns backend names that the reference's emulation header leaves out (no-ops
    or plain memcpy; with FHERMA_GRAPH=0 the backend copies synchronously).
The result is linked with the reference's unmodified harness (main.cpp), so it
reads a point directory and writes c.bin files and results.json like the
solution does.  It runs the reference's kernel bodies on one host thread (its
host copy pool set to two threads that do not spin, so that one process per
core can run side by side).

usage: python build_ref_emulation.py <reference source tree> <output directory>
"""
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))


def rewrite(source):
    """The reference's emulation rewrite of a CUDA source (tests/build_emulation.py)."""
    source = source.replace("#include <cupqc/bigint.hpp>",
                            '#include "tests/cuda_emulation.h"\n#include "cuda_runtime_stubs.h"')
    source = source.replace("#include <cuda_runtime.h>", "")
    source = re.sub(r"__launch_bounds__\([^)]*\)", "", source)
    source = re.sub(r"#if FHERMA_MIN_BLOCKS && FHERMA_TPI==1\s*__global__\s*#else\s*__global__\s*#endif\s*void",
                    "__global__ void", source)
    kernels = list(re.finditer(r"__global__ void (\w+)\([^)]*\)\s*\{", source))
    for m in reversed(kernels):
        start = end = m.end()
        depth = 1
        while depth:
            depth += (source[end] == "{") - (source[end] == "}")
            end += 1
        body = source[start:end - 1]
        body = body.replace("return;", "co_return;")
        body = body.replace("__syncthreads();", "co_await std::suspend_always{};")
        body = body.replace("__shfl_xor_sync(", "co_await emulated_shuffle_xor(")
        head = source[m.start():start].replace("__global__ void", "EmulatedKernel")
        source = source[:m.start()] + head + body + "co_return;\n}" + source[end:]

    def launch(m):
        block = m.group(3).split(",")[0]
        return f"emulate_launch({m.group(2)},{block},[&] {{ return {m.group(1)}({m.group(4)}); }});"

    source, count = re.subn(r"(\w+(?:<[A-Za-z]+(?:,[A-Za-z]+)*>)?)<<<([^,<>]+),\s*([^<>]+)>>>\(([^;]+)\);",
                            launch, source)
    if count != 20:
        raise SystemExit(f"expected the 20 launch sites of rns/solve.cu, found {count}")
    if "<<<" in source:
        raise SystemExit("a launch site was not rewritten")
    return source


def main():
    if len(sys.argv) != 3:
        raise SystemExit(__doc__)
    ref, out = sys.argv[1], sys.argv[2]
    os.makedirs(out, exist_ok=True)
    with open(os.path.join(ref, "rns", "solve.cu")) as f:
        src = rewrite(f.read())
    exe = os.path.join(out, "rns_emulated")
    # the rewritten source is a build intermediate: it lives only for the compile
    with tempfile.TemporaryDirectory() as tmp:
        gen = os.path.join(tmp, "rns_solve_emulated.cpp")
        with open(gen, "w") as f:
            f.write(src)
        # two non-spinning host copy threads (the pool needs an even count): emulated processes share the cores
        cmd = ["g++", "-std=c++20", "-O2", "-w", "-I" + ref, "-I" + HERE, "-DFHERMA_PROFILE=0", "-DFHERMA_GRAPH=0",
               "-DFHERMA_COPY_THREADS=2", "-DFHERMA_SPIN_COPY=0",
               os.path.join(ref, "main.cpp"), gen, "-l:libgmp.so.10", "-pthread", "-o", exe]
        subprocess.run(cmd, check=True)
    print(f"built {exe} (the reference's rns kernels, CPU-emulated)")


if __name__ == "__main__":
    main()
