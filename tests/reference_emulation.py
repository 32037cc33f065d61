"""Runs the reference's own rns kernels, CPU-emulated (oracle/_ref/rns_emulated,
built by oracle/emulation/build_ref_emulation.py from the reference's sources),
on arrays: writes a point directory in the harness format (main.cpp:137-208),
runs the binary, reads the c.bin files back.  Test and benchmark infrastructure:
the reference's CPU path is the checker and the CPU baseline, never the product.

The emulated backend covers what the reference's rns backend covers
(rns/solve.cu:581-587): n a power of two in [2, 32768] and q = 2^868 - c with
0 < c < 2^28, coefficients as 28 u32 words (14 u64 limbs)."""
import json
import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMULATED = os.path.join(ROOT, "oracle", "_ref", "rns_emulated")


def available():
    return os.path.exists(EMULATED)


def write_point(directory, n, q, pairs):
    """The harness layout: manifest.json, point/q.bin, cases/NNNNNN/{a,b}.bin (28 u32 words a coefficient)."""
    os.makedirs(os.path.join(directory, "point"), exist_ok=True)
    with open(os.path.join(directory, "point", "q.bin"), "wb") as f:
        f.write(int(q).to_bytes(112, "little"))
    for idx, (a, b) in enumerate(pairs):
        d = os.path.join(directory, "cases", f"{idx:06d}")
        os.makedirs(d, exist_ok=True)
        for name, x in (("a.bin", a), ("b.bin", b)):
            x = np.ascontiguousarray(x, dtype=np.uint64)
            assert x.shape == (n, 14)
            with open(os.path.join(d, name), "wb") as f:
                f.write(x.tobytes())
    with open(os.path.join(directory, "manifest.json"), "w") as f:
        json.dump({"point": {"N": int(n), "W": 868, "L": 28}, "cases": len(pairs)}, f)


def start(directory):
    """Launch the emulated reference on a point directory (returns the Popen)."""
    return subprocess.Popen([EMULATED, directory], stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True)


def read_results(directory, count, n):
    """(products as (n, 14) uint64 arrays, per-case seconds from results.json)."""
    with open(os.path.join(directory, "out", "results.json")) as f:
        results = json.load(f)
    outs, secs = [], []
    for idx in range(count):
        rec = results["cases"][idx]
        if rec["status"] != "ok":
            raise RuntimeError(f"emulated reference case {idx}: {rec}")
        with open(os.path.join(directory, "out", f"{idx:06d}", "c.bin"), "rb") as f:
            outs.append(np.frombuffer(f.read(), dtype=np.uint64).reshape(n, 14).copy())
        secs.append(rec["seconds"])
    return outs, secs


def multiply(n, q, pairs, timeout=3600):
    """The reference's products of [(a, b)] at (n, q), in one run of the emulated binary."""
    with tempfile.TemporaryDirectory() as tmp:
        write_point(tmp, n, q, pairs)
        p = start(tmp)
        _, err = p.communicate(timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"emulated reference failed ({p.returncode}): {err[-400:]}")
        return read_results(tmp, len(pairs), n)
