"""Known-answer inputs of the reference's end-to-end test, regenerated.

The reference's tests/validate.py:46-59 defines nine deterministic cases per
ring size N (seeded random.Random(20260916 + N)); its golden outputs come from
its Kronecker oracle (tests/validate.py:29-37).  The reference ships no vector
files, so tests/golden/make_golden.py runs that file itself and records the
SHA-256 of every input and output (plus the raw outputs for N <= 32) in
tests/golden/golden.json.  This module rebuilds the same inputs without the
reference present (the case list has to match value for value, so its shape
follows validate.py's), and the tests check the input hashes before trusting
an output hash.
"""
import hashlib
import json
import os
import random

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
WIDTH_BYTES = 112  # 28 u32 words per coefficient (fherma.h:27-42)


def load_golden():
    with open(os.path.join(HERE, "golden.json")) as f:
        return json.load(f)


def reference_cases(n, q):
    """[(label, a, b)] with a, b lists of Python ints, in validate.py's order."""
    rng = random.Random(20260916 + n)
    draw = lambda: [rng.randrange(q) for _ in range(n)]  # noqa: E731
    a, b = draw(), draw()
    out = [("dense-random-1", a, b)]
    a2 = draw()
    b2 = draw()
    out.append(("dense-random-2", a2, b2))
    out.append(("zero", a, [0] * n))
    out.append(("identity", a, [1] + [0] * (n - 1)))
    if n >= 2:
        out.append(("wrap-sign", [0] * (n - 1) + [q - 1], [0, q - 1] + [0] * (n - 2)))
    else:
        out.append(("wrap-sign", [q - 1], [0]))
    out.append(("all-q-minus-one", [q - 1] * n, [q - 1] * n))
    out.append(("alternating", [q - 1 if i % 2 else 0 for i in range(n)], a))
    edges = [0, 1, q - 1, q - 2, 1 << 864, (1 << 864) - 1, 1 << 32, (1 << 32) - 1]
    out.append(("limb-boundaries", [edges[i % len(edges)] for i in range(n)], b))
    out.append(("random-after-edges", b, a))
    return out


def encode(values, width=WIDTH_BYTES):
    return b"".join(int(x).to_bytes(width, "little") for x in values)


def to_limbs(values, limbs=WIDTH_BYTES // 8):
    return np.frombuffer(encode(values, 8 * limbs), dtype=np.uint64).reshape(len(values), limbs).copy()


def sha(data):
    return hashlib.sha256(bytes(data)).hexdigest()


def point_cases(point):
    """Rebuild one golden point: yields (label, a, b, expected) with limb arrays.

    `expected` is a dict with the c hash and, for small N, the c bytes.
    Input hashes are checked against the record before anything is returned.
    """
    n = point["N"]
    q = int(point["q"], 16)
    for rec, (label, a, b) in zip(point["cases"], reference_cases(n, q)):
        assert rec["label"] == label, (rec["label"], label)
        A, B = to_limbs(a), to_limbs(b)
        assert sha(A.tobytes()) == rec["a_sha256"], f"input a of {label} at N={n} does not match the record"
        assert sha(B.tobytes()) == rec["b_sha256"], f"input b of {label} at N={n} does not match the record"
        yield label, A, B, rec
