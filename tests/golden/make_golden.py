"""Regenerate tests/golden/golden.json from the reference's own test oracle.

Run in a container where the reference sources are mounted (read-only):

    python tests/golden/make_golden.py [/path/to/reference]

It imports the reference's tests/validate.py unmodified.  That file needs gmpy2
(absent from the image); a stand-in module with the same three entry points
(mpz.from_bytes, mpz multiplication/to_bytes, is_prime) is injected first,
backed by the system GMP through ctypes (oracle/gmp.py).  For every point it
takes validate.py's modulus(), cases(), oracle() and (N <= 32) schoolbook(),
cross-checks the outputs against the repository's C oracles, and records
SHA-256 hashes of all inputs and outputs, plus raw outputs for N <= 32.
"""
import importlib.util
import json
import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import gmp, oracle  # noqa: E402
from tests.golden.cases import reference_cases, sha, to_limbs  # noqa: E402

POINTS = [  # (N, delta) with delta None -> validate.modulus(N, 868)
    (2, None), (4, None), (32, None), (1024, None), (4096, None), (32768, None),
    (32, 1), (32, 11993087), (32, (1 << 28) - 1), (1024, (1 << 28) - 1),
]


def gmpy2_standin():
    mod = types.ModuleType("gmpy2")

    class mpz(gmp.Mpz):
        pass

    mod.mpz = mpz
    mod.is_prime = lambda value, reps=25: gmp.is_prime(int(value), reps)
    return mod


def load_validate(reference):
    sys.modules["gmpy2"] = gmpy2_standin()
    spec = importlib.util.spec_from_file_location("reference_validate", os.path.join(reference, "tests", "validate.py"))
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py <reference source tree>")
    reference = sys.argv[1]
    validate = load_validate(reference)
    points = []
    for n, delta in POINTS:
        q = validate.modulus(n, 868) if delta is None else (1 << 868) - delta
        ref_cases = list(validate.cases(n, q))
        mine = reference_cases(n, q)
        record = {"N": n, "W": 868, "L": 28, "delta": delta, "q": hex(q), "cases": []}
        for (label, a, b), (label2, a2, b2) in zip(ref_cases, mine):
            assert label == label2 and a == a2 and b == b2, f"case regeneration differs at {label}"
            c = validate.oracle(a, b, q)
            if n <= 32:
                assert c == validate.schoolbook(a, b, q), "reference oracles disagree"
            A, B, C = to_limbs(a), to_limbs(b), to_limbs(c)
            assert (oracle.rns_multiply(A, B, q) == C).all(), f"C RNS oracle differs at N={n} {label}"
            if n <= 1024:
                assert (oracle.schoolbook(A, B, q) == C).all(), f"C schoolbook differs at N={n} {label}"
            entry = {"label": label, "a_sha256": sha(A.tobytes()), "b_sha256": sha(B.tobytes()),
                     "c_sha256": sha(C.tobytes())}
            if n <= 32:
                entry["c_hex"] = C.tobytes().hex()
            record["cases"].append(entry)
            print(f"N={n} delta={delta} {label}: ok", flush=True)
        points.append(record)
    out = {"source": "reference tests/validate.py modulus/cases/oracle/schoolbook, run by tests/golden/make_golden.py",
           "points": points}
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
