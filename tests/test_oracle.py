"""CPU tests of the oracle itself: it must reproduce the reference's golden
vectors (generated by the reference's own tests/validate.py) before any GPU
result is compared with it."""
import hashlib
import os
import subprocess

import numpy as np
import pytest

from oracle import gmp, oracle
from tests.golden.cases import point_cases, sha
from tests.helpers import random_q, uniform_below

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DUMP = os.path.join(ROOT, "oracle", "_ref", "ref_setup_dump")


def test_golden_modulus_for_fherma_point(golden):
    q32768 = [p for p in golden["points"] if p["N"] == 32768 and p["delta"] is None][0]
    assert int(q32768["q"], 16) == (1 << 868) - 11993087  # tests/rns_setup.cpp:8


@pytest.mark.parametrize("n_max", [1024])
def test_rns_oracle_matches_golden(golden, n_max):
    checked = 0
    for point in golden["points"]:
        if point["N"] > n_max:
            continue
        q = int(point["q"], 16)
        for label, a, b, rec in point_cases(point):
            c = oracle.rns_multiply(a, b, q)
            assert sha(c.tobytes()) == rec["c_sha256"], (point["N"], point["delta"], label)
            if "c_hex" in rec:
                assert c.tobytes().hex() == rec["c_hex"]
            checked += 1
    assert checked >= 60


def test_rns_oracle_matches_golden_n32768(golden):
    point = [p for p in golden["points"] if p["N"] == 32768][0]
    q = int(point["q"], 16)
    for idx, (label, a, b, rec) in enumerate(point_cases(point)):
        if idx not in (0, 4, 5, 7):  # dense, wrap-sign, all q-1, limb boundaries
            continue
        assert sha(oracle.rns_multiply(a, b, q).tobytes()) == rec["c_sha256"], label


def test_schoolbook_matches_golden_small(golden):
    for point in golden["points"]:
        if point["N"] > 32:
            continue
        q = int(point["q"], 16)
        for label, a, b, rec in point_cases(point):
            assert oracle.schoolbook(a, b, q).tobytes().hex() == rec["c_hex"], (point["N"], label)


@pytest.mark.parametrize("n,bits", [(2, 3), (4, 64), (8, 65), (64, 200), (128, 517), (256, 868), (512, 896)])
def test_three_oracles_agree_random(n, bits):
    rng = np.random.default_rng(1000 + n + bits)
    q = random_q(rng, bits)
    a, b = uniform_below(rng, q, n), uniform_below(rng, q, n)
    c1 = oracle.rns_multiply(a, b, q)
    assert (c1 == oracle.schoolbook(a, b, q)).all()
    assert (c1 == gmp.kronecker(a, b, q)).all()


def test_rns_oracle_with_reference_prime_rule():
    """The reference's own basis (57 primes < 2^31, = 1 mod 2^16) gives the same products."""
    rng = np.random.default_rng(7)
    q = (1 << 868) - 11993087
    a, b = uniform_below(rng, q, 64), uniform_below(rng, q, 64)
    ref_rule = oracle.rns_multiply(a, b, q, bits=31, order=1 << 16, count=57)
    assert (ref_rule == oracle.rns_multiply(a, b, q)).all()
    assert (ref_rule == gmp.kronecker(a, b, q)).all()


@pytest.mark.skipif(not os.path.exists(REF_DUMP), reason="reference setup not compiled (oracle/_ref)")
@pytest.mark.parametrize("n", [32, 32768])
def test_basis_restatement_matches_reference_setup(n):
    """oracle basis constants == the reference's rns::setup (rns/host_setup.h:61-126)."""
    q = (1 << 868) - 11993087
    words = [(q >> (32 * i)) & 0xFFFFFFFF for i in range(28)]
    out = subprocess.run([REF_DUMP, str(n)] + [format(w, "x") for w in words], check=True,
                         capture_output=True, text=True).stdout.strip().splitlines()
    rows = [list(map(int, line.split())) for line in out[:-1]]
    pmodq = list(map(int, out[-1].split()))
    mine = oracle.basis_dump(n, q, 29, 31, 1 << 16, 57)
    assert len(rows) == 57
    for i, row in enumerate(rows):
        assert row[0] == mine["primes"][i]
        assert row[1] == mine["recip"][i]
        # the reference's forward[1] is psi^1 of its twisted (natural-order) table
        assert row[2] == mine["psi"][i]
        assert row[3:] == list(mine["bases_mod_q"][i])
    # the reference keeps P mod q in q's 28 words; the dump here has a 29th, zero
    assert pmodq == list(mine["product_mod_q"][:len(pmodq)])
    assert not any(mine["product_mod_q"][len(pmodq):])
