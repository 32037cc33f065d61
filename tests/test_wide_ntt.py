"""The direct wide-modulus NTT (PM_WIDE_NTT): the NTT taken modulo q itself, the
reference's wide backend kept for comparison (solve.cu).  It needs a prime
q = 1 (mod 2n); products must equal the oracle's, the reference's golden points
must match by hash, and other moduli must be refused (checked against GMP's
primality test)."""
import numpy as np
import pytest

import polymul
from oracle import gmp, oracle
from tests.golden.cases import point_cases, sha
from tests.helpers import random_q, uniform_below

pytestmark = pytest.mark.gpu

FHERMA_Q = (1 << 868) - 11993087  # prime, = 1 (mod 2^17)


def eligible(q, n):
    return (q - 1) % (2 * n) == 0 and gmp.is_prime(q)


def test_golden_points(cuda, golden):
    used = 0
    for point in golden["points"]:
        q, n = int(point["q"], 16), point["N"]
        if not eligible(q, n):
            with pytest.raises(polymul.PolymulError) as e:
                polymul.Plan(n, q, coef_limbs=14, wide=True)
            assert e.value.status == polymul.PM_ERR_UNSUPPORTED
            continue
        used += 1
        with polymul.Plan(n, q, coef_limbs=14, wide=True) as p:
            for label, a, b, rec in point_cases(point):
                assert sha(p.multiply_host(a, b).tobytes()) == rec["c_sha256"], (n, point["delta"], label)
    assert used >= 6


@pytest.mark.parametrize("n", [2, 64, 1024, 32768])
def test_matches_oracle(cuda, n):
    rng = np.random.default_rng(n + 3)
    a, b = uniform_below(rng, FHERMA_Q, n, 14), uniform_below(rng, FHERMA_Q, n, 14)
    top = np.tile(np.array([(FHERMA_Q - 1 >> (64 * j)) & ((1 << 64) - 1) for j in range(14)], dtype=np.uint64),
                  (n, 1))
    with polymul.Plan(n, FHERMA_Q, coef_limbs=14, wide=True) as p:
        assert (p.multiply_host(a, b) == oracle.rns_multiply(a, b, FHERMA_Q)).all()
        assert (p.multiply_host(top, top) == oracle.rns_multiply(top, top, FHERMA_Q)).all()


def test_batch_and_narrow_prime(cuda):
    torch = cuda
    # a 127-bit prime = 1 mod 2^11 (4 words), batched through the device API
    q = 0
    rng = np.random.default_rng(11)
    while True:
        cand = (int(rng.integers(1 << 62, 1 << 63)) << 64 | int(rng.integers(0, 1 << 63))) >> 11 << 11 | 1
        if cand.bit_length() >= 120 and gmp.is_prime(cand):
            q = cand
            break
    n, count = 1024, 5
    a = np.stack([uniform_below(rng, q, n, 2) for _ in range(count)])
    b = np.stack([uniform_below(rng, q, n, 2) for _ in range(count)])
    da, db = torch.from_numpy(a.view(np.int64)).cuda(), torch.from_numpy(b.view(np.int64)).cuda()
    dc = torch.zeros_like(da)
    with polymul.Plan(n, q, coef_limbs=2, wide=True) as p:
        p.multiply_batch(da.data_ptr(), db.data_ptr(), dc.data_ptr(), count)
        torch.cuda.synchronize()
    c = dc.cpu().numpy().view(np.uint64)
    for k in range(count):
        assert (c[k] == oracle.rns_multiply(a[k], b[k], q)).all(), k


def test_refuses_unsuitable_moduli(cuda):
    rng = np.random.default_rng(4)
    for q, n in [((1 << 868) - 1, 1024), (random_q(rng, 868), 1024), (FHERMA_Q, 65536)]:
        with pytest.raises(polymul.PolymulError) as e:
            polymul.Plan(n, q, coef_limbs=14, wide=True)
        assert e.value.status == polymul.PM_ERR_UNSUPPORTED
