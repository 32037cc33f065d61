"""The quartic factorization (PM_QUARTIC; the reference's best backend,
quartic/host_setup.h, quartic/solve.cu): q = B^4 - delta, 16 primes x 4
channels, evaluation at the roots of Y^4 = delta, interpolation and one INT8
CRT.  Every product against the oracle (the RNS restatement, which does not use
the factorization); parameters outside its coverage are refused."""
import numpy as np
import pytest

import polymul
from oracle import oracle
from tests.helpers import random_q, uniform_below

FHERMA_Q = (1 << 868) - 11993087


@pytest.mark.gpu
@pytest.mark.parametrize("n,q", [(64, FHERMA_Q), (1024, FHERMA_Q), (32768, FHERMA_Q), (4096, (1 << 868) - 1),
                                 (1024, (1 << 864) - 12345), (2048, (1 << 896) - 255)])
def test_quartic_matches_the_oracle(cuda, n, q):
    rng = np.random.default_rng(n + (q & 0xffff))
    with polymul.Plan(n, q, coef_limbs=14, quartic=True) as p:
        assert p.primes == 64  # 16 primes x 4 channels
        for _ in range(2):
            a, b = uniform_below(rng, q, n, 14), uniform_below(rng, q, n, 14)
            assert (p.multiply_host(a, b) == oracle.rns_multiply(a, b, q)).all()


@pytest.mark.gpu
def test_quartic_extreme_coefficients_and_batch(cuda):
    torch = cuda
    n, q = 32768, FHERMA_Q
    rng = np.random.default_rng(7)
    top = np.frombuffer((q - 1).to_bytes(112, "little"), dtype=np.uint64)
    a = np.tile(top, (n, 1)).copy()
    b = a.copy()
    with polymul.Plan(n, q, coef_limbs=14, quartic=True) as p:
        assert (p.multiply_host(a, b) == oracle.rns_multiply(a, b, q)).all()
        count = 3
        A = np.stack([uniform_below(rng, q, n, 14) for _ in range(count)])
        B = np.stack([uniform_below(rng, q, n, 14) for _ in range(count)])
        da = torch.from_numpy(A.view(np.int64)).cuda()
        db = torch.from_numpy(B.view(np.int64)).cuda()
        dc = torch.zeros_like(da)
        p.multiply_batch(da.data_ptr(), db.data_ptr(), dc.data_ptr(), count)
        torch.cuda.synchronize()
        got = dc.cpu().numpy().view(np.uint64)
        for k in range(count):
            assert (got[k] == oracle.rns_multiply(A[k], B[k], q)).all(), k


@pytest.mark.gpu
def test_quartic_refuses_what_it_does_not_cover(cuda):
    cases = [(32768, (1 << 868) - ((1 << 28) - 1)),  # 16 primes too few for n (1 + 3 delta) B^2
             (1024, random_q(np.random.default_rng(3), 868)),  # not 2^k - delta
             (32, FHERMA_Q),  # below n = 64
             (1024, (1 << 866) - 5)]  # bits not a multiple of 4
    for n, q in cases:
        with pytest.raises(polymul.PolymulError) as e:
            polymul.Plan(n, q, coef_limbs=14, quartic=True)
        assert e.value.status == polymul.PM_ERR_UNSUPPORTED, (n, hex(q)[:12])
    with pytest.raises(polymul.PolymulError) as e:
        polymul.Plan(1024, FHERMA_Q, coef_limbs=14, quartic=True, tensor=False)
    assert e.value.status == polymul.PM_ERR_INVALID
