"""Special-form moduli q = 2^k - delta (delta < 2^32, k >= 80) with
PM_SPECIAL_FORM: the CRT reduces by folding 2^k = delta instead of by the
general division (the family the reference's quartic backend targets,
quartic/host_setup.h:41-110; the FHERMA point is q = 2^868 - 11993087).  Every
product must equal the oracle's, and the folding reduction must agree bit for
bit with the general one, on random inputs and on inputs that make the
pre-reduction value as large as it gets (all coefficients q - 1).
"""
import numpy as np
import pytest

import polymul
from oracle import oracle
from tests.helpers import from_ints, uniform_below

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["simt", "tensor"])
def path(request):
    return request.param


def limbs_for(path, bits):
    limbs = (bits + 63) // 64
    return limbs + (limbs % 2) if path == "tensor" else limbs


CASES = [(80, 1), (80, (1 << 32) - 1), (200, 3), (517, (1 << 31) + 11), (868, 1), (868, 11993087),
         (868, (1 << 28) - 1), (868, (1 << 32) - 5), (896, 7), (896, (1 << 32) - 1)]


@pytest.mark.parametrize("k,delta", CASES)
def test_special_form_matches_oracle(cuda, path, k, delta):
    q = (1 << k) - delta
    n = 1024
    limbs = limbs_for(path, k)
    rng = np.random.default_rng(k * 7 + delta % 1000)
    a, b = uniform_below(rng, q, n, limbs), uniform_below(rng, q, n, limbs)
    top = from_ints([q - 1] * n, limbs)
    with polymul.Plan(n, q, coef_limbs=limbs, tensor=(path == "tensor"), special_form=True) as p:
        assert (p.multiply_host(a, b) == oracle.rns_multiply(a, b, q)).all()
        assert (p.multiply_host(top, top) == oracle.rns_multiply(top, top, q)).all()


@pytest.mark.parametrize("k,delta", [(868, 11993087), (896, (1 << 32) - 1)])
def test_special_and_general_reduction_agree(cuda, path, k, delta):
    q = (1 << k) - delta
    n = 32768
    limbs = limbs_for(path, k)
    rng = np.random.default_rng(delta % 997)
    a, b = uniform_below(rng, q, n, limbs), uniform_below(rng, q, n, limbs)
    with polymul.Plan(n, q, coef_limbs=limbs, tensor=(path == "tensor"), special_form=True) as fast, \
            polymul.Plan(n, q, coef_limbs=limbs, tensor=(path == "tensor")) as general:
        c = fast.multiply_host(a, b)
        assert (c == general.multiply_host(a, b)).all()
    m = 2048
    a2, b2 = a[:m], b[:m]
    top = from_ints([q - 1] * m, limbs)
    with polymul.Plan(m, q, coef_limbs=limbs, tensor=(path == "tensor"), special_form=True) as p:
        assert (p.multiply_host(a2, b2) == oracle.rns_multiply(a2, b2, q)).all()
        assert (p.multiply_host(top, top) == oracle.rns_multiply(top, top, q)).all()


def test_flag_is_ignored_for_other_moduli(cuda, path):
    """PM_SPECIAL_FORM on a q that is not 2^k - delta with a small delta: the general reduction runs."""
    from tests.helpers import random_q
    rng = np.random.default_rng(5)
    q = random_q(rng, 868)
    limbs = limbs_for(path, 868)
    a, b = uniform_below(rng, q, 1024, limbs), uniform_below(rng, q, 1024, limbs)
    with polymul.Plan(1024, q, coef_limbs=limbs, tensor=(path == "tensor"), special_form=True) as p:
        assert (p.multiply_host(a, b) == oracle.rns_multiply(a, b, q)).all()
