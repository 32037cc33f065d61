"""Failure detection on the device without a fault: every wait in the library's
kernels is an mbarrier wait with a time limit, after which the kernel records an
error and returns.  Here that wait runs on a barrier nothing arrives at (a
completion that never comes); it must give up after the limit, say so, and leave
the CUDA context able to run products."""
import numpy as np
import pytest

import polymul
from oracle import oracle
from tests.helpers import random_q, uniform_below

pytestmark = pytest.mark.gpu


def test_wait_gives_up_and_context_survives(cuda):
    timed_out, waited_ns = polymul.selftest_bounded_wait(50_000)
    assert timed_out
    assert 50e6 <= waited_ns < 1e9
    # the same context still multiplies
    rng = np.random.default_rng(2)
    q = random_q(rng, 868)
    a, b = uniform_below(rng, q, 1024, 14), uniform_below(rng, q, 1024, 14)
    with polymul.Plan(1024, q, coef_limbs=14, tensor=True) as p:
        assert (p.multiply_host(a, b) == oracle.rns_multiply(a, b, q)).all()
    timed_out, _ = polymul.selftest_bounded_wait(1_000)
    assert timed_out
