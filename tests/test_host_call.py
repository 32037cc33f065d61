"""The single-product host-buffer call (pm_multiply_host, the drop-in's
fherma_run) and its split form pm_multiply_host_begin / _end: pageable and
pinned buffers, the pieces staged by host threads, the product copied out as
it lands; every case against the oracle.  Protocol errors (a second begin, an
end without a begin) are refused without touching the open product."""
import numpy as np
import pytest

import polymul
from oracle import oracle
from tests.helpers import random_q, uniform_below

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [32768, 1024, 2])
def test_split_call_matches_the_oracle(cuda, n):
    rng = np.random.default_rng(600 + n)
    q = random_q(rng, 868)
    with polymul.Plan(n, q, coef_limbs=14) as p:
        for _ in range(2):
            a, b = uniform_below(rng, q, n, 14), uniform_below(rng, q, n, 14)
            want = oracle.rns_multiply(a, b, q)
            p.multiply_host_begin(a, b)
            a[:] = 0  # the inputs are free as soon as begin returns
            b[:] = 0
            assert (p.multiply_host_end() == want).all()


def test_pinned_and_pageable_buffers(cuda):
    torch = cuda
    n = 32768
    rng = np.random.default_rng(611)
    q = random_q(rng, 868)
    a, b = uniform_below(rng, q, n, 14), uniform_below(rng, q, n, 14)
    want = oracle.rns_multiply(a, b, q)
    pa = torch.from_numpy(a.view(np.int64)).pin_memory()
    pb = torch.from_numpy(b.view(np.int64)).pin_memory()
    pc = torch.zeros_like(pa).pin_memory()
    with polymul.Plan(n, q, coef_limbs=14) as p:
        p.multiply_host_ptr(pa.data_ptr(), pb.data_ptr(), pc.data_ptr())  # pinned in, pinned out (direct)
        assert (pc.numpy().view(np.uint64) == want).all()
        c = np.zeros_like(a)
        p.multiply_host_ptr(pa.data_ptr(), b.ctypes.data, c.ctypes.data)  # pinned a, pageable b and c
        assert (c == want).all()
        assert (p.multiply_host(a, b) == want).all()  # all pageable


def test_protocol_errors(cuda):
    n = 1024
    rng = np.random.default_rng(612)
    q = random_q(rng, 868)
    a, b = uniform_below(rng, q, n, 14), uniform_below(rng, q, n, 14)
    with polymul.Plan(n, q, coef_limbs=14) as p:
        with pytest.raises(polymul.PolymulError) as e:
            p.multiply_host_end()
        assert e.value.status == polymul.PM_ERR_INVALID
        p.multiply_host_begin(a, b)
        with pytest.raises(polymul.PolymulError) as e:
            p.multiply_host_begin(a, b)
        assert e.value.status == polymul.PM_ERR_BUSY
        assert (p.multiply_host_end() == oracle.rns_multiply(a, b, q)).all()


def test_pageable_a_with_pinned_b(cuda):
    """b goes to the link first (pinned, one copy) and a is staged after it: a's
    conversion on the side stream then waits behind both copies."""
    torch = cuda
    n = 32768
    rng = np.random.default_rng(613)
    q = random_q(rng, 868)
    a, b = uniform_below(rng, q, n, 14), uniform_below(rng, q, n, 14)
    want = oracle.rns_multiply(a, b, q)
    pb = torch.from_numpy(b.view(np.int64)).pin_memory()
    with polymul.Plan(n, q, coef_limbs=14) as p:
        for _ in range(2):
            c = np.zeros_like(a)
            p.multiply_host_ptr(a.ctypes.data, pb.data_ptr(), c.ctypes.data)
            assert (c == want).all()


@pytest.mark.parametrize("kind", ["k1t", "simt"])
def test_host_call_without_the_conversion_split(cuda, kind):
    """Plans whose conversion takes both polynomials in one launch (the per-group
    tensor conversion K1T, the plain method) run the call unsplit."""
    n = 4096
    rng = np.random.default_rng(614)
    q = random_q(rng, 868)
    with polymul.Plan(n, q, coef_limbs=14, tensor=(kind == "k1t")) as p:
        if kind == "k1t":
            p.set_tuning(conv_whole_basis=0)
        for _ in range(2):
            a, b = uniform_below(rng, q, n, 14), uniform_below(rng, q, n, 14)
            assert (p.multiply_host(a, b) == oracle.rns_multiply(a, b, q)).all()
