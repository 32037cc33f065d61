"""Uneven batches (pm_batch_*): products of different n and q in one CUDA
graph of persistent kernels, bit-exact against per-product plans and the
oracle, before and after the batch autotuner re-shapes the launches."""
import numpy as np
import pytest

import polymul
from oracle import oracle
from tests.helpers import random_q, uniform_below

pytestmark = pytest.mark.gpu


def _products(seed, ns, bits_range=(200, 868)):
    rng = np.random.default_rng(seed)
    qs = [random_q(rng, int(rng.integers(bits_range[0], bits_range[1] + 1))) for _ in ns]
    a = [uniform_below(rng, q, n, 14) for q, n in zip(qs, ns)]
    b = [uniform_below(rng, q, n, 14) for q, n in zip(qs, ns)]
    return qs, a, b


def test_uneven_batch_matches_plans_and_oracle(cuda):
    ns = [1024, 65536, 256, 4096, 32768, 2048, 16384, 1024, 8192, 512, 4096, 32768]
    qs, a, b = _products(4, ns)
    with polymul.Batch(ns, qs) as batch:
        got = batch.multiply_host(a, b)
        for z, (n, q) in enumerate(zip(ns, qs)):
            with polymul.Plan(n, q, 14, tensor=True) as p:
                assert (got[z] == p.multiply_host(a[z], b[z])).all(), (z, n, q.bit_length())
        for z in (2, 3, 9):
            assert (got[z] == oracle.rns_multiply(a[z], b[z], qs[z])).all(), z
        us = batch.autotune(reps=2)
        assert us > 0
        again = batch.multiply_host(a, b)
        for z in range(len(ns)):
            assert (again[z] == got[z]).all(), z


def test_uneven_batch_rejects_small_rings_and_odd_limbs(cuda):
    q = random_q(np.random.default_rng(1), 300)
    with pytest.raises(polymul.PolymulError) as e:
        polymul.Batch([128, 1024], [q, q])
    assert e.value.status == polymul.PM_ERR_UNSUPPORTED
    with pytest.raises(polymul.PolymulError) as e:
        polymul.Batch([1024], [q], coef_limbs=5)
    assert e.value.status == polymul.PM_ERR_UNSUPPORTED
