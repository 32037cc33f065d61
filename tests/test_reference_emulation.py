"""The reference's own rns kernel bodies, run on the CPU by the reference's
coroutine emulation (its tests/build_emulation.py rewrite, built into
oracle/_ref/rns_emulated when the reference's sources are present), as a
second checker beside the oracle:
  - CPU: it reproduces the golden vectors of the reference's validate.py, and
    it agrees with the oracle's restatement on seeded inputs;
  - GPU: this repository's CUDA path (the default, tensor-core plan) returns
    exactly what the reference's kernels return, on seeded inputs at the
    reference's own kind of modulus q = 2^868 - c."""
import numpy as np
import pytest

import polymul
from oracle import oracle
from tests import reference_emulation as emu
from tests.golden.cases import load_golden, point_cases, sha
from tests.helpers import uniform_below

needs_emulation = pytest.mark.skipif(not emu.available(), reason="oracle/_ref/rns_emulated was not built")


def golden_point(n, delta):
    return [p for p in load_golden()["points"] if p["N"] == n and p["delta"] == delta][0]


@needs_emulation
@pytest.mark.parametrize("n,delta,cases", [(32, None, 9), (32, 268435455, 9), (4, None, 9), (1024, None, 2)])
def test_emulated_reference_reproduces_the_golden_vectors(n, delta, cases):
    point = golden_point(n, delta)
    q = int(point["q"], 16)
    rows = list(point_cases(point))[:cases]
    outs, _ = emu.multiply(n, q, [(a, b) for _, a, b, _ in rows])
    for (label, _, _, rec), c in zip(rows, outs):
        assert sha(c.tobytes()) == rec["c_sha256"], label


@needs_emulation
def test_emulated_reference_agrees_with_the_oracle():
    rng = np.random.default_rng(8080)
    n, q = 256, (1 << 868) - 11993087
    pairs = [(uniform_below(rng, q, n, 14), uniform_below(rng, q, n, 14)) for _ in range(2)]
    outs, _ = emu.multiply(n, q, pairs)
    for (a, b), c in zip(pairs, outs):
        assert (c == oracle.rns_multiply(a, b, q)).all()


@needs_emulation
@pytest.mark.gpu
@pytest.mark.parametrize("n,delta", [(4096, 11993087), (2048, (1 << 28) - 1), (64, 1)])
def test_cuda_path_matches_the_reference_kernels(cuda, n, delta):
    rng = np.random.default_rng(n + delta)
    q = (1 << 868) - delta
    a, b = uniform_below(rng, q, n, 14), uniform_below(rng, q, n, 14)
    (want,), _ = emu.multiply(n, q, [(a, b)])
    with polymul.Plan(n, q, coef_limbs=14) as plan:
        assert plan.tensor
        got = plan.multiply_host(a, b)
    assert (got == want).all()
