"""pm_multiply_noalloc, the entry point for callers that cannot allocate
device memory when they multiply (its scratch is a fixed array inside the
library).  Checked bit-exactly against pm_multiply, the entry point that uses
a workspace, on two calls in a row; the second call reuses the array the
first one left behind.  Kept in its own file so pytest collects it last."""
import ctypes

import numpy as np
import pytest

import polymul
from oracle import oracle
from tests.helpers import random_q, uniform_below

pytestmark = pytest.mark.gpu

FHERMA_Q = (1 << 868) - 11993087  # prime, 1 mod 2n for n <= 32768: the wide NTT applies


def _noalloc(plan, a_ptr, b_ptr, c_ptr, stream=0):
    L = polymul.lib()
    L.pm_multiply_noalloc.argtypes = [ctypes.c_void_p] * 5
    polymul.check(L.pm_multiply_noalloc(plan.handle, a_ptr, b_ptr, c_ptr, stream or None))


@pytest.mark.parametrize("tensor", [False, True])
def test_noalloc_matches_workspace_entry_point(cuda, tensor):
    torch = cuda
    n = 8192  # the largest ring the built-in 4 MiB scratch holds at 868 bits
    rng = np.random.default_rng(77 + int(tensor))
    q = random_q(rng, 868)
    with polymul.Plan(n, q, coef_limbs=14, tensor=tensor) as plan:
        assert plan.workspace_bytes <= 4 << 20
        for call in range(2):
            a = torch.from_numpy(uniform_below(rng, q, n, 14).view(np.int64)).cuda()
            b = torch.from_numpy(uniform_below(rng, q, n, 14).view(np.int64)).cuda()
            expect = torch.empty_like(a)
            got = torch.full_like(a, -1)
            plan.multiply(a.data_ptr(), b.data_ptr(), expect.data_ptr())
            _noalloc(plan, a.data_ptr(), b.data_ptr(), got.data_ptr())
            torch.cuda.synchronize()
            assert torch.equal(got, expect), f"call {call}"


def test_noalloc_refuses_plans_above_its_scratch(cuda):
    torch = cuda
    n = 32768
    q = random_q(np.random.default_rng(5), 868)
    with polymul.Plan(n, q, coef_limbs=14) as plan:
        a = torch.zeros((n, 14), dtype=torch.int64, device="cuda")
        with pytest.raises(polymul.PolymulError) as e:
            _noalloc(plan, a.data_ptr(), a.data_ptr(), a.data_ptr())
        assert e.value.status == polymul.PM_ERR_UNSUPPORTED
        assert "4 MiB" in str(e.value)


def test_noalloc_allocates_nothing_and_runs_on_a_side_stream(cuda):
    """The defining property: once the first call has looked the array up, a call
    leaves the device's free memory exactly as it found it.  Also on a stream of
    the caller's own, checked against the oracle."""
    torch = cuda
    n = 4096
    rng = np.random.default_rng(91)
    q = random_q(rng, 868)
    with polymul.Plan(n, q, coef_limbs=14) as plan:
        a_h, b_h = uniform_below(rng, q, n, 14), uniform_below(rng, q, n, 14)
        a = torch.from_numpy(a_h.view(np.int64)).cuda()
        b = torch.from_numpy(b_h.view(np.int64)).cuda()
        c = torch.full_like(a, -1)
        side = torch.cuda.Stream()
        _noalloc(plan, a.data_ptr(), b.data_ptr(), c.data_ptr(), side.cuda_stream)  # first call: address lookup
        side.synchronize()
        free_before, _ = torch.cuda.mem_get_info()
        c.fill_(-1)
        torch.cuda.synchronize()
        _noalloc(plan, a.data_ptr(), b.data_ptr(), c.data_ptr(), side.cuda_stream)
        side.synchronize()
        free_after, _ = torch.cuda.mem_get_info()
        assert free_after == free_before
        expect = oracle.rns_multiply(a_h, b_h, q)
        assert (c.cpu().numpy().view(np.uint64) == expect).all()


def test_noalloc_wide_ntt_plan(cuda):
    """A PM_WIDE_NTT plan: its scratch has another size and 16-byte loads; the
    array serves it too.  Two calls, each against the oracle."""
    torch = cuda
    n = 1024
    rng = np.random.default_rng(93)
    with polymul.Plan(n, FHERMA_Q, coef_limbs=14, wide=True) as plan:
        assert plan.workspace_bytes <= 4 << 20
        for call in range(2):
            a_h, b_h = uniform_below(rng, FHERMA_Q, n, 14), uniform_below(rng, FHERMA_Q, n, 14)
            a = torch.from_numpy(a_h.view(np.int64)).cuda()
            b = torch.from_numpy(b_h.view(np.int64)).cuda()
            c = torch.full_like(a, -1)
            _noalloc(plan, a.data_ptr(), b.data_ptr(), c.data_ptr())
            torch.cuda.synchronize()
            assert (c.cpu().numpy().view(np.uint64) == oracle.rns_multiply(a_h, b_h, FHERMA_Q)).all(), f"call {call}"
