"""pm_multiply_noalloc, the entry point for callers that cannot allocate
device memory when they multiply (its scratch is a fixed array inside the
library).  Checked bit-exactly against pm_multiply, the entry point that uses
a workspace, on two calls in a row; the second call reuses the array the
first one left behind.  Kept in its own file so pytest collects it last."""
import ctypes

import numpy as np
import pytest

import polymul
from tests.helpers import random_q, uniform_below

pytestmark = pytest.mark.gpu


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
