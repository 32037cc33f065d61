"""Device ownership of plans: calls on device pointers run on the plan's own
device (PM_ERR_INVALID from another one, or for another device's memory),
calls on host buffers switch to it for their duration.  The refusals need a
second GPU and are skipped on one; the host-buffer half runs everywhere."""
import numpy as np
import pytest

import polymul
from oracle import oracle
from tests.helpers import random_q, uniform_below

pytestmark = pytest.mark.gpu


def test_host_call_keeps_the_callers_device_and_matches_the_oracle(cuda):
    torch = cuda
    torch.cuda.set_device(0)
    rng = np.random.default_rng(404)
    q = random_q(rng, 868)
    n = 256
    with polymul.Plan(n, q, coef_limbs=14) as plan:
        a, b = uniform_below(rng, q, n, 14), uniform_below(rng, q, n, 14)
        c = plan.multiply_host(a, b)
        assert torch.cuda.current_device() == 0
    assert (c == oracle.rns_multiply(a, b, q)).all()


def test_calls_from_another_device_are_refused(cuda):
    torch = cuda
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    rng = np.random.default_rng(405)
    q = random_q(rng, 868)
    n = 256
    torch.cuda.set_device(0)
    with polymul.Plan(n, q, coef_limbs=14) as plan:
        a0 = torch.zeros((n, 14), dtype=torch.int64, device="cuda:0")
        a1 = torch.zeros((n, 14), dtype=torch.int64, device="cuda:1")
        # device 0 current, operands on device 1: refused before anything runs
        with pytest.raises(polymul.PolymulError) as e:
            plan.multiply(a1.data_ptr(), a1.data_ptr(), a1.data_ptr())
        assert e.value.status == polymul.PM_ERR_INVALID and "device 1" in str(e.value)
        # device 1 current: refused
        torch.cuda.set_device(1)
        with pytest.raises(polymul.PolymulError) as e:
            plan.multiply(a0.data_ptr(), a0.data_ptr(), a0.data_ptr())
        assert e.value.status == polymul.PM_ERR_INVALID
        # host buffers: runs on device 0 and leaves device 1 current
        x, y = uniform_below(rng, q, n, 14), uniform_below(rng, q, n, 14)
        assert (plan.multiply_host(x, y) == oracle.rns_multiply(x, y, q)).all()
        assert torch.cuda.current_device() == 1
        torch.cuda.set_device(0)
