"""The serving loop (pm_server_*): continuous batching of products that arrive
one by one.  Results must be bit-exact and independent of what else was on the
GPU at the same time; admission is bounded by the device arena; waits are
bounded."""
import numpy as np
import pytest

import polymul
from oracle import oracle
from tests.helpers import random_q, uniform_below

pytestmark = pytest.mark.gpu


def _pool(torch, rng, q, n, count):
    a = torch.from_numpy(np.stack([uniform_below(rng, q, n, 14) for _ in range(count)]).view(np.int64)).pin_memory()
    b = torch.from_numpy(np.stack([uniform_below(rng, q, n, 14) for _ in range(count)]).view(np.int64)).pin_memory()
    c = torch.zeros_like(a).pin_memory()
    return a, b, c


@pytest.mark.parametrize("tensor", [True, False])
def test_mixed_stream_matches_plain_path(cuda, tensor):
    torch = cuda
    rng = np.random.default_rng(501 + int(tensor))
    qs = [random_q(rng, 868), (1 << 868) - 11993087]
    sizes = [4096, 16384, 32768, 65536, 4096, 4096, 16384, 32768]
    pools = {}
    with polymul.Server(slots=6, max_group=4, tensor=tensor) as srv:
        tickets = []
        for k, n in enumerate(sizes * 3):
            q = qs[k % 2]
            key = (n, q)
            if key not in pools:
                pools[key] = (_pool(torch, rng, q, n, 3), [0])
            (a, b, c), used = pools[key]
            j = used[0]
            used[0] += 1
            if j >= 3:
                continue
            tickets.append((srv.submit_ptr(n, q, 14, a[j].data_ptr(), b[j].data_ptr(), c[j].data_ptr()), key, j))
        for t, _, _ in tickets:
            srv.wait(t)
        st = srv.stats()
        assert st["completed"] == len(tickets) and st["failed"] == 0
        assert st["p99_us"] >= st["p50_us"] > 0
    for (n, q), ((a, b, c), used) in pools.items():
        with polymul.Plan(n, q, 14, tensor=tensor) as p:
            for j in range(min(used[0], 3)):
                ai, bi = a[j].numpy().view(np.uint64), b[j].numpy().view(np.uint64)
                assert (c[j].numpy().view(np.uint64) == p.multiply_host(ai, bi)).all(), (n, j)


def test_result_same_alone_and_in_the_mix(cuda):
    """A product computed with nothing else on the GPU equals the same product
    computed while many others of other sizes are in flight around it."""
    torch = cuda
    rng = np.random.default_rng(777)
    q = random_q(rng, 868)
    n = 32768
    x_a, x_b, x_c_alone = _pool(torch, rng, q, n, 1)
    x_c_mix = torch.zeros_like(x_c_alone).pin_memory()
    others = {m: _pool(torch, rng, q, m, 4) for m in (4096, 16384, 65536)}
    with polymul.Server(slots=8, max_group=4) as srv:
        srv.wait(srv.submit_ptr(n, q, 14, x_a[0].data_ptr(), x_b[0].data_ptr(), x_c_alone[0].data_ptr()))
        tickets = []
        for j in range(4):
            for m, (a, b, c) in others.items():
                tickets.append(srv.submit_ptr(m, q, 14, a[j].data_ptr(), b[j].data_ptr(), c[j].data_ptr()))
            if j == 2:
                tickets.append(srv.submit_ptr(n, q, 14, x_a[0].data_ptr(), x_b[0].data_ptr(), x_c_mix[0].data_ptr()))
        for t in tickets:
            srv.wait(t)
        assert srv.stats()["peak_inflight"] > 1
    assert torch.equal(x_c_alone, x_c_mix)
    ai, bi = x_a[0].numpy().view(np.uint64), x_b[0].numpy().view(np.uint64)
    assert (x_c_alone[0].numpy().view(np.uint64) == oracle.rns_multiply(ai, bi, q)).all()


def test_admission_by_device_memory(cuda):
    """An arena that holds about two products: everything still completes, never
    more in flight than fits."""
    torch = cuda
    rng = np.random.default_rng(909)
    q = random_q(rng, 868)
    n = 16384
    with polymul.Plan(n, q, 14) as p:
        one = 3 * n * 14 * 8 + p.workspace_bytes
    a, b, c = _pool(torch, rng, q, n, 8)
    with polymul.Server(slots=8, max_group=1, device_budget_bytes=2 * one + 4096) as srv:
        tickets = [srv.submit_ptr(n, q, 14, a[j].data_ptr(), b[j].data_ptr(), c[j].data_ptr()) for j in range(8)]
        for t in tickets:
            srv.wait(t)
        st = srv.stats()
        assert st["completed"] == 8 and st["peak_inflight"] <= 2
    with polymul.Plan(n, q, 14, tensor=True) as p:
        for j in range(8):
            assert (c[j].numpy().view(np.uint64) == p.multiply_host(a[j].numpy().view(np.uint64),
                                                                    b[j].numpy().view(np.uint64))).all()


def test_oversize_request_is_refused(cuda):
    torch = cuda
    q = random_q(np.random.default_rng(3), 868)
    a = torch.zeros((32768, 14), dtype=torch.int64).pin_memory()
    with polymul.Server(slots=2, device_budget_bytes=1 << 20) as srv:
        with pytest.raises(polymul.PolymulError) as e:
            srv.submit_ptr(32768, q, 14, a.data_ptr(), a.data_ptr(), a.data_ptr())
        assert e.value.status == polymul.PM_ERR_BUSY


def test_bounded_wait_times_out_then_drains(cuda):
    torch = cuda
    rng = np.random.default_rng(11)
    q = random_q(rng, 868)
    n = 65536
    a, b, c = _pool(torch, rng, q, n, 2)
    with polymul.Server(slots=1, max_group=1) as srv:
        tickets = [srv.submit_ptr(n, q, 14, a[j % 2].data_ptr(), b[j % 2].data_ptr(), c[j % 2].data_ptr())
                   for j in range(24)]
        with pytest.raises(polymul.PolymulError) as e:
            srv.wait(tickets[-1], timeout_ms=0)
        assert e.value.status == polymul.PM_ERR_TIMEOUT
        srv.drain()
        for t in tickets:
            srv.wait(t)
