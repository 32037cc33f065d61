"""GPU parity through the C ABI, for both conversion/CRT paths: the plain
SIMT one and the tcgen05 INT8 tensor-core one (the NTT kernels are shared).

Bit-exact: every product must equal the oracle's canonical residue in [0, q).
The reference's golden points (tests/golden/golden.json, produced by its own
tests/validate.py) are checked by SHA-256; other sizes and widths against the
C oracle on the same seeded inputs.
"""
import numpy as np
import pytest

import polymul
from oracle import oracle
from tests.golden.cases import point_cases, sha
from tests.helpers import random_q, uniform_below

pytestmark = pytest.mark.gpu


# simt: the plain CUDA-core method; tensor: the tcgen05 path with its default conversion
# (K1W, a coefficient tile through the whole basis); tensor_k1t: the same path with the
# per-prime-group conversion (K1T)
@pytest.fixture(params=["simt", "tensor", "tensor_k1t"])
def path(request):
    return request.param


def make_plan(path, n, q, limbs=None):
    p = polymul.Plan(n, q, coef_limbs=limbs, tensor=(path != "simt"))
    if path == "tensor_k1t":
        p.set_tuning(conv_whole_basis=0)
    return p


def limbs_for(path, bits):
    """u64 limbs per coefficient: the tensor path reads 16-byte coefficient rows."""
    limbs = (bits + 63) // 64
    return limbs + (limbs % 2) if path != "simt" else limbs


def test_golden_points(cuda, golden, path):
    for point in golden["points"]:
        q = int(point["q"], 16)
        with make_plan(path, point["N"], q, 14) as p:
            for label, a, b, rec in point_cases(point):  # same plan reused across cases
                c = p.multiply_host(a, b)
                assert sha(c.tobytes()) == rec["c_sha256"], (point["N"], point["delta"], label)


@pytest.mark.parametrize("n", [2, 4, 8, 16, 32, 64, 128, 256, 512, 2048, 8192, 16384, 65536])
def test_ring_sizes_868(cuda, path, n):
    rng = np.random.default_rng(n)
    q = random_q(rng, 868)
    a, b = uniform_below(rng, q, n, 14), uniform_below(rng, q, n, 14)
    with make_plan(path, n, q, 14) as p:
        assert (p.multiply_host(a, b) == oracle.rns_multiply(a, b, q)).all()


@pytest.mark.parametrize("bits", [3, 31, 64, 65, 129, 200, 257, 384, 517, 640, 700, 800, 867, 896])
def test_widths(cuda, path, bits):
    n = 1024
    rng = np.random.default_rng(bits)
    q = random_q(rng, bits)
    limbs = limbs_for(path, bits)
    a, b = uniform_below(rng, q, n, limbs), uniform_below(rng, q, n, limbs)
    with make_plan(path, n, q, limbs) as p:
        assert (p.multiply_host(a, b) == oracle.rns_multiply(a, b, q)).all()


def test_padded_limbs(cuda, path):
    """Coefficients stored wider than q needs (the fherma layout keeps 28 words for any q)."""
    rng = np.random.default_rng(3)
    q = random_q(rng, 200)
    a, b = uniform_below(rng, q, 256, 14), uniform_below(rng, q, 256, 14)
    with make_plan(path, 256, q, 14) as p:
        c = p.multiply_host(a, b)
    assert (c == oracle.rns_multiply(a, b, q)).all()
    assert not c[:, 4:].any()


def test_edge_values_full_size(cuda, path):
    n = 32768
    q = (1 << 868) - 1  # not prime: any odd q is accepted
    vals = [0, 1, q - 1, q - 2, 1 << 864, (1 << 864) - 1, 1 << 32, (1 << 32) - 1, (1 << 867), 2]
    rng = np.random.default_rng(11)
    idx = rng.integers(0, len(vals), size=n)
    from tests.helpers import from_ints
    a = from_ints([vals[i] for i in idx], 14)
    b = from_ints([vals[i] for i in rng.permutation(idx)], 14)
    with make_plan(path, n, q, 14) as p:
        assert (p.multiply_host(a, b) == oracle.rns_multiply(a, b, q)).all()


def test_device_pointers_and_external_workspace(cuda, path):
    torch = cuda
    n = 4096
    rng = np.random.default_rng(5)
    q = random_q(rng, 868)
    a, b = uniform_below(rng, q, n, 14), uniform_below(rng, q, n, 14)
    expect = oracle.rns_multiply(a, b, q)
    with make_plan(path, n, q, 14) as p:
        da = torch.from_numpy(a.view(np.int64)).cuda()
        db = torch.from_numpy(b.view(np.int64)).cuda()
        dc = torch.empty_like(da)
        ws = torch.empty(p.workspace_bytes, dtype=torch.uint8, device="cuda")
        s = torch.cuda.Stream()
        p.multiply(da.data_ptr(), db.data_ptr(), dc.data_ptr(), ws.data_ptr(), s.cuda_stream)
        s.synchronize()
        assert (dc.cpu().numpy().view(np.uint64) == expect).all()
        # plan-owned workspace on the default stream
        dc.zero_()
        p.multiply(da.data_ptr(), db.data_ptr(), dc.data_ptr())
        torch.cuda.synchronize()
        assert (dc.cpu().numpy().view(np.uint64) == expect).all()


def test_full_size_linearity(cuda, path):
    """Size-independent property at the benchmark size: (a1 + a2) b = a1 b + a2 b (mod q)."""
    from tests.helpers import to_ints, from_ints
    n = 32768
    q = (1 << 868) - 11993087
    rng = np.random.default_rng(21)
    a1, a2, b = (uniform_below(rng, q, n, 14) for _ in range(3))
    s = from_ints([(x + y) % q for x, y in zip(to_ints(a1), to_ints(a2))], 14)
    with make_plan(path, n, q, 14) as p:
        c1, c2, cs = p.multiply_host(a1, b), p.multiply_host(a2, b), p.multiply_host(s, b)
    assert to_ints(cs) == [(x + y) % q for x, y in zip(to_ints(c1), to_ints(c2))]


@pytest.mark.parametrize("n,bits,count", [(32768, 868, 7), (1024, 300, 33), (64, 868, 5), (65536, 868, 3)])
def test_batch_api(cuda, path, n, bits, count):
    """pm_multiply_batch: products back to back, a count that is not a multiple of the group size."""
    torch = cuda
    rng = np.random.default_rng(n + count)
    q = random_q(rng, bits)
    limbs = limbs_for(path, bits)
    a = np.stack([uniform_below(rng, q, n, limbs) for _ in range(count)])
    b = np.stack([uniform_below(rng, q, n, limbs) for _ in range(count)])
    with make_plan(path, n, q, limbs) as p:
        da = torch.from_numpy(a.view(np.int64)).cuda()
        db = torch.from_numpy(b.view(np.int64)).cuda()
        dc = torch.zeros_like(da)
        p.multiply_batch(da.data_ptr(), db.data_ptr(), dc.data_ptr(), count)
        torch.cuda.synchronize()
        got = dc.cpu().numpy().view(np.uint64)
        # caller workspace of exactly one product forces groups of one
        dc2 = torch.zeros_like(da)
        ws = torch.empty(p.workspace_bytes, dtype=torch.uint8, device="cuda")
        p.multiply_batch(da.data_ptr(), db.data_ptr(), dc2.data_ptr(), count, ws.data_ptr(), p.workspace_bytes)
        torch.cuda.synchronize()
        assert (dc2.cpu().numpy().view(np.uint64) == got).all()
    for k in sorted({0, count // 2, count - 1}):
        assert (got[k] == oracle.rns_multiply(a[k], b[k], q)).all(), k


def test_conversion_byte_edges(cuda, path):
    """Coefficients made of 0x00 / 0xFF / 0x80 / 0x7F bytes, the extremes of the
    INT8 digit contraction (the reference checks the same bytes in
    tests/tensor_conversion.cpp:12)."""
    n = 4096
    q = (1 << 868) - 1
    from tests.helpers import from_ints
    patterns = [0, q - 1, int.from_bytes(b"\x80" * 108, "little"), int.from_bytes(b"\x7f" * 108, "little"),
                int.from_bytes(b"\xff" * 108, "little"), (1 << 864) - 1]
    rng = np.random.default_rng(99)
    a = from_ints([patterns[i] for i in rng.integers(0, len(patterns), size=n)], 14)
    b = from_ints([patterns[i] for i in rng.integers(0, len(patterns), size=n)], 14)
    with make_plan(path, n, q, 14) as p:
        assert (p.multiply_host(a, b) == oracle.rns_multiply(a, b, q)).all()


def test_paths_agree_bitwise(cuda):
    """The tensor path is bit-exact against the plain path on the same inputs."""
    n = 32768
    rng = np.random.default_rng(4242)
    q = random_q(rng, 868)
    a, b = uniform_below(rng, q, n, 14), uniform_below(rng, q, n, 14)
    with make_plan("simt", n, q, 14) as p1, make_plan("tensor", n, q, 14) as p2:
        assert (p1.multiply_host(a, b) == p2.multiply_host(a, b)).all()


def test_tensor_path_refuses_odd_limbs(cuda):
    with pytest.raises(polymul.PolymulError) as e:
        make_plan("tensor", 1024, random_q(np.random.default_rng(1), 517), 9)
    assert e.value.status == polymul.PM_ERR_UNSUPPORTED


@pytest.mark.parametrize("pinned", [False, True])
def test_host_batch_pipeline(cuda, path, pinned):
    """pm_multiply_host_batch: host buffers, groups rotating over three streams."""
    torch = cuda
    n, count = 16384, 11
    rng = np.random.default_rng(31 + int(pinned))
    q = random_q(rng, 868)
    a = np.stack([uniform_below(rng, q, n, 14) for _ in range(count)])
    b = np.stack([uniform_below(rng, q, n, 14) for _ in range(count)])
    with make_plan(path, n, q, 14) as p:
        if pinned:
            ha = torch.from_numpy(a.view(np.int64)).pin_memory()
            hb = torch.from_numpy(b.view(np.int64)).pin_memory()
            hc = torch.zeros_like(ha).pin_memory()
            p.multiply_host_batch_ptr(ha.data_ptr(), hb.data_ptr(), hc.data_ptr(), count)
            got = hc.numpy().view(np.uint64)
        else:
            got = p.multiply_host_batch(a, b)
        for k in range(count):
            assert (got[k] == p.multiply_host(a[k], b[k])).all(), k
    for k in (0, count - 1):
        assert (got[k] == oracle.rns_multiply(a[k], b[k], q)).all()


@pytest.mark.parametrize("n", [4096, 16384, 32768, 65536])
def test_tunings_do_not_change_results(cuda, path, n):
    """Every launch shape the autotuner may pick gives the same bits."""
    torch = cuda
    rng = np.random.default_rng(n + 17)
    q = random_q(rng, 868)
    count = 5
    a = torch.from_numpy(np.stack([uniform_below(rng, q, n, 14) for _ in range(count)]).view(np.int64)).cuda()
    b = torch.from_numpy(np.stack([uniform_below(rng, q, n, 14) for _ in range(count)]).view(np.int64)).cuda()
    ref = None
    with make_plan(path, n, q, 14) as p:
        # (row radix, K1T CTAs per SM, K3T CTAs per SM, group, persistent rows, whole-basis conversion)
        shapes = [(8, 4, 2, 0, 1, 0), (4, 4, 2, 0, 1, 0), (8, 2, 1, 1, 1, 0), (4, 3, 1, 2, 1, 0), (8, 4, 2, 5, 1, 0),
                  (8, 4, 2, 0, 0, 0), (4, 4, 2, 3, 0, 0), (8, 4, 2, 3, 1, 0), (16, 3, 2, 0, 1, 0),
                  (16, 3, 2, 3, 1, 0), (16, 3, 2, 2, 0, 0), (16, 3, 2, 0, 1, 1), (16, 3, 2, 1, 1, 1),
                  (8, 3, 1, 3, 0, 1)]
        for shape in shapes:
            p.set_tuning(*shape)
            c = torch.zeros_like(a)
            p.multiply_batch(a.data_ptr(), b.data_ptr(), c.data_ptr(), count)
            torch.cuda.synchronize()
            if ref is None:
                ref = c.clone()
            assert torch.equal(c, ref), shape
        chosen = p.autotune()
        # measured here, or -1: the same plan shape was tuned earlier in this process (its cache)
        assert chosen["row_radix"] in (4, 8, 16) and (chosen["us_per_product"] > 0 or chosen["us_per_product"] == -1)
        c = torch.zeros_like(a)
        p.multiply_batch(a.data_ptr(), b.data_ptr(), c.data_ptr(), count)
        torch.cuda.synchronize()
        assert torch.equal(c, ref)
    for k in (0, count - 1):
        ak, bk = a[k].cpu().numpy().view(np.uint64), b[k].cpu().numpy().view(np.uint64)
        assert (ref[k].cpu().numpy().view(np.uint64) == oracle.rns_multiply(ak, bk, q)).all()


def test_tuning_limits_and_large_default_groups(cuda):
    """pm_plan_set_tuning refuses shapes outside its documented ranges; a batch of more
    products than the default launch group (128) runs in a full group and a tail, with the
    same bits as groups of one and the oracle's."""
    torch = cuda
    rng = np.random.default_rng(77)
    q = random_q(rng, 868)
    n, count = 1024, 131
    with make_plan("tensor", n, q, 14) as p:
        for bad in [dict(row_radix=32), dict(group=257), dict(conv_ctas_per_sm=0), dict(crt_ctas_per_sm=5),
                    dict(row_persistent=2), dict(conv_whole_basis=2)]:
            with pytest.raises(polymul.PolymulError):
                p.set_tuning(**bad)
        p.set_tuning(group=256)
        a = torch.from_numpy(np.stack([uniform_below(rng, q, n, 14) for _ in range(count)]).view(np.int64)).cuda()
        b = torch.from_numpy(np.stack([uniform_below(rng, q, n, 14) for _ in range(count)]).view(np.int64)).cuda()
        outs = []
        for group in (0, 1):
            p.set_tuning(group=group)
            c = torch.zeros_like(a)
            p.multiply_batch(a.data_ptr(), b.data_ptr(), c.data_ptr(), count)
            torch.cuda.synchronize()
            outs.append(c)
        assert torch.equal(outs[0], outs[1])
    for k in (0, 127, 128, count - 1):
        ak, bk = a[k].cpu().numpy().view(np.uint64), b[k].cpu().numpy().view(np.uint64)
        assert (outs[0][k].cpu().numpy().view(np.uint64) == oracle.rns_multiply(ak, bk, q)).all()


def test_bad_device_pointers_are_refused(cuda, path):
    """Misaligned or pageable pointers are caught on the host, before any kernel runs."""
    torch = cuda
    n, limbs = 1024, limbs_for(path, 868)
    rng = np.random.default_rng(8)
    q = random_q(rng, 868)
    a = torch.from_numpy(uniform_below(rng, q, n, limbs).view(np.int64)).cuda()
    b = torch.from_numpy(uniform_below(rng, q, n, limbs).view(np.int64)).cuda()
    c = torch.zeros_like(a)
    raw = torch.zeros(a.numel() * 8 + 64, dtype=torch.uint8, device="cuda")
    host = np.zeros((n, limbs), dtype=np.uint64)  # pageable
    with make_plan(path, n, q, limbs) as p:
        for args in [(a.data_ptr() + 4, b.data_ptr(), c.data_ptr()),
                     (a.data_ptr(), b.data_ptr(), c.data_ptr() + 4),
                     (a.data_ptr(), host.ctypes.data, c.data_ptr())]:
            with pytest.raises(polymul.PolymulError) as e:
                p.multiply(*args)
            assert e.value.status == polymul.PM_ERR_INVALID
        if path != "simt":
            with pytest.raises(polymul.PolymulError) as e:
                p.multiply(raw.data_ptr() + 8, b.data_ptr(), c.data_ptr())
            assert e.value.status == polymul.PM_ERR_INVALID
            with pytest.raises(polymul.PolymulError) as e:
                p.multiply(a.data_ptr(), b.data_ptr(), c.data_ptr(), workspace=raw.data_ptr() + 8)
            assert e.value.status == polymul.PM_ERR_INVALID
        # the plan still works afterwards
        p.multiply(a.data_ptr(), b.data_ptr(), c.data_ptr())
        torch.cuda.synchronize()
        got = c.cpu().numpy().view(np.uint64)
        assert (got == oracle.rns_multiply(a.cpu().numpy().view(np.uint64), b.cpu().numpy().view(np.uint64), q)).all()


@pytest.mark.parametrize("n", [1024, 32768])
@pytest.mark.parametrize("qkind", ["random", "fherma"])
def test_coefficients_that_are_multiples_of_q(cuda, path, n, qkind):
    """a = 1 + X and b alternating (q-1)/2, (q+1)/2: every coefficient c_j, j >= 1, is
    b_j + b_(j-1) = q as an integer, so its residue is 0 while its CRT value is not.
    There the contraction's estimate of the quotient mod q can come out one low, and
    only the final conditional subtraction of q brings the result back to 0."""
    from tests.helpers import from_ints

    rng = np.random.default_rng(700 + n)
    q = random_q(rng, 868) if qkind == "random" else (1 << 868) - 11993087
    a = from_ints([1, 1] + [0] * (n - 2), 14)
    b = from_ints([(q - 1) // 2 if j % 2 == 0 else (q + 1) // 2 for j in range(n)], 14)
    want = oracle.rns_multiply(a, b, q)
    assert (want[1:] == 0).all()
    with make_plan(path, n, q, 14) as p:
        assert (p.multiply_host(a, b) == want).all()
