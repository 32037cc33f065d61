"""CPU tests of the C ABI library: it loads, exports every declared symbol,
rejects bad arguments before touching a GPU, and its host-side basis logic
matches the oracle's restatement of the reference's prime search."""
import ctypes
import os
import re

import pytest

import polymul
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pm_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = polymul.lib()
    names = declared("polymul.h")
    assert len(names) >= 8
    for name in names:
        assert hasattr(lib, name), name


def test_invalid_arguments_fail_before_cuda():
    with pytest.raises(polymul.PolymulError) as e:
        polymul.Plan(24, 101)
    assert e.value.status == polymul.PM_ERR_INVALID
    with pytest.raises(polymul.PolymulError) as e:
        polymul.Plan(32, 100)  # even q
    assert e.value.status == polymul.PM_ERR_INVALID
    with pytest.raises(polymul.PolymulError) as e:
        polymul.Plan(1 << 17, 101)
    assert e.value.status == polymul.PM_ERR_UNSUPPORTED
    with pytest.raises(polymul.PolymulError) as e:
        polymul.Plan(32, (1 << 900) + 1)
    assert e.value.status == polymul.PM_ERR_UNSUPPORTED
    with pytest.raises(polymul.PolymulError):
        polymul.Plan(32, (1 << 868) - 11993087, coef_limbs=13)
    # the two conversion paths exclude each other; unknown flag bits are refused
    for flags in (polymul.PM_CONVERT_TENSOR | polymul.PM_CONVERT_SIMT, 1 << 12):
        h = ctypes.c_void_p()
        qa = polymul.q_limbs_of(101)
        status = polymul.lib().pm_plan_create(ctypes.byref(h), 32, qa.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                              1, 1, flags)
        assert status == polymul.PM_ERR_INVALID and not h.value
    for limit in (0, 2_000_001):
        with pytest.raises(polymul.PolymulError) as e:
            polymul.selftest_bounded_wait(limit)
        assert e.value.status == polymul.PM_ERR_INVALID


def test_status_strings():
    lib = polymul.lib()
    for s in range(7):
        assert lib.pm_status_string(s)


@pytest.mark.parametrize("n,bits", [(2, 868), (32, 868), (1024, 200), (32768, 868), (65536, 868), (4096, 517)])
def test_basis_matches_oracle_rule(n, bits):
    primes = polymul.basis(n, bits)
    q = (1 << bits) - 1  # bit length is all the rule depends on
    dump = oracle.basis_dump(n, q, (bits + 31) // 32, 30, 1 << 17, 0)
    assert primes == list(dump["primes"])
    P = 1
    for p in primes:
        assert p % (1 << 17) == 1 and p < (1 << 30) and p > (1 << 29)
        P *= p
    assert P > 4 * n * (1 << bits) ** 2
    assert P // primes[-1] <= 4 * n * (1 << bits) ** 2  # minimal


def test_fherma_point_basis_size():
    assert len(polymul.basis(32768, 868)) == 59
