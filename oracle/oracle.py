"""TEST INFRASTRUCTURE ONLY: ctypes binding of the C oracle (oracle/polymul_oracle.c).

Coefficient arrays are (n, limbs) uint64, little-endian limbs -- the same bytes
as the reference's N x L x u32 tensors (fherma.h:27-42).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        L.orc_rns_multiply.argtypes = [ctypes.c_uint, u32p, ctypes.c_uint, u32p, u32p, u32p, ctypes.c_uint,
                                       ctypes.c_uint, ctypes.c_uint, ctypes.c_uint32, ctypes.c_uint]
        L.orc_schoolbook.argtypes = [ctypes.c_uint, u32p, ctypes.c_uint, u32p, u32p, u32p, ctypes.c_uint,
                                     ctypes.c_uint]
        L.orc_basis_dump.argtypes = [ctypes.c_uint, u32p, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint32,
                                     ctypes.c_uint, u32p, u32p, u32p, ctypes.POINTER(ctypes.c_uint64), u32p,
                                     ctypes.POINTER(ctypes.c_uint)]
        _LIB = L
    return _LIB


def int_to_words(value, nwords):
    return np.frombuffer(int(value).to_bytes(4 * nwords, "little"), dtype=np.uint32).copy()


def q_words(q):
    q = int(q)
    return int_to_words(q, (q.bit_length() + 31) // 32)


def _p32(x):
    return x.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def _prep(a, b):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    assert a.shape == b.shape and a.ndim == 2
    return a, b


def rns_multiply(a, b, q, threads=None, bits=0, order=0, count=0):
    """The reference's RNS method restated on the CPU (threads over primes)."""
    a, b = _prep(a, b)
    n, limbs = a.shape
    qw = q_words(q)
    c = np.zeros_like(a)
    rc = lib().orc_rns_multiply(n, _p32(qw), len(qw), _p32(a), _p32(b), _p32(c), 2 * limbs,
                                threads or os.cpu_count() or 1, bits, order, count)
    if rc:
        raise RuntimeError(f"orc_rns_multiply failed: {rc}")
    return c


def schoolbook(a, b, q, threads=None):
    a, b = _prep(a, b)
    n, limbs = a.shape
    qw = q_words(q)
    c = np.zeros_like(a)
    rc = lib().orc_schoolbook(n, _p32(qw), len(qw), _p32(a), _p32(b), _p32(c), 2 * limbs,
                              threads or os.cpu_count() or 1)
    if rc:
        raise RuntimeError(f"orc_schoolbook failed: {rc}")
    return c


def basis_dump(n, q, qwords, bits, order, count):
    """Basis constants (primes, recip, psi, (P/p_i) mod q, P mod q) for comparison tests."""
    qw = int_to_words(q, qwords)
    primes = np.zeros(128, np.uint32)
    bases = np.zeros(128 * qwords, np.uint32)
    pmod = np.zeros(qwords, np.uint32)
    recip = np.zeros(128, np.uint64)
    psi = np.zeros(128, np.uint32)
    cnt = ctypes.c_uint(0)
    rc = lib().orc_basis_dump(n, _p32(qw), qwords, bits, order, count, _p32(primes), _p32(bases), _p32(pmod),
                              recip.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), _p32(psi), ctypes.byref(cnt))
    if rc:
        raise RuntimeError(f"orc_basis_dump failed: {rc}")
    k = cnt.value
    return dict(primes=primes[:k].copy(), recip=recip[:k].copy(), psi=psi[:k].copy(),
                bases_mod_q=bases[: k * qwords].reshape(k, qwords).copy(), product_mod_q=pmod.copy())
