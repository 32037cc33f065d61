"""TEST INFRASTRUCTURE ONLY: exact big-integer arithmetic through the system GMP.

GMP (libgmp.so.10, the LGPL runtime in the image) is called through ctypes with
the prototypes of its public manual (mpz_init, mpz_import, mpz_export, mpz_mul,
mpz_probab_prime_p).  It backs two checkers:

* ``kronecker(a, b, q)`` -- the reference's independent oracle restated: pack the
  coefficients into one integer per polynomial with base 2^(8*width),
  B > N*(q-1)^2, multiply once, unpack, fold X^N = -1 (tests/validate.py:29-37).
* ``Mpz`` / ``is_prime`` -- the small surface of gmpy2 that the reference's
  tests/validate.py uses, so that file can be imported unmodified to generate
  golden vectors (tests/golden/make_golden.py).
"""
import ctypes
import ctypes.util

import numpy as np


class _mpz_t(ctypes.Structure):
    _fields_ = [("alloc", ctypes.c_int), ("size", ctypes.c_int), ("d", ctypes.c_void_p)]


def _load():
    for name in ("libgmp.so.10", ctypes.util.find_library("gmp")):
        if not name:
            continue
        try:
            return ctypes.CDLL(name)
        except OSError:
            continue
    raise OSError("libgmp runtime not found")


_gmp = _load()
_P = ctypes.POINTER(_mpz_t)


def _fn(name, argtypes, restype=None):
    f = getattr(_gmp, name)  # looked up by string: a __name inside a class would be mangled
    f.argtypes = argtypes
    f.restype = restype
    return f


_init = _fn("__gmpz_init", [_P])
_clear = _fn("__gmpz_clear", [_P])
_import = _fn("__gmpz_import", [_P, ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t, ctypes.c_int,
                                ctypes.c_size_t, ctypes.c_void_p])
_export = _fn("__gmpz_export", [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t), ctypes.c_int,
                                ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t, _P], ctypes.c_void_p)
_mul = _fn("__gmpz_mul", [_P, _P, _P])
_sizeinbase = _fn("__gmpz_sizeinbase", [_P, ctypes.c_int], ctypes.c_size_t)
_probab_prime = _fn("__gmpz_probab_prime_p", [_P, ctypes.c_int], ctypes.c_int)


class Mpz:
    """Non-negative GMP integer with just the operations validate.py needs."""

    def __init__(self):
        self._z = _mpz_t()
        _init(ctypes.byref(self._z))

    def __del__(self):
        try:
            _clear(ctypes.byref(self._z))
        except Exception:
            pass

    @classmethod
    def from_bytes(cls, data, byteorder="little"):
        assert byteorder == "little"
        z = cls()
        buf = ctypes.create_string_buffer(bytes(data), len(data))
        _import(ctypes.byref(z._z), len(data), -1, 1, 0, 0, buf)
        return z

    @classmethod
    def from_int(cls, value):
        value = int(value)
        assert value >= 0
        return cls.from_bytes(value.to_bytes(max(1, (value.bit_length() + 7) // 8), "little"))

    def __mul__(self, other):
        if not isinstance(other, Mpz):
            other = Mpz.from_int(other)
        r = Mpz()
        _mul(ctypes.byref(r._z), ctypes.byref(self._z), ctypes.byref(other._z))
        return r

    __rmul__ = __mul__

    def nbytes(self):
        return (_sizeinbase(ctypes.byref(self._z), 2) + 7) // 8

    def to_bytes(self, length, byteorder="little"):
        assert byteorder == "little"
        need = self.nbytes()
        if need > length:
            raise OverflowError("int too big to convert")
        buf = ctypes.create_string_buffer(max(need, 1))
        count = ctypes.c_size_t(0)
        _export(buf, ctypes.byref(count), -1, 1, 0, 0, ctypes.byref(self._z))
        return buf.raw[: count.value] + b"\x00" * (length - count.value)

    def __int__(self):
        return int.from_bytes(self.to_bytes(self.nbytes() or 1), "little")


def is_prime(value, reps=25):
    z = Mpz.from_int(int(value))
    return _probab_prime(ctypes.byref(z._z), int(reps)) > 0


def kronecker(a, b, q):
    """c = a*b mod (X^n+1, q); a, b: (n, limbs) uint64 arrays; returns the same shape."""
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    n, limbs = a.shape
    q = int(q)
    stride = limbs * 8
    width = max(((n * (q - 1) ** 2).bit_length() + 7) // 8, stride)

    def pack(x):
        raw = np.zeros((n, width), dtype=np.uint8)
        raw[:, :stride] = x.view(np.uint8).reshape(n, stride)
        return Mpz.from_bytes(raw.tobytes())

    prod = (pack(a) * pack(b)).to_bytes(2 * n * width)
    raw = np.frombuffer(prod, dtype=np.uint8).reshape(2 * n, width)
    out = np.zeros((n, limbs), dtype=np.uint64)
    view = out.view(np.uint8).reshape(n, stride)
    for k in range(n):
        lo = int.from_bytes(raw[k].tobytes(), "little")
        hi = int.from_bytes(raw[k + n].tobytes(), "little")
        view[k] = np.frombuffer(((lo - hi) % q).to_bytes(stride, "little"), dtype=np.uint8)
    return out
