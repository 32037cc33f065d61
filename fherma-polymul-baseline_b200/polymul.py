"""Python binding of libpolymul (include/polymul.h) over ctypes.

Host-side mirror of the reference's solution interface for the tests and the
benchmark: ``Plan`` plays fherma_init / fherma_free (fherma.h:44,46) and
``Plan.multiply_host`` plays fherma_run (fherma.h:45) on (n, limbs) uint64
coefficient arrays.  Errors raise ``PolymulError`` carrying the library's
status code and message, the way the reference raises std::runtime_error
(rns/solve.cu:421-423).

The library must be built (``make -C fherma-polymul-baseline_b200``); there is
no fallback -- a missing library is an ImportError-class failure.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpolymul.so")

PM_OK = 0
PM_ERR_INVALID = 1
PM_ERR_UNSUPPORTED = 2
PM_ERR_CUDA = 3
PM_ERR_NO_MEMORY = 4
PM_ERR_TIMEOUT = 5
PM_ERR_BUSY = 6
PM_CONVERT_DEFAULT = 0
PM_CONVERT_TENSOR = 1
PM_CONVERT_SIMT = 8
PM_SPECIAL_FORM = 2
PM_WIDE_NTT = 4
PM_QUARTIC = 16

_lib = None


class PolymulError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


class PlanInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("q_bits", ctypes.c_uint32), ("coef_limbs", ctypes.c_uint32),
                ("primes", ctypes.c_uint32), ("convert", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("workspace_bytes", ctypes.c_size_t)]


class Tuning(ctypes.Structure):
    _fields_ = [("row_radix", ctypes.c_uint32), ("conv_ctas_per_sm", ctypes.c_uint32),
                ("crt_ctas_per_sm", ctypes.c_uint32), ("group", ctypes.c_uint32), ("row_persistent", ctypes.c_uint32),
                ("conv_whole_basis", ctypes.c_uint32), ("us_per_product", ctypes.c_double)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_uint32), ("max_group", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("device_budget_bytes", ctypes.c_size_t)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64),
                ("groups", ctypes.c_uint64), ("peak_inflight", ctypes.c_uint32), ("peak_group", ctypes.c_uint32),
                ("arena_bytes", ctypes.c_size_t), ("arena_used", ctypes.c_size_t), ("p50_us", ctypes.c_double),
                ("p99_us", ctypes.c_double), ("mean_us", ctypes.c_double), ("max_us", ctypes.c_double),
                ("products_per_s", ctypes.c_double)]


def lib():
    """Load libpolymul.so once; raises OSError when it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: build it with make -C {HERE}")
        L = ctypes.CDLL(LIB_PATH)
        vp, u32, u64p = ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64)
        L.pm_plan_create.argtypes = [ctypes.POINTER(vp), u32, u64p, u32, u32, u32]
        L.pm_plan_get_info.argtypes = [vp, ctypes.POINTER(PlanInfo)]
        L.pm_plan_destroy.argtypes = [vp]
        L.pm_multiply.argtypes = [vp, vp, vp, vp, vp, vp]
        L.pm_multiply_host.argtypes = [vp, vp, vp, vp]
        L.pm_multiply_host_begin.argtypes = [vp, vp, vp]
        L.pm_multiply_host_end.argtypes = [vp, vp]
        L.pm_multiply_host_batch.argtypes = [vp, vp, vp, vp, u32]
        L.pm_multiply_batch.argtypes = [vp, vp, vp, vp, u32, vp, ctypes.c_size_t, vp]
        L.pm_batch_workspace_size.argtypes = [vp, u32, ctypes.POINTER(ctypes.c_size_t)]
        L.pm_basis_query.argtypes = [u32, u32, ctypes.POINTER(u32), u32, ctypes.POINTER(u32)]
        L.pm_server_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(ServerConfig)]
        L.pm_server_submit.argtypes = [vp, u32, u64p, u32, u32, vp, vp, vp, ctypes.POINTER(ctypes.c_uint64)]
        L.pm_server_wait.argtypes = [vp, ctypes.c_uint64, u32]
        L.pm_server_drain.argtypes = [vp, u32]
        L.pm_server_get_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
        L.pm_server_reset_stats.argtypes = [vp]
        L.pm_server_destroy.argtypes = [vp]
        L.pm_plan_autotune.argtypes = [vp, u32, ctypes.POINTER(Tuning)]
        L.pm_plan_set_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
        L.pm_batch_create.argtypes = [ctypes.POINTER(vp), u32, ctypes.POINTER(u32), ctypes.POINTER(u64p),
                                      ctypes.POINTER(u32), u32]
        L.pm_batch_buffers.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp), u64p]
        L.pm_batch_copy_in.argtypes = [vp, vp, vp, vp]
        L.pm_batch_copy_out.argtypes = [vp, vp, vp]
        L.pm_batch_run.argtypes = [vp, vp]
        L.pm_batch_check.argtypes = [vp]
        L.pm_batch_autotune.argtypes = [vp, u32, ctypes.POINTER(ctypes.c_double)]
        L.pm_batch_destroy.argtypes = [vp]
        L.pm_status_string.restype = ctypes.c_char_p
        L.pm_status_string.argtypes = [ctypes.c_int]
        L.pm_last_error.restype = ctypes.c_char_p
        L.pm_kernel_launch_count.restype = ctypes.c_uint64
        L.pm_profile_enable.argtypes = [ctypes.c_uint32]
        L.pm_profile_read.argtypes = [ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_uint64),
                                      ctypes.POINTER(ctypes.c_double), ctypes.c_uint32, ctypes.POINTER(u32)]
        _lib = L
    return _lib


def check(status):
    if status != PM_OK:
        raise PolymulError(status, lib().pm_last_error().decode(errors="replace"))


def q_limbs_of(q):
    q = int(q)
    limbs = max(1, (q.bit_length() + 63) // 64)
    return np.frombuffer(q.to_bytes(8 * limbs, "little"), dtype=np.uint64).copy()


def basis(n, q_bits):
    """Primes of the RNS basis for (n, q_bits); needs no GPU."""
    buf = (ctypes.c_uint32 * 128)()
    count = ctypes.c_uint32(0)
    check(lib().pm_basis_query(n, q_bits, buf, 128, ctypes.byref(count)))
    return [buf[i] for i in range(count.value)]


def launch_count():
    return int(lib().pm_kernel_launch_count())


def profile_enable(capacity):
    """Record device time of each library kernel launch (up to `capacity` launches)."""
    check(lib().pm_profile_enable(capacity))


def profile_read():
    """{kernel name: (launches, total device ms)} since profile_enable."""
    cap = 64
    names = (ctypes.c_char_p * cap)()
    launches = (ctypes.c_uint64 * cap)()
    ms = (ctypes.c_double * cap)()
    count = ctypes.c_uint32(0)
    check(lib().pm_profile_read(names, launches, ms, cap, ctypes.byref(count)))
    return {names[i].decode(): (int(launches[i]), float(ms[i])) for i in range(min(cap, count.value))}


def selftest_bounded_wait(limit_us):
    """Run the library's bounded device wait on a barrier nothing arrives at; returns
    (timed_out, waited_ns)."""
    t = ctypes.c_uint32(0)
    w = ctypes.c_uint64(0)
    check(lib().pm_selftest_bounded_wait(ctypes.c_uint32(limit_us), ctypes.byref(t), ctypes.byref(w)))
    return bool(t.value), w.value


class Plan:
    """A product plan for (n, q): basis, CRT constants, workspace, staging."""

    def __init__(self, n, q, coef_limbs=None, tensor=None, special_form=False, wide=False, quartic=False):
        """tensor: None lets the library choose (the tensor path when coef_limbs is even),
        True asks for the tcgen05 conversion/CRT, False for the plain method."""
        self.q = int(q)
        qarr = q_limbs_of(self.q)
        self.n = int(n)
        self.coef_limbs = int(coef_limbs) if coef_limbs else len(qarr)
        self._h = ctypes.c_void_p()
        check(lib().pm_plan_create(ctypes.byref(self._h), self.n,
                                   qarr.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), len(qarr),
                                   self.coef_limbs, self._convert_flag(tensor)
                                   | (PM_SPECIAL_FORM if special_form else 0) | (PM_WIDE_NTT if wide else 0)
                                   | (PM_QUARTIC if quartic else 0)))
        info = PlanInfo()
        check(lib().pm_plan_get_info(self._h, ctypes.byref(info)))
        self.info = info
        self.primes = info.primes
        self.workspace_bytes = info.workspace_bytes
        self.tensor = info.convert == PM_CONVERT_TENSOR

    @staticmethod
    def _convert_flag(tensor):
        if tensor is None:
            return PM_CONVERT_DEFAULT
        return PM_CONVERT_TENSOR if tensor else PM_CONVERT_SIMT

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().pm_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _shape_ok(self, x):
        x = np.ascontiguousarray(x, dtype=np.uint64)
        if x.shape != (self.n, self.coef_limbs):
            raise PolymulError(PM_ERR_INVALID, f"expected shape {(self.n, self.coef_limbs)}, got {x.shape}")
        return x

    def multiply_host(self, a, b, out=None):
        """c = a*b mod (X^n+1, q) for host arrays; synchronous."""
        a, b = self._shape_ok(a), self._shape_ok(b)
        c = np.empty_like(a) if out is None else out
        check(lib().pm_multiply_host(self._h, a.ctypes.data, b.ctypes.data, c.ctypes.data))
        return c

    def multiply_host_begin(self, a, b):
        """First half of multiply_host: stage a, b and queue the product; returns at once."""
        a, b = self._shape_ok(a), self._shape_ok(b)
        check(lib().pm_multiply_host_begin(self._h, a.ctypes.data, b.ctypes.data))

    def multiply_host_end(self, out=None):
        """Second half: wait for the product and copy it out."""
        c = np.empty((self.n, self.coef_limbs), dtype=np.uint64) if out is None else out
        check(lib().pm_multiply_host_end(self._h, c.ctypes.data))
        return c

    def multiply_host_ptr(self, a_ptr, b_ptr, c_ptr):
        """Same on raw host pointers (e.g. pinned torch tensors); synchronous."""
        check(lib().pm_multiply_host(self._h, a_ptr, b_ptr, c_ptr))

    def autotune(self, reps=3):
        """Time candidate launch shapes and keep the fastest; returns them as a dict."""
        t = Tuning()
        check(lib().pm_plan_autotune(self._h, reps, ctypes.byref(t)))
        return {name: getattr(t, name) for name, _ in Tuning._fields_}

    def set_tuning(self, row_radix=16, conv_ctas_per_sm=3, crt_ctas_per_sm=2, group=0, row_persistent=1,
                   conv_whole_basis=1):
        t = Tuning(row_radix, conv_ctas_per_sm, crt_ctas_per_sm, group, row_persistent, conv_whole_basis, 0.0)
        check(lib().pm_plan_set_tuning(self._h, ctypes.byref(t)))

    def multiply_host_batch(self, a, b, out=None):
        """(count, n, limbs) host arrays -> products, pipelined over three streams; synchronous."""
        a = np.ascontiguousarray(a, dtype=np.uint64)
        b = np.ascontiguousarray(b, dtype=np.uint64)
        if a.shape != b.shape or a.ndim != 3 or a.shape[1:] != (self.n, self.coef_limbs):
            raise PolymulError(PM_ERR_INVALID, f"expected (count, {self.n}, {self.coef_limbs}) arrays")
        c = np.empty_like(a) if out is None else out
        check(lib().pm_multiply_host_batch(self._h, a.ctypes.data, b.ctypes.data, c.ctypes.data, a.shape[0]))
        return c

    def multiply_host_batch_ptr(self, a_ptr, b_ptr, c_ptr, count):
        """Same on raw host pointers (e.g. pinned torch tensors)."""
        check(lib().pm_multiply_host_batch(self._h, a_ptr, b_ptr, c_ptr, count))

    def multiply_batch(self, a_ptr, b_ptr, c_ptr, count, workspace=0, workspace_bytes=0, stream=0):
        """count products stored back to back on the device (asynchronous)."""
        check(lib().pm_multiply_batch(self._h, a_ptr, b_ptr, c_ptr, count, workspace or None, workspace_bytes,
                                      stream or None))

    def batch_workspace_size(self, count):
        out = ctypes.c_size_t(0)
        check(lib().pm_batch_workspace_size(self._h, count, ctypes.byref(out)))
        return out.value

    def multiply(self, a_ptr, b_ptr, c_ptr, workspace=0, stream=0):
        """Asynchronous product on device pointers (ints) on a CUDA stream handle."""
        check(lib().pm_multiply(self._h, a_ptr, b_ptr, c_ptr, workspace or None, stream or None))


class Server:
    """Continuous-batching serving loop (pm_server_*): submit host buffers, wait on tickets."""

    def __init__(self, slots=8, max_group=8, tensor=True, device_budget_bytes=0):
        cfg = ServerConfig(slots, max_group, PM_CONVERT_TENSOR if tensor else PM_CONVERT_SIMT, 0,
                           device_budget_bytes)
        self._h = ctypes.c_void_p()
        check(lib().pm_server_create(ctypes.byref(self._h), ctypes.byref(cfg)))
        self._q = {}

    def submit_ptr(self, n, q, coef_limbs, a_ptr, b_ptr, c_ptr):
        """Queue one product on host pointers (keep the buffers alive); returns a ticket."""
        qa = self._q.get(q)
        if qa is None:
            qa = self._q[q] = q_limbs_of(q)
        t = ctypes.c_uint64(0)
        check(lib().pm_server_submit(self._h, n, qa.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), len(qa),
                                     coef_limbs, a_ptr, b_ptr, c_ptr, ctypes.byref(t)))
        return t.value

    def wait(self, ticket, timeout_ms=60000):
        check(lib().pm_server_wait(self._h, ticket, timeout_ms))

    def drain(self, timeout_ms=600000):
        check(lib().pm_server_drain(self._h, timeout_ms))

    def stats(self):
        st = ServerStats()
        check(lib().pm_server_get_stats(self._h, ctypes.byref(st)))
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}

    def reset_stats(self):
        check(lib().pm_server_reset_stats(self._h))

    def close(self):
        if self._h:
            lib().pm_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Batch:
    """Uneven batch (pm_batch_*): products of different n and q run as one CUDA graph."""

    def __init__(self, ns, qs, coef_limbs=14):
        count = len(ns)
        self.ns = [int(n) for n in ns]
        self.coef_limbs = int(coef_limbs)
        self._qarr = [q_limbs_of(q) for q in qs]
        n_arr = (ctypes.c_uint32 * count)(*self.ns)
        q_ptrs = (ctypes.POINTER(ctypes.c_uint64) * count)(
            *[qa.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)) for qa in self._qarr])
        ql = (ctypes.c_uint32 * count)(*[len(qa) for qa in self._qarr])
        self._h = ctypes.c_void_p()
        check(lib().pm_batch_create(ctypes.byref(self._h), count, n_arr, q_ptrs, ql, self.coef_limbs))
        offs = (ctypes.c_uint64 * count)()
        a, b, c = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        check(lib().pm_batch_buffers(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), offs))
        self.offsets = [int(o) for o in offs]
        self.words = sum(n * self.coef_limbs for n in self.ns)
        self.a_ptr, self.b_ptr, self.c_ptr = a.value, b.value, c.value

    def pack(self, arrays):
        """List of (n_z, limbs) arrays -> one packed uint64 array in the batch's layout."""
        out = np.zeros(self.words, dtype=np.uint64)
        for off, arr in zip(self.offsets, arrays):
            flat = np.ascontiguousarray(arr, dtype=np.uint64).ravel()
            out[off:off + flat.size] = flat
        return out

    def unpack(self, packed):
        return [packed[off:off + n * self.coef_limbs].reshape(n, self.coef_limbs)
                for off, n in zip(self.offsets, self.ns)]

    def copy_in(self, a_packed_ptr, b_packed_ptr, stream=0):
        check(lib().pm_batch_copy_in(self._h, a_packed_ptr, b_packed_ptr, stream or None))

    def copy_out(self, c_packed_ptr, stream=0):
        check(lib().pm_batch_copy_out(self._h, c_packed_ptr, stream or None))

    def run(self, stream=0):
        check(lib().pm_batch_run(self._h, stream or None))

    def check_errors(self):
        check(lib().pm_batch_check(self._h))

    def autotune(self, reps=3):
        us = ctypes.c_double(0)
        check(lib().pm_batch_autotune(self._h, reps, ctypes.byref(us)))
        return us.value

    def multiply_host(self, a_list, b_list):
        """Synchronous convenience: host arrays in, list of products out."""
        import torch

        a = self.pack(a_list)
        b = self.pack(b_list)
        c = np.zeros_like(a)
        self.copy_in(a.ctypes.data, b.ctypes.data)
        self.run()
        self.copy_out(c.ctypes.data)
        torch.cuda.synchronize()
        self.check_errors()
        return self.unpack(c)

    def close(self):
        if self._h:
            lib().pm_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
