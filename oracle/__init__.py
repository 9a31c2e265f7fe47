"""Python bindings for the oracle libraries (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` may
import this package, and only as the checker or as the timed CPU baseline.
The product (``bluecrunch_b200``) never imports it.

Two libraries are wrapped:

* ``restated()``  -> oracle/_build/libbcoracle.so, the plain-C restatement of
  the reference multiply path (bc_oracle.c), plus an exact FP64-free NTT
  multiply and modular checksums.
* ``reference(kind)`` -> oracle/_ref/{serial,omp}/libbcref.so, the reference's
  own C sources compiled by oracle/Makefile (present only where the reference
  sources were available at build time; the build output travels with the
  repository snapshot).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_u32p = ctypes.POINTER(ctypes.c_uint32)
_sz = ctypes.c_size_t


def _ptr(a):
    return a.ctypes.data_as(_u32p)


class _Restated:
    def __init__(self, path):
        self.lib = lib = ctypes.CDLL(path)
        lib.bco_width.restype = ctypes.c_int
        lib.bco_width.argtypes = [_sz]
        lib.bco_fft_length.restype = _sz
        lib.bco_fft_length.argtypes = [_sz]
        for name in ("bco_fft_mul",):
            fn = getattr(lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = [_u32p, _sz, _u32p, _sz, _u32p, _sz]
        lib.bco_fft_mul_width.restype = ctypes.c_double
        lib.bco_fft_mul_width.argtypes = [_u32p, _sz, _u32p, _sz, _u32p, _sz, ctypes.c_int]
        lib.bco_basecase_mul.restype = None
        lib.bco_basecase_mul.argtypes = [_u32p, _sz, _u32p, _sz, _u32p, _sz]
        lib.bco_ntt_mul.restype = ctypes.c_int
        lib.bco_ntt_mul.argtypes = [_u32p, _sz, _u32p, _sz, _u32p, _sz]
        lib.bco_checksum.restype = ctypes.c_uint32
        lib.bco_checksum.argtypes = [_u32p, _sz, ctypes.c_uint32]
        lib.bco_modcheck.restype = ctypes.c_int
        lib.bco_modcheck.argtypes = [_u32p, _sz, _u32p, _sz, _u32p, _sz, ctypes.c_int]
        c128 = ctypes.POINTER(ctypes.c_double)
        lib.bco_int_to_fft.restype = _sz
        lib.bco_int_to_fft.argtypes = [c128, _sz, _u32p, _sz, ctypes.c_int]
        lib.bco_fft_to_int.restype = None
        lib.bco_fft_to_int.argtypes = [c128, _sz, _u32p, _sz, ctypes.c_int]
        lib.bco_fft_forward.restype = None
        lib.bco_fft_forward.argtypes = [c128, _sz]
        lib.bco_fft_inverse.restype = None
        lib.bco_fft_inverse.argtypes = [c128, _sz]

    # -- thin numpy-friendly wrappers -------------------------------------
    def width(self, CL):
        return self.lib.bco_width(CL)

    def fft_length(self, n):
        return self.lib.bco_fft_length(n)

    def _mul(self, fn, a, b, CL, square):
        a = np.ascontiguousarray(a, dtype=np.uint32)
        b = a if square else np.ascontiguousarray(b, dtype=np.uint32)
        c = np.zeros(CL, dtype=np.uint32)
        r = fn(_ptr(c), CL, _ptr(a), a.size, _ptr(b), b.size)
        return c, r

    def fft_mul(self, a, b, CL=None, square=False):
        CL = CL or (len(a) + (len(a) if square else len(b)))
        return self._mul(self.lib.bco_fft_mul, a, b, CL, square)[0]

    def fft_mul_width(self, a, b, width, CL=None, square=False):
        a = np.ascontiguousarray(a, dtype=np.uint32)
        b = a if square else np.ascontiguousarray(b, dtype=np.uint32)
        CL = CL or (a.size + b.size)
        c = np.zeros(CL, dtype=np.uint32)
        err = self.lib.bco_fft_mul_width(_ptr(c), CL, _ptr(a), a.size, _ptr(b), b.size, width)
        return c, err

    def basecase_mul(self, a, b, CL=None):
        CL = CL or (len(a) + len(b))
        return self._mul(self.lib.bco_basecase_mul, a, b, CL, False)[0]

    def ntt_mul(self, a, b, CL=None, square=False):
        CL = CL or (len(a) + (len(a) if square else len(b)))
        c, r = self._mul(self.lib.bco_ntt_mul, a, b, CL, square)
        if r != 0:
            raise ValueError("operands too large for the NTT oracle")
        return c

    def checksum(self, a, p=0x9F063B05):
        a = np.ascontiguousarray(a, dtype=np.uint32)
        return self.lib.bco_checksum(_ptr(a), a.size, p)

    def modcheck(self, c, a, b, nprimes=4):
        a = np.ascontiguousarray(a, dtype=np.uint32)
        b = np.ascontiguousarray(b, dtype=np.uint32)
        c = np.ascontiguousarray(c, dtype=np.uint32)
        return bool(self.lib.bco_modcheck(_ptr(c), c.size, _ptr(a), a.size, _ptr(b), b.size, nprimes))

    def int_to_fft(self, words, length, b, alloc=None):
        words = np.ascontiguousarray(words, dtype=np.uint32)
        out = np.zeros(alloc or max(length, 1), dtype=np.complex128)
        n = self.lib.bco_int_to_fft(out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), length,
                                    _ptr(words), words.size, b)
        return out, n

    def fft_to_int(self, points, length, nwords, b):
        points = np.ascontiguousarray(points, dtype=np.complex128)
        out = np.zeros(nwords, dtype=np.uint32)
        self.lib.bco_fft_to_int(points.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), length,
                                _ptr(out), nwords, b)
        return out

    def fft_forward(self, x):
        x = np.array(x, dtype=np.complex128)
        self.lib.bco_fft_forward(x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), x.size)
        return x

    def fft_inverse(self, x):
        x = np.array(x, dtype=np.complex128)
        self.lib.bco_fft_inverse(x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), x.size)
        return x


class _Reference:
    """The reference's own multiply (bigfloat/mul.c:108-174) via oracle/_ref."""

    def __init__(self, path):
        self.lib = lib = ctypes.CDLL(path)
        lib._fft_mul.restype = ctypes.c_int
        lib._fft_mul.argtypes = [_u32p, _sz, _u32p, _sz, _u32p, _sz]
        lib.bcref_fft_mul_par.restype = ctypes.c_int
        lib.bcref_fft_mul_par.argtypes = [_u32p, _sz, _u32p, _sz, _u32p, _sz]
        lib.fft_ensure_table.restype = None
        lib.fft_ensure_table.argtypes = [_sz]
        lib.bcref_threads.restype = ctypes.c_int
        self.table_len = 0

    def ensure_table(self, length):
        # fft/table.c:211-228; tables are global and cumulative.
        if length > self.table_len:
            self.lib.fft_ensure_table(length)
            self.table_len = length

    def threads(self):
        return self.lib.bcref_threads()

    def fft_mul(self, a, b, CL=None, square=False, parallel=False):
        a = np.ascontiguousarray(a, dtype=np.uint32)
        b = a if square else np.ascontiguousarray(b, dtype=np.uint32)
        CL = CL or (a.size + b.size)
        width = restated().width(CL)
        if width < 7:
            raise ValueError("reference multiply aborts for CL > 4e6 (needs %d-bit packers)" % width)
        length = restated().fft_length(int(32.0 / width * CL))
        self.ensure_table(length)
        c = np.zeros(CL, dtype=np.uint32)
        fn = self.lib.bcref_fft_mul_par if parallel else self.lib._fft_mul
        fn(_ptr(c), CL, _ptr(a), a.size, _ptr(b), b.size)
        return c


_cache = {}


def restated_path():
    return os.path.join(HERE, "_build", "libbcoracle.so")


def reference_path(kind="serial"):
    return os.path.join(HERE, "_ref", kind, "libbcref.so")


def reference_cli(kind="serial"):
    return os.path.join(HERE, "_ref", kind, "bluecrunch_ref")


def restated():
    if "restated" not in _cache:
        _cache["restated"] = _Restated(restated_path())
    return _cache["restated"]


def have_reference(kind="serial"):
    return os.path.exists(reference_path(kind))


def reference(kind="serial"):
    key = "ref-" + kind
    if key not in _cache:
        _cache[key] = _Reference(reference_path(kind))
    return _cache[key]


def convert_trunc(y, n, k, alpha):
    """k base-10^9 digits of the fraction y (uint32 limbs below the point) by
    the reference's convert_trunc rounds (bigfloat/radix.c:41-91): multiply
    the window by 10^9 (its top limb cleared first, the carry out dropped),
    take limb n - floor(alpha*(i-1)) of the window, then slide the window up
    by floor(alpha*i) - floor(alpha*(i-1)) limbs.  Pure Python: small cases."""
    import math
    t = [int(v) for v in y] + [0]
    base, tl = 0, len(t)
    s = [0] * k
    for i in range(1, k + 1):
        t[base + tl - 1] = 0
        c = 0
        for j in range(base, base + tl):
            v = t[j] * 1000000000 + c
            t[j] = v & 0xFFFFFFFF
            c = v >> 32
        ni_1 = int(float(n) - math.floor(alpha * float(i - 1)))
        ni = int(float(n) - math.floor(alpha * float(i)))
        s[k - i] = t[base + ni_1]
        base += ni_1 - ni
        tl = ni + 1
        t[base + tl - 1] = 0
    return np.array(s, dtype=np.uint32)


def splitmix64(seed, n):
    """SplitMix64 stream as uint64 (the synthetic-operand generator)."""
    out = np.empty(n, dtype=np.uint64)
    x = np.uint64(seed)
    with np.errstate(over="ignore"):
        idx = np.arange(1, n + 1, dtype=np.uint64)
        z = x + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        out[:] = z ^ (z >> np.uint64(31))
    return out


def random_limbs(seed, n):
    """n uint32 limbs from SplitMix64, top limb forced nonzero."""
    v = splitmix64(seed, (n + 1) // 2).view(np.uint32)[:n].copy()
    if n:
        v[-1] |= 1
    return v
