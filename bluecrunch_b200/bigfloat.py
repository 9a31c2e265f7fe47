"""ctypes binding of the bigfloat C API (include/bigfloat.h).

The prototypes are the reference's (include/bigfloat.h:17-45 of bluecrunch),
so ``bind(path)`` works for ``libbluecrunch.so`` (this package, products on
the GPU) and for any other library exporting the same functions.  Values
cross the boundary as little-endian uint32 limb arrays plus a limb exponent:
value = +-sum coef[i] * 2^(32*(i+exp)).
"""
import ctypes

import numpy as np

from . import HOST_LIB


class BF(ctypes.Structure):
    """_bigfloat_struct (include/bigfloat.h:6-13)."""
    _fields_ = [("coef", ctypes.POINTER(ctypes.c_uint32)), ("exp", ctypes.c_int64),
                ("len", ctypes.c_size_t), ("sign", ctypes.c_int)]


_P = ctypes.POINTER(BF)
_SZ = ctypes.c_size_t
_SIGS = {
    "bigfloat_new": (None, [_P]),
    "bigfloat_free": (None, [_P]),
    "bigfloat_zero": (None, [_P]),
    "bigfloat_alloc": (None, [_P, _SZ]),
    "bigfloat_copy": (None, [_P, _P]),
    "bigfloat_set": (None, [_P, ctypes.c_uint32]),
    "bigfloat_add": (None, [_P, _P, _P, _SZ]),
    "bigfloat_sub": (None, [_P, _P, _P, _SZ]),
    "bigfloat_mul": (None, [_P, _P, _P, _SZ]),
    "bigfloat_div": (None, [_P, _P, _P, _SZ]),
    "bigfloat_rcp": (None, [_P, _P, _SZ]),
    "bigfloat_exp": (None, [_P, _P, ctypes.c_uint64]),
    "bigfloat_radix": (None, [_P, _P]),
    "bigfloat_to_string": (_SZ, [ctypes.c_char_p, _P, _SZ, ctypes.c_int]),
}


class Lib:
    """The bigfloat functions of one shared library, with argtypes set."""

    def __init__(self, path=HOST_LIB):
        self.path = path
        self.dll = ctypes.CDLL(path)
        for name, (res, args) in _SIGS.items():
            fn = getattr(self.dll, name)
            fn.restype = res
            fn.argtypes = args
            setattr(self, name[len("bigfloat_"):], fn)
        libc = ctypes.CDLL(None)
        libc.malloc.restype = ctypes.c_void_p
        libc.malloc.argtypes = [ctypes.c_size_t]
        self._malloc = libc.malloc

    def make(self, limbs=None, exp=0, sign=1):
        """A new bigfloat owning a malloc'd copy of ``limbs`` (freed by
        bigfloat_free, like every coefficient array of the C library)."""
        x = BF()
        self.new(x)
        if limbs is not None and len(limbs):
            a = np.ascontiguousarray(limbs, dtype=np.uint32)
            mem = self._malloc(a.nbytes)
            if not mem:
                raise MemoryError("malloc(%d)" % a.nbytes)
            ctypes.memmove(mem, a.ctypes.data, a.nbytes)
            self.free(x)
            x.coef = ctypes.cast(mem, ctypes.POINTER(ctypes.c_uint32))
            x.len, x.exp, x.sign = a.size, exp, sign
        return x

    def string(self, x, digits, base=10):
        """bigfloat_to_string (bigfloat/string.c:62-125) into a bytes object."""
        buf = ctypes.create_string_buffer(digits + 32)
        n = self.to_string(buf, x, digits, base)
        return buf.raw[:n]


def limbs(x):
    """Copy of the coefficient array of a BF."""
    if not x.len:
        return np.zeros(0, dtype=np.uint32)
    return np.ctypeslib.as_array(x.coef, (x.len,)).copy()


def value(x):
    """(sign, exp, integer of the limbs)."""
    return x.sign, x.exp, int.from_bytes(limbs(x).astype("<u4").tobytes(), "little")
