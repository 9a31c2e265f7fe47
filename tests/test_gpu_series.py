"""GPU: binary splitting of e's series in device memory (bc_gpu_e_series)
against exact Python integers: P/Q = sum_{j=a+1}^{b} 1/((a+1)..j), Q =
(a+1)..b, the values of the reference's e_BSR (main.c:63-109)."""
import ctypes

import numpy as np
import pytest

import bluecrunch_b200 as bc

pytestmark = pytest.mark.gpu


def _exact(a, b):
    P, Q = 1, a + 1
    for k in range(a + 2, b + 1):
        P = P * k + 1
        Q = Q * k
    return P, Q


def _series(a, b):
    lib = bc._lib()
    fn = lib.bc_gpu_e_series
    p, q = ctypes.POINTER(ctypes.c_uint32)(), ctypes.POINTER(ctypes.c_uint32)()
    pl, ql = ctypes.c_size_t(), ctypes.c_size_t()
    r = fn(a, b, ctypes.byref(p), ctypes.byref(pl), ctypes.byref(q), ctypes.byref(ql))
    assert r == 0, bc_err(r)
    P = np.ctypeslib.as_array(p, (pl.value,)).copy()
    Q = np.ctypeslib.as_array(q, (ql.value,)).copy()
    libc = ctypes.CDLL(None)
    libc.free(p)
    libc.free(q)
    return P, Q


def bc_err(r):
    return bc._lib().bc_gpu_strerror(r)


@pytest.mark.parametrize("a,b", [(0, 1), (0, 2), (0, 63), (0, 64), (0, 65), (5, 77), (0, 1000), (1000, 1129),
                                 (0, 1023), (0, 1024), (0, 1025), (0, 3073), (0, 20000), (123456, 160000),
                                 (0, 300000), (2**31 - 5000, 2**31), (4000000000, 4000003000)])
def test_series_exact(gpu, a, b):
    P, Q = _series(a, b)
    wp, wq = _exact(a, b)
    assert P[-1] != 0 and Q[-1] != 0  # no top zero limbs
    assert bc.to_int(P) == wp and bc.to_int(Q) == wq
