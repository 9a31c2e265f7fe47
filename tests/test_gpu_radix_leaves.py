"""GPU: leaves of the binary-to-decimal conversion (bc_gpu_radix_leaves)
against the reference's convert_trunc rounds restated in the oracle
(bigfloat/radix.c:41-91), digit for digit."""
import ctypes
import math

import numpy as np
import pytest

import oracle
import bluecrunch_b200 as bc

pytestmark = pytest.mark.gpu
ALPHA = math.log(1e9) / math.log(4294967296.0)


class Leaf(ctypes.Structure):
    _fields_ = [("y", ctypes.c_void_p), ("len", ctypes.c_size_t), ("n", ctypes.c_size_t), ("k", ctypes.c_size_t),
                ("s", ctypes.c_void_p)]


def _gpu_leaves(cases):
    arr = (Leaf * len(cases))()
    outs = []
    for i, (y, n, k) in enumerate(cases):
        s = np.zeros(k, dtype=np.uint32)
        outs.append(s)
        arr[i] = Leaf(y.ctypes.data, y.size, n, k, s.ctypes.data)
    r = bc._lib().bc_gpu_radix_leaves(ctypes.cast(arr, ctypes.c_void_p), len(cases), ALPHA)
    assert r == 0, r
    return outs


def test_leaves_match_restated_rounds(gpu):
    rng = np.random.default_rng(3)
    cases = []
    for i in range(60):
        k = int(rng.integers(1, 200))
        n = int(math.floor((k * math.log(1e9) + math.log(4.0) + math.log(1000.0)) / math.log(4294967296.0) + 1))
        ln = n + int(rng.integers(0, 2))  # y has n limbs, or n + 1 with an integer limb on top
        y = oracle.random_limbs(900 + i, ln)
        cases.append((y, n, k))
    # edge fractions: all ones, all zeros below the top, single limb
    cases.append((np.full(40, 0xFFFFFFFF, dtype=np.uint32), 40, 42))
    cases.append((np.zeros(30, dtype=np.uint32), 30, 20))
    cases.append((np.array([0x80000000], dtype=np.uint32), 1, 1))
    outs = _gpu_leaves(cases)
    for (y, n, k), got in zip(cases, outs):
        want = oracle.convert_trunc(y, n, k, ALPHA)
        assert np.array_equal(got, want), (len(y), n, k)


def test_leaves_full_size(gpu):
    # leaves of the conversion's own size (1000 digits, 936 limbs), many at once
    k = 1000
    n = int(math.floor((k * math.log(1e9) + math.log(4.0) + math.log(1000.0)) / math.log(4294967296.0) + 1))
    cases = [(oracle.random_limbs(70 + i, n), n, k) for i in range(300)]
    outs = _gpu_leaves(cases)
    for (y, n, k), got in list(zip(cases, outs))[:3]:
        assert np.array_equal(got, oracle.convert_trunc(y, n, k, ALPHA))
    assert all(int(o.max()) < 10**9 for o in outs)
