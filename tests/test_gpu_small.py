"""GPU: many small exact products in one launch (bc_gpu_mul_small_batch).

The reference computes products below 100 output limbs on the CPU with its
basecase / Karatsuba code (bigfloat/mul.c:176-553, dispatch mul.c:640-648).
Here a batch of them is one schoolbook kernel: checked against Python
integers for every operand length up to the 256-limb maximum, truncated and
zero-padded outputs, carry-heavy operands and zero operands; and
bigfloat_mul_batch, which now sends the small products of a large batch to
that kernel, is checked against bigfloat_mul item by item."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle
import bluecrunch_b200 as bc

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _exact(a, b, CL):
    x = bc.to_int(a) * bc.to_int(b)
    return bc.from_int(x % (1 << (32 * CL)), CL)


def test_small_batch_matches_exact_products(gpu):
    rng = np.random.default_rng(11)
    items = []
    for k in range(600):
        al = int(rng.integers(1, 257))
        bl = int(rng.integers(1, 257))
        a = oracle.random_limbs(2 * k + 1, al)
        b = oracle.random_limbs(2 * k + 2, bl)
        if k % 7 == 0:
            a[:] = 0xFFFFFFFF  # every column sum near its maximum, long carries
            b[:] = 0xFFFFFFFF
        mode = k % 3
        CL = al + bl if mode == 0 else (max(1, (al + bl) // 2) if mode == 1 else min(512, al + bl + 9))
        items.append((a, b, CL))
    items += [(np.full(256, 0xFFFFFFFF, np.uint32), np.full(256, 0xFFFFFFFF, np.uint32), 512),
              (np.array([7], np.uint32), np.array([9], np.uint32), 1),
              (np.array([0xFFFFFFFF], np.uint32), np.array([0xFFFFFFFF], np.uint32), 2)]
    outs = gpu.mul_small_batch(items)
    for (a, b, CL), c in zip(items, outs):
        assert np.array_equal(c, _exact(a, b, CL)), (a.size, b.size, CL)


def test_small_batch_zero_operand_and_limits(gpu):
    a = oracle.random_limbs(5, 40)
    outs = gpu.mul_small_batch([(a, np.zeros(0, np.uint32), 30), (a, a, None)])
    assert not outs[0].any()
    assert np.array_equal(outs[1], _exact(a, a, 80))
    with pytest.raises(bc.BcError):  # operand above 256 limbs
        gpu.mul_small_batch([(oracle.random_limbs(6, 257), a, None)])
    with pytest.raises(bc.BcError):  # product above 512 limbs
        gpu.mul_small_batch([(a, a, 513)])
    assert gpu.mul_small_batch([]) == []


_BATCH = r"""
import ctypes, hashlib, sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {golden!r})
import numpy as np
import oracle
from bluecrunch_b200.bigfloat import Lib, BF, limbs

class Item(ctypes.Structure):
    _fields_ = [("target", ctypes.POINTER(BF)), ("a", ctypes.POINTER(BF)), ("b", ctypes.POINTER(BF)),
                ("p", ctypes.c_size_t)]

lib = Lib()
lib.dll.bigfloat_mul_batch.argtypes = [ctypes.POINTER(Item), ctypes.c_size_t]
rng = np.random.default_rng(3)
xs, ys, ps = [], [], []
for k in range(1200):  # small products (below 100 output limbs) and a few large ones
    n = int(rng.integers(2, 48)) if k % 50 else int(rng.integers(200, 3000))
    m = int(rng.integers(2, 48)) if k % 50 else int(rng.integers(200, 3000))
    xs.append(lib.make(oracle.random_limbs(7 * k + 1, n), exp=-int(rng.integers(0, n)), sign=k % 2))
    ys.append(lib.make(oracle.random_limbs(7 * k + 2, m), exp=-int(rng.integers(0, m))))
    ps.append(int(rng.integers(1, n + m + 2)))
tb = [lib.make() for _ in xs]
items = (Item * len(xs))(*[Item(ctypes.pointer(t), ctypes.pointer(x), ctypes.pointer(y), p)
                           for t, x, y, p in zip(tb, xs, ys, ps)])
lib.dll.bigfloat_mul_batch(items, len(xs))
bad = 0
for t, x, y, p in zip(tb, xs, ys, ps):
    s = lib.make()
    lib.mul(s, x, y, p)
    same = (t.exp, t.len, t.sign) == (s.exp, s.len, s.sign) and np.array_equal(limbs(t), limbs(s))
    bad += not same
    lib.free(s)
print("BAD", bad)
"""


def test_mul_batch_small_products_match_single_products():
    # 1,176 small products (sent to the schoolbook kernel as one batch) and
    # 24 large ones; every result equals bigfloat_mul's (the small ones of
    # single calls stay on the host, as in the reference)
    code = _BATCH.format(root=ROOT, golden=os.path.join(ROOT, "tests", "golden"))
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip().splitlines()[-1] == "BAD 0", p.stdout[-2000:]
