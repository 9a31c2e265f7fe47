"""Failure paths made on the host, never by faulting the GPU.

* BC_VERIFY=1 (every GPU product checked modulo two primes, the reference's
  DEBUG check of bigfloat/mul.c:650-658) aborts the program when a result is
  corrupted on the host after the GPU returned it (BC_FAULT_FLIP_PRODUCT);
* a device arena capped below what a product needs (bc_gpu_config.arena_bytes)
  gives BC_ERR_NOMEM and leaves the engine usable;
* lengths no transform can hold are refused with BC_ERR_TOO_LARGE before any
  memory is touched.

The GPU tests run their cases in child processes so the session's engine
keeps its own configuration.  The check function itself is exercised on the
CPU (no GPU needed)."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_product_check_detects_a_flipped_bit():
    import bluecrunch_b200 as bc
    import oracle
    lib = ctypes.CDLL(bc.HOST_LIB)
    f = lib.bc_host_product_check
    f.restype = ctypes.c_uint64
    u32p = ctypes.POINTER(ctypes.c_uint32)
    f.argtypes = [u32p, ctypes.c_size_t] * 3
    a, b = oracle.random_limbs(5, 3000), oracle.random_limbs(6, 2000)
    c = bc.from_int(bc.to_int(a) * bc.to_int(b), 5000)
    p = lambda x: x.ctypes.data_as(u32p)  # noqa: E731
    assert f(p(c), 5000, p(a), 3000, p(b), 2000) == 0
    for limb, bit in ((0, 0), (2500, 7), (4999, 31)):
        bad = c.copy()
        bad[limb] ^= np.uint32(1 << bit)
        assert f(p(bad), 5000, p(a), 3000, p(b), 2000) == 0x9F063B05
    assert f(p(c), 4000, p(a), 3000, p(b), 2000) == 0  # CL < AL + BL: not checkable, passes


_VERIFY = r"""
import sys
sys.path.insert(0, {root!r})
import oracle
from bluecrunch_b200.bigfloat import Lib, limbs
import bluecrunch_b200 as bc
lib = Lib()
a, b = oracle.random_limbs(1, 5000), oracle.random_limbs(2, 4000)
x, y, z = lib.make(a), lib.make(b), lib.make()
lib.mul(z, x, y, 0)
assert bc.to_int(limbs(z)) == bc.to_int(a) * bc.to_int(b)
print("PRODUCT OK")
"""


@pytest.mark.gpu
@pytest.mark.parametrize("flip", [False, True])
def test_verify_aborts_on_a_corrupted_product(flip):
    env = dict(os.environ, BC_VERIFY="1")
    env.pop("BC_FAULT_FLIP_PRODUCT", None)
    if flip:
        env["BC_FAULT_FLIP_PRODUCT"] = "1"
    p = subprocess.run([sys.executable, "-c", _VERIFY.format(root=ROOT)], env=env, capture_output=True, text=True,
                       timeout=300)
    if flip:
        assert p.returncode != 0 and "PRODUCT OK" not in p.stdout
        assert "fails the modular check" in p.stderr, p.stderr[-1000:]
    else:
        assert p.returncode == 0 and "PRODUCT OK" in p.stdout, p.stderr[-1000:]


_ARENA = r"""
import sys
sys.path.insert(0, {root!r})
import numpy as np
import oracle
import bluecrunch_b200 as bc
bc.init(0, arena_bytes=16 << 20)
a = oracle.random_limbs(3, 1 << 21)
try:
    bc.mul(a, a[: 1 << 20])
    print("NO ERROR")
except bc.BcError as e:
    print("CODE", e.code)
s = oracle.random_limbs(4, 1000)
c = bc.mul(s, s[:700])
assert np.array_equal(c, bc.from_int(bc.to_int(s) * bc.to_int(s[:700]), 1700))
print("SMALL OK")
"""


@pytest.mark.gpu
def test_capped_arena_gives_nomem_and_the_engine_stays_usable():
    p = subprocess.run([sys.executable, "-c", _ARENA.format(root=ROOT)], capture_output=True, text=True,
                       timeout=300)
    assert p.returncode == 0, p.stderr[-1500:]
    assert "CODE -2" in p.stdout and "SMALL OK" in p.stdout, p.stdout


@pytest.mark.gpu
def test_oversized_lengths_are_refused_before_any_access(gpu):
    lib = gpu._lib()
    buf = np.zeros(16, dtype=np.uint32)
    big = 1 << 31  # 2^31 limbs per operand: more digits than 2^31 complex points can hold
    rc = lib.bc_gpu_mul(buf.ctypes.data, 2 * big, buf.ctypes.data, big, buf.ctypes.data + 4, big, None)
    assert rc == -7  # BC_ERR_TOO_LARGE
    # the engine keeps working
    a = np.arange(1, 301, dtype=np.uint32)
    assert np.array_equal(gpu.mul(a, a[:200]), gpu.from_int(gpu.to_int(a) * gpu.to_int(a[:200]), 500))
