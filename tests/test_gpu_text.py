"""GPU: decimal text of a conversion rendered on the device.

* bc_gpu_decimal_write against Python's formatting: nine zero-padded
  characters per base-10^9 limb, most significant first (the reference's
  printing loop, bigfloat/string.c:93-111), cut at any byte, at any file
  offset, from host or device limbs, across several staging chunks;
* bigfloat_radix_device + bc_dec_device_write against bigfloat_radix +
  bigfloat_to_string (the reference's pair, bigfloat/radix.c:321-360 and
  bigfloat/string.c:62-125): the same bytes for random fractions and for
  every kind of cut the string layout has.
The e CLI writes e.txt through this path; tests/test_gpu_e.py checks those
files against the published md5s."""
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


def _limbs_below_1e9(seed, n):
    x = oracle.random_limbs(seed, n).astype(np.uint64)
    return (x * 1000000000 >> 32).astype(np.uint32)  # uniform in [0, 10^9)


def _text(limbs, top, n, maxbytes):
    """Nine characters per limb of limbs[top], limbs[top-1], ... (numpy, vectorised)."""
    if n == 0 or maxbytes == 0:
        return b""
    v = limbs[top - n + 1:top + 1][::-1].astype(np.int64)
    digits = np.empty((n, 9), dtype=np.uint8)
    for d in range(8, -1, -1):
        digits[:, d] = (v % 10).astype(np.uint8) + ord("0")
        v //= 10
    return digits.tobytes()[:maxbytes]


def _write(tmp_path, limbs, top, n, maxbytes, offset, name):
    path = str(tmp_path / name)
    fd = os.open(path, os.O_WRONLY | os.O_CREAT | os.O_TRUNC, 0o644)
    try:
        bc.decimal_write(limbs, top, n, maxbytes, fd, offset)
    finally:
        os.close(fd)
    return open(path, "rb").read()


@pytest.mark.parametrize("n,top_extra,cut,offset", [
    (1, 0, 9, 0), (1, 5, 4, 2), (7, 3, 63, 0), (1023, 0, 10 ** 9, 1), (1024, 0, 9216, 2), (1025, 9, 9000, 0),
    (3000, 17, 26999, 3), (3000, 0, 1, 0), (100000, 11, 10 ** 7, 2)])
def test_decimal_text_matches_python(gpu, tmp_path, n, top_extra, cut, offset):
    limbs = _limbs_below_1e9(n + top_extra, n + top_extra)
    top = n - 1 + top_extra
    got = _write(tmp_path, limbs, top, n, cut, offset, "t.txt")
    want = _text(limbs, top, n, cut)
    assert got[:offset] == b"\0" * offset  # pwrite at the offset leaves a hole before it
    assert got[offset:] == want


def test_decimal_text_edge_values_and_nothing_to_write(gpu, tmp_path):
    limbs = np.array([0, 999999999, 1, 100000000, 10, 999999990], dtype=np.uint32)
    got = _write(tmp_path, limbs, 5, 6, 10 ** 6, 0, "e.txt")
    assert got == b"999999990000000010100000000000000001999999999000000000"
    assert _write(tmp_path, limbs, 5, 0, 100, 0, "z.txt") == b""
    assert _write(tmp_path, limbs, 5, 6, 0, 0, "c.txt") == b""
    with pytest.raises(bc.BcError):  # n limbs below top do not exist
        _write(tmp_path, limbs, 2, 4, 100, 0, "bad.txt")


def test_decimal_text_from_device_limbs_across_chunks(gpu, tmp_path):
    # 20,000,000 limbs = 180 MB of text: three 64 MiB staging chunks, the
    # last partial; the limbs are read from device memory
    torch = pytest.importorskip("torch")
    n = 20_000_000
    limbs = _limbs_below_1e9(77, n)
    dev = torch.from_numpy(limbs.view(np.int32)).cuda()
    cut = 9 * n - 5
    got = _write(tmp_path, dev, n - 1, n, cut, 2, "big.txt")
    assert len(got) == 2 + cut
    want = _text(limbs, n - 1, n, cut)
    step = 1 << 24
    for i in range(0, cut, step):
        assert got[2 + i:2 + i + step] == want[i:i + step], "first difference in bytes %d.." % i


_CONVERT = r"""
import ctypes, os, sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {golden!r})
import numpy as np
import oracle
from bluecrunch_b200.bigfloat import Lib, BF
lib = Lib()

class Dec(ctypes.Structure):
    _fields_ = [("dev", ctypes.c_void_p), ("len", ctypes.c_size_t), ("exp", ctypes.c_int64), ("top", ctypes.c_uint32)]

lib.dll.bigfloat_radix_device.restype = ctypes.c_int
lib.dll.bigfloat_radix_device.argtypes = [ctypes.POINTER(Dec), ctypes.POINTER(BF)]
lib.dll.bc_dec_device_write.restype = ctypes.c_int
lib.dll.bc_dec_device_write.argtypes = [ctypes.POINTER(Dec), ctypes.c_size_t, ctypes.c_int]
lib.dll.bc_dec_device_free.argtypes = [ctypes.POINTER(Dec)]
out = []
for seed, n, cuts in {cases!r}:
    xl = oracle.random_limbs(seed, n)
    xl[-1] = 2
    x = lib.make(xl, exp=-(n - 1))
    dec = lib.make()
    lib.radix(dec, x)
    d = Dec()
    assert lib.dll.bigfloat_radix_device(ctypes.byref(d), ctypes.byref(x)) == 0
    for digits in cuts:
        host = lib.string(dec, digits)
        path = os.path.join({tmp!r}, "d%d_%d.txt" % (seed, digits))
        fd = os.open(path, os.O_WRONLY | os.O_CREAT | os.O_TRUNC, 0o644)
        rc = lib.dll.bc_dec_device_write(ctypes.byref(d), digits, fd)
        os.close(fd)
        dev = open(path, "rb").read()
        out.append((seed, n, digits, rc, len(host), host == dev))
    lib.dll.bc_dec_device_free(ctypes.byref(d))
    lib.free(x)
    lib.free(dec)
print(repr(out))
"""


def test_device_conversion_prints_like_the_host_pair(tmp_path):
    # fractions of 300 ... 110,000 limbs with integer part 2 (the only one
    # the reference prints, bigfloat/string.c:40-61); digit counts that cut
    # inside the head, inside a limb, at a limb boundary, and beyond the
    # converted digits
    cases = []
    for seed, n in ((1, 300), (2, 4000), (3, 110_000)):
        full = int((n - 1) * 32 * 0.30102999566398120) - 20
        cases.append((seed, n, [1, 2, 3, 4, 12, 13, 20, full // 2, full - 1, full, full + 2, 10 * full]))
    code = _CONVERT.format(root=ROOT, golden=os.path.join(ROOT, "tests", "golden"), cases=cases, tmp=str(tmp_path))
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    res = eval(p.stdout.strip().splitlines()[-1])
    assert len(res) == sum(len(c[2]) for c in cases)
    for seed, n, digits, rc, hlen, same in res:
        assert rc == 0 and same, (seed, n, digits, rc, hlen)
