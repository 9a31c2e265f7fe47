"""GPU: Newton reciprocal and division and radix conversion of random
bigfloats through the host library (products on the GPU), against the
reference's own results (tests/golden/newton_radix.json, generated by
tests/golden/make_newton_radix.py from the reference's bigfloat/rcp.c,
div.c, radix.c and string.c), plus a 50-million-digit case beyond the
reference's reach checked by modular verification of every product and by
x * rcp(x) = 1 - eps."""
import hashlib
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

from make_newton_radix import decimal_digits, operands, record  # noqa: E402

GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "newton_radix.json")))["cases"]

pytestmark = pytest.mark.gpu


def _lib():
    from bluecrunch_b200.bigfloat import Lib
    return Lib()


@pytest.mark.parametrize("case", GOLD, ids=lambda c: "n%d" % c["n"])
@pytest.mark.parametrize("driver", ["tree", "levels", "percall"])
def test_matches_reference(case, driver, monkeypatch):
    monkeypatch.delenv("BC_RADIX_PERCALL", raising=False)
    monkeypatch.delenv("BC_RADIX_LEVELS", raising=False)
    if driver == "percall":
        if case["n"] > 110_000:
            pytest.skip("per-call driver checked on the smaller cases")
        monkeypatch.setenv("BC_RADIX_PERCALL", "1")
    elif driver == "levels":
        monkeypatch.setenv("BC_RADIX_LEVELS", "1")
    lib = _lib()
    n = case["n"]
    xl, yl = operands(case["seed"], n)
    x = lib.make(xl, exp=-(n - 1))
    y = lib.make(yl, exp=-(n - 1))
    r, q, d = lib.make(), lib.make(), lib.make()
    lib.rcp(r, x, n)
    assert record(r) == case["rcp"]
    lib.div(q, y, x, n)
    assert record(q) == case["div"]
    lib.radix(d, x)
    assert record(d) == case["radix"]
    s = lib.string(d, decimal_digits(n), 10)
    assert s[:24].decode() == case["string_head"]
    assert hashlib.sha256(s).hexdigest() == case["string_sha256"]
    for z in (x, y, r, q, d):
        lib.free(z)


_BIG = r"""
import sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {golden!r})
from bluecrunch_b200.bigfloat import Lib, value
from make_newton_radix import operands, decimal_digits
n = {n}
lib = Lib()
xl, yl = operands(7, n)
x = lib.make(xl, exp=-(n - 1)); r = lib.make(); m = lib.make(); d = lib.make()
if {with_rcp}:
    lib.rcp(r, x, n)
    lib.mul(m, x, r, 0)
    s, e, v = value(m)
    one = 1 << (-32 * e)
    err = abs(v - one)
    assert s == 1 and err * (1 << (32 * (n - 2))) <= one, "x*rcp(x) too far from 1"
lib.radix(d, x)
out = lib.string(d, decimal_digits(n), 10)
# a truncated output is "2." and digits - 3 digits (bigfloat/string.c:117-121)
assert out.startswith(b"2.") and len(out) == decimal_digits(n) - 1 and out[2:].isdigit(), (len(out), out[:30])
open({path!r}, "wb").write(out)
print("OK", r.len, d.len)
"""

# The exact decimal expansion of x = X / 2^E (E = 32(n-1)) is the digit
# string of X * 5^E with the point after its first digit.  Computed with the
# decimal module (libmpdec, transform multiplication) from str(X), so it
# shares nothing with the library under test.
_EXACT = r"""
import sys, decimal
sys.set_int_max_str_digits(0)
sys.path.insert(0, {root!r}); sys.path.insert(0, {golden!r})
from make_newton_radix import operands, decimal_digits
n = {n}
xl, _ = operands(7, n)
X = int.from_bytes(xl.astype("<u4").tobytes(), "little")
E = 32 * (n - 1)
decimal.setcontext(decimal.Context(prec=decimal.MAX_PREC, Emax=decimal.MAX_EMAX, Emin=decimal.MIN_EMIN))
full = str(decimal.Decimal(str(X)) * decimal.Decimal(5) ** E)
assert len(full) == E + 1 and full[0] == "2"
keep = decimal_digits(n) - 3
open({path!r}, "wb").write(("2." + full[1:1 + keep]).encode())
print("OK", len(full))
"""


def _first_difference(a, b):
    if len(a) != len(b):
        return "lengths %d and %d" % (len(a), len(b))
    step = 1 << 20
    for i in range(0, len(a), step):
        if a[i:i + step] != b[i:i + step]:
            j = next(k for k in range(i, min(i + step, len(a))) if a[k] != b[k])
            return "first difference at %d of %d: %r vs %r" % (j, len(a), a[j:j + 20], b[j:j + 20])
    return None


def test_fifty_million_digits_verified(tmp_path):
    """C4: a random 50,000,000-digit bigfloat (5,190,471 limbs): reciprocal at
    full precision (|x*rcp(x) - 1| <= 2^(-32(n-2))) and conversion to decimal,
    every GPU product checked modulo primes (BC_VERIFY=1 aborts on a
    mismatch).  All 49,999,566 output digits are compared with (1) the exact
    expansion of x truncated to the same length and (2) the per-call radix
    driver (the reference's recursion, bigfloat/radix.c:228-318, with host
    leaves as bigfloat/radix.c:41-91 computes them).

    Truncation rule: bigfloat_to_string (bigfloat/string.c:62-125) prints
    "2." and D - 3 digits, D = decimal_digits(n) = floor((n-1) 32 log10 2) - 20;
    the 20 digits of margin absorb the truncations of the conversion tree, so
    the printed digits equal the exact expansion truncated to that length
    (the reference's own output satisfies this at every pinned size,
    300 to 600,000 limbs)."""
    n = 5_190_471
    golden = os.path.join(ROOT, "tests", "golden")
    exact_path, tree_path, percall_path = (str(tmp_path / f) for f in ("exact.txt", "tree.txt", "percall.txt"))
    exact = subprocess.Popen([sys.executable, "-c", _EXACT.format(root=ROOT, golden=golden, n=n, path=exact_path)],
                             stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
    try:
        for path, extra, with_rcp in ((tree_path, {}, True), (percall_path, {"BC_RADIX_PERCALL": "1"}, False)):
            code = _BIG.format(root=ROOT, golden=golden, n=n, path=path, with_rcp=with_rcp)
            env = dict(os.environ, BC_VERIFY="1", **extra)
            if not extra:
                env.pop("BC_RADIX_PERCALL", None)
            env.pop("BC_RADIX_LEVELS", None)
            p = subprocess.run([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                               text=True, timeout=1200)
            assert p.returncode == 0, p.stderr[-2000:]
            assert p.stdout.strip().splitlines()[-1].startswith("OK"), p.stdout[-2000:]
        out, err = exact.communicate(timeout=1500)
        assert exact.returncode == 0, err[-2000:]
    finally:
        if exact.poll() is None:
            exact.kill()
    want = open(exact_path, "rb").read()
    tree = open(tree_path, "rb").read()
    percall = open(percall_path, "rb").read()
    assert len(want) == decimal_digits(n) - 1  # "2." and 49,999,566 digits
    assert _first_difference(tree, want) is None, _first_difference(tree, want)
    assert _first_difference(percall, want) is None, _first_difference(percall, want)


_DEV_VS_HOST = r"""
import sys, hashlib, os
sys.path.insert(0, {root!r}); sys.path.insert(0, {golden!r})
from bluecrunch_b200.bigfloat import Lib, limbs
import oracle
lib = Lib()
out = []
for seed, n, p, e in {cases!r}:
    xl = oracle.random_limbs(seed, n); xl[-1] |= 1
    yl = oracle.random_limbs(seed ^ 0x77, n + 3)
    x = lib.make(xl, exp=e); y = lib.make(yl, exp=-(n + 3) // 2)
    r, q = lib.make(), lib.make()
    lib.rcp(r, x, p)
    lib.div(q, y, x, p)
    for z in (r, q):
        out.append((int(z.exp), int(z.len), int(z.sign), hashlib.sha256(limbs(z).astype("<u4").tobytes()).hexdigest()))
    for z in (x, y, r, q):
        lib.free(z)
print(repr(out))
"""


def test_device_newton_matches_host_newton():
    # the Newton levels of 2^16 limbs and more run in device memory
    # (bc_gpu_newton); BC_NEWTON_HOST=1 runs every level through the host
    # library: both must give the same limbs, exponent and sign, for
    # reciprocals and quotients of assorted sizes, precisions and exponents
    import subprocess
    cases = [(11, 70_000, 66_000, -69_999), (12, 300_000, 300_000, -5), (13, 150_000, 400_000, 3),
             (14, 1_000_000, 700_000, -1_000_000),
             (15, 5_190_471, 5_190_471, -(5_190_471 - 1))]  # the 50,000,000-digit precision
    code = _DEV_VS_HOST.format(root=ROOT, golden=os.path.join(ROOT, "tests", "golden"), cases=cases)
    res = []
    for host in (False, True):
        env = dict(os.environ)
        env.pop("BC_NEWTON_HOST", None)
        if host:
            env["BC_NEWTON_HOST"] = "1"
        p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900)
        assert p.returncode == 0, p.stderr[-2000:]
        res.append(p.stdout.strip().splitlines()[-1])
    assert res[0] == res[1]
