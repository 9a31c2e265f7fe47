"""CPU: the host C library (include/bigfloat.h) on sizes whose products all
stay below 100 limbs, where bigfloat_mul never calls the GPU (the reference's
own host range, bigfloat/mul.c:640-648)."""
import ctypes
import hashlib
import os
import subprocess
import tempfile

import numpy as np
import pytest

import bluecrunch_b200 as bc
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run_e(digits, tmp, per_call=False):
    # host tree and the reference's recursive conversion: at these sizes every
    # product and the conversion's single leaf stay on the host
    cmd = [bc.CLI, str(digits)] + (["--per-call"] if per_call else ["--levels"])
    env = dict(os.environ, BC_RADIX_PERCALL="1")
    subprocess.run(cmd, cwd=tmp, check=True, stdout=subprocess.DEVNULL, timeout=120, env=env)
    return open(os.path.join(tmp, "e.txt"), "rb").read(), open(os.path.join(tmp, "e-hex.txt"), "rb").read()


@pytest.mark.parametrize("digits", [10, 50, 100, 200, 250, 400])
def test_e_small_matches_true_digits(digits):
    import mpmath
    mpmath.mp.dps = digits + 30
    want = mpmath.nstr(mpmath.e, digits + 10, strip_zeros=False)
    with tempfile.TemporaryDirectory() as d:
        dec, hexs = _run_e(digits, d)
        dec2, hex2 = _run_e(digits, d, per_call=True)
    assert want.startswith(dec.decode())
    if digits >= 50:  # below that the output stops at a whole limb, as the reference's does
        assert len(dec) == digits + 2
    assert (dec, hexs) == (dec2, hex2)


@pytest.mark.parametrize("digits", [50, 100, 200, 400])
def test_e_small_matches_reference_build(digits):
    if not os.path.exists(oracle.reference_cli("serial")):
        pytest.skip("reference build not present")
    with tempfile.TemporaryDirectory() as d:
        mine = _run_e(digits, d)
        subprocess.run([oracle.reference_cli("serial"), str(digits)], cwd=d, check=True,
                       stdout=subprocess.DEVNULL)
        ref = (open(os.path.join(d, "e.txt"), "rb").read(), open(os.path.join(d, "e-hex.txt"), "rb").read())
    assert mine == ref


class BF(ctypes.Structure):
    _fields_ = [("coef", ctypes.POINTER(ctypes.c_uint32)), ("exp", ctypes.c_int64),
                ("len", ctypes.c_size_t), ("sign", ctypes.c_int)]


def _host():
    lib = ctypes.CDLL(bc.HOST_LIB)
    P = ctypes.POINTER(BF)
    for n in ("bigfloat_new", "bigfloat_free", "bigfloat_zero"):
        getattr(lib, n).argtypes = [P]
    lib.bigfloat_set.argtypes = [P, ctypes.c_uint32]
    lib.bigfloat_exp.argtypes = [P, P, ctypes.c_uint64]
    lib.bigfloat_mul.argtypes = [P, P, P, ctypes.c_size_t]
    lib.bigfloat_add.argtypes = [P, P, P, ctypes.c_size_t]
    lib.bigfloat_sub.argtypes = [P, P, P, ctypes.c_size_t]
    lib.bigfloat_radix.argtypes = [P, P]
    return lib


def _val(x):
    return int.from_bytes(np.ctypeslib.as_array(x.coef, (x.len,)).astype("<u4").tobytes(), "little") if x.len else 0


def test_power_known_answer():
    # test/test_bigfloat_exp.c: 0x1234^0xd7 has 82 limbs (all products < 100 limbs)
    lib = _host()
    a, b = BF(), BF()
    lib.bigfloat_new(a); lib.bigfloat_new(b)
    lib.bigfloat_set(a, 0x1234)
    lib.bigfloat_exp(b, a, 0xD7)
    assert b.len == 82 and b.exp == 0 and b.sign == 1
    assert _val(b) == 0x1234 ** 0xD7


def test_in_place_square_regression():
    # test/test_regression.c:40-67: bigfloat_mul(a, a, a, 0) in place
    lib = _host()
    a = BF()
    lib.bigfloat_new(a)
    arr = (ctypes.c_uint32 * 4)(0x44210000, 0xb1514c28, 0xce88deb8, 0x2)
    lib.bigfloat_set(a, 1)
    libc = ctypes.CDLL(None)
    libc.malloc.restype = ctypes.c_void_p
    mem = libc.malloc(16)
    ctypes.memmove(mem, arr, 16)
    a.coef = ctypes.cast(mem, ctypes.POINTER(ctypes.c_uint32))
    a.len, a.exp, a.sign = 4, 0, 1
    lib.bigfloat_mul(a, a, a, 0)
    got = list(np.ctypeslib.as_array(a.coef, (a.len,)))
    assert got == [0x0, 0xf4718c41, 0x21c8adaa, 0x28b6543c, 0x68a5465b, 0xe0c40a81, 0x7]


def test_add_sub_truncation_semantics():
    # precision p keeps p+2 limbs (bigfloat/addsub.c:83-86): exponent top-(p+2)
    lib = _host()
    x, y, t = BF(), BF(), BF()
    for z in (x, y, t):
        lib.bigfloat_new(z)
    lib.bigfloat_set(x, 7)
    lib.bigfloat_set(y, 5)
    y.exp = -10
    lib.bigfloat_add(t, x, y, 3)
    assert t.len == 5 and t.exp == 1 - 5 and _val(t) == 7 << (32 * 4)
    lib.bigfloat_sub(t, x, y, 0)
    assert t.exp == -10 and t.len == 11 and t.sign == 1


@pytest.mark.parametrize("kind", ["random", "carry_runs"])
def test_long_add_sub_parallel_chunks(kind):
    # bigfloat_add / bigfloat_sub above 2^20 limbs run in parallel chunks; the
    # carry and borrow chains across chunk boundaries must match the serial loop
    from bluecrunch_b200.bigfloat import Lib, value
    import oracle
    lib = Lib()
    n = 1_500_000
    a = oracle.random_limbs(77, n)
    b = oracle.random_limbs(78, n - 5)
    if kind == "carry_runs":
        a[: n - 10] = 0xFFFFFFFF  # a carry from the bottom crosses every chunk
        b[:] = 0
        b[0] = 1
    x, y = lib.make(a, exp=-3), lib.make(b, exp=-3)
    t = lib.make()
    lib.add(t, x, y, 0)
    ia, ib = value(x)[2], value(y)[2]
    s, e, v = value(t)
    assert s == 1 and e == -3 and v == ia + ib
    lib.sub(t, x, y, 0)
    s, e, v = value(t)
    assert s == 1 and e == -3 and v == ia - ib
    # borrow through a long run of zeros
    z = np.zeros(n, dtype=np.uint32)
    z[-1] = 5
    zz = lib.make(z, exp=-3)
    one = lib.make(np.array([1], dtype=np.uint32), exp=-3)
    lib.sub(t, zz, one, 0)
    assert value(t)[2] == value(zz)[2] - 1
    for q in (x, y, t, zz, one):
        lib.free(q)


@pytest.mark.parametrize("seed", range(6))
def test_add_sub_windows_random(seed):
    # random operand placements (overlapping, nested, disjoint with a gap),
    # lengths on both sides of the 2^20-limb parallel threshold and
    # precisions that cut into either operand, against Python integers: the
    # limbs are the exact sum / difference of the operands' limbs at or
    # above bot = top - (p + 2) (all limbs when p = 0)
    # (bigfloat/addsub.c:65-181)
    from bluecrunch_b200.bigfloat import Lib, value
    import oracle
    lib = Lib()
    rng = np.random.default_rng(1000 + seed)
    big = seed >= 4
    for case in range(4 if big else 40):
        la = int(rng.integers(1, 3_000_000 if big else 300))
        lb = int(rng.integers(1, 3_000_000 if big else 300))
        ea = int(rng.integers(-2 * la, la))
        eb = ea + int(rng.integers(-la - lb - 50, la + lb + 50))
        a = oracle.random_limbs(seed * 1000 + 2 * case, la)
        b = oracle.random_limbs(seed * 1000 + 2 * case + 1, lb)
        a[-1] |= 1
        b[-1] |= 1
        if case % 3 == 0:
            a[: la // 2] = 0xFFFFFFFF  # long carry and borrow runs
        x, y, t = lib.make(a, exp=ea), lib.make(b, exp=eb), lib.make()
        top = max(ea + la, eb + lb)
        bot_full = min(ea, eb)
        p = 0 if case % 2 == 0 else int(rng.integers(1, top - bot_full + 3))
        bot = bot_full if p == 0 or top - bot_full <= p + 2 else top - (p + 2)
        # the result's exponent is top - (p + 2) whenever p > 0, also when
        # nothing was cut (the reference sets it so, bigfloat/addsub.c:108,
        # and its limbs still start at bot)
        e_want = bot_full if p == 0 else top - (p + 2)

        def trunc(limbs, e):
            k = max(0, bot - e)
            if k >= len(limbs):
                return 0
            return int.from_bytes(limbs[k:].astype("<u4").tobytes(), "little") << (32 * (e + k - bot))

        ia, ib = trunc(a, ea), trunc(b, eb)
        lib.add(t, x, y, p)
        s, e, v = value(t)
        assert (s, e, v) == (1, e_want, ia + ib), (case, la, lb, ea, eb, p)
        lib.sub(t, x, y, p)
        s, e, v = value(t)
        full_a = int.from_bytes(a.astype("<u4").tobytes(), "little") << (32 * (ea - bot_full))
        full_b = int.from_bytes(b.astype("<u4").tobytes(), "little") << (32 * (eb - bot_full))
        if full_a == full_b:
            continue
        want = ia - ib if full_a > full_b else ib - ia
        if want:
            # sign field: 1 positive, 0 negative (include/bigfloat.h)
            assert (e, v) == (e_want, want) and s == (1 if full_a > full_b else 0), (case, la, lb, ea, eb, p)
        for q in (x, y, t):
            lib.free(q)


def _string_loop(limbs, exp, digits, base):
    """bigfloat/string.c:62-125 as its sequential loop: head, limbs from the
    top down to min_c until `digits` characters, then the truncation."""
    if len(limbs) == 0:
        return b"0", 1
    s = bytearray()
    mag = len(limbs) + exp
    c = len(limbs) - 1
    if mag == 1:
        assert limbs[c] == 2
        s += b"2"
    s += b"."
    per = 8 if base == 10 else 9
    min_c = len(limbs) - digits // per - 1 if len(limbs) > digits // per else 0
    while c > min_c:
        c -= 1
        s += (b"%09d" % limbs[c]) if base == 10 else (b"%08x" % limbs[c])
        if len(s) >= digits:
            break
    if len(s) + 1 > digits:
        return bytes(s[:digits - 1]), digits - 1
    return bytes(s), len(s)


def test_to_string_matches_the_sequential_loop():
    # the layout is computed up front so that limbs print in parallel; it
    # must reproduce the loop's stopping point and its final truncation for
    # every length, exponent and digit count, in both bases
    from bluecrunch_b200.bigfloat import Lib
    lib = Lib()
    rng = np.random.default_rng(5)
    for trial in range(400):
        n = int(rng.integers(1, 40))
        base = 10 if trial % 2 else 16
        lim = rng.integers(0, 10 ** 9 if base == 10 else 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
        exp = -(n - 1) if trial % 3 else -int(rng.integers(n, n + 3))  # integer part 2, or none
        if exp == -(n - 1):
            lim[-1] = 2
        digits = int(rng.integers(1, 9 * n + 30))
        x = lib.make(lim, exp=exp)
        got = lib.string(x, digits, base)
        want, wlen = _string_loop([int(v) for v in lim], exp, digits, base)
        lib.free(x)
        assert got == want[:wlen], (n, exp, digits, base)
