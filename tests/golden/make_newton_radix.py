#!/usr/bin/env python3
"""Regenerate tests/golden/newton_radix.json with the reference's own
Newton reciprocal, division and radix conversion.

The reference's bigfloat library (bigfloat/rcp.c:15-101, bigfloat/div.c:14-27,
bigfloat/radix.c:228-360, bigfloat/string.c:62-125, with its own _fft_mul,
bigfloat/mul.c:108-174), built by oracle/Makefile, runs on seeded random
operands of the shape
bigfloat_radix accepts (n limbs, exp = -(n-1): one integer limb, 2 for x):

    r = rcp(x, n);  q = div(y, x, n);  d = radix(x);  s = to_string(d, D, 10)

and the file stores (exp, len, sign, sha256 of the limbs) of r, q and d and
the sha256 of s.  Sizes stay below the reference multiply's reach
(CL <= 4e6 limbs, bigfloat/mul.c:117-118).

Two builds run every case: oracle/_ref/exactsmall (the reference with its
products below 100 limbs on its own exact schoolbook, oracle/ref_exact_small.c)
gives the stored values, since every product of this implementation is exact;
oracle/_ref/serial (as shipped, small products through the inexact
_karatzuba_mul, bigfloat/mul.c:367-553) is recorded beside them as
"shipped_agrees" per result.

Usage:  python tests/golden/make_newton_radix.py
"""
import ctypes
import hashlib
import json
import math
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from bluecrunch_b200.bigfloat import Lib, limbs  # noqa: E402

# (seed, n limbs)
CASES = [(101, 300), (102, 4_000), (103, 25_000), (104, 110_000), (105, 600_000)]


def operands(seed, n):
    """x, y: n random limbs, exponent -(n-1).  x's integer limb is 2 (x in
    [2, 3), the shape of e): the reference prints only that integer part
    (bigfloat/string.c:40-61 aborts on any other)."""
    x = oracle.random_limbs(seed, n)
    x[-1] = 2
    return x, oracle.random_limbs(seed ^ 0x5EED, n)


def decimal_digits(n):
    """Digits printed from the radix-converted x: what n-1 fractional limbs hold, less a margin."""
    return int((n - 1) * 32 * math.log10(2)) - 20


def record(x):
    c = limbs(x)
    return {"exp": int(x.exp), "len": int(x.len), "sign": int(x.sign),
            "sha256": hashlib.sha256(c.astype("<u4").tobytes()).hexdigest()}


def run_case(lib, seed, n):
    xl, yl = operands(seed, n)
    x = lib.make(xl, exp=-(n - 1))
    y = lib.make(yl, exp=-(n - 1))
    r, q, d = lib.make(), lib.make(), lib.make()
    t0 = time.perf_counter()
    lib.rcp(r, x, n)
    lib.div(q, y, x, n)
    lib.radix(d, x)
    s = lib.string(d, decimal_digits(n), 10)
    dt = time.perf_counter() - t0
    out = {"seed": seed, "n": n, "digits": decimal_digits(n), "rcp": record(r), "div": record(q),
           "radix": record(d), "string_sha256": hashlib.sha256(s).hexdigest(),
           "string_head": s[:24].decode()}
    for z in (x, y, r, q, d):
        lib.free(z)
    return out, dt


def run_in_child(kind, i):
    out = subprocess.run([sys.executable, os.path.abspath(__file__), "--case", kind, str(i)], check=True,
                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True).stdout
    return json.loads([ln for ln in out.splitlines() if ln.startswith("JSON ")][0][5:])


def main():
    if len(sys.argv) == 4 and sys.argv[1] == "--case":
        # One case per process: the reference keeps its radix table's exponent
        # list in a global that its free_radix_conversion does not clear
        # (bigfloat/radix.c:93-98,207-226), so a second conversion in the same
        # process starts from a stale list.
        lib = Lib(oracle.reference_path(sys.argv[2]))
        lib.dll.fft_ensure_table.argtypes = [ctypes.c_size_t]
        lib.dll.fft_ensure_table(1 << 23)  # main.c:190-200 sizes this from the digit count
        seed, n = CASES[int(sys.argv[3])]
        c, dt = run_case(lib, seed, n)
        c["seconds"] = round(dt, 3)
        print("JSON " + json.dumps(c))
        return
    for kind in ("exactsmall", "serial"):
        if not os.path.exists(oracle.reference_path(kind)):
            sys.exit("build the reference first: make -C oracle ref")
    cases = []
    for i in range(len(CASES)):
        c = run_in_child("exactsmall", i)
        shipped = run_in_child("serial", i)
        c["shipped_agrees"] = {k: c[k] == shipped[k] for k in ("rcp", "div", "radix", "string_sha256")}
        print("n=%d: %.2f s  %s  shipped agrees: %s" % (c["n"], c.pop("seconds"), c["string_head"],
                                                       c["shipped_agrees"]))
        cases.append(c)
    with open(os.path.join(HERE, "newton_radix.json"), "w") as f:
        json.dump({"source": "reference bigfloat_rcp/div/radix/to_string via oracle/_ref/exactsmall/libbcref.so",
                   "cases": cases}, f, indent=1)


if __name__ == "__main__":
    main()
