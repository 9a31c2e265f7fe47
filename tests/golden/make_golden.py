#!/usr/bin/env python3
"""Regenerate tests/golden/*.json from the reference (run in a container that
has the reference sources; the GPU box only reads the committed JSON).

Sources:
* known answers parsed (as text) from the reference's own unit tests:
  test/test_fft.c:22-39, test/test_int_to_fft.c:9-56 (tests fft_to_int),
  test/test_fft_to_int.c:20-90 (tests int_to_fft), test/test_regression.c:40-67,
  test/test_bigfloat_exp.c:5-118;
* md5sums.txt:1-8 (md5 of e.txt for 1e3..1e9 digits);
* products computed by the reference's own _fft_mul (bigfloat/mul.c:108-174)
  built by oracle/Makefile into oracle/_ref/serial/libbcref.so, on seeded
  SplitMix64 operands (oracle.random_limbs), stored as sha256 of the output;
* e.txt / e-hex.txt md5 from the reference CLI build for 1e3..1e5 digits.

Usage:  python tests/golden/make_golden.py [--ref DIR]

DIR is the reference source tree: $BC_REFERENCE_SRC, else a directory
named "reference" beside this repository.
"""
import argparse
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

import oracle  # noqa: E402

# (seed, AL, BL, CL, square) — CL >= 100 is the reference multiply's domain
# (bigfloat/mul.c:640-649 sends smaller products elsewhere).
PRODUCT_CASES = [
    (11, 50, 50, 100, False),
    (12, 64, 37, 101, False),
    (13, 100, 100, 200, False),
    (14, 333, 333, 666, True),
    (15, 1000, 1000, 2000, False),
    (16, 1000, 125, 1125, False),
    (17, 1024, 1024, 2048, True),
    (18, 2047, 2049, 4096, False),
    (19, 4500, 4500, 9000, False),
    (20, 4096, 4096, 8192, False),
    (21, 12000, 12000, 24000, False),
    (22, 16384, 2048, 18432, False),
    (23, 16384, 16384, 32768, False),
    (24, 16384, 16384, 32768, True),
    (25, 40000, 40000, 80000, False),
    (26, 65536, 65536, 131072, False),
    (27, 131072, 16384, 147456, False),
    (28, 140000, 140000, 280000, True),
    (29, 262144, 262144, 524288, False),
    (30, 100, 100, 300, False),      # CL > AL+BL: high words zero
    (31, 700, 300, 1000, False),
]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()


def parse_hex_asserts(text, var):
    pat = re.compile(r"assert\(%s\[(\d+)\]\s*==\s*(0x[0-9a-fA-F]+)\)" % re.escape(var))
    return {int(i): int(v, 16) for i, v in pat.findall(text)}


def known_answers(ref):
    kat = {}
    t = open(os.path.join(ref, "test", "test_fft.c")).read()
    kat["fft4"] = {
        "source": "test/test_fft.c:22-39",
        "input": [1, 2, 3, 4],
        # +i sign convention, digit-reversed output; inverse is unscaled
        "forward": [[10, 0], [-2, 0], [-2, -2], [-2, 2]],
        "inverse_of_forward": [[4, 0], [8, 0], [12, 0], [16, 0]],
    }
    assert "values[2], -2-2*I" in t and "values[3], -2+2*I" in t and "values[3], 16" in t

    t = open(os.path.join(ref, "test", "test_int_to_fft.c")).read()
    cases = []
    for blk in re.split(r"\n  //", t):
        m = re.search(r"complex double T\[16\] = \{([^}]*)\}", blk)
        if not m:
            continue
        pts = [int(x, 16) for x in m.group(1).split(",")]
        nw = int(re.search(r"uint32_t words\[(\d+)\]", blk).group(1))
        words = parse_hex_asserts(blk, "words")
        cases.append({"points_x16": pts, "length": 16, "bits": 12, "nwords": nw,
                      "words": [words[i] for i in range(nw)]})
    kat["fft_to_int"] = {"source": "test/test_int_to_fft.c:9-56", "cases": cases}

    t = open(os.path.join(ref, "test", "test_fft_to_int.c")).read()
    cases = []
    for blk in re.split(r"\n  //", t):
        m = re.search(r"uint32_t words\[\] = \{([^}]*)\}", blk)
        if not m:
            continue
        words = [int(x, 16) for x in m.group(1).split(",")]
        bits = int(re.search(r"int_to_fft\(T, \d+, words, \d+, (\d+)\)", blk).group(1))
        pts = {}
        for i, v in re.findall(r"assert_fp\(T\[(\d+)\], (0x[0-9a-fA-F]+)\)", blk):
            pts[int(i)] = int(v, 16)
        zero_from = int(re.search(r"for\(size_t i=(\d+);i<16", blk).group(1))
        cases.append({"words": words, "bits": bits,
                      "points": [pts[i] for i in range(len(pts))], "zero_from": zero_from,
                      "note": "entries at or beyond zero_from are only asserted by the reference "
                              "test (test_fft_to_int.c:92, beyond the length argument; a test bug)"})
    kat["int_to_fft"] = {"source": "test/test_fft_to_int.c:20-90", "cases": cases}

    t = open(os.path.join(ref, "test", "test_regression.c")).read()
    live = t.split("*/", 1)[1]
    inp = [int(v, 16) for v in re.findall(r"a->coef\[\d\] = (0x[0-9a-fA-F]+);", live)]
    out = parse_hex_asserts(live.split("bigfloat_mul")[1], "a->coef")
    kat["square4"] = {"source": "test/test_regression.c:40-67", "a": inp,
                      "result": [out[i] for i in range(len(out))]}

    t = open(os.path.join(ref, "test", "test_bigfloat_exp.c")).read()
    coef = parse_hex_asserts(t, "b->coef")
    ln = int(re.search(r"assert\(b->len\s*==\s*(\d+)\)", t).group(1))
    base = int(re.search(r"bigfloat_set\(a, (0x[0-9a-fA-F]+)\)", t).group(1), 16)
    ex = int(re.search(r"bigfloat_exp\(b, a, (0x[0-9a-fA-F]+)\)", t).group(1), 16)
    kat["pow"] = {"source": "test/test_bigfloat_exp.c:5-118", "base": base, "exp": ex, "len": ln,
                  "top_words": {str(k): v for k, v in sorted(coef.items())}}
    return kat


def md5sums(ref):
    out = {}
    for line in open(os.path.join(ref, "md5sums.txt")):
        if "=" not in line:
            continue
        n, h = line.split("=")
        nbytes = int(n.strip().replace(".", ""))
        out[str(nbytes - 2)] = h.strip()
    return {"source": "md5sums.txt:1-8", "digits_to_md5": out}


def product_vectors():
    F = oracle.reference("serial")
    R = oracle.restated()
    vec = []
    for seed, al, bl, cl, sq in PRODUCT_CASES:
        a = oracle.random_limbs(seed, al)
        b = a if sq else oracle.random_limbs(seed + 1000, bl)
        c = F.fft_mul(a, b, cl, square=sq)
        assert np.array_equal(c, R.ntt_mul(a, b, cl, square=sq)), (seed, al, bl)
        vec.append({"seed_a": seed, "seed_b": None if sq else seed + 1000, "AL": al, "BL": bl,
                    "CL": cl, "square": sq, "sha256": sha(c), "width_ref": R.width(cl),
                    "low_words": [int(x) for x in c[:4]], "high_words": [int(x) for x in c[-4:]]})
    return {"source": "bigfloat/mul.c:108-174 via oracle/_ref/serial/libbcref.so",
            "generator": "oracle.random_limbs(seed, n) (SplitMix64, top limb |= 1)",
            "cases": vec}


def e_cli_md5():
    out = {}
    cli = oracle.reference_cli("serial")
    with tempfile.TemporaryDirectory() as d:
        for n in (1000, 10000, 100000):
            subprocess.run([cli, str(n)], cwd=d, check=True, stdout=subprocess.DEVNULL)
            out[str(n)] = {
                "e.txt": hashlib.md5(open(os.path.join(d, "e.txt"), "rb").read()).hexdigest(),
                "e-hex.txt": hashlib.md5(open(os.path.join(d, "e-hex.txt"), "rb").read()).hexdigest(),
            }
    return {"source": "main.c:111-167 via oracle/_ref/serial/bluecrunch_ref", "digits": out}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("BC_REFERENCE_SRC") or os.path.join(ROOT, "..", "reference"))
    args = ap.parse_args()
    blobs = {
        "known_answers.json": known_answers(args.ref),
        "e_md5.json": {"published": md5sums(args.ref), "reference_cli": e_cli_md5()},
        "products.json": product_vectors(),
    }
    for name, obj in blobs.items():
        with open(os.path.join(HERE, name), "w") as fh:
            json.dump(obj, fh, indent=1, sort_keys=True)
            fh.write("\n")
        print("wrote", name)


if __name__ == "__main__":
    main()
