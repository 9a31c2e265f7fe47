"""CPU: the device carry arithmetic (run records, 192-bit signed add with
carry out, bit extraction), compiled for the host from the same headers and
checked against Python integers for every digit width 8..24."""
import os
import random
import shutil
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.fixture(scope="module")
def checker():
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    d = tempfile.mkdtemp()
    exe = os.path.join(d, "carry_check")
    subprocess.check_call([NVCC, "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a", "-I" + os.path.join(ROOT, "bluecrunch_b200", "csrc"),
                           "-o", exe, os.path.join(ROOT, "tests", "carry_host_check.cu")])
    yield exe
    shutil.rmtree(d)


def run(exe, lines):
    out = subprocess.run([exe], input="\n".join(lines) + "\n", capture_output=True, text=True, check=True).stdout
    return out.strip().split("\n")


def words(x):
    return [(x >> (64 * i)) & ((1 << 64) - 1) for i in range(3)]


def test_add_with_carry_all_widths(checker):
    rng = random.Random(5)
    cases, expect = [], []
    for b in range(8, 25):
        nbits = 8 * b
        for _ in range(300):
            kind = rng.random()
            if kind < 0.3:
                h = (1 << nbits) - 1 - rng.randrange(0, 1 << 20)   # near all-ones
            elif kind < 0.6:
                h = rng.randrange(0, 1 << 20)                      # near zero
            else:
                h = rng.randrange(0, 1 << nbits)
            v = rng.randrange(-(1 << 62), 1 << 62)
            if rng.random() < 0.3:
                v = rng.choice([-1, 0, 1])
            s = h + v
            carry, hp = s >> nbits, s % (1 << nbits)
            cases.append("A %d %x %x %x %d" % (nbits, *words(h), v))
            expect.append((carry, hp, hp == 0, hp == (1 << nbits) - 1))
    for line, (carry, hp, z, o) in zip(run(checker, cases), expect):
        c, h0, h1, h2, iz, io = line.split()
        got = int(h0, 16) | (int(h1, 16) << 64) | (int(h2, 16) << 128)
        assert (int(c), got, bool(int(iz)), bool(int(io))) == (carry, hp, z, o), line


def test_run_records_and_bit_extraction(checker):
    rng = random.Random(9)
    cases, expect = [], []
    for b in range(8, 25):
        for _ in range(100):
            cs = [rng.randrange(-(1 << 52), 1 << 52) for _ in range(8)]
            v = sum(c << (b * u) for u, c in enumerate(cs))
            cases.append("R %d %s" % (b, " ".join(map(str, cs))))
            expect.append((v % (1 << (8 * b)), v >> (8 * b)))
    for line, (h, c) in zip(run(checker, cases), expect):
        h0, h1, h2, cc = line.split()
        assert int(h0, 16) | (int(h1, 16) << 64) | (int(h2, 16) << 128) == h and int(cc) == c
    cases, expect = [], []
    for _ in range(500):
        x = rng.randrange(0, 1 << 192)
        off = rng.randrange(0, 200)
        cases.append("W %x %x %x %d" % (*words(x), off))
        expect.append((x >> off) & 0xFFFFFFFF)
    for line, e in zip(run(checker, cases), expect):
        assert int(line, 16) == e
