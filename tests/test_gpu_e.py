"""GPU: e to N digits through the host C library and the GPU multiply,
against the md5 of e.txt published with the reference (md5sums.txt:1-8)."""
import hashlib
import json
import os
import subprocess
import tempfile

import pytest

import bluecrunch_b200 as bc

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
MD5 = json.load(open(os.path.join(HERE, "golden", "e_md5.json")))["published"]["digits_to_md5"]


def _e(digits, per_call=False, env=None, levels=False):
    with tempfile.TemporaryDirectory() as d:
        cmd = [bc.CLI, str(digits)] + (["--per-call"] if per_call else []) + (["--levels"] if levels else [])
        e = dict(os.environ, **(env or {}))
        res = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=900, env=e)
        assert res.returncode == 0, "bluecrunch %s failed (%d): %s" % (digits, res.returncode, res.stderr[-2000:])
        out = res.stdout
        dec = open(os.path.join(d, "e.txt"), "rb").read()
        hexs = open(os.path.join(d, "e-hex.txt"), "rb").read()
    return hashlib.md5(dec).hexdigest(), hashlib.md5(hexs).hexdigest(), out


@pytest.mark.parametrize("digits", [1000, 10000, 100000, 1000000])
def test_e_batched_matches_published_md5(digits):
    md5, _, _ = _e(digits)  # the splitting tree in device memory
    assert md5 == MD5[str(digits)]
    if digits <= 100000:
        md5, _, _ = _e(digits, levels=True)  # host tree, batched levels
        assert md5 == MD5[str(digits)]
    if digits >= 100000:
        md5, _, _ = _e(digits, env={"BC_RADIX_LEVELS": "1"})  # conversion levels merged on the host
        assert md5 == MD5[str(digits)]


def test_e_per_call_1e6_matches_batched():
    # one GPU product per _fft_mul call, the reference's own recursion
    a = _e(1000000, per_call=True)
    b = _e(1000000, env={"BC_RADIX_PERCALL": "1"})
    assert a[0] == MD5["1000000"] and a[:2] == b[:2]


def test_e_hex_matches_reference_cli():
    ref = json.load(open(os.path.join(HERE, "golden", "e_md5.json")))["reference_cli"]["digits"]
    for digits, h in ref.items():
        dec, hexs, _ = _e(int(digits))
        assert dec == h["e.txt"] and hexs == h["e-hex.txt"]


def test_e_1e7_matches_published_md5():
    md5, _, _ = _e(10000000)
    assert md5 == MD5["10000000"]


def test_e_1e9_matches_published_md5():
    # e to 10^9 digits end to end (series, division and conversion in device
    # memory), against the md5 published with the reference
    md5, _, out = _e(1000000000)
    assert md5 == MD5["1000000000"], out[-2000:]
