"""GPU: the drop-in check with the reference's own host code.

oracle/_ref/gpurelink/bluecrunch_gpu is the reference's CLI built from its
sources (main.c, bigfloat/*.c, util/, OpenMP tasks for its Cilk spawns) with
one change: _fft_mul (include/mul.h:3) comes from
bluecrunch_b200/shim/gpu_fft_mul.c, which calls bc_gpu_mul in libbcgpu.so
(oracle/Makefile, target gpu-relink).  Its e.txt must match the published
md5 (md5sums.txt of the reference) at 10^6 digits, and at 10^8 digits, a
size the reference's CPU _fft_mul cannot reach (bigfloat/mul.c:117-118,
fft/convert.c:66-68 abort above CL = 4e6 limbs)."""
import hashlib
import json
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "gpurelink", "bluecrunch_gpu")
PUB = json.load(open(os.path.join(ROOT, "tests", "golden", "e_md5.json")))["published"]["digits_to_md5"]

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("digits", [1_000_000, 100_000_000])
def test_reference_cli_on_gpu_multiply_matches_published_md5(digits):
    if not os.path.exists(BIN):
        pytest.skip("oracle/_ref/gpurelink was not built (reference sources absent at build time)")
    env = dict(os.environ, BC_TUNE_FILE=os.path.join(ROOT, "bluecrunch_b200", "tune", "widths.txt"))
    with tempfile.TemporaryDirectory() as d:
        p = subprocess.run([BIN, str(digits)], cwd=d, env=env, capture_output=True, text=True, timeout=1500)
        assert p.returncode == 0, (p.stdout[-1500:], p.stderr[-1500:])
        h = hashlib.md5()
        with open(os.path.join(d, "e.txt"), "rb") as f:
            for blk in iter(lambda: f.read(1 << 24), b""):
                h.update(blk)
    assert h.hexdigest() == PUB[str(digits)], p.stdout[-1500:]
