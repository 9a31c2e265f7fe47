"""CPU: bench.py's pieces that need no GPU — the byte formula's width (the
engine's length choice restated in Python, so the reference arm never loads
the engine) and the reference arm's isolation from this repository's native
libraries."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _sizes():
    out = []
    for n in [1, 7, 50, 100, 999, 4096, 5000, 65536, 10**5, 2**20, 3 * 2**20 + 5, 2**22, 2**24, 2**26, 2**27]:
        out += [(n, n), (n, max(1, n // 8)), (n, max(1, n // 2)), (n, 1)]
    return out


@pytest.mark.parametrize("al,bl", _sizes())
def test_formula_plan_matches_engine_plan(al, bl):
    import bench
    import bluecrunch_b200 as bc
    p = bc.plan(al, bl)
    M, b = bench.formula_plan(al, bl)
    assert M == p["fft_points"], (al, bl)
    assert b == bc.width_limit(M)


def test_formula_lengths_match_engine_lengths():
    import bench
    import bluecrunch_b200 as bc
    assert bench._lengths() == bc.lengths()


_PROBE = r"""
import sys, types, json, io, contextlib
sys.path.insert(0, {root!r})
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"]
import bench
buf = io.StringIO()
with contextlib.redirect_stdout(buf):
    bench.main()
maps = open("/proc/self/maps").read()
line = [l for l in buf.getvalue().splitlines() if l.startswith("{{")][0]
print(json.dumps({{"line": json.loads(line), "bcgpu": "libbcgpu.so" in maps,
                   "bluecrunch": "libbluecrunch.so" in maps, "engine_imported": "bluecrunch_b200" in sys.modules}}))
"""


def test_reference_arm_loads_no_engine_library():
    p = subprocess.run([sys.executable, "-c", _PROBE.format(root=ROOT)], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    res = json.loads(p.stdout.strip().splitlines()[-1])
    assert not res["bcgpu"] and not res["bluecrunch"] and not res["engine_imported"], res
    ln = res["line"]
    if "unavailable" not in ln:
        assert ln["config"]["width_for_formula"] == 18 and ln["config"]["AL"] == 2**20
