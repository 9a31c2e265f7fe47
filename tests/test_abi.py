"""CPU: the C-ABI libraries load and export every declared symbol; planning
and width logic (no GPU calls)."""
import ctypes
import os
import re

import pytest

import bluecrunch_b200 as bc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", text, re.M))


def test_gpu_library_exports_header():
    names = _declared("bc_gpu.h")
    assert "bc_gpu_mul" in names and "bc_gpu_mul_batch" in names
    lib = ctypes.CDLL(bc.GPU_LIB)
    for n in names:
        assert hasattr(lib, n), n
    assert set(bc.GPU_SYMBOLS) >= names


def test_host_library_exports_reference_prototypes():
    lib = ctypes.CDLL(bc.HOST_LIB)
    for header in ("bigfloat.h", "mul.h", "bench.h"):
        for n in _declared(header):
            assert hasattr(lib, n), (header, n)


def test_strerror_and_uninitialised_calls():
    lib = bc._lib()
    for code in range(0, -10, -1):
        assert lib.bc_gpu_strerror(code)
    # nothing initialised in this process: calls report, never abort
    assert lib.bc_gpu_sync() in (bc.BC_OK, -6)


@pytest.mark.parametrize("n", [1, 50, 100, 999, 4096, 10**5, 2**20, 3 * 2**20 + 5, 2**26])
def test_plans_fit_and_are_exact_sized(n):
    for (al, bl) in [(n, n), (n, max(1, n // 8)), (n, 1)]:
        p = bc.plan(al, bl)
        M, b = p["fft_points"], p["width"]
        assert 8 <= b <= 24
        assert p["digits_a"] == -(-32 * al // b) and p["digits_b"] == -(-32 * bl // b)
        # acyclic product must fit the 2M real coefficients
        assert p["digits_a"] + p["digits_b"] - 1 <= 2 * M
        assert b <= bc.width_limit(M)
        assert p["levels"] in (1, 2, 3)
        assert p["L1"] * p["L2"] * max(p["Lr"], 1) == M


def test_lengths_are_2k_3x2k_5x2k():
    L = bc.lengths()
    assert L == sorted(L) and L[0] == 256 and L[-1] == 1 << 30
    for M in L:
        m = M // 3 if M % 3 == 0 else (M // 5 if M % 5 == 0 else M)
        assert m & (m - 1) == 0
    # every 2^k; 5*2^k from 1280 on except 10240 (no split: a 160-point row is
    # not whole 8-line swizzle atoms, 1280 threads are too many for the
    # one-CTA kernel)
    for k in range(8, 31):
        assert (1 << k) in L, k
    for k in range(8, 28):
        assert ((5 << k) in L) == ((5 << k) != 10240), k


def test_width_table_monotone():
    bc.load_width_table()
    prev = 99
    for M in bc.lengths():
        w = bc.width_limit(M)
        assert w <= prev + 1  # non-increasing up to one-step noise
        prev = w


def test_pipelined_launch_shapes_consistent():
    # every supported length: TMA boxes deliver exactly the bytes each kernel
    # waits for and tiles cover the rows (checked again before every launch)
    assert bc._lib().bc_gpu_check_shapes() == 0


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the behaviour without a GPU")
def test_no_gpu_no_fallback():
    # without an sm_100 device the engine refuses (BC_ERR_NO_DEVICE) and a
    # product raises; there is no CPU path that would compute it instead
    import numpy as np
    with pytest.raises(bc.BcError) as e:
        bc.init(0)
    assert e.value.code == -8
    with pytest.raises(bc.BcError):
        bc.mul(np.arange(1, 300, dtype=np.uint32), np.arange(1, 300, dtype=np.uint32))


@pytest.mark.skipif(_has_gpu(), reason="checks the behaviour without a GPU")
def test_host_fft_mul_aborts_without_gpu():
    # the reference's _fft_mul entry point (include/mul.h) aborts with a
    # message when the GPU engine is unavailable, as the reference aborts on
    # the widths it cannot pack; it never computes the product on the CPU
    import subprocess
    import sys
    code = (
        "import ctypes, numpy as np, bluecrunch_b200 as bc\n"
        "lib = ctypes.CDLL(bc.HOST_LIB)\n"
        "a = np.arange(1, 2001, dtype=np.uint32); c = np.zeros(4000, dtype=np.uint32)\n"
        "p = lambda x: x.ctypes.data_as(ctypes.c_void_p)\n"
        "lib._fft_mul(p(c), ctypes.c_size_t(4000), p(a), ctypes.c_size_t(2000), p(a), ctypes.c_size_t(2000))\n"
        "print('computed')\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and "computed" not in r.stdout
    assert "GPU" in r.stderr


def test_shape_candidates_and_table():
    # every length of two or more levels offers its built-in split among the
    # candidates; a candidate can be set and reset, anything else is refused
    lib = bc._lib()
    for M in (1 << 13, 3 << 14, 1 << 20, 1 << 22, 1 << 25, 3 << 25, 1 << 28):
        p = bc.plan(M // 2, M // 2, M)
        if p["fft_points"] != M:
            continue
        cands = bc.shape_candidates(M)
        assert (p["levels"], p["L1"], p["L2"], p["Lr"]) in cands, (M, p, cands)
        for lv, L1, L2, Lr in cands:
            assert lv == p["levels"] and L1 * L2 * Lr == M
        lv, L1, L2, Lr = cands[-1]
        bc.set_shape(M, L1, L2, Lr)
        q = bc.plan(M // 2, M // 2, M)
        assert (q["L1"], q["L2"], q["Lr"]) == (L1, L2, Lr)
        assert lib.bc_gpu_check_shapes() == 0
        bc.set_shape(M)
        assert lib.bc_gpu_set_shape(M, 3, 5, 7) == -1
    # the committed table holds candidates only
    if os.path.exists(bc.SHAPE_FILE):
        assert lib.bc_gpu_load_shape_table(bc.SHAPE_FILE.encode()) == 0
        assert lib.bc_gpu_check_shapes() == 0
        for M in bc.lengths():
            bc.set_shape(M)


def test_ctypes_structs_match_the_header(tmp_path):
    """The Python mirrors of bc_batch_stats, bc_mul_stats, bc_mul_desc and
    bc_plan_info have the C compiler's size and field offsets, and the batch
    flags have the header's values."""
    import subprocess
    structs = {"bc_batch_stats": bc.BatchStats, "bc_mul_stats": bc.MulStats, "bc_mul_desc": bc.MulDesc,
               "bc_plan_info": bc.PlanInfo}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "bc_gpu.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append('printf("%s sizeof %%zu\\n", sizeof(%s));' % (cname, cname))
        for f, _ in py._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, f, cname, f))
    lines.append('printf("flags %d %d %d\\n", BC_BATCH_HOST_OPERANDS, BC_BATCH_DEVICE_OPERANDS, BC_BATCH_GRAPH);')
    lines.append("return 0; }")
    src, exe = tmp_path / "layout.c", tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.check_call(["gcc", "-std=c11", "-I" + os.path.join(ROOT, "include"), "-o", str(exe), str(src)])
    got = {}
    for ln in subprocess.check_output([str(exe)], text=True).splitlines():
        k, v = ln.rsplit(" ", 1) if not ln.startswith("flags") else (ln[:5], ln[6:])
        got[k] = v
    for cname, py in structs.items():
        assert int(got[cname + " sizeof"]) == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got["%s %s" % (cname, f)]) == getattr(py, f).offset, (cname, f)
    assert got["flags"].split() == [str(bc.BATCH_HOST_OPERANDS), str(bc.BATCH_DEVICE_OPERANDS), str(bc.BATCH_GRAPH)]
