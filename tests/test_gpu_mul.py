"""GPU parity: bc_gpu_mul / bc_gpu_mul_batch (the device side of _fft_mul,
bigfloat/mul.c:108-174) against the oracle.  Bit-exact throughout."""
import json
import os

import numpy as np
import pytest

from conftest import exact, limbs

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _check(gpu, orc, a, b, CL=None, square=False):
    CL = CL or (len(a) + len(b))
    c, st = gpu.mul(a, None if square else b, CL=CL, square=square, want_stats=True)
    if CL <= 20000:
        want = exact(a, a if square else b, CL)
    else:
        want = orc.ntt_mul(a, a if square else b, CL)
    assert np.array_equal(c, want), (len(a), len(b), CL, st)
    assert st["max_round_err"] < 0.25
    return st


@pytest.mark.parametrize("al,bl", [(1, 1), (1, 7), (3, 5), (13, 100), (50, 50), (100, 100), (255, 257),
                                   (1000, 1000), (1000, 125), (4096, 4096), (6000, 3000)])
def test_small_and_medium(gpu, orc, al, bl):
    _check(gpu, orc, limbs(al * 7 + 1, al), limbs(bl * 7 + 2, bl))


@pytest.mark.parametrize("al,bl", [(10000, 10000), (16384, 16384), (40000, 5000), (65536, 65536),
                                   (100000, 100000), (131072, 16384), (262144, 262144)])
def test_two_level(gpu, orc, al, bl):
    _check(gpu, orc, limbs(al + 11, al), limbs(bl + 13, bl))


@pytest.mark.parametrize("al", [1 << 19, 1 << 20, 3 << 19])
def test_three_level(gpu, orc, al):
    _check(gpu, orc, limbs(al + 17, al), limbs(al + 19, al))


@pytest.mark.parametrize("al,bl,sq", [(1 << 21, 1 << 21, False), (1 << 22, 1 << 22, False), (1 << 22, 1 << 19, False),
                                      (1 << 22, 1 << 22, True), (3 << 20, 3 << 20, False)])
def test_three_level_rows_of_1024(gpu, orc, al, bl, sq):
    # transforms of 2^22 and more points run their 1024-point rows on the
    # one-warp-per-row kernel (k2_rows_w1024), squaring included
    a = limbs(al + 29, al)
    b = a if sq else limbs(bl + 31, bl)
    st = _check(gpu, orc, a, b, square=sq)
    assert st["fft_points"] >= 1 << 21


_ROWS_BLOCK = r"""
import sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import numpy as np
import bluecrunch_b200 as bc
import oracle
from conftest import limbs
bc.init(0)
n = 1 << 21
a, b = limbs(101, n), limbs(102, n)
c = bc.mul(a, b, CL=2 * n)
assert np.array_equal(c, oracle.restated().ntt_mul(a, b, 2 * n))
s = bc.mul(a, None, CL=2 * n, square=True)
assert np.array_equal(s, oracle.restated().ntt_mul(a, a, 2 * n))
print("OK")
"""


def test_block_row_kernel_for_1024_point_rows():
    # BC_ROWS_WARP=0 keeps the 8-points-per-thread row kernel k2_rows<1024>
    import subprocess
    import sys
    root = os.path.dirname(HERE)
    env = dict(os.environ, BC_ROWS_WARP="0")
    p = subprocess.run([sys.executable, "-c", _ROWS_BLOCK.format(root=root, tests=HERE)], env=env,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0 and p.stdout.strip().endswith("OK"), p.stderr[-2000:]


_FUSED = r"""
import sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import numpy as np
import bluecrunch_b200 as bc
import oracle
from conftest import limbs
bc.init(0)
R = oracle.restated()
# M = 2^22 (64 x 64 x 1024), 2^23 (128 x 64 x 1024), 2^24 (128 x 128 x 1024):
# splits with 1024-point rows, which the fused kernel covers (the tuned
# table may prefer others)
for M, L1, L2 in ((1 << 22, 64, 64), (1 << 23, 128, 64), (1 << 24, 128, 128)):
    bc.set_shape(M, L1, L2, 1024)
for n in (1 << 21, 1 << 22, 1 << 23):
    a, b = limbs(n + 1, n), limbs(n + 2, n)
    c, st = bc.mul(a, b, CL=2 * n, want_stats=True)
    assert bc.plan(n, n)["levels"] == 3
    ok = np.array_equal(c, R.ntt_mul(a, b, 2 * n)) if n <= (1 << 21) else R.modcheck(c, a, b, 4)
    assert ok, n
    s = bc.mul(a, None, CL=2 * n, square=True)
    assert (np.array_equal(s, R.ntt_mul(a, a, 2 * n)) if n <= (1 << 21) else R.modcheck(s, a, a, 4)), n
bc.time_kernels(True)
bc.mul(a, b, CL=2 * n)
assert "mid_fused" in [k for k, _ in bc.kernel_times()], bc.kernel_times()
print("OK")
"""


def test_fused_middle_pass():
    # BC_FUSED=1: the three-level middle (column pass, row products, inverse
    # column pass) in one persistent cooperative kernel (k4_mid_fused)
    import subprocess
    import sys
    root = os.path.dirname(HERE)
    env = dict(os.environ, BC_FUSED="1")
    p = subprocess.run([sys.executable, "-c", _FUSED.format(root=root, tests=HERE)], env=env,
                       capture_output=True, text=True, timeout=900)
    assert p.returncode == 0 and p.stdout.strip().endswith("OK"), p.stderr[-2000:]


@pytest.mark.parametrize("bl,als", [(3000, [2900, 3000, 3100, 1000]),            # one length, two levels
                                    (300000, [290000, 310000, 300000]),         # two levels
                                    (2 << 20, [(2 << 20) - 5000, 2 << 20, (2 << 20) + 7])])  # three levels
def test_shared_b_transform(gpu, orc, bl, als):
    # items of a batch whose B is the same device array share one B slot
    # (packed and transformed once, at the widest of their widths); every
    # product must stay exact, also beside items with their own B and squares
    torch = pytest.importorskip("torch")
    import numpy as np
    b = limbs(bl + 5, bl)
    db = torch.from_numpy(b.view(np.int32)).cuda()
    items, outs, want = [], [], []
    for k, al in enumerate(als):
        a = limbs(al + 11 * k, al)
        da = torch.from_numpy(a.view(np.int32)).cuda()
        dc = torch.zeros(al + bl, dtype=torch.int32, device="cuda")
        items.append((da, db, dc))
        want.append((a, b))
    other = limbs(bl + 77, bl)
    do = torch.from_numpy(other.view(np.int32)).cuda()
    dco = torch.zeros(2 * bl, dtype=torch.int32, device="cuda")
    dsq = torch.zeros(2 * bl, dtype=torch.int32, device="cuda")
    descs = (gpu.MulDesc * (len(items) + 2))()
    for i, (da, dbb, dc) in enumerate(items):
        descs[i] = gpu.MulDesc(dc.data_ptr(), dc.numel(), da.data_ptr(), da.numel(), dbb.data_ptr(), dbb.numel())
    descs[len(items)] = gpu.MulDesc(dco.data_ptr(), 2 * bl, do.data_ptr(), bl, db.data_ptr(), bl)
    descs[len(items) + 1] = gpu.MulDesc(dsq.data_ptr(), 2 * bl, db.data_ptr(), bl, db.data_ptr(), bl)
    gpu.mul_batch_desc(descs, len(items) + 2)
    torch.cuda.synchronize()
    for (a, bb), (_, _, dc) in zip(want, items):
        got = dc.cpu().numpy().view(np.uint32)
        if a.size + bb.size <= 1 << 20:
            assert np.array_equal(got, exact(a, bb, a.size + bb.size)), (a.size, bb.size)
        else:
            assert orc.modcheck(got, a, bb, 4), (a.size, bb.size)
    got_o = dco.cpu().numpy().view(np.uint32)
    got_s = dsq.cpu().numpy().view(np.uint32)
    if 2 * bl <= 1 << 20:
        assert np.array_equal(got_o, exact(other, b, 2 * bl)) and np.array_equal(got_s, exact(b, b, 2 * bl))
    else:
        assert orc.modcheck(got_o, other, b, 4) and orc.modcheck(got_s, b, b, 4)


@pytest.mark.parametrize("M", [1280, 2560, 5120, 20480, 40960, 163840, 5 << 18, 5 << 20, 5 << 22])
@pytest.mark.parametrize("kind", ["product", "square", "unbalanced"])
def test_lengths_with_factor_five(gpu, orc, M, kind):
    # transform lengths 5*2^k (a radix-5 first stage in the row or one-CTA
    # transform) between 2^k and 3*2^k; each forced at its width limit
    b = gpu.width_limit(M)
    n = (M * b) // 32 - 3
    a = limbs(M + 1, n)
    bb = a if kind == "square" else limbs(M + 2, n if kind == "product" else n // 3)
    gpu.force_plan(M, b)
    try:
        c, st = gpu.mul(a, None if kind == "square" else bb, CL=a.size + bb.size, square=kind == "square",
                        want_stats=True)
    finally:
        gpu.force_plan(0, 0)
    assert st["fft_points"] == M and st["max_round_err"] < 0.25, st
    if a.size + bb.size <= 1 << 21:
        assert np.array_equal(c, orc.ntt_mul(a, bb, a.size + bb.size)), (M, kind)
    else:
        assert orc.modcheck(c, a, bb, 4), (M, kind)


@pytest.mark.parametrize("al,bl", [(1 << 21, 1 << 19), (1 << 22, 1 << 20)])
def test_unbalanced_product_takes_a_five_length(gpu, orc, al, bl):
    # 1:4 products: CL = 1.25 * AL fits 5*2^k points, between the 2^(k+2)
    # that is too short and the 3*2^(k+1) the 2^k / 3*2^k lengths would take
    a, b = limbs(al + 1, al), limbs(bl + 2, bl)
    c, st = gpu.mul(a, b, want_stats=True)
    assert st["fft_points"] % 5 == 0, st
    assert orc.modcheck(c, a, b, 4)


@pytest.mark.parametrize("n", [100, 2048, 30000, 1 << 18, 1 << 20])
def test_squaring(gpu, orc, n):
    a = limbs(n + 23, n)
    _check(gpu, orc, a, a, square=True)


def test_golden_products(gpu):
    import hashlib
    import oracle
    g = json.load(open(os.path.join(HERE, "golden", "products.json")))
    for case in g["cases"]:
        a = oracle.random_limbs(case["seed_a"], case["AL"])
        b = a if case["square"] else oracle.random_limbs(case["seed_b"], case["BL"])
        c = gpu.mul(a, None if case["square"] else b, CL=case["CL"], square=case["square"])
        assert hashlib.sha256(c.astype("<u4").tobytes()).hexdigest() == case["sha256"], case


def test_edge_values(gpu, orc):
    # structured operands put every balanced digit near +-2^(b-1); at the
    # widths tuned on random data some of these exceed the rounding limit and
    # the library redoes them with narrower digits — results stay exact
    for n in (100, 5000, 70000):
        ones = np.full(n, 0xFFFFFFFF, dtype=np.uint32)
        _check(gpu, orc, ones, ones)
        _check(gpu, orc, ones, ones, square=True)
        alt = np.tile(np.array([0x80008000, 0x7FFF7FFF], dtype=np.uint32), n // 2)
        _check(gpu, orc, alt, alt)
        z = np.zeros(n, dtype=np.uint32); z[-1] = 1
        _check(gpu, orc, z, ones)


def test_truncated_and_padded_outputs(gpu, orc):
    a, b = limbs(5, 3000), limbs(6, 2000)
    _check(gpu, orc, a, b, CL=6000)      # CL > AL+BL: high words zero
    _check(gpu, orc, a, b, CL=2500)      # CL < AL+BL: low words only
    _check(gpu, orc, a, b, CL=1)


def test_zero_length(gpu):
    c = gpu.mul(np.zeros(0, dtype=np.uint32), limbs(1, 10), CL=12)
    assert not c.any()


def test_batch_matches_single(gpu, orc):
    rng = np.random.default_rng(7)
    items = []
    for i in range(40):
        al = int(np.exp(rng.uniform(np.log(64), np.log(60000))))
        bl = int(np.exp(rng.uniform(np.log(64), np.log(60000))))
        a = limbs(1000 + i, al)
        b = a if i % 5 == 0 else limbs(2000 + i, bl)
        items.append((a, None if i % 5 == 0 else b, None))
    outs, st = gpu.mul_batch(items, want_stats=True)
    for (a, b, _), c in zip(items, outs):
        bb = a if b is None else b
        assert np.array_equal(c, orc.ntt_mul(a, bb, len(a) + len(bb)))
    assert st["classes"] >= 2


def test_device_pointers_and_aliasing(gpu, orc):
    torch = pytest.importorskip("torch")
    a, b = limbs(31, 50000), limbs(32, 40000)
    da = torch.from_numpy(a.view(np.int32)).cuda()
    db = torch.from_numpy(b.view(np.int32)).cuda()
    dc = torch.zeros(90000, dtype=torch.int32, device="cuda")
    gpu.mul(da, db, CL=90000, out=dc)
    want = orc.ntt_mul(a, b)
    assert np.array_equal(dc.cpu().numpy().view(np.uint32), want)
    # in place: C aliases A (bigfloat_mul's in-place path, bigfloat/mul.c:609-627)
    buf = torch.zeros(90000, dtype=torch.int32, device="cuda")
    buf[:50000] = da
    gpu.mul(buf[:50000], db, CL=90000, out=buf)
    assert np.array_equal(buf.cpu().numpy().view(np.uint32), want)


def test_batch_spanning_several_staging_chunks(gpu, orc):
    """Pageable operands and results of one batch crossing in 64 MiB chunks:
    items larger than a chunk, items straddling chunk boundaries, small ones
    between them; each product checked modulo primes (sizes beyond the NTT's
    few-second range)."""
    sizes = [(9_000_000, 8_000_000), (300, 200), (17_000_000, 5_000_000), (1, 1), (4_000_000, 4_000_001),
             (2_500, 70_000)]
    items = [(limbs(500 + i, al), limbs(600 + i, bl), None) for i, (al, bl) in enumerate(sizes)]
    outs, st = gpu.mul_batch(items, want_stats=True)
    for (a, b, _), c in zip(items, outs):
        assert len(c) == len(a) + len(b)
        assert orc.modcheck(c, a, b, 4)
    small = items[1]
    assert np.array_equal(outs[1], exact(small[0], small[1], len(small[0]) + len(small[1])))


def test_pinned_host_operands_large(gpu, orc):
    # one large product with both operands and the result in pinned host
    # memory: B crosses on its own stream while the outer pass packs A
    import torch
    n = 1 << 21
    a, b = limbs(n + 41, n), limbs(n + 43, n - 5)
    ha = torch.from_numpy(a.view(np.int32)).pin_memory()
    hb = torch.from_numpy(b.view(np.int32)).pin_memory()
    hc = torch.zeros(a.size + b.size, dtype=torch.int32).pin_memory()
    for _ in range(2):
        gpu.mul(ha, hb, CL=a.size + b.size, out=hc)
        assert np.array_equal(hc.numpy().view(np.uint32), orc.ntt_mul(a, b, a.size + b.size))


@pytest.mark.parametrize("al,bl,sq", [(1 << 26, 1 << 26, False), (1 << 27, 1 << 24, False), (1 << 26, 1 << 26, True)])
def test_full_size_products_modular(gpu, orc, al, bl, sq):
    # the sweep's largest sizes (2^26 and 2^27 limbs, transforms of 2^27 and
    # 2^28 points): too large for an exact reference product in a test, so
    # size-independent properties instead — the product agrees with A*B
    # modulo four primes (FP64-free, seeded from the reference's CHECKPRIME),
    # and its top limbs are zero exactly where AL + BL exceeds the product's
    # length
    a = limbs(al + 51, al)
    b = a if sq else limbs(bl + 53, bl)
    c, st = gpu.mul(a, None if sq else b, CL=al + bl, square=sq, want_stats=True)
    assert st["max_round_err"] < 0.25 and st["fft_points"] >= 1 << 27
    assert orc.modcheck(c, a, b, 4)
    # one flipped bit of A: the new product passes the same check and
    # differs from the old one (the check is not blind to the input)
    if not sq:
        j = al // 3
        a2 = a.copy()
        a2[j] ^= 1  # flip the lowest bit of limb j
        c2 = gpu.mul(a2, b, CL=al + bl)
        assert orc.modcheck(c2, a2, b, 4)
        assert not np.array_equal(c, c2)


def test_bounded_wait_runs_out_without_a_fault(gpu, orc):
    # a carry lookback whose predecessor never publishes (its tile is never
    # taken): the bounded spin gives up, flags the sum and the kernel ends;
    # the host gets BC_ERR_TIMEOUT and the context stays usable
    import ctypes
    secs = ctypes.c_double(0.0)
    rc = gpu._lib().bc_gpu_selftest_wait(ctypes.byref(secs))
    assert rc == -4, rc  # BC_ERR_TIMEOUT
    assert 0.0 < secs.value < 60.0, secs.value
    _check(gpu, orc, limbs(5, 5000), limbs(6, 4000))
