"""GPU: bc_gpu_mul_noalloc, the allocation-free product for callers that
cannot allocate device memory (under a pool or allocator that owns the
device, or in hosts that forbid cudaMalloc after start-up).

Called through the C ABI with device buffers the test allocates itself; the
result must equal the allocating entry point's (bc_gpu_mul) and the exact
product (Python integers), bit for bit, on two calls in a row, and the calls
must not change the device's free memory.  Collected last so a run that
stops at the first failure has run every other test; passes alone in a fresh
process too."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _limbs(seed, n):
    rng = np.random.default_rng(seed)
    v = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    v[-1] |= 1
    return v


def test_noalloc_matches_bc_gpu_mul_twice():
    torch = pytest.importorskip("torch")
    import bluecrunch_b200 as bc
    bc.init(0)
    lib = bc._lib()
    stream = torch.cuda.current_stream().cuda_stream
    cases = [(5000, 3000, 8000), (60000, 60000, 120000), (1000, 1000, 2000), (40000, 5000, 45000)]
    for rep in range(2):  # two calls in a row per shape
        for k, (al, bl, cl) in enumerate(cases):
            a, b = _limbs(10 * k + 1, al), _limbs(10 * k + 2, bl)
            want = bc.mul(a, b, CL=cl)
            da = torch.from_numpy(a.view(np.int32)).cuda()
            db = torch.from_numpy(b.view(np.int32)).cuda()
            out = torch.full((cl,), -1, dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            rc = lib.bc_gpu_mul_noalloc(out.data_ptr(), cl, da.data_ptr(), al, db.data_ptr(), bl, stream)
            torch.cuda.synchronize()
            free_after = torch.cuda.mem_get_info()[0]
            assert rc == 0, bc.BcError(rc)
            got = out.cpu().numpy().view(np.uint32)
            assert np.array_equal(got, want), (rep, al, bl)
            exact = bc.from_int(bc.to_int(a) * bc.to_int(b) % (1 << (32 * cl)), cl)
            assert np.array_equal(got, exact), (rep, al, bl)
            if rep == 1:  # kernels are loaded by now: the call itself allocates nothing
                assert free_after == free_before


def test_noalloc_square_and_limits():
    torch = pytest.importorskip("torch")
    import bluecrunch_b200 as bc
    bc.init(0)
    lib = bc._lib()
    a = _limbs(7, 20000)
    da = torch.from_numpy(a.view(np.int32)).cuda()
    out = torch.zeros(40000, dtype=torch.int32, device="cuda")
    assert lib.bc_gpu_mul_noalloc(out.data_ptr(), 40000, da.data_ptr(), 20000, da.data_ptr(), 20000, None) == 0
    assert np.array_equal(out.cpu().numpy().view(np.uint32), bc.mul(a, square=True))
    big = torch.zeros(70000, dtype=torch.int32, device="cuda")
    res = torch.zeros(140000, dtype=torch.int32, device="cuda")
    assert lib.bc_gpu_mul_noalloc(res.data_ptr(), 140000, big.data_ptr(), 70000, big.data_ptr(), 70000, None) \
        == -7  # BC_ERR_TOO_LARGE beyond 131072 limbs
    assert lib.bc_gpu_mul_noalloc(da.data_ptr(), 40000, da.data_ptr(), 20000, da.data_ptr(), 20000, None) \
        == -1  # BC_ERR_INVALID: output overlaps an input
