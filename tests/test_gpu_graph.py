"""GPU parity of the graph form of a batch (BC_BATCH_GRAPH): the passes of
every length bucket captured into one CUDA graph and started with one
cudaGraphLaunch.  Every product must equal the exact product and the plain
batch's output; a second batch of the same lengths must reuse the kept
executable graph (updated in place), a batch of other lengths must get a new
one."""
import numpy as np
import pytest

from conftest import limbs

pytestmark = pytest.mark.gpu


def _device_batch(gpu, torch, shapes, seed):
    """shapes: (AL, BL or None for a square, shares_b_with or None).  Operands
    in one device pool (items with shares_b_with use that item's B array);
    returns descs, the pool, the output pool, host operands and offsets."""
    host, offs, tot = [], [], 0
    for i, (al, bl, share) in enumerate(shapes):
        a = limbs(seed + 2 * i, al)
        b = None if bl is None else (host[share][1] if share is not None else limbs(seed + 2 * i + 1, bl))
        host.append((a, b))
    parts, pos = [], 0
    for a, b in host:
        parts.append(a)
        offs.append([pos, None])
        pos += a.size
        if b is not None:
            parts.append(b)
            offs[-1][1] = pos
            pos += b.size
    pool = torch.from_numpy(np.concatenate(parts).view(np.int32)).cuda()
    CLs = [a.size + (a.size if b is None else b.size) for a, b in host]
    out = torch.zeros(sum(CLs), dtype=torch.int32, device="cuda")
    descs = (gpu.MulDesc * len(shapes))()
    o = 0
    for i, ((al, bl, share), (a, b)) in enumerate(zip(shapes, host)):
        pa = pool.data_ptr() + 4 * offs[i][0]
        if b is None:
            pb, blen = pa, al
        else:
            src = offs[share][1] if share is not None else offs[i][1]
            pb, blen = pool.data_ptr() + 4 * src, b.size
        descs[i] = gpu.MulDesc(out.data_ptr() + 4 * o, CLs[i], pa, al, pb, blen)
        o += CLs[i]
    return descs, pool, out, host, CLs


def _outputs(out, CLs):
    h = out.cpu().numpy().view(np.uint32)
    res, o = [], 0
    for CL in CLs:
        res.append(h[o:o + CL].copy())
        o += CL
    return res


SHAPES = [(3000, 2000, None), (3100, None, None), (70_000, 65_000, None), (40_000, 41_000, 2),
          (300_000, 280_000, None), (120, 90, None), (9000, 9000, None), (1 << 17, None, None)]


def test_graph_batch_matches_plain_batch_and_exact(gpu, orc):
    torch = pytest.importorskip("torch")
    descs, pool, out, host, CLs = _device_batch(gpu, torch, SHAPES, 7100)
    st = gpu.mul_batch_desc(descs, len(SHAPES), gpu.BATCH_GRAPH)
    torch.cuda.synchronize()
    got = _outputs(out, CLs)
    assert st["graph_launches"] >= 1 and st["graph_nodes"] >= st["launches"] >= st["classes"] >= 4
    out.zero_()
    st_plain = gpu.mul_batch_desc(descs, len(SHAPES))
    torch.cuda.synchronize()
    plain = _outputs(out, CLs)
    assert st_plain["graph_launches"] == 0
    for (a, b), g_, p_ in zip(host, got, plain):
        assert np.array_equal(g_, p_)
        bb = a if b is None else b
        if a.size + bb.size <= 200_000:
            assert np.array_equal(g_, orc.ntt_mul(a, bb, a.size + bb.size))
        else:
            assert orc.modcheck(g_, a, bb, 4)


def test_graph_kept_for_same_lengths_and_renewed_for_others(gpu, orc):
    torch = pytest.importorskip("torch")
    # first batch: instantiates (or updates a graph kept from an earlier test)
    d1, p1, o1, h1, c1 = _device_batch(gpu, torch, SHAPES, 8100)
    gpu.mul_batch_desc(d1, len(SHAPES), gpu.BATCH_GRAPH)
    # same lengths, other operands in other buffers: the kept graph is updated
    d2, p2, o2, h2, c2 = _device_batch(gpu, torch, SHAPES, 9100)
    st2 = gpu.mul_batch_desc(d2, len(SHAPES), gpu.BATCH_GRAPH)
    assert st2["graph_launches"] == 1 and st2["graph_updates"] == 1
    # other lengths: a new graph
    other = [(5000, 4000, None), (200_000, None, None), (777, 555, None)]
    d3, p3, o3, h3, c3 = _device_batch(gpu, torch, other, 10100)
    st3 = gpu.mul_batch_desc(d3, len(other), gpu.BATCH_GRAPH)
    assert st3["graph_launches"] == 1 and st3["graph_updates"] == 0
    torch.cuda.synchronize()
    for out, CLs, host in ((o1, c1, h1), (o2, c2, h2), (o3, c3, h3)):
        for (a, b), c in zip(host, _outputs(out, CLs)):
            bb = a if b is None else b
            assert orc.modcheck(c, a, bb, 4)
    # and the first batch once more through the (renewed) graph, exact
    o1.zero_()
    gpu.mul_batch_desc(d1, len(SHAPES), gpu.BATCH_GRAPH)
    torch.cuda.synchronize()
    for (a, b), c in zip(h1, _outputs(o1, c1)):
        bb = a if b is None else b
        if a.size + bb.size <= 200_000:
            assert np.array_equal(c, orc.ntt_mul(a, bb, a.size + bb.size))
        else:
            assert orc.modcheck(c, a, bb, 4)
