"""Width autotuner: per transform length M, the widest balanced digit width b
whose measured max |x - round(x)| on seeded random operands stays below the
target (default 0.125, half the library's 0.25 retry threshold).

The FP64 rounding error of the convolution grows by ~4x per extra bit of b,
so one measurement at a probe width predicts the limit; the prediction is then
verified (and stepped down until it holds).  Results go to tune/widths.txt,
which bc_gpu_init loads (bluecrunch_b200.init passes it; C callers set
BC_TUNE_FILE or bc_gpu_config.tune_path).

  python -m bluecrunch_b200.tune.autotune [--max-log2 29] [--target 0.125]

With --shapes it tunes the decomposition instead: for every length of two or
more levels, each valid split (bc_gpu_shape_candidates: L1 x Lr or
L1 x L2 x Lr over the compiled pass lengths) runs a full-size product of
seeded random operands on the GPU (CUDA events, modular check of the
result), and the fastest goes to tune/shapes.txt, which bc_gpu_init loads
from beside the width table.

  python -m bluecrunch_b200.tune.autotune --shapes [--max-log2 28]
"""
import argparse
import datetime
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def random_limbs(seed, n):
    rng = np.random.default_rng(seed)
    v = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    v[-1] |= 1
    return v


def measure(bc, torch, M, b, seed=1):
    n = max(1, (M * b) // 32)
    a = random_limbs(seed * 7919 + M, n)
    c = random_limbs(seed * 7919 + M + 1, n)
    bc.force_plan(M, b)
    try:
        da = torch.from_numpy(a.view(np.int32)).cuda()
        db = torch.from_numpy(c.view(np.int32)).cuda()
        out = torch.empty(2 * n, dtype=torch.int32, device="cuda")
        _, st = bc.mul(da, db, CL=2 * n, out=out, want_stats=True)
    finally:
        bc.force_plan(0, 0)
    assert st["fft_points"] == M, (st, M)
    return st["max_round_err"]


def time_shape(bc, torch, M, shape, reps):
    """Device time (ms) of one full-size product at length M with the given
    decomposition, and whether the result passes the modular check."""
    _, L1, L2, Lr = shape
    bc.set_shape(M, L1, L2, Lr)
    b = bc.width_limit(M)
    n = max(1, (M * b) // 32)
    a = random_limbs(M + 11, n)
    c = random_limbs(M + 13, n)
    bc.force_plan(M, b)
    try:
        da = torch.from_numpy(a.view(np.int32)).cuda()
        db = torch.from_numpy(c.view(np.int32)).cuda()
        out = torch.empty(2 * n, dtype=torch.int32, device="cuda")
        _, st = bc.mul(da, db, CL=2 * n, out=out, want_stats=True)  # warm (tables, arena)
        assert st["fft_points"] == M
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            bc.mul(da, db, CL=2 * n, out=out)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        ok = True
        try:
            import oracle
            ok = oracle.restated().modcheck(out.cpu().numpy().view(np.uint32), a, c, 2)
        except (ImportError, OSError):
            pass
        return ms, ok
    finally:
        bc.force_plan(0, 0)
        bc.set_shape(M)


def tune_shapes(bc, torch, args):
    """Per transform length of two or more levels, time every decomposition
    (bc_gpu_shape_candidates) on a full-size product and keep the fastest."""
    lines = []
    for M in bc.lengths():
        if M > (1 << args.max_log2):
            break
        cands = bc.shape_candidates(M)
        if len(cands) < 2:
            continue
        reps = 8 if M <= (1 << 22) else 3
        res = []
        for sh in cands:
            try:
                ms, ok = time_shape(bc, torch, M, sh, reps)
            except bc.BcError as exc:  # a split whose product is refused or wrong is not a candidate
                print("M=%d %s failed: %s" % (M, sh, exc), flush=True)
                ms, ok = float("inf"), False
            if not ok:
                print("M=%d %s: wrong product" % (M, sh), flush=True)
            res.append((ms if ok else float("inf"), sh))
        res.sort()
        best = res[0][1]
        desc = ", ".join("%dx%dx%d %.4f" % (s[1], s[2], s[3], t) for t, s in res)
        lines.append((M, best, desc))
        print("M=%-10d best %s   (%s)" % (M, best, desc), flush=True)
        torch.cuda.empty_cache()
    with open(args.out, "w") as fh:
        fh.write("# transform_points L1 L2 Lr  (bluecrunch_b200/tune/autotune.py --shapes, %s, %s);\n"
                 "# each line's comment lists every decomposition timed (ms per full-size product)\n"
                 % (torch.cuda.get_device_name(0), datetime.date.today().isoformat()))
        for M, (_, L1, L2, Lr), desc in lines:
            fh.write("%d %d %d %d  # %s\n" % (M, L1, L2, Lr, desc))
    print("wrote", args.out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--max-log2", type=int, default=29)
    ap.add_argument("--target", type=float, default=0.125)
    ap.add_argument("--shapes", action="store_true",
                    help="tune the decomposition of every length instead of the widths")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    import torch
    import bluecrunch_b200 as bc

    if args.shapes:
        args.out = args.out or os.path.join(HERE, "shapes.txt")
        bc.init(0)  # the tuned widths; the shapes under test are set one by one
        for M in bc.lengths():
            bc.set_shape(M)  # start from the built-in decompositions
        tune_shapes(bc, torch, args)
        return
    args.out = args.out or os.path.join(HERE, "widths.txt")

    bc.init(0, tune_path="")  # start from the built-in defaults
    lines = []
    for M in bc.lengths():
        if M > (1 << args.max_log2):
            break
        probe = min(24, bc.width_limit(M) + 2)
        err = measure(bc, torch, M, probe)
        guess = probe + int(math.floor(math.log(args.target / max(err, 1e-12), 4)))
        b = max(8, min(24, guess))
        e = measure(bc, torch, M, b, seed=2)
        while e >= args.target and b > 8:
            b -= 1
            e = measure(bc, torch, M, b, seed=2)
        # one step wider must fail the target for the limit to be the widest
        if b < 24:
            e_up = measure(bc, torch, M, b + 1, seed=3)
            if e_up < args.target:
                b += 1
                e = e_up
        lines.append((M, b, e, probe, err))
        print("M=%-10d b=%2d err=%.4f (probe b=%d err=%.3g)" % (M, b, e, probe, err), flush=True)
        torch.cuda.empty_cache()
    with open(args.out, "w") as fh:
        fh.write("# transform_points width_limit max_round_err_at_limit  "
                 "(bluecrunch_b200/tune/autotune.py, target %.3f, %s, %s)\n"
                 % (args.target, torch.cuda.get_device_name(0), datetime.date.today().isoformat()))
        for M, b, e, _, _ in lines:
            fh.write("%d %d %.6f\n" % (M, b, e))
    print("wrote", args.out)


if __name__ == "__main__":
    main()
