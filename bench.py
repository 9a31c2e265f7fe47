#!/usr/bin/env python3
"""Benchmark: exact bigfloat multiply throughput on B200 (and the reference
CPU multiply beside it).

Workload (the "single exact bigfloat multiply" configuration): A, B of
2^24 uniformly random base-2^32 limbs each (SplitMix64, seed 0xB1C0FFEE ^
log2(len), top limb nonzero), C = A*B of 2^25 limbs, bit-exact.  One step is
one product.  Operands and FFT work buffers (GBs) are far larger than the
126 MB L2, so no flush is needed between steps.

Metric: exact-multiply GB/s by the fixed algorithmic-bytes formula
    bytes = 4(AL+BL+CL) + (3-s) * 2 * 32 * Nc,  Nc = ceil(32 CL / b)/2
with b the width limit of the chosen transform length (the widest digits
that pass the 0.25 rounding-error criterion) and s = 1 for squaring.
`value` times device-resident operands; `e2e` times the C ABI call with
pinned host buffers (copies inside the timed region).

Reference arm (--impl reference): the reference's own _fft_mul compiled from
its sources (oracle/_ref, OpenMP tasks over all host threads), on the largest
size its packers support (2^20 x 2^20 limbs; it aborts for CL > 4e6), same
formula and unit.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

SEED = 0xB1C0FFEE
HEADLINE_LOG2 = 24
REF_LOG2 = 20


def alg_bytes(AL, BL, CL, b, square):
    nc = math.ceil(32 * CL / b) / 2
    return 4 * (AL + BL + CL) + (3 - (1 if square else 0)) * 2 * 32 * nc


# ---------------------------------------------------------------- formula width
# The byte formula's b is the width limit of the transform length the engine
# picks for a product.  The reference arm must not load the engine, so the
# length choice (shape_for / lengths / make_plan in csrc/bc_gpu.cu) is
# restated here over the same width table; tests/test_bench_contract.py checks
# it against bc_gpu_plan for many sizes.
_ROW_LENS = (128, 192, 256, 320, 384, 512, 640, 768, 1024, 1280, 1536, 2048, 2560, 3072, 4096)
_SMALL_LENS = (256, 512, 768, 1024, 1280, 1536, 2048, 2560, 3072, 4096, 5120)
_OUTER_LENS = (64, 128, 256, 512)
_ROW_PREF = (1024, 768, 1536, 512, 2048, 3072, 4096, 1280, 640, 2560)
_MAX_M = 1 << 30


def _pass_tile_w(L):
    return 1024 // L if 1024 // L >= 8 else 8


def _pow2part(x):
    return x & -x


def shape_levels(M):
    """Levels of the kernel shape for transform length M (0: no shape)."""
    if M < 256 or M > _MAX_M:
        return 0
    p2 = M // 3 if M % 3 == 0 else (M // 5 if M % 5 == 0 else M)
    if p2 & (p2 - 1):
        return 0
    if M <= 5120:
        return 1 if M in _SMALL_LENS else 0
    for L1 in _OUTER_LENS:
        if M % L1 == 0 and (M // L1) in _ROW_LENS and _pow2part(M // L1) >= _pass_tile_w(L1):
            return 2
    for Lr in _ROW_PREF:
        if M % Lr:
            continue
        R = M // Lr
        for L1 in _OUTER_LENS:
            if R % L1:
                continue
            L2 = R // L1
            if L2 < 64 or L2 > 512 or (L2 & (L2 - 1)) or L2 > L1:
                continue
            if _pow2part(Lr) < _pass_tile_w(L2) or _pow2part(L2 * Lr) < _pass_tile_w(L1):
                continue
            return 3
    return 0


def _lengths():
    out = []
    p = 256
    while p <= _MAX_M:
        for m in (p, 3 * p // 2, 5 * p // 4):
            if m <= _MAX_M and shape_levels(m):
                out.append(m)
        p *= 2
    return sorted(set(out))


def _width_table(path=os.path.join(ROOT, "bluecrunch_b200", "tune", "widths.txt")):
    table = {}
    if os.path.exists(path):
        for ln in open(path):
            f = ln.split()
            if len(f) >= 2 and not ln.startswith("#") and 8 <= int(f[1]) <= 24:
                table[int(f[0])] = int(f[1])
    return table


def width_limit_of(M, table=None):
    table = _width_table() if table is None else table
    default = max(8, min(24, math.floor(23.0 - 0.3 * math.log2(M))))
    if M in table:
        return table[M]
    longer = [k for k in table if k > M]
    if longer:  # the width of the next longer tuned length
        return min(table[min(longer)], default + 4)
    return default


def formula_plan(AL, BL, CL=None, square=False):
    """(M, width limit at M) of the product, as the engine plans it."""
    CL = CL or AL + BL
    AL, BL = min(AL, CL), min(BL, CL)
    table = _width_table()
    nd = lambda x, b: (32 * x + b - 1) // b  # noqa: E731
    best = None
    first_fit = 0
    for M in _lengths():
        if first_fit and M > 4 * first_fit:
            break
        bmax = min(width_limit_of(M, table), 24)
        if bmax < 8 or nd(AL, bmax) + nd(BL, bmax) > 2 * M + 1:
            continue
        first_fit = first_fit or M
        cost = M * (2 if shape_levels(M) == 3 else 1)
        if best is not None and cost >= best[0]:
            continue
        best = (cost, M)
    if best is None:
        raise ValueError("no transform length fits %d x %d limbs" % (AL, BL))
    return best[1], width_limit_of(best[1], table)


def operands(log2n, square=False, ratio=1):
    import oracle
    n = 1 << log2n
    a = oracle.random_limbs(SEED ^ log2n, n)
    b = a if square else oracle.random_limbs((SEED ^ log2n) + 1, n // ratio)
    return a, b


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class Clocks:
    """Samples SM clock, power and clock-event reasons every 10 ms during the
    timed region through NVML (read-only queries), falling back to
    `nvidia-smi -lms 200`.  The first sample is taken before __enter__
    returns, so even a short timed region is covered."""

    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index=0, period_s=0.01):
        self.index = index
        self.period = period_s
        self.rows = []  # (sm_mhz, max_mhz, watts, set of reason names)
        self.proc = None
        self.stop = threading.Event()
        self.thread = None
        self.source = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            ids = [x for x in vis.split(",") if x.strip().isdigit()]
            phys = int(ids[self.index]) if self.index < len(ids) else self.index
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(phys)

    def _nvml_loop(self, nv, h):
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while True:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                w = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((float(sm), float(mx), w, {n for n, b in bits.items() if rs & b}))
            except Exception:
                pass
            if self.stop.wait(self.period):
                break

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.source = "nvml 10 ms"
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self.thread.start()
        except Exception:
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            try:
                self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                              "--format=csv,noheader,nounits", "-lms", "200"],
                                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.source = "nvidia-smi 200 ms"
                self.thread = threading.Thread(target=self._smi_read, daemon=True)
                self.thread.start()
            except OSError:
                self.proc = None
        t0 = time.perf_counter()
        while self.thread is not None and not self.rows and time.perf_counter() - t0 < 3.0:
            time.sleep(0.005)
        return self

    def _smi_read(self):
        for line in self.proc.stdout:
            r = [x.strip() for x in line.split(",")]
            try:
                reasons = {n for i, n in enumerate(self.NAMES) if len(r) > 5 + i and r[5 + i].lower().startswith("active")}
                self.rows.append((float(r[1]), float(r[2]), float(r[3]), reasons))
            except (ValueError, IndexError):
                pass

    def __exit__(self, *exc):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        reasons = set()
        for r in self.rows:
            reasons |= r[3]
        return {"sm_mhz": float(np.median([r[0] for r in self.rows])), "sm_max_mhz": max(r[1] for r in self.rows),
                "power_w_median": round(float(np.median([r[2] for r in self.rows])), 1),
                "reasons": sorted(reasons), "samples": len(self.rows), "source": self.source}


# ---------------------------------------------------------------- reference arm
def time_reference(log2n=REF_LOG2, reps=3, kind="omp"):
    import oracle
    ref = oracle.reference(kind)
    a, b = operands(log2n)
    CL = a.size + b.size
    ref.fft_mul(a, b, CL, parallel=(kind == "omp"))  # warm (tables)
    t0 = time.perf_counter()
    for _ in range(reps):
        ref.fft_mul(a, b, CL, parallel=(kind == "omp"))
    dt = (time.perf_counter() - t0) / reps
    return a.size, b.size, CL, dt, ref.threads()


def reference_cli_e(digits, threads=None):
    """e to `digits` digits by the reference's own CLI (main.c:169-219) built
    from its sources into oracle/_ref/omp (OpenMP tasks in place of Cilk
    spawns, all host threads unless `threads`), wall time and md5 of e.txt."""
    import hashlib
    import tempfile
    import oracle
    cli = oracle.reference_cli("omp")
    if not os.path.exists(cli):
        return None
    env = dict(os.environ)
    nthr = threads or os.cpu_count() or 1
    env["OMP_NUM_THREADS"] = str(nthr)
    with tempfile.TemporaryDirectory() as d:
        t0 = time.perf_counter()
        res = subprocess.run([cli, str(digits)], cwd=d, capture_output=True, text=True, timeout=1800, env=env)
        wall = time.perf_counter() - t0
        if res.returncode != 0:
            return {"digits": digits, "mode": "reference CLI", "error": res.stderr[-300:]}
        md5 = hashlib.md5(open(os.path.join(d, "e.txt"), "rb").read()).hexdigest()
    pub = json.load(open(os.path.join(ROOT, "tests", "golden", "e_md5.json")))["published"]["digits_to_md5"]
    return {"digits": digits, "mode": "reference CLI (oracle/_ref/omp/bluecrunch_ref, %d threads)" % nthr,
            "wall_s": round(wall, 3), "threads": nthr, "md5": md5, "md5_matches_published": pub.get(str(digits)) == md5}


def reference_arm(args):
    """The reference's own _fft_mul (bigfloat/mul.c:108-174), compiled from its
    sources into oracle/_ref/omp, timed on all host threads.  Loads nothing of
    this repository's engine: the byte formula's width comes from
    formula_plan (the engine's length choice restated over its width table)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    if not oracle.have_reference("omp"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (reference sources absent at build time)"}))
        return
    K, W = args.steps, args.warmup
    ref = oracle.reference("omp")
    a, b = operands(REF_LOG2)
    CL = a.size + b.size
    for _ in range(W):
        ref.fft_mul(a, b, CL, parallel=True)
    t0 = time.perf_counter()
    for _ in range(K):
        ref.fft_mul(a, b, CL, parallel=True)
    dt = (time.perf_counter() - t0) / K
    _, b_alg = formula_plan(a.size, b.size, CL)
    gbs = alg_bytes(a.size, b.size, CL, b_alg, False) / dt / 1e9
    threads = ref.threads()
    print(json.dumps({
        "impl": "reference", "metric": "exact_mul_GBps", "value": round(gbs, 4), "unit": "GB/s",
        "higher_is_better": True, "n_gpus": args.gpus, "steps": K, "warmup": W,
        "ms_per_step": round(dt * 1e3, 3), "dtype": "f64", "data": "synthetic",
        "scaling": "weak",
        "config": {"workload": "exact multiply 2^20 x 2^20 limbs (largest size the reference packers support)",
                   "AL": a.size, "BL": b.size, "CL": CL, "width_for_formula": b_alg},
        "cpu_baseline": {"value": round(gbs, 4), "unit": "GB/s", "cores": threads, "kind": "reference",
                         "sample": "reference _fft_mul (bigfloat/mul.c:108-174) from oracle/_ref, OpenMP tasks, "
                                   "%d threads, %d timed multiplies of 2^20 x 2^20 limbs" % (threads, K)},
        "e2e": {"value": round(gbs, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ---------------------------------------------------------------- batched products
def batched_workload(n=8192, lo=128, hi=262144, seed=0xB1C0FFEE, sibling=False):
    """n independent products; AL, BL log-uniform in [lo, hi] limbs (or BL =
    AL*U(0.875, 1.125) for the sibling variant that mimics a splitting level)."""
    rng = np.random.default_rng(seed)
    al = np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.int64)
    if sibling:
        bl = np.maximum(1, (al * rng.uniform(0.875, 1.125, n)).astype(np.int64))
    else:
        bl = np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.int64)
    return al, bl


def run_batched(bc, torch, stream, n=8192, sibling=False, per_call=True, reps=2):
    import oracle
    al, bl = batched_workload(n, sibling=sibling)
    tot = int(al.sum() + bl.sum())
    pool = torch.from_numpy(oracle.random_limbs(0x5EED ^ n, tot).view(np.int32)).cuda()
    out = torch.zeros(tot, dtype=torch.int32, device="cuda")
    descs = (bc.MulDesc * n)()
    offs = np.concatenate([[0], np.cumsum(al + bl)])
    base_in, base_out = pool.data_ptr(), out.data_ptr()
    nbytes = 0
    for i in range(n):
        a0, b0 = int(offs[i]), int(offs[i] + al[i])
        CL = int(al[i] + bl[i])
        descs[i] = bc.MulDesc(base_out + 4 * int(offs[i]), CL, base_in + 4 * a0, int(al[i]),
                              base_in + 4 * b0, int(bl[i]))
        p = bc.plan(int(al[i]), int(bl[i]), CL)
        nbytes += alg_bytes(int(al[i]), int(bl[i]), CL, bc.width_limit(p["fft_points"]), False)
    bc.mul_batch_desc(descs, n)  # warm
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        st = bc.mul_batch_desc(descs, n)
    e1.record(stream)
    torch.cuda.synchronize()
    batched_ms = e0.elapsed_time(e1) / reps
    # spot check: modular check of a few items against the oracle
    R = oracle.restated()
    pool_h = pool.cpu().numpy().view(np.uint32)
    out_h = out.cpu().numpy().view(np.uint32)
    ok = True
    for i in np.random.default_rng(1).choice(n, 16, replace=False):
        a = pool_h[offs[i]:offs[i] + al[i]]
        b = pool_h[offs[i] + al[i]:offs[i + 1]]
        c = out_h[offs[i]:offs[i + 1]]
        ok &= R.modcheck(c, a, b, 2)
    res = {"items": n, "sibling": sibling, "total_limbs_in": tot, "classes": st["classes"],
           "launches_per_batch": st["launches"], "batched_ms": round(batched_ms, 3),
           "batched_GBps": round(nbytes / (batched_ms * 1e-3) / 1e9, 1),
           "products_per_s": round(n / (batched_ms * 1e-3), 1), "modcheck_sample_ok": bool(ok)}
    # the same batch as one CUDA graph launch (BC_BATCH_GRAPH): the first call
    # instantiates, the timed ones update the kept executable graph in place
    out.zero_()
    bc.mul_batch_desc(descs, n, bc.BATCH_GRAPH)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        sg = bc.mul_batch_desc(descs, n, bc.BATCH_GRAPH)
    e1.record(stream)
    torch.cuda.synchronize()
    graph_ms = e0.elapsed_time(e1) / reps
    out_g = out.cpu().numpy().view(np.uint32)
    gok = bool(np.array_equal(out_g, out_h))
    res.update({"graph_ms": round(graph_ms, 3), "graph_launches_per_batch": sg["graph_launches"],
                "graph_kernel_nodes": sg["graph_nodes"], "graph_updated_in_place": sg["graph_updates"] == 1,
                "graph_GBps": round(nbytes / (graph_ms * 1e-3) / 1e9, 1), "graph_equals_batched": gok})
    if per_call:
        out.zero_()
        lib = bc._lib()
        torch.cuda.synchronize()
        e0.record(stream)
        for i in range(n):
            d = descs[i]
            rc = lib.bc_gpu_mul(d.C, d.CL, d.A, d.AL, d.B, d.BL, None)
            if rc:
                raise bc.BcError(rc)
        e1.record(stream)
        torch.cuda.synchronize()
        per_ms = e0.elapsed_time(e1)
        res.update({"per_call_ms": round(per_ms, 3), "speedup_batched_vs_per_call": round(per_ms / batched_ms, 2)})
    del pool, out
    torch.cuda.empty_cache()
    return res


# ---------------------------------------------------------------- GPU arm
def run_e(digits, extra=()):
    """e to `digits` decimal digits through the CLI (the reference's main.c
    flow: binary splitting, Newton division, radix conversion, output files),
    wall time of the whole process and the md5 of e.txt against the
    published value (md5sums.txt of the reference)."""
    import hashlib
    import tempfile
    cli = os.path.join(ROOT, "bluecrunch_b200", "bluecrunch")
    pub = json.load(open(os.path.join(ROOT, "tests", "golden", "e_md5.json")))["published"]["digits_to_md5"]
    with tempfile.TemporaryDirectory() as d:
        t0 = time.perf_counter()
        res = subprocess.run([cli, str(digits), *extra], cwd=d, capture_output=True, text=True, timeout=1800)
        wall = time.perf_counter() - t0
        if res.returncode != 0:
            return {"digits": digits, "mode": " ".join(extra) or "default", "error": res.stderr[-300:]}
        h = hashlib.md5()
        with open(os.path.join(d, "e.txt"), "rb") as f:
            for blk in iter(lambda: f.read(1 << 24), b""):
                h.update(blk)
    phases = parse_phases(res.stdout)
    md5 = h.hexdigest()
    out = {"digits": digits, "mode": " ".join(extra) or "tree in device memory", "wall_s": round(wall, 3),
           "phases_s": phases, "md5": md5, "md5_matches_published": pub.get(str(digits)) == md5}
    if "Starting GPU engine" in phases:
        # process start and GPU context creation vary by a few seconds between
        # fresh processes; the rest is the computation and the output files
        out["wall_after_engine_start_s"] = round(wall - phases["Starting GPU engine"], 3)
    return out


PHASES = ("Starting GPU engine", "Summing", "Dividing", "Converting to decimal", "Writing hex digits",
          "Writing decimal digits")


def parse_phases(text):
    """Phase times of the CLI's output (timers.c format): "<name>... done [s
    seconds]" on one line, or "<name>..." then inner phases and an indented
    "Done [s seconds]" at the phase's own indentation."""
    phases, open_at = {}, {}
    for raw in text.splitlines():
        ind = len(raw) - len(raw.lstrip(" "))
        ln = raw.strip()
        for name in PHASES:
            if ln.startswith(name + "..."):
                if "[" in ln:
                    try:
                        phases[name] = float(ln.rsplit("[", 1)[1].split()[0])
                    except ValueError:
                        pass
                else:
                    open_at[ind] = name
        # "Done [..]" closes the phase opened at its indentation; a bare
        # "done [..]" (the phase's line was broken by diagnostic output) the
        # latest one
        key = ind if ln.startswith("Done [") else (max(open_at) if open_at and ln.startswith("done [") else None)
        if key is not None and key in open_at:
            try:
                phases[open_at.pop(key)] = float(ln.split("[", 1)[1].split()[0])
            except ValueError:
                pass
    return phases


def same_config_mul(bc, torch, stream, cpu, log2n=REF_LOG2, reps=20):
    """The reference arm's workload (2^20 x 2^20 limbs) on this engine:
    device-resident (CUDA events) and end to end through bc_gpu_mul with
    pinned and with pageable host buffers (copies inside the timed region)."""
    import oracle
    a, b = operands(log2n)
    AL, BL = a.size, b.size
    CL = AL + BL
    _, b_alg = formula_plan(AL, BL, CL)
    nbytes = alg_bytes(AL, BL, CL, b_alg, False)
    da = torch.from_numpy(a.view(np.int32)).cuda()
    db = torch.from_numpy(b.view(np.int32)).cuda()
    dc = torch.zeros(CL, dtype=torch.int32, device="cuda")
    for _ in range(3):
        bc.mul(da, db, CL=CL, out=dc)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        bc.mul(da, db, CL=CL, out=dc)
    e1.record(stream)
    torch.cuda.synchronize()
    dev_ms = e0.elapsed_time(e1) / reps
    want = dc.cpu().numpy().view(np.uint32).copy()
    ok = oracle.restated().modcheck(want, a, b, 4)
    res = {"workload": "exact multiply 2^20 x 2^20 limbs (the reference arm's and cpu_baseline's workload)",
           "unit": "GB/s", "higher_is_better": True, "width_for_formula": b_alg,
           "gpu_device": {"value": round(nbytes / (dev_ms * 1e-3) / 1e9, 2), "ms_per_step": round(dev_ms, 4)},
           "modcheck": bool(ok)}
    ha = torch.from_numpy(a.view(np.int32)).pin_memory()
    hb = torch.from_numpy(b.view(np.int32)).pin_memory()
    hc = torch.zeros(CL, dtype=torch.int32).pin_memory()
    for kind, (xa, xb, xc) in (("pinned", (ha, hb, hc)),
                               ("pageable", (a, b, np.zeros(CL, dtype=np.uint32)))):
        bc.mul(xa, xb, CL=CL, out=xc)
        t0 = time.perf_counter()
        for _ in range(reps):
            bc.mul(xa, xb, CL=CL, out=xc)
        e_ms = (time.perf_counter() - t0) * 1e3 / reps
        got = xc.numpy().view(np.uint32) if hasattr(xc, "numpy") else xc
        res["gpu_e2e_" + kind] = {"value": round(nbytes / (e_ms * 1e-3) / 1e9, 2), "ms_per_step": round(e_ms, 4),
                                  "h2d_bytes_per_step": 4 * (AL + BL), "d2h_bytes_per_step": 4 * CL,
                                  "matches_device_result": bool(np.array_equal(got, want))}
    res["reference"] = {"value": cpu["value"], "cores": cpu["cores"], "sample": cpu["sample"]}
    res["gpu_e2e_pageable_over_reference"] = round(res["gpu_e2e_pageable"]["value"] / cpu["value"], 1)
    res["gpu_device_over_reference"] = round(res["gpu_device"]["value"] / cpu["value"], 1)
    del da, db, dc
    return res


def gpu_arm(args):
    import torch
    import bluecrunch_b200 as bc
    import oracle

    from bluecrunch_b200.replicas import Replicas, job_throughput
    ranks = Replicas()  # N ranks = N independent replicas; no collective on the data path
    world, rank, local = ranks.world, ranks.rank, ranks.local
    torch.cuda.set_device(local)
    bc.init(local)
    stream = torch.cuda.current_stream()
    bc.set_stream(stream.cuda_stream)

    K, W = args.steps, args.warmup
    log2n = args.log2
    a, b = operands(log2n)
    AL, BL = a.size, b.size
    CL = AL + BL
    p = bc.plan(AL, BL, CL)
    b_alg = bc.width_limit(p["fft_points"])
    nbytes = alg_bytes(AL, BL, CL, b_alg, False)

    da = torch.from_numpy(a.view(np.int32)).cuda()
    db = torch.from_numpy(b.view(np.int32)).cuda()
    dc = torch.zeros(CL, dtype=torch.int32, device="cuda")
    want_sum = None
    # correctness of this exact workload: modular check (FP64-free) on the result
    c, st = bc.mul(da, db, CL=CL, out=dc, want_stats=True)
    host_c = dc.cpu().numpy().view(np.uint32)
    assert oracle.restated().modcheck(host_c, a, b, 4), "GPU product fails the modular check"

    def barrier():
        ranks.barrier()
        torch.cuda.synchronize()

    for _ in range(W):
        bc.mul(da, db, CL=CL, out=dc)
    barrier()
    with Clocks(local) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            bc.mul(da, db, CL=CL, out=dc)
        e1.record(stream)
        barrier()
    ms = e0.elapsed_time(e1) / K
    # per-kernel times (CUDA events after each launch on the library's
    # stream) from a second pass over the same K products, so the event
    # bookkeeping stays out of the timed pass above
    kern = {}
    per_product = 0
    bc.time_kernels(True)
    for _ in range(K):
        bc.mul(da, db, CL=CL, out=dc)
        kt = bc.kernel_times()
        per_product = len(kt)
        for name, kms in kt:
            kern.setdefault(name, []).append(kms)
    bc.time_kernels(False)
    barrier()
    launches = K * per_product  # kernels of this library launched in the timed pass
    ms = ranks.max(ms)
    value = job_throughput(nbytes, ms, world) / 1e9

    # ---- e2e: pinned host buffers through the C ABI, copies in the timed region
    ha = torch.from_numpy(a.view(np.int32)).pin_memory()
    hb = torch.from_numpy(b.view(np.int32)).pin_memory()
    hc = torch.zeros(CL, dtype=torch.int32).pin_memory()
    bc.mul(ha, hb, CL=CL, out=hc)
    barrier()
    t0 = time.perf_counter()
    for _ in range(max(1, K)):
        bc.mul(ha, hb, CL=CL, out=hc)
    e2e_ms = ranks.max((time.perf_counter() - t0) * 1e3 / max(1, K))
    assert np.array_equal(hc.numpy().view(np.uint32), host_c)
    e2e = job_throughput(nbytes, e2e_ms, world) / 1e9

    # ---- roofline of the dominant kernel (algorithmic bytes per launch)
    M = p["fft_points"]
    per_kernel_bytes = {
        "outer_fwd": 4 * (AL + BL) + 2 * 16 * M,
        "mid_fwd": 2 * 2 * 16 * M,
        "rows": 3 * 16 * M,
        "mid_inv": 2 * 16 * M,
        "outer_inv": 16 * M + 8 * M,
        "carry": 8 * M + 4 * CL,
        "small": 4 * (AL + BL + CL),
    }
    avg = {k: float(np.mean(v)) for k, v in kern.items()}
    dom = max(avg, key=avg.get) if avg else None
    peak, peak_kind = peaks()
    roof = None
    if dom:
        achieved = per_kernel_bytes.get(dom, 0) / (avg[dom] * 1e-3) / 1e9
        # DRAM bytes per launch are not measurable without a profiler: the
        # figure comes from the stored ncu capture of this kernel and length
        traffic, traffic_src = None, None
        tf = os.path.join(ROOT, "profiles", "ncu_traffic.json")
        if os.path.exists(tf):
            tj = json.load(open(tf))
            tr = tj.get(dom)
            if tr and tr.get("fft_points") == M:
                traffic = tr.get("dram_bytes_per_launch")
                traffic_src = "stored ncu capture (profiles/ncu_traffic.json, %s), not measured in this run" % (
                    tr.get("captured") or tj.get("captured") or "date not recorded")
        roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_kind": peak_kind, "traffic": traffic,
                "traffic_source": traffic_src,
                "algorithmic_bytes_per_launch": per_kernel_bytes.get(dom),
                "kernel_ms": {k: round(v, 4) for k, v in avg.items()},
                "kernel_share": {k: round(v / sum(avg.values()), 4) for k, v in avg.items()}}

    # ---- sweep (device-resident, a few steps each)
    sweep = []
    # the per-GPU characterisations (sweep, batches, e) run at N = 1 only: with
    # N ranks the other ranks would wait for them at the closing barrier
    if not args.no_sweep and rank == 0 and world == 1:
        for lg, ratio, sq in [(14, 1, False), (16, 1, False), (18, 1, False), (20, 1, False), (22, 1, False),
                              (24, 1, False), (26, 1, False), (27, 1, False),
                              (20, 8, False), (24, 8, False), (27, 8, False),
                              (20, 1, True), (24, 1, True), (27, 1, True)]:
            try:
                sa, sb = operands(lg, square=sq, ratio=ratio)
                sCL = sa.size + sb.size
                xa = torch.from_numpy(sa.view(np.int32)).cuda()
                xb = xa if sq else torch.from_numpy(sb.view(np.int32)).cuda()
                xc = torch.zeros(sCL, dtype=torch.int32, device="cuda")
                _, s0 = bc.mul(xa, None if sq else xb, CL=sCL, square=sq, out=xc, want_stats=True)
                reps = 5 if lg <= 24 else 2
                torch.cuda.synchronize()
                f0 = torch.cuda.Event(enable_timing=True)
                f1 = torch.cuda.Event(enable_timing=True)
                f0.record(stream)
                for _ in range(reps):
                    bc.mul(xa, None if sq else xb, CL=sCL, square=sq, out=xc)
                f1.record(stream)
                torch.cuda.synchronize()
                sms = f0.elapsed_time(f1) / reps
                sp = bc.plan(sa.size, sb.size, sCL, square=sq)
                sb_alg = bc.width_limit(sp["fft_points"])
                g = alg_bytes(sa.size, sb.size, sCL, sb_alg, sq) / (sms * 1e-3) / 1e9
                ok = oracle.restated().modcheck(xc.cpu().numpy().view(np.uint32), sa, sa if sq else sb, 2)
                sweep.append({"AL": sa.size, "BL": sb.size, "square": sq, "M": sp["fft_points"],
                              "levels": sp["levels"], "width": s0["width"], "max_round_err": s0["max_round_err"],
                              "ms": round(sms, 4), "GBps": round(g, 1), "frac_hbm": round(g / peak, 4),
                              "modcheck": ok})
                del xa, xb, xc
                torch.cuda.empty_cache()
            except Exception as exc:  # report, keep going
                sweep.append({"log2": lg, "ratio": ratio, "square": sq, "error": str(exc)[:200]})

    # ---- batched uneven products (8192 per launch sequence) vs per-call launches
    batched = []
    if not args.no_batched and rank == 0 and world == 1:
        for sib in (False, True):
            try:
                batched.append(run_batched(bc, torch, stream, n=args.batch_items, sibling=sib))
            except Exception as exc:
                batched.append({"sibling": sib, "error": str(exc)[:300]})

    # ---- e to N digits end to end (CLI), default mode and, smaller, per call
    e_runs = []
    e_list = [int(x) for x in str(args.e_digits).split(",") if x.strip() and int(x) > 0]
    if rank == 0 and world == 1 and e_list:
        for nd in e_list:
            e_runs.append(run_e(nd))
        if args.e_per_call:
            pc = run_e(args.e_per_call, ("--per-call",))
            pc["mode"] = "one GPU product per call (--per-call)"
            same = [x for x in e_runs if x.get("digits") == args.e_per_call and "wall_s" in x]
            if not same:
                same = [run_e(args.e_per_call)]
                e_runs.append(same[0])
            if "wall_s" in pc and "wall_s" in same[0]:
                pc["per_call_over_tree"] = round(pc["wall_s"] / same[0]["wall_s"], 2)
                pc["same_md5"] = pc.get("md5") == same[0].get("md5")
            e_runs.append(pc)

    # ---- CPU baseline: the reference multiply on the host cores, bounded sample
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        import oracle as orc
        if orc.have_reference("omp"):
            # a bounded sample of about 10 s of CPU work (0.4 s per product on 16 threads)
            nrep = 24
            ral, rbl, rcl, rdt, thr = time_reference(REF_LOG2, reps=nrep, kind="omp")
            rp = bc.plan(ral, rbl, rcl)
            rb_alg = bc.width_limit(rp["fft_points"])
            cpu = {"value": round(alg_bytes(ral, rbl, rcl, rb_alg, False) / rdt / 1e9, 4), "unit": "GB/s",
                   "cores": thr, "kind": "reference",
                   "sample": "reference _fft_mul from oracle/_ref (OpenMP tasks, %d threads), %d multiplies of "
                             "2^20 x 2^20 limbs (largest size it supports), %.3f s each" % (thr, nrep, rdt)}
        else:
            sa, sb = operands(16)
            t0 = time.perf_counter()
            orc.restated().fft_mul(sa, sb)
            dt = time.perf_counter() - t0
            rp = bc.plan(sa.size, sb.size, sa.size + sb.size)
            cpu = {"value": round(alg_bytes(sa.size, sb.size, sa.size + sb.size, bc.width_limit(rp["fft_points"]), False) / dt / 1e9, 4),
                   "unit": "GB/s", "cores": 1, "kind": "port", "sample": "oracle restatement, one 2^16 x 2^16 multiply"}

    # ---- same-workload pairs with the reference, at the sizes it can run:
    # (1) the exact multiply of 2^20 x 2^20 limbs (the cpu_baseline workload),
    #     device-resident and through the C ABI with host buffers;
    # (2) e to 10^7 digits by this repository's CLI and by the reference CLI.
    same = []
    if rank == 0 and world == 1 and not args.no_cpu and cpu and cpu.get("kind") == "reference":
        try:
            same.append(same_config_mul(bc, torch, stream, cpu))
        except Exception as exc:
            same.append({"workload": "exact multiply 2^20 x 2^20 limbs", "error": str(exc)[:300]})
        if args.e_same:
            g = run_e(args.e_same)
            r = reference_cli_e(args.e_same)
            pair = {"workload": "e to %d decimal digits, end to end (CLI, output files, md5)" % args.e_same,
                    "unit": "s", "higher_is_better": False, "gpu": g, "reference": r}
            if r and g.get("wall_s") and r.get("wall_s"):
                pair["reference_over_gpu"] = round(r["wall_s"] / g["wall_s"], 2)
                pair["same_digits"] = g.get("md5") == r.get("md5")
            same.append(pair)

    if rank == 0:
        line = {
            "metric": "exact_mul_GBps", "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": round(ms, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "exact multiply 2^%d x 2^%d limbs (SplitMix64 seeded, uniform limbs)" % (log2n, log2n),
                       "AL": AL, "BL": BL, "CL": CL, "fft_points": M, "levels": p["levels"],
                       "width": st["width"], "width_for_formula": b_alg, "max_round_err": st["max_round_err"],
                       "l2": "inputs and work buffers larger than L2 (no flush)",
                       "parallelism": "replicas" if world > 1 else "single"},
            "e2e": {"value": round(e2e, 2), "unit": "GB/s", "ms_per_step": round(e2e_ms, 3),
                    "h2d_bytes_per_step": 4 * (AL + BL), "d2h_bytes_per_step": 4 * CL,
                    "path": "bc_gpu_mul with pinned host buffers"},
            "roofline": roof,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "sweep": sweep,
            "batched": batched,
            "e": e_runs,
            "same_config": same,
        }
        print(json.dumps(line), flush=True)
    ranks.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bluecrunch_b200")
    ap.add_argument("--log2", type=int, default=HEADLINE_LOG2)
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-items", type=int, default=8192)
    ap.add_argument("--e-digits", default="100000000,1000000000",
                    help="e to these numbers of digits, comma-separated (0: skip)")
    ap.add_argument("--e-per-call", type=int, default=1000000000,
                    help="also e to this many digits with one GPU product per call (0: skip); the default-mode "
                         "run of the same size comes from --e-digits")
    ap.add_argument("--e-same", type=int, default=10000000,
                    help="e to this many digits by this CLI and by the reference CLI (same workload; 0: skip)")
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
