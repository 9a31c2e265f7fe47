"""bluecrunch_b200 — exact big-integer multiply on B200 for bluecrunch's e.

Python view of the native libraries built in this directory:

* ``libbcgpu.so``      — the CUDA engine behind include/bc_gpu.h (the device
  side of the reference's ``_fft_mul``, bigfloat/mul.c:108-174);
* ``libbluecrunch.so`` — the host C bigfloat library (include/bigfloat.h,
  include/mul.h) whose ``_fft_mul`` forwards to the engine.

Operands are little-endian base-2^32 limb arrays (numpy ``uint32``, or CUDA
tensors whose ``data_ptr()`` is passed through as device memory).  There is
no CPU fallback: if the native library is missing or no sm_100 GPU is present
the calls raise.
"""
import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
GPU_LIB = os.path.join(PKG, "libbcgpu.so")
HOST_LIB = os.path.join(PKG, "libbluecrunch.so")
CLI = os.path.join(PKG, "bluecrunch")

BC_OK = 0
ERRORS = {
    -1: "BC_ERR_INVALID", -2: "BC_ERR_NOMEM", -3: "BC_ERR_CUDA", -4: "BC_ERR_TIMEOUT",
    -5: "BC_ERR_PRECISION", -6: "BC_ERR_NOT_INIT", -7: "BC_ERR_TOO_LARGE",
    -8: "BC_ERR_NO_DEVICE", -9: "BC_ERR_CARRY", -10: "BC_ERR_IO",
}

_u32p = ctypes.POINTER(ctypes.c_uint32)
_sz = ctypes.c_size_t


class BcError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        msg = _lib().bc_gpu_strerror(code).decode() if _LIB else ERRORS.get(code, str(code))
        super().__init__("%s (%s)%s" % (ERRORS.get(code, code), msg, (": " + what) if what else ""))


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("arena_bytes", _sz), ("tune_path", ctypes.c_char_p),
                ("max_round_err", ctypes.c_double), ("verbose", ctypes.c_int)]


class MulStats(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("retries", ctypes.c_int), ("fft_points", _sz),
                ("max_round_err", ctypes.c_double), ("device_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double)]


class MulDesc(ctypes.Structure):
    _fields_ = [("C", ctypes.c_void_p), ("CL", _sz), ("A", ctypes.c_void_p), ("AL", _sz),
                ("B", ctypes.c_void_p), ("BL", _sz)]


class BatchStats(ctypes.Structure):
    _fields_ = [("items", _sz), ("classes", _sz), ("launches", _sz), ("retries", ctypes.c_int),
                ("max_round_err", ctypes.c_double), ("device_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double), ("h2d_bytes", _sz), ("d2h_bytes", _sz),
                ("graph_launches", _sz), ("graph_nodes", _sz), ("graph_updates", _sz)]


BATCH_HOST_OPERANDS, BATCH_DEVICE_OPERANDS, BATCH_GRAPH = 1, 2, 4


class PlanInfo(ctypes.Structure):
    _fields_ = [("fft_points", _sz), ("width", ctypes.c_int), ("levels", ctypes.c_int),
                ("L1", ctypes.c_int), ("L2", ctypes.c_int), ("Lr", ctypes.c_int),
                ("digits_a", _sz), ("digits_b", _sz), ("out_words", _sz), ("work_bytes", _sz)]


# Every symbol include/bc_gpu.h declares, with its ctypes signature.
GPU_SYMBOLS = {
    "bc_gpu_init": (ctypes.c_int, [ctypes.POINTER(Config)]),
    "bc_gpu_shutdown": (ctypes.c_int, []),
    "bc_gpu_mul": (ctypes.c_int, [ctypes.c_void_p, _sz, ctypes.c_void_p, _sz, ctypes.c_void_p, _sz,
                                  ctypes.POINTER(MulStats)]),
    "bc_gpu_mul_batch": (ctypes.c_int, [ctypes.POINTER(MulDesc), _sz, ctypes.POINTER(BatchStats)]),
    "bc_gpu_mul_batch_flags": (ctypes.c_int, [ctypes.POINTER(MulDesc), _sz, ctypes.c_uint, ctypes.POINTER(BatchStats)]),
    "bc_gpu_radix_leaves": (ctypes.c_int, [ctypes.c_void_p, _sz, ctypes.c_double]),
    "bc_gpu_radix_tree": (ctypes.c_int, [ctypes.c_void_p, _sz, ctypes.c_void_p, _sz, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_int, ctypes.c_double, ctypes.c_void_p]),
    "bc_gpu_selftest_wait": (ctypes.c_int, [ctypes.POINTER(ctypes.c_double)]),
    "bc_gpu_newton": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                     _sz, ctypes.c_void_p]),
    "bc_gpu_radix_tree_pow": (ctypes.c_int, [ctypes.c_void_p, _sz, ctypes.c_void_p, _sz, ctypes.c_void_p, _sz,
                                             ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p]),
    "bc_gpu_e_series": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ctypes.POINTER(ctypes.c_uint32)),
                                       ctypes.POINTER(_sz), ctypes.POINTER(ctypes.POINTER(ctypes.c_uint32)),
                                       ctypes.POINTER(_sz)]),
    "bc_gpu_mul_small_batch": (ctypes.c_int, [ctypes.POINTER(MulDesc), _sz]),
    "bc_gpu_decimal_write": (ctypes.c_int, [ctypes.c_void_p, _sz, _sz, _sz, ctypes.c_int, ctypes.c_longlong]),
    "bc_gpu_device_alloc": (ctypes.c_int, [_sz, ctypes.POINTER(ctypes.c_void_p)]),
    "bc_gpu_device_free": (ctypes.c_int, [ctypes.c_void_p]),
    "bc_gpu_copy": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, _sz]),
    "bc_gpu_set_stream": (ctypes.c_int, [ctypes.c_void_p]),
    "bc_gpu_plan": (ctypes.c_int, [_sz, _sz, _sz, ctypes.c_int, ctypes.POINTER(PlanInfo)]),
    "bc_gpu_width_limit": (ctypes.c_int, [_sz]),
    "bc_gpu_set_width_limit": (ctypes.c_int, [_sz, ctypes.c_int]),
    "bc_gpu_force_width": (ctypes.c_int, [ctypes.c_int]),
    "bc_gpu_force_plan": (ctypes.c_int, [_sz, ctypes.c_int]),
    "bc_gpu_lengths": (ctypes.c_int, [ctypes.POINTER(_sz), ctypes.c_int]),
    "bc_gpu_check_shapes": (ctypes.c_int, []),
    "bc_gpu_load_width_table": (ctypes.c_int, [ctypes.c_char_p]),
    "bc_gpu_shape_candidates": (ctypes.c_int, [_sz, ctypes.POINTER(ctypes.c_int), ctypes.c_int]),
    "bc_gpu_set_shape": (ctypes.c_int, [_sz, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "bc_gpu_load_shape_table": (ctypes.c_int, [ctypes.c_char_p]),
    "bc_gpu_mul_noalloc": (ctypes.c_int, [ctypes.c_void_p, _sz, ctypes.c_void_p, _sz, ctypes.c_void_p, _sz,
                                          ctypes.c_void_p]),
    "bc_gpu_sync": (ctypes.c_int, []),
    "bc_gpu_last_error": (ctypes.c_int, []),
    "bc_gpu_last_cuda_error": (ctypes.c_int, []),
    "bc_gpu_strerror": (ctypes.c_char_p, [ctypes.c_int]),
    "bc_gpu_time_kernels": (ctypes.c_int, [ctypes.c_int]),
    "bc_gpu_kernel_times": (ctypes.c_int, [ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_double),
                                           ctypes.c_int]),
}

_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(GPU_LIB):
            raise OSError("native library %s is missing: run `python -m bluecrunch_b200.build`" % GPU_LIB)
        lib = ctypes.CDLL(GPU_LIB)
        for name, (res, args) in GPU_SYMBOLS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def _check(code, what=""):
    if code != BC_OK:
        raise BcError(code, what)


def init(device=0, arena_bytes=0, tune_path=None, max_round_err=0.25, verbose=0):
    global _widths_loaded
    if tune_path is None:
        default = os.path.join(PKG, "tune", "widths.txt")
        tune_path = default if os.path.exists(default) else None
    _widths_loaded = bool(tune_path)
    cfg = Config(device, arena_bytes, tune_path.encode() if tune_path else None, max_round_err, verbose)
    _check(_lib().bc_gpu_init(ctypes.byref(cfg)), "bc_gpu_init")


def shutdown():
    _check(_lib().bc_gpu_shutdown())


def _ptr_len(x):
    """(pointer, length, keepalive) for a numpy uint32 array or a CUDA tensor."""
    if hasattr(x, "data_ptr"):  # torch tensor (device or host)
        return x.data_ptr(), x.numel(), x
    x = np.ascontiguousarray(x, dtype=np.uint32)
    return x.ctypes.data, x.size, x


def mul(a, b=None, CL=None, square=False, out=None, want_stats=False):
    """C = A*B mod 2^(32*CL) (CL defaults to AL+BL).  Squares when b is None
    or square=True (the same buffer is passed twice, as _fft_mul detects)."""
    pa, al, ka = _ptr_len(a)
    if square or b is None:
        pb, bl, kb = pa, al, ka
    else:
        pb, bl, kb = _ptr_len(b)
    if CL is None:
        CL = al + bl
    if out is None:
        out = np.zeros(CL, dtype=np.uint32)
    pc, cl, kc = _ptr_len(out)
    if cl < CL:
        raise ValueError("output buffer too small")
    st = MulStats()
    _check(_lib().bc_gpu_mul(pc, CL, pa, al, pb, bl, ctypes.byref(st)), "bc_gpu_mul")
    del ka, kb, kc
    if want_stats:
        return out, {k: getattr(st, k) for k, _ in MulStats._fields_}
    return out


def mul_batch(items, want_stats=False):
    """items: list of (a, b_or_None, CL_or_None).  Returns the list of outputs."""
    descs = (MulDesc * len(items))()
    keep, outs = [], []
    for i, (a, b, CL) in enumerate(items):
        pa, al, ka = _ptr_len(a)
        if b is None:
            pb, bl, kb = pa, al, ka
        else:
            pb, bl, kb = _ptr_len(b)
        CL = CL or (al + bl)
        out = np.zeros(CL, dtype=np.uint32)
        outs.append(out)
        keep += [ka, kb]
        descs[i] = MulDesc(out.ctypes.data, CL, pa, al, pb, bl)
    st = BatchStats()
    _check(_lib().bc_gpu_mul_batch(descs, len(items), ctypes.byref(st)), "bc_gpu_mul_batch")
    if want_stats:
        return outs, {k: getattr(st, k) for k, _ in BatchStats._fields_}
    return outs


def mul_small_batch(items):
    """Exact small products in one launch (bc_gpu_mul_small_batch): items are
    (a, b, CL_or_None) of numpy uint32 limbs, at most 256 limbs per operand
    and 512 per product.  Returns the list of outputs."""
    descs = (MulDesc * max(len(items), 1))()
    keep, outs = [], []
    for i, (a, b, CL) in enumerate(items):
        a = np.ascontiguousarray(a, dtype=np.uint32)
        b = np.ascontiguousarray(b, dtype=np.uint32)
        CL = (a.size + b.size) if CL is None else CL
        out = np.zeros(max(CL, 1), dtype=np.uint32)
        keep += [a, b]
        outs.append(out[:CL])
        descs[i] = MulDesc(out.ctypes.data, CL, a.ctypes.data, a.size, b.ctypes.data, b.size)
    _check(_lib().bc_gpu_mul_small_batch(descs, len(items)), "bc_gpu_mul_small_batch")
    del keep
    return outs


def decimal_write(limbs, top, n, maxbytes, fd, offset=0):
    """Nine decimal characters per limb for limbs[top], limbs[top-1], ...,
    limbs[top-n+1], cut at maxbytes bytes, written at byte `offset` of the
    open file descriptor fd (bc_gpu_decimal_write).  limbs: numpy uint32 or
    a CUDA tensor (device memory)."""
    p, _, keep = _ptr_len(limbs)
    _check(_lib().bc_gpu_decimal_write(p, top, n, maxbytes, fd, offset), "bc_gpu_decimal_write")
    del keep


def mul_batch_desc(descs, n, flags=0):
    """Raw batch call on a prepared (MulDesc * n) array (bc_gpu_mul_batch, or
    bc_gpu_mul_batch_flags with `flags`, e.g. BATCH_GRAPH); returns stats dict."""
    st = BatchStats()
    if flags:
        _check(_lib().bc_gpu_mul_batch_flags(descs, n, flags, ctypes.byref(st)), "bc_gpu_mul_batch_flags")
    else:
        _check(_lib().bc_gpu_mul_batch(descs, n, ctypes.byref(st)), "bc_gpu_mul_batch")
    return {k: getattr(st, k) for k, _ in BatchStats._fields_}


TUNE_FILE = os.path.join(PKG, "tune", "widths.txt")
_widths_loaded = False


def load_width_table(path=TUNE_FILE):
    """Load the tuned width table into the library (no GPU needed)."""
    global _widths_loaded
    _check(_lib().bc_gpu_load_width_table(path.encode()), "bc_gpu_load_width_table")
    _widths_loaded = True


def plan(AL, BL, CL=None, square=False):
    if not _widths_loaded and os.path.exists(TUNE_FILE):
        load_width_table()
    info = PlanInfo()
    _check(_lib().bc_gpu_plan(AL, BL, CL or (AL + BL), int(square), ctypes.byref(info)), "bc_gpu_plan")
    return {k: getattr(info, k) for k, _ in PlanInfo._fields_}


def width_limit(M):
    return _lib().bc_gpu_width_limit(M)


def set_width_limit(M, width):
    _check(_lib().bc_gpu_set_width_limit(M, width))


def force_width(width):
    _check(_lib().bc_gpu_force_width(width))


def force_plan(fft_points, width):
    _check(_lib().bc_gpu_force_plan(fft_points, width))


def shape_candidates(M):
    """Valid decompositions of transform length M: list of (levels, L1, L2, Lr)."""
    n = _lib().bc_gpu_shape_candidates(M, None, 0)
    buf = (ctypes.c_int * (4 * max(n, 1)))()
    _lib().bc_gpu_shape_candidates(M, buf, n)
    return [tuple(buf[4 * i:4 * i + 4]) for i in range(n)]


def set_shape(M, L1=0, L2=0, Lr=0):
    """Run transform length M as L1 x L2 x Lr (L2 = 1: two levels); zeros: built-in."""
    _check(_lib().bc_gpu_set_shape(M, L1, L2, Lr), "bc_gpu_set_shape")


SHAPE_FILE = os.path.join(PKG, "tune", "shapes.txt")


def lengths():
    """Supported transform lengths M (2^k and 3*2^k with a kernel shape)."""
    n = _lib().bc_gpu_lengths(None, 0)
    buf = (_sz * n)()
    _lib().bc_gpu_lengths(buf, n)
    return list(buf)


def set_stream(ptr):
    _check(_lib().bc_gpu_set_stream(ctypes.c_void_p(ptr)))


def time_kernels(on=True):
    _check(_lib().bc_gpu_time_kernels(int(on)))


def kernel_times():
    n = _lib().bc_gpu_kernel_times(None, None, 0)
    names = (ctypes.c_char_p * max(n, 1))()
    ms = (ctypes.c_double * max(n, 1))()
    _lib().bc_gpu_kernel_times(names, ms, n)
    return [(names[i].decode(), ms[i]) for i in range(n)]


def to_int(words):
    """Python int of a little-endian uint32 limb array (test helper)."""
    return int.from_bytes(np.ascontiguousarray(words, dtype="<u4").tobytes(), "little")


def from_int(x, n):
    return np.frombuffer(int(x).to_bytes(4 * n, "little"), dtype="<u4").copy()
