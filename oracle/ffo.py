"""ctypes binding of the CPU restatement (oracle/liboracle.so). Test infrastructure only:
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it as the checker."""
import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


class Counters(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ("sums", "map_probes", "mr_calls", "mr_mulmods", "splits", "abop_calls",
                 "trial_steps", "divisors", "errors")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class Geometry(ctypes.Structure):
    _fields_ = [("sum_start", ctypes.c_uint32), ("sum_limit", ctypes.c_uint32),
                ("max_generated_prime", ctypes.c_uint32), ("product_limit", ctypes.c_uint64),
                ("prime_limit", ctypes.c_uint64), ("num_primes_requested", ctypes.c_uint64),
                ("max_prime_map_value", ctypes.c_uint64), ("prime_map_bytes", ctypes.c_uint64),
                ("sqrt_limit", ctypes.c_uint64), ("pmap_sum_limit", ctypes.c_uint64),
                ("renormalised", ctypes.c_int), ("too_big", ctypes.c_int)]


_lib = None
u8p = ctypes.POINTER(ctypes.c_uint8)
u32p = ctypes.POINTER(ctypes.c_uint32)
u64p = ctypes.POINTER(ctypes.c_uint64)


def build():
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        sig = {
            "ffo_isqrt64": (ctypes.c_uint64, [ctypes.c_uint64]),
            "ffo_geometry_headers": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32,
                                                    ctypes.POINTER(Geometry), ctypes.c_char_p,
                                                    ctypes.c_size_t]),
            "ffo_parse_args": (None, [ctypes.c_int, ctypes.c_int32, ctypes.c_int32, u32p, u32p]),
            "ffo_schedule": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                            ctypes.c_uint32, u32p, u32p, ctypes.c_int]),
            "ffo_segment_fill": (None, [ctypes.c_uint64, ctypes.c_uint64, u32p, ctypes.c_uint32, u8p]),
            "ffo_slab_relative": (None, [ctypes.c_uint64, ctypes.c_uint64, u32p, ctypes.c_uint32, u8p]),
            "ffo_odd_primes": (ctypes.c_uint64, [ctypes.c_uint64, u32p, ctypes.c_uint64]),
            "ffo_build_map": (ctypes.c_int, [ctypes.c_uint64, u8p, ctypes.c_int]),
            "ffo_miller_rabin": (ctypes.c_int, [ctypes.c_uint64]),
            "ffo_create": (ctypes.c_void_p, [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int]),
            "ffo_destroy": (None, [ctypes.c_void_p]),
            "ffo_map_bound": (ctypes.c_uint64, [ctypes.c_void_p]),
            "ffo_is_prime": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
            "ffo_eval_sum": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, u32p, u32p,
                                            ctypes.POINTER(Counters)]),
            "ffo_eval_range": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                              u64p, ctypes.c_int, ctypes.POINTER(Counters)]),
            "ffo_format_line": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                               ctypes.c_uint32, ctypes.c_uint32, ctypes.c_char_p,
                                               ctypes.c_size_t]),
            "ffo_run": (ctypes.c_void_p, [ctypes.c_int, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_uint64, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(Counters)]),
            "ffo_free": (None, [ctypes.c_void_p]),
            "ffo_emit": (ctypes.c_void_p, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int32,
                                           ctypes.c_int32, u64p, ctypes.c_uint32, ctypes.c_uint64,
                                           ctypes.POINTER(ctypes.c_size_t)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def run(*args, map_bound=0, threads=8):
    """ff_seg's stdout (timing lines normalised to N) for the positional arguments."""
    lib = load()
    n = ctypes.c_size_t()
    k = Counters()
    a = list(args) + [0, 0]
    p = lib.ffo_run(len(args), a[0], a[1], map_bound, threads, ctypes.byref(n), ctypes.byref(k))
    if not p:
        raise ValueError(f"oracle cannot run {args}")
    try:
        return ctypes.string_at(p, n.value)
    finally:
        lib.ffo_free(p)


def run_counted(*args, map_bound=0, threads=8):
    lib = load()
    n = ctypes.c_size_t()
    k = Counters()
    a = list(args) + [0, 0]
    p = lib.ffo_run(len(args), a[0], a[1], map_bound, threads, ctypes.byref(n), ctypes.byref(k))
    if not p:
        raise ValueError(f"oracle cannot run {args}")
    try:
        return ctypes.string_at(p, n.value), k.as_dict()
    finally:
        lib.ffo_free(p)


class Context:
    """A bitmap up to map_bound (0: the reference's full map for max_sum) + trial primes."""

    def __init__(self, max_sum, map_bound=0, threads=8):
        self.lib = load()
        self.h = self.lib.ffo_create(max_sum, map_bound, threads)
        if not self.h:
            raise ValueError("oracle context")

    def close(self):
        if self.h:
            self.lib.ffo_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def is_prime(self, n):
        return bool(self.lib.ffo_is_prime(self.h, n))

    def eval_sum(self, s):
        lo, hi = ctypes.c_uint32(), ctypes.c_uint32()
        k = Counters()
        r = self.lib.ffo_eval_sum(self.h, s, ctypes.byref(lo), ctypes.byref(hi), ctypes.byref(k))
        return (lo.value, hi.value) if r else None

    def eval_range(self, lo, hi, threads=8):
        """Packed (low<<32|high or 0) per odd sum lo..hi."""
        import numpy as np
        n = (hi - lo) // 2 + 1
        out = np.zeros(n, dtype=np.uint64)
        k = Counters()
        rc = self.lib.ffo_eval_range(self.h, lo, hi, out.ctypes.data_as(u64p), threads, ctypes.byref(k))
        if rc:
            raise ValueError("eval_range")
        return out, k.as_dict()

    def emit(self, args, rec, rec_lo):
        """ff_seg's stdout (timing lines as N) for the argument list from per-sum records
        rec (numpy uint64, rec[(s - rec_lo)/2]) that cover its schedule."""
        import numpy as np
        rec = np.ascontiguousarray(rec, dtype=np.uint64)
        a = list(args) + [0, 0]
        n = ctypes.c_size_t()
        p = self.lib.ffo_emit(self.h, len(args), a[0], a[1], rec.ctypes.data_as(u64p), rec_lo,
                              len(rec), ctypes.byref(n))
        if not p:
            raise ValueError(f"records do not cover the schedule of {args}")
        try:
            return ctypes.string_at(p, n.value)
        finally:
            self.lib.ffo_free(p)


def odd_primes(limit):
    import numpy as np
    lib = load()
    n = lib.ffo_odd_primes(limit, None, 0)
    out = np.zeros(max(n, 1), dtype=np.uint32)
    lib.ffo_odd_primes(limit, out.ctypes.data_as(u32p), n)
    return out[:n]


def slab_relative(seg_lo, seg_hi, primes):
    """SieveSlabRun's expected output ((seg_hi+15)>>4 bytes)."""
    import numpy as np
    lib = load()
    pr = np.ascontiguousarray(primes, dtype=np.uint32)
    out = np.zeros((seg_hi + 15) >> 4, dtype=np.uint8)
    lib.ffo_slab_relative(seg_lo, seg_hi, pr.ctypes.data_as(u32p), len(pr), out.ctypes.data_as(u8p))
    return out


def build_map(mpv, threads=8):
    import numpy as np
    lib = load()
    out = np.zeros((mpv + 1 + 15) >> 4, dtype=np.uint8)
    lib.ffo_build_map(mpv, out.ctypes.data_as(u8p), threads)
    return out


def schedule(sum_start, sum_limit, mpv, threads=31):
    lib = load()
    cap = 8 * threads + 8
    f = (ctypes.c_uint32 * cap)()
    l = (ctypes.c_uint32 * cap)()
    n = lib.ffo_schedule(sum_start, sum_limit, mpv, threads, f, l, cap)
    if n < 0:
        raise ValueError("schedule")
    return [(f[i], l[i]) for i in range(n)]


def geometry(sum_start, sum_limit):
    lib = load()
    g = Geometry()
    buf = ctypes.create_string_buffer(4096)
    n = lib.ffo_geometry_headers(sum_start, sum_limit, ctypes.byref(g), buf, len(buf))
    return g, buf.raw[:max(n, 0)]


def parse_args(*args):
    lib = load()
    s, l = ctypes.c_uint32(), ctypes.c_uint32()
    a = list(args) + [0, 0]
    lib.ffo_parse_args(len(args), a[0], a[1], ctypes.byref(s), ctypes.byref(l))
    return s.value, l.value


def miller_rabin(n):
    return bool(load().ffo_miller_rabin(n))
