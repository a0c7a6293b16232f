"""ctypes binding of the C ABI in include/ffb200.h (lib/libffb200.so).

The Python side is a thin caller of the library: every computation happens in the CUDA
kernels behind the C entry points. Loading fails loudly when the library has not been
built (there is no fallback).
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libffb200.so")

u8p = ctypes.POINTER(ctypes.c_uint8)
u32p = ctypes.POINTER(ctypes.c_uint32)
u64p = ctypes.POINTER(ctypes.c_uint64)


class GpuRecord(ctypes.Structure):
    """source/m4/gpu_search_kernel.h:37-42 (sizeof 32)."""
    _fields_ = [("sum", ctypes.c_uint32), ("low", ctypes.c_uint64),
                ("high", ctypes.c_uint64), ("tag", ctypes.c_uint8)]


class FfbBatchInfo(ctypes.Structure):
    _fields_ = [("ranges", ctypes.c_uint32), ("intervals", ctypes.c_uint32),
                ("sums", ctypes.c_uint64), ("mapMaxValue", ctypes.c_uint64),
                ("mapBytes", ctypes.c_uint64), ("sieveTileBytes", ctypes.c_uint32),
                ("searchWarps", ctypes.c_uint32), ("autotuned", ctypes.c_int),
                ("sieveMs", ctypes.c_float), ("searchMs", ctypes.c_float),
                ("searchChunk", ctypes.c_uint32), ("searchGroup", ctypes.c_uint32)]


class FfbGeometry(ctypes.Structure):
    _fields_ = [("sumStart", ctypes.c_uint32), ("sumLimit", ctypes.c_uint32),
                ("maxPrimeMapValue", ctypes.c_uint64), ("mapBytes", ctypes.c_uint64),
                ("numPrimesRequested", ctypes.c_uint64), ("pmapSumLimit", ctypes.c_uint64)]


class FfbBudget(ctypes.Structure):
    """source/budget.h:23-33 (DeviceBudget)."""
    _fields_ = [("fraction", ctypes.c_double), ("freeQueried", ctypes.c_ulonglong),
                ("freeUsed", ctypes.c_ulonglong), ("cap", ctypes.c_ulonglong),
                ("budget", ctypes.c_ulonglong), ("scratch", ctypes.c_ulonglong),
                ("headroom", ctypes.c_ulonglong), ("backing", ctypes.c_ulonglong),
                ("slabCount", ctypes.c_ulonglong)]


class FfbServeConfig(ctypes.Structure):
    _fields_ = [("vramBudgetBytes", ctypes.c_uint64), ("vramFraction", ctypes.c_double),
                ("slots", ctypes.c_uint32), ("launchWork", ctypes.c_uint32),
                ("launchSums", ctypes.c_uint32), ("searchWarps", ctypes.c_uint32),
                ("warmLimit", ctypes.c_uint32)]


class FfbServeChunk(ctypes.Structure):
    _fields_ = [("request", ctypes.c_uint64), ("seq", ctypes.c_uint32), ("status", ctypes.c_int32),
                ("text", ctypes.c_void_p), ("len", ctypes.c_size_t)]


class FfbPeaks(ctypes.Structure):
    """Measured on-chip peaks (ffb_measure_peaks), operations per second."""
    _fields_ = [("imad32PerS", ctypes.c_double), ("alu32PerS", ctypes.c_double),
                ("mul64PerS", ctypes.c_double), ("intOpsPerS", ctypes.c_double),
                ("atomsConflictFreePerS", ctypes.c_double), ("atomsRandomPerS", ctypes.c_double),
                ("smemRmwPerS", ctypes.c_double), ("sms", ctypes.c_int), ("clockMhz", ctypes.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class FfbServeRequestInfo(ctypes.Structure):
    _fields_ = [("sumStart", ctypes.c_uint32), ("sumLimit", ctypes.c_uint32),
                ("sums", ctypes.c_uint64), ("textBytes", ctypes.c_uint64),
                ("bodyHash", ctypes.c_uint64), ("submitUs", ctypes.c_double),
                ("admitUs", ctypes.c_double), ("firstChunkUs", ctypes.c_double),
                ("doneUs", ctypes.c_double), ("launches", ctypes.c_uint32),
                ("state", ctypes.c_int32)]


class FfbServeInfo(ctypes.Structure):
    _fields_ = [("budget", FfbBudget), ("mapBytes", ctypes.c_uint64),
                ("mapMaxValue", ctypes.c_uint64), ("requests", ctypes.c_uint64),
                ("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64),
                ("launches", ctypes.c_uint64), ("sumsRequested", ctypes.c_uint64),
                ("sumsSearched", ctypes.c_uint64), ("chunks", ctypes.c_uint64),
                ("textBytes", ctypes.c_uint64), ("slots", ctypes.c_uint32),
                ("maxQueued", ctypes.c_uint32), ("sieveMs", ctypes.c_double),
                ("searchMs", ctypes.c_double), ("stage1Probes", ctypes.c_uint64),
                ("stage2Items", ctypes.c_uint64), ("mrCandidates", ctypes.c_uint64),
                ("mrBase2Passed", ctypes.c_uint64)]


# name -> (restype, argtypes); every symbol include/ffb200.h declares
SIGNATURES = {
    "SieveSlabRun_sm_100a": (ctypes.c_int, [ctypes.c_int, u32p, ctypes.c_uint32, ctypes.c_uint64,
                                            ctypes.c_uint64, u8p]),
    "SieveSlabGetLaunchFn_sm_100a": (ctypes.c_void_p, [ctypes.c_int]),
    "SieveSlabRun_sm_120": (ctypes.c_int, [ctypes.c_int, u32p, ctypes.c_uint32, ctypes.c_uint64,
                                           ctypes.c_uint64, u8p]),
    "SieveSlabGetLaunchFn_sm_120": (ctypes.c_void_p, [ctypes.c_int]),
    "SieveSlabGetLaunchFn_gfx1201": (ctypes.c_void_p, [ctypes.c_int]),
    "SieveSlabEngineRun_sm_100a": (ctypes.c_int, [ctypes.c_int, u32p, ctypes.c_uint32,
                                                  ctypes.c_uint64, u8p]),
    "SieveSlabEngineGetLaunchFn_sm_100a": (ctypes.c_void_p, [ctypes.c_int]),
    "SieveSlabEngineRun_sm_120": (ctypes.c_int, [ctypes.c_int, u32p, ctypes.c_uint32,
                                                 ctypes.c_uint64, u8p]),
    "SieveSlabEngineGetLaunchFn_sm_120": (ctypes.c_void_p, [ctypes.c_int]),
    "SieveSlabEngineGetLaunchFn_gfx1201": (ctypes.c_void_p, [ctypes.c_int]),
    "SievePoolGet_sm_100a": (ctypes.c_void_p, [ctypes.c_int]),
    "SievePoolGet_sm_120": (ctypes.c_void_p, [ctypes.c_int]),
    "SievePoolGet_gfx1201": (ctypes.c_void_p, [ctypes.c_int]),
    "SearchKernelRun_sm_100a": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                                               ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p,
                                               ctypes.c_void_p]),
    "SearchKernelGetLaunchFn_sm_100a": (ctypes.c_void_p, [ctypes.c_int]),
    "SearchKernelRun_sm_120": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                                              ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p,
                                              ctypes.c_void_p]),
    "SearchKernelGetLaunchFn_sm_120": (ctypes.c_void_p, [ctypes.c_int]),
    "SearchKernelGetLaunchFn_gfx1201": (ctypes.c_void_p, [ctypes.c_int]),
    "GpuSearchLaunch": (ctypes.c_int, [ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p,
                                       ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                       ctypes.c_void_p, ctypes.c_void_p]),
    "ffb_format_line": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_char_p, ctypes.c_size_t]),
    "ffb_geometry": (ctypes.c_int, [ctypes.c_int, ctypes.c_int32, ctypes.c_int32,
                                    ctypes.POINTER(FfbGeometry), ctypes.c_char_p, ctypes.c_size_t]),
    "ffb_schedule": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                    ctypes.c_uint32, u32p, u32p, ctypes.c_int]),
    "ffb_sieve_map_async": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.c_void_p,
                                           ctypes.c_void_p]),
    "ffb_sieve_map_tiled_async": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.c_void_p,
                                                 ctypes.c_uint32, ctypes.c_void_p]),
    "ffb_search_async": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                                        ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p,
                                        ctypes.c_void_p]),
    "ffb_take_errors": (ctypes.c_int, [ctypes.c_int, u32p]),
    "ffb_sieve_map_range_async": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64,
                                                 ctypes.c_void_p, ctypes.c_void_p]),
    "ffb_measure_peaks": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(FfbPeaks)]),
    "ffb_probe_bound": (ctypes.c_uint64, [ctypes.c_uint32]),
    "ffb_search_stats": (ctypes.c_int, [ctypes.c_int, u64p, ctypes.c_int]),
    "ffb_search_shape_async": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                                              ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p,
                                              ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                              ctypes.c_void_p]),
    "ffb_search_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                                          ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p]),
    "ffb_context_create": (ctypes.c_void_p, [ctypes.c_int]),
    "ffb_context_destroy": (None, [ctypes.c_void_p]),
    "ffb_context_set_map_budget": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "ffb_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int32, ctypes.c_int32,
                               ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t)]),
    "ffb_free": (None, [ctypes.c_void_p]),
    "ffb_map_dump": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int32, ctypes.c_int32,
                                    ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_uint64),
                                    ctypes.c_char_p, ctypes.c_size_t]),
    "ffb_emit": (ctypes.c_int, [ctypes.c_int, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double, ctypes.c_double,
                                ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t)]),
    "ffb_batch_create": (ctypes.c_void_p, [ctypes.c_int, ctypes.c_uint32,
                                           ctypes.POINTER(ctypes.c_int32),
                                           ctypes.POINTER(ctypes.c_int32), ctypes.c_int]),
    "ffb_batch_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "ffb_batch_collect": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                         ctypes.POINTER(ctypes.c_size_t)]),
    "ffb_batch_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(FfbBatchInfo)]),
    "ffb_batch_destroy": (None, [ctypes.c_void_p]),
    "ffb_compute_budget": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_double, ctypes.c_uint64,
                                          ctypes.c_uint64, ctypes.c_uint64,
                                          ctypes.POINTER(FfbBudget)]),
    "ffb_shrink_budget": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_double, ctypes.c_uint64,
                                         ctypes.c_uint64, ctypes.c_uint64,
                                         ctypes.POINTER(FfbBudget)]),
    "ffb_serve_create": (ctypes.c_void_p, [ctypes.c_int, ctypes.POINTER(FfbServeConfig)]),
    "ffb_serve_submit": (ctypes.c_int64, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int32,
                                          ctypes.c_int32]),
    "ffb_serve_next": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(FfbServeChunk), ctypes.c_int]),
    "ffb_serve_request_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64,
                                              ctypes.POINTER(FfbServeRequestInfo)]),
    "ffb_serve_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(FfbServeInfo)]),
    "ffb_serve_drain": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "ffb_serve_destroy": (None, [ctypes.c_void_p]),
}

_lib = None


def load():
    """The library handle with argument types set; raises if the library is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built (run `make -C ff-gpu_b200`)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def geometry(*args):
    """ffb_geometry for 0, 1 or 2 atoi()-style positional arguments -> (FfbGeometry, header)."""
    lib = load()
    g = FfbGeometry()
    buf = ctypes.create_string_buffer(4096)
    a = list(args) + [0, 0]
    n = lib.ffb_geometry(len(args), a[0], a[1], ctypes.byref(g), buf, len(buf))
    if n < 0:
        raise ValueError(buf.value.decode())
    return g, buf.raw[:n]


def schedule(sum_start, sum_limit, mpv, threads=31):
    lib = load()
    cap = 8 * threads + 8
    f = (ctypes.c_uint32 * cap)()
    l = (ctypes.c_uint32 * cap)()
    n = lib.ffb_schedule(sum_start, sum_limit, mpv, threads, f, l, cap)
    if n < 0:
        raise ValueError("schedule failed")
    return [(f[i], l[i]) for i in range(n)]


def format_line(count, s, low, high, low_prime, high_prime):
    lib = load()
    buf = ctypes.create_string_buffer(256)
    n = lib.ffb_format_line(count, s, low, high, int(low_prime), int(high_prime), buf, len(buf))
    return buf.raw[:n]


def run(*args, ctx=None):
    """The full ff_sieve stdout for the positional arguments, as bytes."""
    lib = load()
    p = ctypes.c_void_p()
    n = ctypes.c_size_t()
    rc = lib.ffb_run(ctx, len(args), *(list(args) + [0, 0])[:2], ctypes.byref(p), ctypes.byref(n))
    if rc != 0:
        raise RuntimeError(f"ffb_run{args} failed")
    try:
        return ctypes.string_at(p, n.value)
    finally:
        lib.ffb_free(p)


def emit(args, records, rec_lo, prime_us=0.0, freud_us=0.0):
    """ffb_emit: ff_seg's stdout from packed records (numpy uint64/int64 array, odd sums from
    rec_lo) computed elsewhere."""
    import numpy as np
    lib = load()
    rec = np.ascontiguousarray(records).view(np.uint64)
    p = ctypes.c_void_p()
    n = ctypes.c_size_t()
    a = [int(x) for x in args] + [0, 0]
    rc = lib.ffb_emit(len(args), a[0], a[1], rec.ctypes.data, rec_lo, rec.size, prime_us,
                      freud_us, ctypes.byref(p), ctypes.byref(n))
    if rc != 0:
        raise ValueError(f"ffb_emit{tuple(args)} failed")
    try:
        return ctypes.string_at(p, n.value)
    finally:
        lib.ffb_free(p)


def map_dump(*args, dev=0):
    """ffb_map_dump: (map bytes, header text) of `ff_seg --dump-map <file> <args>`."""
    lib = load()
    p = ctypes.c_void_p()
    n = ctypes.c_uint64()
    hdr = ctypes.create_string_buffer(4096)
    a = [int(x) for x in args] + [0, 0]
    if lib.ffb_map_dump(dev, len(args), a[0], a[1], ctypes.byref(p), ctypes.byref(n), hdr,
                        len(hdr)) != 0:
        raise RuntimeError(f"ffb_map_dump{args} failed")
    try:
        return ctypes.string_at(p, n.value), hdr.value
    finally:
        lib.ffb_free(p)


def take_errors(dev=0):
    lib = load()
    f = ctypes.c_uint32()
    if lib.ffb_take_errors(dev, ctypes.byref(f)) != 0:
        raise RuntimeError("ffb_take_errors failed")
    return f.value


class Batch:
    """ffb_batch_*: many ranges (start, limit) evaluated together; .run() -> list of texts."""

    def __init__(self, ranges, dev=0, autotune=True):
        self.lib = load()
        n = len(ranges)
        self.n = n
        s = (ctypes.c_int32 * n)(*[int(a) for a, _ in ranges])
        l = (ctypes.c_int32 * n)(*[int(b) for _, b in ranges])
        self.h = self.lib.ffb_batch_create(dev, n, s, l, 1 if autotune else 0)
        if not self.h:
            raise RuntimeError("ffb_batch_create failed")

    def launch(self, stream=None):
        if self.lib.ffb_batch_launch(self.h, stream) != 0:
            raise RuntimeError("ffb_batch_launch failed")

    def collect(self):
        p = ctypes.c_void_p()
        off = (ctypes.c_size_t * (self.n + 1))()
        if self.lib.ffb_batch_collect(self.h, ctypes.byref(p), off) != 0:
            raise RuntimeError("ffb_batch_collect failed")
        try:
            raw = ctypes.string_at(p, off[self.n])
        finally:
            self.lib.ffb_free(p)
        return [raw[off[i]:off[i + 1]] for i in range(self.n)]

    def run(self):
        self.launch()
        return self.collect()

    def info(self):
        i = FfbBatchInfo()
        self.lib.ffb_batch_info(self.h, ctypes.byref(i))
        return {n: getattr(i, n) for n, _ in i._fields_}

    def close(self):
        if self.h:
            self.lib.ffb_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _struct_dict(st):
    out = {}
    for n, _ in st._fields_:
        v = getattr(st, n)
        out[n] = _struct_dict(v) if isinstance(v, ctypes.Structure) else v
    return out


def compute_budget(free_bytes, fraction=0.90, cap=0, scratch=0, slab=1 << 30, shrink=False):
    """computeBudget / shrinkFractionForAlloc of the reference as a dict."""
    lib = load()
    b = FfbBudget()
    fn = lib.ffb_shrink_budget if shrink else lib.ffb_compute_budget
    if fn(free_bytes, fraction, cap, scratch, slab, ctypes.byref(b)) != 0:
        raise ValueError("bad budget arguments")
    return _struct_dict(b)


class Server:
    """ffb_serve_*: submit(start, limit) -> id; next() -> (id, seq, status, bytes) chunks."""

    def __init__(self, dev=0, budget_bytes=8 << 30, fraction=0.90, slots=0, launch_work=0,
                 launch_sums=0, warps=0, warm_limit=0):
        self.lib = load()
        cfg = FfbServeConfig(budget_bytes, fraction, slots, launch_work, launch_sums, warps,
                             warm_limit)
        self.h = self.lib.ffb_serve_create(dev, ctypes.byref(cfg))
        if not self.h:
            raise RuntimeError("ffb_serve_create failed")

    def submit(self, *args):
        a = [int(x) for x in args] + [0, 0]
        rid = self.lib.ffb_serve_submit(self.h, len(args), a[0], a[1])
        if rid < 0:
            raise ValueError(f"request {args} rejected")
        return rid

    def next(self, timeout_ms=-1, keep_text=True):
        """(request, seq, status, text or length) or None on timeout."""
        c = FfbServeChunk()
        if self.lib.ffb_serve_next(self.h, ctypes.byref(c), timeout_ms) != 1:
            return None
        try:
            body = ctypes.string_at(c.text, c.len) if (keep_text and c.text) else c.len
        finally:
            if c.text:
                self.lib.ffb_free(c.text)
        return c.request, c.seq, c.status, body

    def collect(self, ids, timeout_ms=600000):
        """Texts of the given requests (bytes, None when failed), in the order of ids."""
        want = set(ids)
        parts = {i: [] for i in ids}
        failed = set()
        done = set()
        while done | failed != want:
            got = self.next(timeout_ms)
            if got is None:
                raise TimeoutError("no output within the timeout")
            rid, seq, status, text = got
            if rid not in parts:
                continue
            if status < 0:
                failed.add(rid)
                continue
            if seq != len(parts[rid]):
                raise RuntimeError(f"request {rid}: chunk {seq} out of order")
            parts[rid].append(text)
            if status == 1:
                done.add(rid)
        return [None if i in failed else b"".join(parts[i]) for i in ids]

    def request_info(self, rid):
        o = FfbServeRequestInfo()
        if self.lib.ffb_serve_request_info(self.h, rid, ctypes.byref(o)) != 0:
            raise KeyError(rid)
        return _struct_dict(o)

    def info(self):
        o = FfbServeInfo()
        self.lib.ffb_serve_info(self.h, ctypes.byref(o))
        return _struct_dict(o)

    def drain(self, timeout_ms=-1):
        return self.lib.ffb_serve_drain(self.h, timeout_ms) == 0

    def close(self):
        if self.h:
            self.lib.ffb_serve_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def measure_peaks(dev=0):
    """ffb_measure_peaks as a dict (operations per second)."""
    p = FfbPeaks()
    if load().ffb_measure_peaks(dev, ctypes.byref(p)) != 0:
        raise RuntimeError("ffb_measure_peaks failed")
    return p.as_dict()
