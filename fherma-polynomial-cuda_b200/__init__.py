"""Python host mirror of the B200 negacyclic product (ctypes over libnegacyclic.so).

Mirrors the reference plugin interface (src/fherma.h:46-48):

    state = fherma_init(Point(N, W, L, q))     # parameter-only plan
    out   = fherma_run(state, Inputs(a, b))    # Outputs(c), c = a*b mod (X^N+1, q)
    fherma_free(state)

with numpy [N][L] uint32 arrays in place of fherma::Tensor<uint32_t>, and
RuntimeError where the reference throws std::runtime_error. `Plan` is the
lower-level handle over the C ABI (include/negacyclic.h). Every call goes to
the CUDA library; there is no CPU implementation here, and importing fails
if the library has not been built.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "libnegacyclic.so")
SHIM_LIBRARY = os.path.join(HERE, "libfherma_negacyclic.so")

OK, EINVAL, ENOFIELDS, ESIZE, ECUDA, ENOMEM, ENODEV, EBUSY = range(8)
GEMM_AUTO, GEMM_SIMT, GEMM_TENSOR, GEMM_TENSOR_SINGLE = 0, 1, 2, 3
STATUS_REDUCE, STATUS_GEMM_MASK = 0x1, 0x1ffff00

EXPORTED = [
    "negacyclic_last_error", "negacyclic_init", "negacyclic_get_info", "negacyclic_run",
    "negacyclic_run_device", "negacyclic_free", "negacyclic_host_plan", "negacyclic_debug_read",
    "negacyclic_gemm_u8", "negacyclic_run_device_timed", "negacyclic_work_bytes", "negacyclic_bind_work",
    "negacyclic_pipeline_status", "negacyclic_run_begin", "negacyclic_run_finish",
    "negacyclic_prepare_host", "negacyclic_run_device_static", "negacyclic_plan_status",
    "negacyclic_gemm_u8_withheld", "negacyclic_batch_status", "negacyclic_host_touch",
    "negacyclic_batch_create", "negacyclic_batch_io", "negacyclic_batch_get_info", "negacyclic_batch_run_device",
    "negacyclic_batch_run", "negacyclic_batch_run_one", "negacyclic_batch_run_plain", "negacyclic_batch_free",
    "negacyclic_server_create", "negacyclic_server_open_session", "negacyclic_server_submit",
    "negacyclic_server_wait", "negacyclic_server_get_stats", "negacyclic_server_free",
]
STAGES = ["pad", "convert", "forward", "pointwise", "inverse", "transpose", "crt", "reduce"]


class Options(ctypes.Structure):
    _fields_ = [("split", ctypes.c_uint32), ("gemm", ctypes.c_uint32), ("device", ctypes.c_int32),
                ("external_work", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 4)]


class Info(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint32) for name in
                ("n", "w", "limbs", "primes", "padded_primes", "split", "n_sub", "words", "gemm", "q_bits")] + \
               [("device_bytes", ctypes.c_uint64), ("table_bytes", ctypes.c_uint64),
                ("kernels_per_product", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class PointSpec(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("w", ctypes.c_uint32), ("limbs", ctypes.c_uint32),
                ("q", ctypes.c_void_p)]


class BatchOptions(ctypes.Structure):
    _fields_ = [("lanes", ctypes.c_uint32), ("tune", ctypes.c_uint32), ("device", ctypes.c_int32),
                ("reserved0", ctypes.c_uint32), ("tune_cache", ctypes.c_char_p), ("reserved", ctypes.c_uint32 * 4)]


class BatchInstance(ctypes.Structure):
    _fields_ = [("plan", Info), ("lane", ctypes.c_uint32), ("requested_gemm", ctypes.c_uint32),
                ("tuned_ms", ctypes.c_double), ("phase", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class ServerOptions(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_uint64), ("slots", ctypes.c_uint32), ("device", ctypes.c_int32),
                ("max_queue", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 3)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64), ("queued", ctypes.c_uint64),
                ("resident_bytes", ctypes.c_uint64), ("in_flight_bytes", ctypes.c_uint64),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
                ("products_per_s", ctypes.c_double), ("rejected", ctypes.c_uint64), ("max_queued", ctypes.c_uint64)]


_lib = None


def library() -> ctypes.CDLL:
    """Loads libnegacyclic.so (built by `make -C fherma-polynomial-cuda_b200`)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY):
            raise ImportError(f"CUDA library not built: {LIBRARY} (run __graft_entry__.build())")
        lib = ctypes.CDLL(LIBRARY)
        u32, p = ctypes.c_uint32, ctypes.c_void_p
        lib.negacyclic_last_error.restype = ctypes.c_char_p
        lib.negacyclic_init.argtypes = [u32, u32, u32, p, ctypes.POINTER(Options), ctypes.POINTER(p)]
        lib.negacyclic_get_info.argtypes = [p, ctypes.POINTER(Info)]
        lib.negacyclic_run.argtypes = [p, p, p, p]
        lib.negacyclic_run_device.argtypes = [p, p, p, p, p]
        lib.negacyclic_free.argtypes = [p]
        lib.negacyclic_free.restype = None
        lib.negacyclic_host_plan.argtypes = [u32, u32, p, u32, u32, p, p, p, p, p, p, p]
        lib.negacyclic_debug_read.argtypes = [p, ctypes.c_int, p, ctypes.POINTER(ctypes.c_size_t)]
        lib.negacyclic_gemm_u8.argtypes = [p, p, p, u32, u32, u32, u32, p]
        lib.negacyclic_run_device_timed.argtypes = [p, p, p, p, p, ctypes.POINTER(ctypes.c_float)]
        lib.negacyclic_work_bytes.argtypes = [p]
        lib.negacyclic_work_bytes.restype = ctypes.c_size_t
        lib.negacyclic_bind_work.argtypes = [p, p, ctypes.c_size_t]
        lib.negacyclic_pipeline_status.argtypes = [ctypes.POINTER(u32)]
        lib.negacyclic_run_begin.argtypes = [p, p, p]
        lib.negacyclic_run_finish.argtypes = [p, p]
        lib.negacyclic_prepare_host.argtypes = [p]
        lib.negacyclic_run_device_static.argtypes = [p, p, p, p, p]
        lib.negacyclic_plan_status.argtypes = [p, ctypes.POINTER(u32)]
        lib.negacyclic_gemm_u8_withheld.argtypes = [p, p, p, u32, u32, u32, u32, ctypes.c_uint64, u32,
                                                    ctypes.POINTER(u32), ctypes.POINTER(ctypes.c_double)]
        lib.negacyclic_batch_status.argtypes = [p, p]
        lib.negacyclic_host_touch.argtypes = [p, p, ctypes.c_size_t]
        pp = ctypes.POINTER(p)
        lib.negacyclic_batch_create.argtypes = [ctypes.POINTER(PointSpec), u32, ctypes.POINTER(BatchOptions),
                                                ctypes.POINTER(p)]
        lib.negacyclic_batch_io.argtypes = [p, u32, pp, pp, pp]
        lib.negacyclic_batch_get_info.argtypes = [p, u32, ctypes.POINTER(BatchInstance)]
        lib.negacyclic_batch_run_device.argtypes = [p, p]
        lib.negacyclic_batch_run.argtypes = [p, pp, pp, pp]
        lib.negacyclic_batch_run_one.argtypes = [p, u32, p]
        lib.negacyclic_batch_run_plain.argtypes = [p, pp, pp, pp]
        lib.negacyclic_batch_free.argtypes = [p]
        lib.negacyclic_batch_free.restype = None
        lib.negacyclic_server_create.argtypes = [ctypes.POINTER(ServerOptions), ctypes.POINTER(p)]
        lib.negacyclic_server_open_session.argtypes = [p, u32, u32, p, p, u32, ctypes.POINTER(u32)]
        lib.negacyclic_server_submit.argtypes = [p, u32, u32, p, p, p, ctypes.POINTER(ctypes.c_uint64)]
        lib.negacyclic_server_wait.argtypes = [p, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
        lib.negacyclic_server_get_stats.argtypes = [p, ctypes.POINTER(ServerStats)]
        lib.negacyclic_server_free.argtypes = [p]
        lib.negacyclic_server_free.restype = None
        _lib = lib
    return _lib


def last_error() -> str:
    return library().negacyclic_last_error().decode()


def _check(status: int, what: str):
    if status != OK:
        raise RuntimeError(f"{what}: {last_error()} (status {status})")


def _u32(array) -> np.ndarray:
    return np.ascontiguousarray(array, dtype=np.uint32)


class Plan:
    """One point (N, W, L, q): plan tables on the device, products on demand."""

    def __init__(self, n: int, w: int, limbs: int, q, split: int = 0, gemm: int = GEMM_AUTO, device: int = -1,
                 external_work: bool = False):
        q = _u32(q)
        if q.shape != (limbs,):
            raise RuntimeError("q must hold L words")
        opts = Options(split, gemm, device, int(external_work))
        handle = ctypes.c_void_p()
        _check(library().negacyclic_init(n, w, limbs, q.ctypes.data, ctypes.byref(opts), ctypes.byref(handle)),
               "negacyclic_init")
        self._handle = handle
        self.n, self.limbs = n, limbs

    @property
    def handle(self) -> ctypes.c_void_p:
        if not self._handle:
            raise RuntimeError("plan is closed")
        return self._handle

    def info(self) -> dict:
        info = Info()
        _check(library().negacyclic_get_info(self.handle, ctypes.byref(info)), "negacyclic_get_info")
        return {name: getattr(info, name) for name, _ in Info._fields_}

    def run(self, a, b, out: np.ndarray | None = None) -> np.ndarray:
        """Host arrays in, host array out ([N][L] uint32)."""
        a, b = _u32(a), _u32(b)
        shape = (self.n, self.limbs)
        if a.shape != shape or b.shape != shape:
            raise RuntimeError("wrong input size")
        c = np.empty(shape, dtype=np.uint32) if out is None else out
        _check(library().negacyclic_run(self.handle, a.ctypes.data, b.ctypes.data, c.ctypes.data), "negacyclic_run")
        return c

    def run_device(self, a_ptr: int, b_ptr: int, c_ptr: int, stream: int = 0):
        """Device pointers ([N][L] uint32 each), enqueued on `stream`."""
        _check(library().negacyclic_run_device(self.handle, a_ptr, b_ptr, c_ptr, stream), "negacyclic_run_device")

    def run_device_static(self, a_ptr: int, b_ptr: int, c_ptr: int, stream: int = 0):
        """run_device with no allocation: the work space is the library's static device array
        (NEGACYCLIC_STATIC_WORK_BYTES, shared by every such call; order calls on one stream)."""
        _check(library().negacyclic_run_device_static(self.handle, a_ptr, b_ptr, c_ptr, stream),
               "negacyclic_run_device_static")

    def run_device_timed(self, a_ptr: int, b_ptr: int, c_ptr: int, stream: int = 0) -> dict:
        """run_device, synchronously, returning per-stage milliseconds (CUDA events on `stream`)."""
        ms = (ctypes.c_float * len(STAGES))()
        _check(library().negacyclic_run_device_timed(self.handle, a_ptr, b_ptr, c_ptr, stream, ms),
               "negacyclic_run_device_timed")
        return dict(zip(STAGES, list(ms)))

    def status(self) -> int:
        """The plan's device status word (STATUS_* bits; 0 = sound) after a device sync; clears it."""
        flags = ctypes.c_uint32()
        _check(library().negacyclic_plan_status(self.handle, ctypes.byref(flags)), "negacyclic_plan_status")
        return flags.value

    def work_bytes(self) -> int:
        return int(library().negacyclic_work_bytes(self.handle))

    def bind_work(self, d_work: int, nbytes: int):
        _check(library().negacyclic_bind_work(self.handle, d_work, nbytes), "negacyclic_bind_work")

    def debug_read(self, which: int) -> bytes:
        size = ctypes.c_size_t(0)
        _check(library().negacyclic_debug_read(self.handle, which, None, ctypes.byref(size)), "debug_read")
        buf = ctypes.create_string_buffer(size.value)
        _check(library().negacyclic_debug_read(self.handle, which, buf, ctypes.byref(size)), "debug_read")
        return buf.raw

    def close(self):
        if self._handle:
            library().negacyclic_free(self._handle)
            self._handle = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pipeline_status() -> int:
    """Tensor-core GEMM status word of the current device (nonzero: a wait timed out); clears it."""
    flags = ctypes.c_uint32()
    _check(library().negacyclic_pipeline_status(ctypes.byref(flags)), "negacyclic_pipeline_status")
    return flags.value


def gemm_u8_withheld(a_ptr: int, b_ptr: int, d_ptr: int, m: int, n: int, k: int, engine: int, limit_cycles: int,
                     withheld_step: int):
    """(status, flags, elapsed_ms) of the tensor GEMM run with one pipeline stage withheld from the
    first CTA (pair), every wait bounded by limit_cycles (negacyclic_gemm_u8_withheld)."""
    flags, ms = ctypes.c_uint32(), ctypes.c_double()
    status = library().negacyclic_gemm_u8_withheld(a_ptr, b_ptr, d_ptr, m, n, k, engine, limit_cycles, withheld_step,
                                                   ctypes.byref(flags), ctypes.byref(ms))
    return status, flags.value, ms.value


def host_plan(n: int, limbs: int, q, split: int = 0) -> dict:
    """Host-only plan constants (no GPU): primes, split, N', finish factors, M_k, (-P) mod q."""
    q = _u32(q)
    lib = library()
    r, s, ns = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    _check(lib.negacyclic_host_plan(n, limbs, q.ctypes.data, split, 0, ctypes.byref(r), ctypes.byref(s),
                                    ctypes.byref(ns), None, None, None, None), "negacyclic_host_plan")
    primes = np.zeros(r.value, np.uint32)
    finish = np.zeros(r.value, np.uint32)
    crt = np.zeros((r.value, limbs), np.uint32)
    minus_p = np.zeros(limbs, np.uint32)
    _check(lib.negacyclic_host_plan(n, limbs, q.ctypes.data, split, r.value, ctypes.byref(r), ctypes.byref(s),
                                    ctypes.byref(ns), primes.ctypes.data, finish.ctypes.data, crt.ctypes.data,
                                    minus_p.ctypes.data), "negacyclic_host_plan")
    return {"primes": primes, "split": s.value, "n_sub": ns.value, "finish": finish, "crt_mod_q": crt,
            "minus_p_mod_q": minus_p}


class Batch:
    """Many products of uneven (N, W, q) in one graph launch (negacyclic_batch_*)."""

    def __init__(self, points, lanes: int = 0, tune: bool = False, tune_cache: str | None = None, device: int = -1):
        """points: iterable of (n, w, limbs, q)."""
        points = list(points)
        self._q = [_u32(q) for (_, _, _, q) in points]
        specs = (PointSpec * len(points))(*[PointSpec(n, w, limbs, q.ctypes.data)
                                            for (n, w, limbs, _), q in zip(points, self._q)])
        opts = BatchOptions(lanes, int(tune), device, 0, tune_cache.encode() if tune_cache else None)
        handle = ctypes.c_void_p()
        _check(library().negacyclic_batch_create(specs, len(points), ctypes.byref(opts), ctypes.byref(handle)),
               "negacyclic_batch_create")
        self._handle = handle
        self.shapes = [(n, limbs) for (n, _, limbs, _) in points]

    def __len__(self):
        return len(self.shapes)

    def io(self, index: int):
        """Device pointers (a, b, c) of instance `index`."""
        ptrs = [ctypes.c_void_p() for _ in range(3)]
        _check(library().negacyclic_batch_io(self._handle, index, *[ctypes.byref(x) for x in ptrs]),
               "negacyclic_batch_io")
        return tuple(int(x.value) for x in ptrs)

    def info(self, index: int) -> dict:
        inst = BatchInstance()
        _check(library().negacyclic_batch_get_info(self._handle, index, ctypes.byref(inst)), "negacyclic_batch_get_info")
        out = {name: getattr(inst.plan, name) for name, _ in Info._fields_}
        out.update(lane=inst.lane, requested_gemm=inst.requested_gemm, tuned_ms=inst.tuned_ms, phase=inst.phase)
        return out

    def run_device(self, stream: int = 0):
        _check(library().negacyclic_batch_run_device(self._handle, stream), "negacyclic_batch_run_device")

    def status(self) -> np.ndarray:
        """Every instance's device status word after a device sync (0 = sound); clears them."""
        flags = np.zeros(len(self.shapes), np.uint32)
        _check(library().negacyclic_batch_status(self._handle, flags.ctypes.data), "negacyclic_batch_status")
        return flags

    def run_one(self, index: int, stream: int = 0):
        """Instance `index` alone on `stream` (the plain per-call path)."""
        _check(library().negacyclic_batch_run_one(self._handle, index, stream), "negacyclic_batch_run_one")

    def run(self, a_list, b_list, c_list=None, plain: bool = False):
        """Host arrays in and out; plain=True runs one negacyclic_run per instance instead."""
        a_list = [_u32(a) for a in a_list]
        b_list = [_u32(b) for b in b_list]
        if c_list is None:
            c_list = [np.empty(shape, np.uint32) for shape in self.shapes]
        arr = lambda xs: (ctypes.c_void_p * len(xs))(*[x.ctypes.data for x in xs])  # noqa: E731
        fn = library().negacyclic_batch_run_plain if plain else library().negacyclic_batch_run
        _check(fn(self._handle, arr(a_list), arr(b_list), arr(c_list)), "negacyclic_batch_run")
        return c_list

    def close(self):
        if self._handle:
            library().negacyclic_batch_free(self._handle)
            self._handle = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Server:
    """Request loop with continuous batching (negacyclic_server_*)."""

    def __init__(self, hbm_budget: int = 0, slots: int = 0, device: int = -1, max_queue: int = 0):
        opts = ServerOptions(hbm_budget, slots, device, max_queue)
        handle = ctypes.c_void_p()
        _check(library().negacyclic_server_create(ctypes.byref(opts), ctypes.byref(handle)), "negacyclic_server_create")
        self._handle = handle
        self._keep = {}  # request id -> host buffers kept alive until wait()

    def open_session(self, w: int, limbs: int, q, ns=()) -> int:
        q = _u32(q)
        ns = np.ascontiguousarray(ns, dtype=np.uint32)
        session = ctypes.c_uint32()
        _check(library().negacyclic_server_open_session(self._handle, w, limbs, q.ctypes.data,
                                                        ns.ctypes.data if ns.size else None, ns.size,
                                                        ctypes.byref(session)), "negacyclic_server_open_session")
        return session.value

    def submit(self, session: int, a, b, out=None) -> int:
        """Request id, or None when the server's queue is full (the request was refused)."""
        a, b = _u32(a), _u32(b)
        c = np.empty_like(a) if out is None else out
        rid = ctypes.c_uint64()
        status = library().negacyclic_server_submit(self._handle, session, a.shape[0], a.ctypes.data, b.ctypes.data,
                                                    c.ctypes.data, ctypes.byref(rid))
        if status == EBUSY:
            return None
        _check(status, "negacyclic_server_submit")
        self._keep[rid.value] = (a, b, c)
        return rid.value

    def wait(self, request: int, timeout_ms: float = 0.0):
        """(result, latency_ms) of a submitted request."""
        latency = ctypes.c_double()
        status = library().negacyclic_server_wait(self._handle, request, timeout_ms, ctypes.byref(latency))
        a, b, c = self._keep.pop(request)
        _check(status, "negacyclic_server_wait")
        return c, latency.value

    def stats(self) -> dict:
        st = ServerStats()
        _check(library().negacyclic_server_get_stats(self._handle, ctypes.byref(st)), "negacyclic_server_get_stats")
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}

    def close(self):
        if self._handle:
            library().negacyclic_server_free(self._handle)
            self._handle = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---- the reference's plugin interface, in Python -------------------------------------------

@dataclass
class Point:
    N: int
    W: int
    L: int
    q: np.ndarray


@dataclass
class Inputs:
    a: np.ndarray
    b: np.ndarray


@dataclass
class Outputs:
    c: np.ndarray


def fherma_init(point: Point) -> Plan:
    plan = Plan(point.N, point.W, point.L, point.q)
    _check(library().negacyclic_prepare_host(plan.handle), "negacyclic_prepare_host")
    return plan


def fherma_run(state: Plan, inputs: Inputs) -> Outputs:
    return Outputs(state.run(inputs.a, inputs.b))


def fherma_free(state: Plan):
    state.close()
