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

OK, EINVAL, ENOFIELDS, ESIZE, ECUDA, ENOMEM, ENODEV = range(7)
GEMM_AUTO, GEMM_SIMT, GEMM_TENSOR, GEMM_TENSOR_SINGLE = 0, 1, 2, 3

EXPORTED = [
    "negacyclic_last_error", "negacyclic_init", "negacyclic_get_info", "negacyclic_run",
    "negacyclic_run_device", "negacyclic_free", "negacyclic_host_plan", "negacyclic_debug_read",
    "negacyclic_gemm_u8", "negacyclic_run_device_timed",
]
STAGES = ["pad", "convert", "forward", "pointwise", "inverse", "transpose", "crt", "reduce"]


class Options(ctypes.Structure):
    _fields_ = [("split", ctypes.c_uint32), ("gemm", ctypes.c_uint32), ("device", ctypes.c_int32),
                ("reserved", ctypes.c_uint32 * 5)]


class Info(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint32) for name in
                ("n", "w", "limbs", "primes", "padded_primes", "split", "n_sub", "words", "gemm", "q_bits")] + \
               [("device_bytes", ctypes.c_uint64), ("table_bytes", ctypes.c_uint64),
                ("kernels_per_product", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


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

    def __init__(self, n: int, w: int, limbs: int, q, split: int = 0, gemm: int = GEMM_AUTO, device: int = -1):
        q = _u32(q)
        if q.shape != (limbs,):
            raise RuntimeError("q must hold L words")
        opts = Options(split, gemm, device)
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

    def run_device_timed(self, a_ptr: int, b_ptr: int, c_ptr: int, stream: int = 0) -> dict:
        """run_device, synchronously, returning per-stage milliseconds (CUDA events on `stream`)."""
        ms = (ctypes.c_float * len(STAGES))()
        _check(library().negacyclic_run_device_timed(self.handle, a_ptr, b_ptr, c_ptr, stream, ms),
               "negacyclic_run_device_timed")
        return dict(zip(STAGES, list(ms)))

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
    return Plan(point.N, point.W, point.L, point.q)


def fherma_run(state: Plan, inputs: Inputs) -> Outputs:
    return Outputs(state.run(inputs.a, inputs.b))


def fherma_free(state: Plan):
    state.close()
