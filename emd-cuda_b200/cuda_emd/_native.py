"""ctypes binding of libemdb200.so (C ABI in include/emdb200.h).

There is no fallback: if the library is missing or no CUDA device is present,
using the binding raises.  Build the library with
``python emd-cuda_b200/build.py``.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# EMDB_LIB overrides the library path (a measurement build, e.g. one with
# EMDB_LOAD_CLOCKS=1); the default is the in-tree product build
LIB_PATH = os.environ.get("EMDB_LIB") or os.path.join(os.path.dirname(HERE), "lib", "libemdb200.so")

EMDB_OK = 0
EMDB_ERR_INVALID = 1
EMDB_ERR_CUDA = 2
EMDB_ERR_NOMEM = 3
EMDB_ERR_UNSUPPORTED = 4
EMDB_ERR_DEVICE = 5
STATUS_STALE_ENVELOPE = 1
STATUS_TOO_LONG = 2

# Every symbol include/emdb200.h declares (checked by the CPU test suite).
EXPORTS = ("emdb_version", "emdb_plan_create", "emdb_plan_destroy", "emdb_plan_set_arena",
           "emdb_plan_set_variant", "emdb_plan_set_max_ctas", "emdb_plan_phase_clocks",
           "emdb_plan_query", "emdb_run", "emdb_run_ragged", "emdb_envelope", "emdb_status",
           "emdb_last_error", "emdb_features", "emdb_mlp_num_params", "emdb_mlp_forward",
           "emdb_mlp_backward", "emdb_mlp_adam", "emdb_mlp_infer_bf16", "emdb_check_division",
           "emdb_plan_counters", "emdb_run_noalloc", "emdb_run_host", "emdb_min_arena",
           "emdb_host_bytes", "emdb_host_register", "emdb_host_unregister",
           "emdb_notify_create", "emdb_notify_reset", "emdb_notify_destroy",
           "emdb_run_ragged_notify", "emdb_pass_placement", "emdb_noalloc_status",
           "emdb_pack_rows", "emdb_run_f32", "emdb_run_ragged_f32", "emdb_envelope_f32",
           "emdb_plan_query_f32", "emdb_plan_set_tail")


class EmdbConfig(ctypes.Structure):
    _fields_ = [("max_extrema", ctypes.c_int), ("nbsym", ctypes.c_int),
                ("max_iteration", ctypes.c_int), ("max_imfs", ctypes.c_int),
                ("threads_per_block", ctypes.c_int)]


_lib = None
_lock = threading.Lock()


def lib_path() -> str:
    return LIB_PATH


def load() -> ctypes.CDLL:
    """Load the library (once).  Raises OSError if it is not built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.isfile(LIB_PATH):
            raise OSError(f"{LIB_PATH} is not built; run `python emd-cuda_b200/build.py`")
        L = ctypes.CDLL(LIB_PATH)
        P, I, VP = ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p
        L.emdb_version.restype = I
        L.emdb_plan_create.argtypes = [ctypes.POINTER(EmdbConfig), I, ctypes.POINTER(VP)]
        L.emdb_plan_destroy.argtypes = [VP]
        L.emdb_plan_set_arena.argtypes = [VP, I]
        L.emdb_plan_set_variant.argtypes = [VP, I]
        L.emdb_plan_set_max_ctas.argtypes = [VP, I]
        L.emdb_plan_set_tail.argtypes = [VP, I]
        L.emdb_plan_phase_clocks.argtypes = [VP, P, I, I]
        L.emdb_plan_query.argtypes = [VP, I, ctypes.POINTER(I), ctypes.POINTER(I), ctypes.POINTER(I)]
        L.emdb_run.argtypes = [VP, P, P, I, I, P, P, P, P, P, P, VP]
        L.emdb_run_f32.argtypes = [VP, P, P, I, I, P, P, P, P, P, P, VP]
        L.emdb_plan_query_f32.argtypes = [VP, I, ctypes.POINTER(I), ctypes.POINTER(I),
                                          ctypes.POINTER(I)]
        L.emdb_run_host.argtypes = [VP, P, P, I, I, P, P, P, P, P, P, VP]
        L.emdb_min_arena.argtypes = [I, ctypes.POINTER(I)]
        L.emdb_notify_create.argtypes = [I, I, ctypes.POINTER(VP),
                                         ctypes.POINTER(ctypes.POINTER(ctypes.c_uint))]
        L.emdb_notify_reset.argtypes = [VP, I, VP]
        L.emdb_notify_destroy.argtypes = [VP]
        L.emdb_run_ragged_notify.argtypes = [VP, P, P, I, I, P, I, P, P, P, P, P, P, P, VP, I, VP]
        L.emdb_host_register.argtypes = [VP, ctypes.c_size_t, I]
        L.emdb_host_unregister.argtypes = [VP]
        L.emdb_host_bytes.argtypes = [VP, ctypes.POINTER(ctypes.c_ulonglong),
                                      ctypes.POINTER(ctypes.c_ulonglong)]
        L.emdb_run_ragged.argtypes = [VP, P, P, I, I, P, I, P, P, P, P, P, P, P, VP]
        L.emdb_run_ragged_f32.argtypes = [VP, P, P, I, I, P, I, P, P, P, P, P, P, P, VP]
        L.emdb_envelope.argtypes = [VP, P, P, I, I, P, P, P, P, P, P, P, P, P, VP]
        L.emdb_envelope_f32.argtypes = [VP, P, P, I, I, P, P, P, P, P, P, P, P, P, VP]
        L.emdb_status.argtypes = [VP, ctypes.POINTER(I), VP]
        L.emdb_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        L.emdb_run_noalloc.argtypes = [ctypes.POINTER(EmdbConfig), P, P, I, I, P, P, P, P, P, P, VP]
        L.emdb_noalloc_status.argtypes = [ctypes.POINTER(I), VP]
        L.emdb_pack_rows.argtypes = [P, P, P, P, I, I, P, VP]
        L.emdb_plan_counters.argtypes = [VP, ctypes.POINTER(ctypes.c_ulonglong),
                                         ctypes.POINTER(ctypes.c_ulonglong), I]
        L.emdb_check_division.argtypes = [I, ctypes.c_longlong, ctypes.c_ulonglong, P]
        for name in EXPORTS:
            getattr(L, name).restype = I
        _lib = L
        return L


PLACEMENTS = {0: "shared", 1: "split", 2: "slab", 3: "borrow", 4: "park", 5: "compact borrow",
              -1: "does not fit"}


def pass_placement(cfg: EmdbConfig, N: int, arena_bytes: int, n_max: int, n_min: int) -> int:
    """Knot placement of one sift pass (see emdb_pass_placement); no GPU needed."""
    L = load()
    out = ctypes.c_int()
    check(L.emdb_pass_placement(ctypes.byref(cfg), int(N), int(arena_bytes), int(n_max),
                                int(n_min), ctypes.byref(out)), "emdb_pass_placement")
    return out.value


def last_error() -> str:
    L = load()
    buf = ctypes.create_string_buffer(1024)
    L.emdb_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


class EmdbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def check(rc: int, what: str) -> None:
    """Map a C-ABI return code to the reference's exception types."""
    if rc == EMDB_OK:
        return
    msg = f"{what}: {last_error()}"
    if rc in (EMDB_ERR_INVALID, EMDB_ERR_UNSUPPORTED):
        raise ValueError(msg)
    if rc == EMDB_ERR_NOMEM:
        raise MemoryError(msg)
    raise EmdbError(rc, msg)


class Notify:
    """Per-trace completion flags (emdb_notify): ``flags`` is a live NumPy view
    of page-locked host memory the kernel writes; flags[b] = 1 + the rows of
    trace b that may hold data, once trace b is complete (0 before)."""

    def __init__(self, capacity: int, device: int):
        self.L = load()
        self.capacity = int(capacity)
        h = ctypes.c_void_p()
        ptr = ctypes.POINTER(ctypes.c_uint)()
        check(self.L.emdb_notify_create(self.capacity, int(device), ctypes.byref(h),
                                        ctypes.byref(ptr)), "emdb_notify_create")
        self.handle = h
        self.flags = np.ctypeslib.as_array(ptr, shape=(self.capacity,))

    def reset(self, n: int, stream: int) -> None:
        """Zero the first n counters and flags (no launch using them may run)."""
        check(self.L.emdb_notify_reset(self.handle, int(n), stream), "emdb_notify_reset")

    def __del__(self):
        try:
            if self.handle:
                self.L.emdb_notify_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class Plan:
    """Owns one emdb_plan (device scratch + config) for one CUDA device."""

    def __init__(self, cfg: EmdbConfig, device: int):
        self.L = load()
        self.device = device
        h = ctypes.c_void_p()
        check(self.L.emdb_plan_create(ctypes.byref(cfg), device, ctypes.byref(h)), "emdb_plan_create")
        self.handle = h

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.L.emdb_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_arena(self, arena_bytes: int) -> None:
        check(self.L.emdb_plan_set_arena(self.handle, int(arena_bytes)), "emdb_plan_set_arena")

    def set_variant(self, min_ctas_per_sm: int) -> None:
        check(self.L.emdb_plan_set_variant(self.handle, int(min_ctas_per_sm)), "emdb_plan_set_variant")

    def set_tail(self, yield_below: int) -> None:
        """Tail migration (emdb_plan_set_tail): 0 off, -1 below the SM count,
        > 0 below that many traces in flight."""
        check(self.L.emdb_plan_set_tail(self.handle, int(yield_below)), "emdb_plan_set_tail")

    def set_max_ctas(self, max_ctas: int) -> None:
        check(self.L.emdb_plan_set_max_ctas(self.handle, int(max_ctas)), "emdb_plan_set_max_ctas")

    def query(self, max_n: int, f32: bool = False) -> tuple[int, int, int]:
        """(arena bytes, CTAs per SM, grid) the plan's launches use for traces
        up to max_n (f32: the FP32 kernels)."""
        a, c, g = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        fn = self.L.emdb_plan_query_f32 if f32 else self.L.emdb_plan_query
        check(fn(self.handle, int(max_n), ctypes.byref(a), ctypes.byref(c), ctypes.byref(g)),
              "emdb_plan_query")
        return a.value, c.value, g.value

    def host_bytes(self) -> tuple[int, int]:
        """(host->device, device->host) bytes of the last host-pipeline call."""
        a, b = ctypes.c_ulonglong(), ctypes.c_ulonglong()
        check(self.L.emdb_host_bytes(self.handle, ctypes.byref(a), ctypes.byref(b)),
              "emdb_host_bytes")
        return a.value, b.value

    def min_arena(self, max_n: int) -> int:
        """Smallest arena that holds a trace of max_n samples (knots all spilled)."""
        a = ctypes.c_int()
        check(self.L.emdb_min_arena(int(max_n), ctypes.byref(a)), "emdb_min_arena")
        return a.value

    def counters(self, reset: bool = False) -> tuple[int, int]:
        """(sift passes, passes spilled to the global slab) since creation / last reset."""
        a, b = ctypes.c_ulonglong(), ctypes.c_ulonglong()
        check(self.L.emdb_plan_counters(self.handle, ctypes.byref(a), ctypes.byref(b), int(reset)),
              "emdb_plan_counters")
        return a.value, b.value

    PHASES = ("load", "trace", "fill", "mirror", "spline rows", "pcr", "diagonal", "evaluation",
              "lane sums", "trees+scan", "per-IMF", "rest")

    def phase_clocks(self, reset: bool = False) -> dict:
        """Cycle counts by phase (emdb_plan_phase_clocks); non-zero only in a
        library built with EMDB_LOAD_CLOCKS=1."""
        buf = (ctypes.c_ulonglong * len(self.PHASES))()
        check(self.L.emdb_plan_phase_clocks(self.handle, ctypes.cast(buf, ctypes.c_void_p),
                                            len(self.PHASES), int(reset)), "emdb_plan_phase_clocks")
        return dict(zip(self.PHASES, (int(v) for v in buf)))

    def status(self, stream: int) -> int:
        s = ctypes.c_int()
        check(self.L.emdb_status(self.handle, ctypes.byref(s), ctypes.c_void_p(stream)), "emdb_status")
        return s.value


def check_division(mode: int, n: int, seed: int = 0) -> tuple[int, int, int]:
    """Self-test: mismatches of the kernels' own divisions vs the hardware
    division, three counters per mode (mode 0/1: the reciprocal-based
    division of the evaluation; mode 2: the PCR rows' branch-free division;
    modes 3/4: the FP32 kernels' float quotients against the float division;
    the header documents the cases)."""
    L = load()
    out = (ctypes.c_ulonglong * 3)()
    check(L.emdb_check_division(int(mode), int(n), int(seed), out), "emdb_check_division")
    return tuple(int(v) for v in out)
