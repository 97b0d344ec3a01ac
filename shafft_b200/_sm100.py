"""ctypes binding of libshafft_sm100.so (the kernel library's C ABI,
include/shafft_sm100.h).

The product path is C/C++/CUDA; this module only forwards plain pointers
and sizes.  It fails loudly when the shared library has not been built:
there is no fallback implementation.
"""
from __future__ import annotations

import ctypes
import json
import os

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
SM100_LIB = os.path.join(LIB_DIR, "libshafft_sm100.so")

_lib = None


class Sm100Error(RuntimeError):
    pass


def load():
    """Load libshafft_sm100.so (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(SM100_LIB):
        raise Sm100Error(
            f"{SM100_LIB} is not built; run __graft_entry__.build() "
            "(python -c 'import __graft_entry__ as g; g.build()')")
    lib = ctypes.CDLL(SM100_LIB, mode=ctypes.RTLD_GLOBAL)
    vp = ctypes.c_void_p
    i64p = ctypes.POINTER(ctypes.c_int64)
    lib.shafft_sm100_plan_create_nd.argtypes = [ctypes.POINTER(vp), ctypes.c_int, i64p, ctypes.c_int]
    lib.shafft_sm100_plan_create_nd_ex.argtypes = [ctypes.POINTER(vp), ctypes.c_int, i64p, ctypes.c_int,
                                                   ctypes.c_int]
    lib.shafft_sm100_plan_query_ex.argtypes = [ctypes.c_int, i64p, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_char_p, ctypes.c_int]
    lib.shafft_sm100_plan_create_1d.argtypes = [ctypes.POINTER(vp), ctypes.c_int64, ctypes.c_int]
    lib.shafft_sm100_plan_destroy.argtypes = [vp]
    lib.shafft_sm100_set_stream.argtypes = [vp, vp]
    lib.shafft_sm100_execute.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_double, vp]
    lib.shafft_sm100_scale.argtypes = [vp, ctypes.c_size_t, ctypes.c_int, ctypes.c_double, vp]
    lib.shafft_sm100_plan_elements.argtypes = [vp]
    lib.shafft_sm100_plan_elements.restype = ctypes.c_int64
    lib.shafft_sm100_plan_passes.argtypes = [vp]
    lib.shafft_sm100_plan_launches.argtypes = [vp]
    lib.shafft_sm100_plan_device_bytes.argtypes = [vp]
    lib.shafft_sm100_plan_device_bytes.restype = ctypes.c_size_t
    lib.shafft_sm100_plan_query.argtypes = [ctypes.c_int, i64p, ctypes.c_int, ctypes.c_char_p,
                                            ctypes.c_int]
    lib.shafft_sm100_plan_describe.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
    lib.shafft_sm100_execute_step.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_int, ctypes.c_double, vp]
    lib.shafft_sm100_step_bytes.argtypes = [vp, ctypes.c_int]
    lib.shafft_sm100_step_bytes.restype = ctypes.c_int64
    lib.shafft_sm100_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int,
                                              ctypes.POINTER(ctypes.c_int), i64p, ctypes.c_int,
                                              ctypes.c_int]
    lib.shafft_sm100_batch_execute.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                               ctypes.c_int, ctypes.c_double, vp]
    lib.shafft_sm100_batch_destroy.argtypes = [vp]
    lib.shafft_sm100_batch_status.argtypes = [vp]
    lib.shafft_sm100_batch_set_wait_limit.argtypes = [vp, ctypes.c_uint]
    lib.shafft_sm100_batch_bytes.argtypes = [vp]
    lib.shafft_sm100_batch_bytes.restype = ctypes.c_int64
    lib.shafft_sm100_batch_describe.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
    lib.shafft_sm100_plan_status.argtypes = [vp]
    lib.shafft_sm100_tma_launch_count.argtypes = []
    lib.shafft_sm100_tma_launch_count.restype = ctypes.c_int64
    lib.shafft_sm100_server_create.argtypes = [ctypes.POINTER(vp), ctypes.c_size_t, ctypes.c_int]
    lib.shafft_sm100_server_submit.argtypes = [vp, ctypes.c_int, i64p, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_double, vp, vp, ctypes.POINTER(ctypes.c_uint64)]
    lib.shafft_sm100_server_wait.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double)]
    lib.shafft_sm100_server_stats.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
    lib.shafft_sm100_server_reset_stats.argtypes = [vp]
    lib.shafft_sm100_server_destroy.argtypes = [vp]
    lib.shafft_sm100_rplan_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, i64p, ctypes.c_int]
    lib.shafft_sm100_rplan_destroy.argtypes = [vp]
    lib.shafft_sm100_rplan_spectrum_elements.argtypes = [vp]
    lib.shafft_sm100_rplan_spectrum_elements.restype = ctypes.c_int64
    lib.shafft_sm100_execute_r2c.argtypes = [vp, vp, vp, ctypes.c_double, vp]
    lib.shafft_sm100_execute_c2r.argtypes = [vp, vp, vp, ctypes.c_double, vp]
    lib.shafft_sm100_check_guards.argtypes = []
    lib.shafft_sm100_malloc.argtypes = [ctypes.POINTER(vp), ctypes.c_size_t]
    lib.shafft_sm100_free.argtypes = [vp]
    lib.shafft_sm100_memcpy.argtypes = [vp, vp, ctypes.c_size_t, ctypes.c_int, vp]
    lib.shafft_sm100_stream_sync.argtypes = [vp]
    lib.shafft_sm100_last_error_message.restype = ctypes.c_char_p
    lib.shafft_sm100_version.restype = ctypes.c_char_p
    _lib = lib
    return lib


def _check(rc, what):
    if rc != 0:
        msg = load().shafft_sm100_last_error_message().decode(errors="replace")
        raise Sm100Error(f"{what} failed rc={rc}: {msg}")


# plan flags (shafft_sm100.h)
PLAN_TENSOR_CORE = 1
PLAN_TC_PRIME_AXES = 2
PLAN_MEASURE = 4


def plan_query_mapped(dims, axes, precision=0, load_map=None, store_map=None) -> dict:
    """Planning-only description of an axis-subset plan with exchange block
    maps (shafft_sm100_plan_query_mapped); "fused" = bit 0 load, bit 1 store."""
    lib = load()
    d = (ctypes.c_int64 * len(dims))(*[int(x) for x in dims])
    a = (ctypes.c_int * len(axes))(*[int(x) for x in axes])
    lm = None if load_map is None else (ctypes.c_int64 * 4)(*load_map)
    sm = None if store_map is None else (ctypes.c_int64 * 4)(*store_map)
    buf = ctypes.create_string_buffer(1 << 16)
    _check(lib.shafft_sm100_plan_query_mapped(len(dims), d, int(precision), len(axes), a, lm, sm, buf, len(buf)),
           "plan_query_mapped")
    return json.loads(buf.value.decode())


def plan_query(dims, precision=0, flags=0) -> dict:
    """Host-only planner query (no GPU needed)."""
    lib = load()
    d = (ctypes.c_int64 * len(dims))(*dims)
    buf = ctypes.create_string_buffer(1 << 16)
    _check(lib.shafft_sm100_plan_query_ex(len(dims), d, precision, flags, buf, len(buf)), "plan_query")
    return json.loads(buf.value.decode())


class Plan:
    """Owning handle of a shafft_sm100 plan (device tables + scratch)."""

    def __init__(self, dims, precision=0, flags=0):
        lib = load()
        self._lib = lib
        self.dims = tuple(int(x) for x in dims)
        self.precision = int(precision)
        self.flags = int(flags)
        h = ctypes.c_void_p()
        d = (ctypes.c_int64 * len(self.dims))(*self.dims)
        _check(lib.shafft_sm100_plan_create_nd_ex(ctypes.byref(h), len(self.dims), d, self.precision,
                                                  self.flags), "plan_create_nd")
        self.handle = h

    def execute(self, src_ptr: int, dst_ptr: int, direction: int = 0, scale: float = 1.0,
                stream: int = 0):
        _check(self._lib.shafft_sm100_execute(self.handle, ctypes.c_void_p(src_ptr),
                                              ctypes.c_void_p(dst_ptr), int(direction),
                                              float(scale), ctypes.c_void_p(stream)), "execute")

    def execute_step(self, step: int, src_ptr: int, dst_ptr: int, direction: int = 0,
                     scale: float = 1.0, stream: int = 0):
        _check(self._lib.shafft_sm100_execute_step(self.handle, int(step), ctypes.c_void_p(src_ptr),
                                                   ctypes.c_void_p(dst_ptr), int(direction),
                                                   float(scale), ctypes.c_void_p(stream)),
               "execute_step")

    def step_bytes(self, step: int) -> int:
        return int(self._lib.shafft_sm100_step_bytes(self.handle, int(step)))

    def status(self):
        """Synchronises and raises if a device-side wait of the last executes gave up."""
        _check(self._lib.shafft_sm100_stream_sync(None), "stream_sync")
        _check(self._lib.shafft_sm100_plan_status(self.handle), "plan_status")

    def describe(self) -> dict:
        buf = ctypes.create_string_buffer(1 << 16)
        _check(self._lib.shafft_sm100_plan_describe(self.handle, buf, len(buf)), "describe")
        return json.loads(buf.value.decode())

    @property
    def launches(self) -> int:
        return self._lib.shafft_sm100_plan_launches(self.handle)

    @property
    def passes(self) -> int:
        return self._lib.shafft_sm100_plan_passes(self.handle)

    @property
    def device_bytes(self) -> int:
        """Device memory the plan holds (tables and scratch)."""
        return int(self._lib.shafft_sm100_plan_device_bytes(self.handle))

    def destroy(self):
        if self.handle:
            self._lib.shafft_sm100_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class RPlan:
    """Real-to-complex / complex-to-real plan (shafft_sm100_rplan_*): real
    tensor `dims` (last length even) <-> its half spectrum (..., L/2 + 1)."""

    def __init__(self, dims, precision=0):
        lib = load()
        self._lib = lib
        self.dims = tuple(int(x) for x in dims)
        self.precision = int(precision)
        h = ctypes.c_void_p()
        d = (ctypes.c_int64 * len(self.dims))(*self.dims)
        _check(lib.shafft_sm100_rplan_create(ctypes.byref(h), len(self.dims), d, self.precision),
               "rplan_create")
        self.handle = h

    @property
    def spectrum_elements(self) -> int:
        return int(self._lib.shafft_sm100_rplan_spectrum_elements(self.handle))

    def r2c(self, real_ptr: int, spec_ptr: int, scale: float = 1.0, stream: int = 0):
        _check(self._lib.shafft_sm100_execute_r2c(self.handle, ctypes.c_void_p(real_ptr),
                                                  ctypes.c_void_p(spec_ptr), float(scale),
                                                  ctypes.c_void_p(stream)), "execute_r2c")

    def c2r(self, spec_ptr: int, real_ptr: int, scale: float = 1.0, stream: int = 0):
        _check(self._lib.shafft_sm100_execute_c2r(self.handle, ctypes.c_void_p(spec_ptr),
                                                  ctypes.c_void_p(real_ptr), float(scale),
                                                  ctypes.c_void_p(stream)), "execute_c2r")

    def destroy(self):
        if self.handle:
            self._lib.shafft_sm100_rplan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def tma_launch_count() -> int:
    """Column passes this process ran through the bulk-tensor-copy kernel."""
    return int(load().shafft_sm100_tma_launch_count())


def scale(ptr: int, count: int, precision: int, factor: float, stream: int = 0):
    _check(load().shafft_sm100_scale(ctypes.c_void_p(ptr), count, precision, factor,
                                     ctypes.c_void_p(stream)), "scale")


class Batch:
    """Many independent transforms of different shapes, one launch per execute
    (shafft_sm100_batch_*)."""

    def __init__(self, shapes, precision=0, autotune=False):
        lib = load()
        self._lib = lib
        self.shapes = [tuple(int(d) for d in s) for s in shapes]
        self.precision = int(precision)
        nd = (ctypes.c_int * len(self.shapes))(*[len(s) for s in self.shapes])
        flat = [d for s in self.shapes for d in s]
        dims = (ctypes.c_int64 * len(flat))(*flat)
        h = ctypes.c_void_p()
        _check(lib.shafft_sm100_batch_create(ctypes.byref(h), len(self.shapes), nd, dims,
                                             self.precision, 1 if autotune else 0), "batch_create")
        self.handle = h

    def execute(self, src_ptrs, dst_ptrs, direction=0, scale=1.0, stream=0):
        n = len(self.shapes)
        s = (ctypes.c_void_p * n)(*src_ptrs)
        d = (ctypes.c_void_p * n)(*dst_ptrs)
        _check(self._lib.shafft_sm100_batch_execute(self.handle, s, d, int(direction), float(scale),
                                                    ctypes.c_void_p(stream)), "batch_execute")

    def status(self):
        _check(self._lib.shafft_sm100_batch_status(self.handle), "batch_status")

    def set_wait_limit(self, polls: int):
        """Bound of each tile's wait for the previous pass (0 = default)."""
        _check(self._lib.shafft_sm100_batch_set_wait_limit(self.handle, int(polls)), "set_wait_limit")

    @property
    def alg_bytes(self) -> int:
        return int(self._lib.shafft_sm100_batch_bytes(self.handle))

    def describe(self) -> dict:
        buf = ctypes.create_string_buffer(4096)
        _check(self._lib.shafft_sm100_batch_describe(self.handle, buf, len(buf)), "describe")
        return json.loads(buf.value.decode())

    def destroy(self):
        if self.handle:
            self._lib.shafft_sm100_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Server:
    """Request loop with continuous admission (shafft_sm100_server_*)."""

    def __init__(self, budget_bytes, streams=4):
        lib = load()
        self._lib = lib
        h = ctypes.c_void_p()
        _check(lib.shafft_sm100_server_create(ctypes.byref(h), int(budget_bytes), int(streams)),
               "server_create")
        self.handle = h

    def submit(self, dims, precision, direction, scale, host_in_ptr, host_out_ptr) -> int:
        d = (ctypes.c_int64 * len(dims))(*dims)
        rid = ctypes.c_uint64()
        _check(self._lib.shafft_sm100_server_submit(self.handle, len(dims), d, int(precision),
                                                    int(direction), float(scale),
                                                    ctypes.c_void_p(host_in_ptr),
                                                    ctypes.c_void_p(host_out_ptr), ctypes.byref(rid)),
               "server_submit")
        return rid.value

    def wait(self, rid) -> float:
        lat = ctypes.c_double()
        _check(self._lib.shafft_sm100_server_wait(self.handle, ctypes.c_uint64(rid), ctypes.byref(lat)),
               "server_wait")
        return lat.value

    def stats(self) -> dict:
        buf = ctypes.create_string_buffer(1024)
        _check(self._lib.shafft_sm100_server_stats(self.handle, buf, len(buf)), "server_stats")
        return json.loads(buf.value.decode())

    def reset_stats(self):
        self._lib.shafft_sm100_server_reset_stats(self.handle)

    def destroy(self):
        if self.handle:
            self._lib.shafft_sm100_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
