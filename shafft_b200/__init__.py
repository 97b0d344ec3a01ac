"""shafft_b200 -- SHAFFT's C2C/Z2Z hot path on one NVIDIA B200 (sm_100a).

The product is native: ``lib/libshafft.so`` (the SHAFFT C++ API and C ABI,
include/shafft/shafft.h) on top of ``lib/libshafft_sm100.so`` (hand-written
sm_100a kernels, include/shafft_sm100.h).  This module is a thin ctypes
mirror of the reference's plan interface -- the same names, argument meaning
and status codes as ``shafft::FFTND`` / ``shafft::FFT1D`` and the C functions
``shafftNDCreate/NDInit/Plan/SetBuffers/Execute/Normalize/...`` -- so that
tests and the benchmark read like the reference's own tests.  It has no
compute of its own and raises if the native libraries are missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _sm100  # noqa: F401  (kernel-library binding)

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
SHAFFT_LIB = os.path.join(LIB_DIR, "libshafft.so")

# shafft_t / shafft_direction_t / shafft_status_t (include/shafft/shafft.h)
C2C, Z2Z = 0, 1
FORWARD, BACKWARD = 0, 1
LAYOUT_REDISTRIBUTED, LAYOUT_INITIAL = 0, 1
TENSOR_LAYOUT_CURRENT, TENSOR_LAYOUT_INITIAL, TENSOR_LAYOUT_REDISTRIBUTED = 0, 1, 2
MAXIMIZE_NDA, MINIMIZE_NDA = 0, 1
STATUS = {
    0: "SUCCESS", 1: "ERR_NULLPTR", 2: "ERR_INVALID_COMM", 3: "ERR_NO_BUFFER",
    4: "ERR_PLAN_NOT_INIT", 5: "ERR_INVALID_DIM", 6: "ERR_DIM_MISMATCH",
    7: "ERR_INVALID_DECOMP", 8: "ERR_INVALID_FFTTYPE", 9: "ERR_ALLOC", 10: "ERR_BACKEND",
    11: "ERR_MPI", 12: "ERR_INVALID_LAYOUT", 13: "ERR_SIZE_OVERFLOW", 14: "ERR_NOT_IMPL",
    15: "ERR_INVALID_STATE", 16: "ERR_INTERNAL",
}
for _code, _name in STATUS.items():
    globals()[_name] = _code

# single-rank MPI shim handles (include/mpi_shim/mpi.h)
MPI_COMM_NULL = 0
MPI_COMM_WORLD = 0x44000000
MPI_COMM_SELF = 0x44000001

_lib = None


class ShafftError(RuntimeError):
    def __init__(self, status, what, message=""):
        super().__init__(f"{what}: {STATUS.get(status, status)} ({status}) {message}".rstrip())
        self.status = status


def load():
    """Load libshafft.so (and through it libshafft_sm100.so)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(SHAFFT_LIB):
        raise ShafftError(ERR_INTERNAL, "load",  # noqa: F821
                          f"{SHAFFT_LIB} not built; run __graft_entry__.build()")
    lib = ctypes.CDLL(SHAFFT_LIB, mode=ctypes.RTLD_GLOBAL)
    vp, vpp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)
    ip = ctypes.POINTER(ctypes.c_int)
    szp = ctypes.POINTER(ctypes.c_size_t)
    sig = {
        "shafftNDCreate": [vpp],
        "shafftNDInit": [vp, ctypes.c_int, ip, ip, ctypes.c_int, ctypes.c_int, ctypes.c_int],
        "shafft1DCreate": [vpp],
        "shafft1DInit": [vp, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int,
                         ctypes.c_int],
        "shafftPlan": [vp],
        "shafftDestroy": [vpp],
        "shafftGetLayout": [vp, szp, szp, ctypes.c_int],
        "shafftGetAxes": [vp, ip, ip, ctypes.c_int],
        "shafftGetAllocSize": [vp, szp],
        "shafftGetGlobalSize": [vp, szp],
        "shafftIsConfigured": [vp, ip],
        "shafftIsActive": [vp, ip],
        "shafftSetBuffers": [vp, vp, vp],
        "shafftGetBuffers": [vp, vpp, vpp],
        "shafftExecute": [vp, ctypes.c_int],
        "shafftExecuteNormalized": [vp, ctypes.c_int],
        "shafftNormalize": [vp],
        "shafftSetStream": [vp, vp],
        "shafftGetCommunicator": [vp, ip],
        "shafftConfigurationND": [ctypes.c_int, ip, ctypes.c_int, ip, ip, szp, szp, ip, ctypes.c_int,
                                  ctypes.c_size_t, ctypes.c_int],
        "shafftConfiguration1D": [ctypes.c_size_t, szp, szp, szp, ctypes.c_int, ctypes.c_int],
        "shafftAllocBufferF": [ctypes.c_size_t, vpp],
        "shafftAllocBufferD": [ctypes.c_size_t, vpp],
        "shafftFreeBufferF": [vp],
        "shafftFreeBufferD": [vp],
        "shafftCopyToBufferF": [vp, vp, ctypes.c_size_t],
        "shafftCopyToBufferD": [vp, vp, ctypes.c_size_t],
        "shafftCopyFromBufferF": [vp, vp, ctypes.c_size_t],
        "shafftCopyFromBufferD": [vp, vp, ctypes.c_size_t],
        "shafftLastErrorMessage": [ctypes.c_char_p, ctypes.c_int],
        "shafftLastErrorStatus": [],
        "shafftLastErrorSource": [],
        "shafftLastErrorDomainCode": [],
        "shafftClearLastError": [],
        "shafftErrorSourceName": [ctypes.c_int],
        "shafftGetBackendName": [],
        "shafftGetVersion": [ip, ip, ip],
        "shafftGetVersionString": [],
        "shafftFinalize": [],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    lib.shafftErrorSourceName.restype = ctypes.c_char_p
    lib.shafftGetBackendName.restype = ctypes.c_char_p
    lib.shafftGetVersionString.restype = ctypes.c_char_p
    lib.shafftClearLastError.restype = None
    lib.shafftGetVersion.restype = None
    _lib = lib
    return lib


def last_error_message() -> str:
    buf = ctypes.create_string_buffer(512)
    load().shafftLastErrorMessage(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int, what: str):
    if rc != 0:
        raise ShafftError(rc, what, last_error_message())
    return rc


def _iarr(vals):
    return (ctypes.c_int * max(1, len(vals)))(*vals)


# ---------------------------------------------------------------------------
# Buffers (allocBuffer / freeBuffer / copyToBuffer / copyFromBuffer)
# ---------------------------------------------------------------------------

class DeviceBuffer:
    """Device buffer of `count` complex elements from shafftAllocBufferF/D."""

    def __init__(self, count: int, precision: int = C2C):
        self.count = int(count)
        self.precision = precision
        p = ctypes.c_void_p()
        f = load().shafftAllocBufferD if precision == Z2Z else load().shafftAllocBufferF
        check(f(self.count, ctypes.byref(p)), "allocBuffer")
        self.ptr = p.value or 0

    @property
    def dtype(self):
        return np.complex128 if self.precision == Z2Z else np.complex64

    def upload(self, host: np.ndarray):
        a = np.ascontiguousarray(host, dtype=self.dtype).ravel()
        assert a.size <= self.count
        f = load().shafftCopyToBufferD if self.precision == Z2Z else load().shafftCopyToBufferF
        check(f(ctypes.c_void_p(self.ptr), a.ctypes.data_as(ctypes.c_void_p), a.size), "copyToBuffer")

    def download(self, count=None) -> np.ndarray:
        n = self.count if count is None else int(count)
        out = np.empty(n, dtype=self.dtype)
        f = load().shafftCopyFromBufferD if self.precision == Z2Z else load().shafftCopyFromBufferF
        check(f(out.ctypes.data_as(ctypes.c_void_p), ctypes.c_void_p(self.ptr), n), "copyFromBuffer")
        return out

    def free(self):
        if self.ptr:
            f = load().shafftFreeBufferD if self.precision == Z2Z else load().shafftFreeBufferF
            f(ctypes.c_void_p(self.ptr))
            self.ptr = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def download_ptr(ptr: int, count: int, precision: int) -> np.ndarray:
    dt = np.complex128 if precision == Z2Z else np.complex64
    out = np.empty(int(count), dtype=dt)
    f = load().shafftCopyFromBufferD if precision == Z2Z else load().shafftCopyFromBufferF
    check(f(out.ctypes.data_as(ctypes.c_void_p), ctypes.c_void_p(ptr), int(count)), "copyFromBuffer")
    return out


# ---------------------------------------------------------------------------
# Plans (mirror of shafft::FFTND / shafft::FFT1D over the C ABI)
# ---------------------------------------------------------------------------

class _Plan:
    _create = None

    def __init__(self):
        self._lib = load()
        self.handle = ctypes.c_void_p()
        check(getattr(self._lib, self._create)(ctypes.byref(self.handle)), self._create)

    # lifecycle -------------------------------------------------------------
    def plan(self) -> int:
        return self._lib.shafftPlan(self.handle)

    def release(self):
        if self.handle:
            h = ctypes.c_void_p(self.handle.value)
            self._lib.shafftDestroy(ctypes.byref(h))
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    # buffers ---------------------------------------------------------------
    def set_buffers(self, data: int, work: int) -> int:
        return self._lib.shafftSetBuffers(self.handle, ctypes.c_void_p(data), ctypes.c_void_p(work))

    def get_buffers(self):
        d, w = ctypes.c_void_p(), ctypes.c_void_p()
        rc = self._lib.shafftGetBuffers(self.handle, ctypes.byref(d), ctypes.byref(w))
        return rc, (d.value or 0), (w.value or 0)

    def set_stream(self, stream: int) -> int:
        return self._lib.shafftSetStream(self.handle, ctypes.c_void_p(stream))

    # compute ---------------------------------------------------------------
    def execute(self, direction: int) -> int:
        return self._lib.shafftExecute(self.handle, int(direction))

    def execute_normalized(self, direction: int) -> int:
        return self._lib.shafftExecuteNormalized(self.handle, int(direction))

    def normalize(self) -> int:
        return self._lib.shafftNormalize(self.handle)

    # queries ---------------------------------------------------------------
    def alloc_size(self) -> int:
        n = ctypes.c_size_t()
        rc = self._lib.shafftGetAllocSize(self.handle, ctypes.byref(n))
        return n.value if rc == 0 else 0

    def global_size(self) -> int:
        n = ctypes.c_size_t()
        rc = self._lib.shafftGetGlobalSize(self.handle, ctypes.byref(n))
        return n.value if rc == 0 else 0

    def is_configured(self) -> bool:
        v = ctypes.c_int()
        self._lib.shafftIsConfigured(self.handle, ctypes.byref(v))
        return bool(v.value)

    def is_active(self) -> bool:
        v = ctypes.c_int()
        self._lib.shafftIsActive(self.handle, ctypes.byref(v))
        return bool(v.value)


class FFTND(_Plan):
    """shafft::FFTND over the C ABI: init(commDims, dims, precision) ->
    plan() -> set_buffers() -> execute()/normalize()."""
    _create = "shafftNDCreate"

    def init(self, comm_dims, dims, precision=C2C, comm=MPI_COMM_WORLD,
             output_policy=LAYOUT_REDISTRIBUTED) -> int:
        self.dims = tuple(int(d) for d in dims)
        self.precision = precision
        return self._lib.shafftNDInit(self.handle, len(dims), _iarr(comm_dims), _iarr(dims),
                                      int(precision), int(comm), int(output_policy))

    def get_layout(self, layout=TENSOR_LAYOUT_CURRENT):
        n = len(self.dims)
        sub = (ctypes.c_size_t * n)()
        off = (ctypes.c_size_t * n)()
        rc = self._lib.shafftGetLayout(self.handle, sub, off, layout)
        return rc, list(sub), list(off)

    def get_axes(self, layout=TENSOR_LAYOUT_CURRENT):
        n = len(self.dims)
        ca = (ctypes.c_int * n)()
        da = (ctypes.c_int * max(1, n))()
        rc = self._lib.shafftGetAxes(self.handle, ca, da, layout)
        return rc, list(ca), []


class FFT1D(_Plan):
    """shafft::FFT1D over the C ABI."""
    _create = "shafft1DCreate"

    def init(self, n, local_n=None, local_start=0, precision=C2C, comm=MPI_COMM_WORLD) -> int:
        self.dims = (int(n),)
        self.precision = precision
        return self._lib.shafft1DInit(self.handle, int(n), int(n if local_n is None else local_n),
                                      int(local_start), int(precision), int(comm))


def configuration_nd(dims, precision=C2C, comm_dims=None, nda=0, strategy=MAXIMIZE_NDA,
                     mem_limit=0, comm=MPI_COMM_WORLD):
    """shafftConfigurationND: returns (rc, commDims, nda, subsize, offset, commSize)."""
    lib = load()
    n = len(dims)
    cd = _iarr(comm_dims if comm_dims is not None else [0] * n)
    nd = ctypes.c_int(nda)
    sub = (ctypes.c_size_t * n)()
    off = (ctypes.c_size_t * n)()
    cs = ctypes.c_int()
    rc = lib.shafftConfigurationND(n, _iarr(dims), precision, cd, ctypes.byref(nd), sub, off,
                                   ctypes.byref(cs), strategy, mem_limit, comm)
    return rc, list(cd)[:n], nd.value, list(sub), list(off), cs.value


def configuration_1d(n, precision=C2C, comm=MPI_COMM_WORLD):
    lib = load()
    ln, ls, al = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
    rc = lib.shafftConfiguration1D(int(n), ctypes.byref(ln), ctypes.byref(ls), ctypes.byref(al),
                                   precision, comm)
    return rc, ln.value, ls.value, al.value


def backend_name() -> str:
    return load().shafftGetBackendName().decode()


def version_string() -> str:
    return load().shafftGetVersionString().decode()


def native_libraries():
    """Paths of the native libraries this package loads."""
    return [SHAFFT_LIB, _sm100.SM100_LIB, os.path.join(LIB_DIR, "libshafft_mpishim.so")]
