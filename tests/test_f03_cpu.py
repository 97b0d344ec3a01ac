"""Fortran 2003 binding entry points of libshafft.so (include/shafft/shafft_f03.h),
driven through ctypes the way the reference's Fortran module calls them
(src/f03/shafft.f03 binds to these names; src/f03/shafftf03.cpp:11-344 is
the reference's implementation).  No gfortran is installed, so the module
itself is not compiled here; these tests pin the C side it links against:
Fortran communicator handles, heap configuration objects, the field
accessors and setters, string truncation, and NULL safety.  Host-only."""
import ctypes
import os

import pytest

import shafft_b200 as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sz = ctypes.c_size_t
vp = ctypes.c_void_p


@pytest.fixture(scope="module")
def lib():
    L = S.load()
    M = ctypes.CDLL(os.path.join(ROOT, "shafft_b200", "lib", "libshafft_mpishim.so"))
    for name in ("shafftConfigNDAllocf03", "shafftConfig1DAllocf03"):
        getattr(L, name).restype = vp
    for name in ("shafftConfigNDGetAllocElements", "shafftConfigNDGetMemLimit", "shafftConfigNDGetHostnameLen",
                 "shafftConfigNDGetDeviceNameLen", "shafftConfig1DGetGlobalSize",
                 "shafftConfig1DGetAllocElements", "shafftConfig1DGetHostnameLen",
                 "shafftConfig1DGetDeviceNameLen", "shafftConfig1DGetInitialLocalSize",
                 "shafftConfig1DGetInitialLocalStart", "shafftConfig1DGetOutputLocalSize",
                 "shafftConfig1DGetOutputLocalStart"):
        getattr(L, name).restype = sz
        getattr(L, name).argtypes = [vp]
    L.shafftConfigNDSetMemLimit.argtypes = [vp, sz]
    M.MPI_Comm_c2f.restype = ctypes.c_int
    M.MPI_Comm_c2f.argtypes = [ctypes.c_int]
    return L, M


def world_handle(M):
    return ctypes.c_int(M.MPI_Comm_c2f(0x44000000))  # MPI_COMM_WORLD of the shim


def test_nd_config_object_roundtrip(lib):
    L, M = lib
    cfg = vp(L.shafftConfigNDAllocf03())
    assert cfg.value
    shape = (sz * 3)(64, 48, 40)
    fh = world_handle(M)
    rc = L.shafftConfigNDInitf03(cfg, 3, shape, S.C2C, None, 0, 1, S.LAYOUT_REDISTRIBUTED, sz(0),
                                 ctypes.byref(fh))
    assert rc == 0
    assert L.shafftConfigNDGetNdim(cfg) == 3
    assert L.shafftConfigNDGetPrecision(cfg) == S.C2C
    assert L.shafftConfigNDGetIsActive(cfg) == 1
    assert L.shafftConfigNDGetActiveSize(cfg) == 1 and L.shafftConfigNDGetCommSize(cfg) == 1
    assert L.shafftConfigNDGetStrategy(cfg) == 1
    assert L.shafftConfigNDGetAllocElements(cfg) == 64 * 48 * 40
    out = (sz * 3)()
    L.shafftConfigNDGetGlobalShape(cfg, out)
    assert list(out) == [64, 48, 40]
    L.shafftConfigNDGetInitialSubsize(cfg, out)
    assert list(out) == [64, 48, 40]
    L.shafftConfigNDGetOutputOffset(cfg, out)
    assert list(out) == [0, 0, 0]
    cd = (ctypes.c_int * 3)()
    L.shafftConfigNDGetCommDims(cfg, cd)
    assert list(cd) == [1, 1, 1]
    # communicators come back as Fortran handles of the config's own comms
    assert L.shafftConfigNDGetWorldComm(cfg) != 0 and L.shafftConfigNDGetActiveComm(cfg) != 0
    # setters, then re-resolve
    L.shafftConfigNDSetStrategy(cfg, 0)
    L.shafftConfigNDSetMemLimit(cfg, sz(1 << 40))
    L.shafftConfigNDSetHintNda(cfg, 0)
    assert L.shafftConfigNDGetStrategy(cfg) == 0 and L.shafftConfigNDGetMemLimit(cfg) == 1 << 40
    assert L.shafftConfigNDResolvef03(cfg) == 0
    # plan from the config
    plan = vp()
    assert L.shafftNDCreate(ctypes.byref(plan)) == 0
    assert L.shafftNDInitFromConfigf03(plan, cfg) == 0
    comm = ctypes.c_int(0)
    assert L.shafftGetCommunicatorf03(plan, ctypes.byref(comm)) == 0 and comm.value != 0
    assert L.shafftDestroy(ctypes.byref(plan)) == 0
    L.shafftConfigNDRelease(cfg)
    L.shafftConfigNDFreef03(cfg)


def test_string_getters_truncate_like_the_reference(lib):
    L, M = lib
    cfg = vp(L.shafftConfigNDAllocf03())
    fh = world_handle(M)
    shape = (sz * 2)(16, 16)
    assert L.shafftConfigNDInitf03(cfg, 2, shape, S.Z2Z, None, 0, 0, S.LAYOUT_INITIAL, sz(0),
                                   ctypes.byref(fh)) == 0
    n = L.shafftConfigNDGetHostnameLen(cfg)
    assert n >= 1
    full = ctypes.create_string_buffer(n + 8)
    L.shafftConfigNDGetHostname(cfg, full, sz(n + 8))
    assert len(full.value) == n                    # NUL after the copy
    short = ctypes.create_string_buffer(b"#" * 4, 4)
    L.shafftConfigNDGetHostname(cfg, short, sz(1))
    assert short.raw[0:1] == full.value[0:1] and short.raw[1:2] == b"#"  # exactly maxLen bytes, no NUL
    L.shafftConfigNDRelease(cfg)
    L.shafftConfigNDFreef03(cfg)


def test_nd_init_and_configuration_wrappers(lib):
    L, M = lib
    fh = world_handle(M)
    size = (ctypes.c_int * 3)(64, 64, 32)
    cd = (ctypes.c_int * 3)(0, 0, 0)
    nda = ctypes.c_int(0)
    sub = (sz * 3)()
    off = (sz * 3)()
    cs = ctypes.c_int(0)
    rc = L.shafftConfigurationNDf03(3, size, S.C2C, cd, ctypes.byref(nda), sub, off, ctypes.byref(cs), 1,
                                    sz(0), ctypes.byref(fh))
    assert rc == 0 and list(cd) == [1, 1, 1] and list(sub) == [64, 64, 32] and cs.value == 1
    plan = vp()
    assert L.shafftNDCreate(ctypes.byref(plan)) == 0
    pol = ctypes.c_int(S.LAYOUT_REDISTRIBUTED)
    assert L.shafftNDInitf03(plan, 3, cd, size, S.C2C, None, ctypes.byref(pol)) == S.ERR_NULLPTR
    assert L.shafftNDInitf03(plan, 3, cd, size, S.C2C, ctypes.byref(fh), None) == S.ERR_NULLPTR
    assert L.shafftNDInitf03(plan, 3, cd, size, S.C2C, ctypes.byref(fh), ctypes.byref(pol)) == 0
    alloc = sz(0)
    assert L.shafftGetAllocSize(plan, ctypes.byref(alloc)) == 0 and alloc.value == 64 * 64 * 32
    assert L.shafftDestroy(ctypes.byref(plan)) == 0


def test_fft1d_wrappers_and_config(lib):
    L, M = lib
    fh = world_handle(M)
    ln, ls, la = sz(0), sz(0), sz(0)
    assert L.shafftConfiguration1Df03(sz(1000003), ctypes.byref(ln), ctypes.byref(ls), ctypes.byref(la),
                                      S.C2C, ctypes.byref(fh)) == 0
    assert (ln.value, ls.value, la.value) == (1000003, 0, 1000003)
    plan = vp()
    assert L.shafft1DCreate(ctypes.byref(plan)) == 0
    assert L.shafft1DInitf03(plan, sz(4096), sz(4096), sz(0), S.Z2Z, ctypes.byref(fh)) == 0
    assert L.shafftDestroy(ctypes.byref(plan)) == 0
    cfg = vp(L.shafftConfig1DAllocf03())
    assert L.shafftConfig1DInitf03(cfg, sz(4096), S.Z2Z, ctypes.byref(fh)) == 0
    assert L.shafftConfig1DResolvef03(cfg) == 0
    assert L.shafftConfig1DGetGlobalSize(cfg) == 4096 and L.shafftConfig1DGetPrecision(cfg) == S.Z2Z
    assert L.shafftConfig1DGetAllocElements(cfg) == 4096 and L.shafftConfig1DGetIsActive(cfg) == 1
    assert L.shafftConfig1DGetInitialLocalSize(cfg) == 4096 and L.shafftConfig1DGetInitialLocalStart(cfg) == 0
    assert L.shafftConfig1DGetOutputLocalSize(cfg) == 4096 and L.shafftConfig1DGetOutputLocalStart(cfg) == 0
    assert L.shafftConfig1DGetWorldComm(cfg) != 0
    plan = vp()
    assert L.shafft1DCreate(ctypes.byref(plan)) == 0
    assert L.shafft1DInitFromConfigf03(plan, cfg) == 0
    assert L.shafftDestroy(ctypes.byref(plan)) == 0
    L.shafftConfig1DRelease(cfg)
    L.shafftConfig1DFreef03(cfg)


def test_null_configs_are_safe(lib):
    L, M = lib
    assert L.shafftConfigNDGetNdim(None) == 0 and L.shafftConfig1DGetStatus(None) == 0
    assert L.shafftConfigNDGetAllocElements(None) == 0 and L.shafftConfig1DGetGlobalSize(None) == 0
    assert L.shafftConfigNDGetWorldComm(None) == M.MPI_Comm_c2f(0)  # MPI_COMM_NULL's handle
    buf = ctypes.create_string_buffer(b"x" * 4, 4)
    L.shafftConfigNDGetHostname(None, buf, sz(4))
    L.shafftConfigNDGetGlobalShape(None, None)
    L.shafftConfigNDSetHintCommDims(None, None)
    assert buf.raw == b"x" * 4
    fh = world_handle(M)
    assert L.shafftConfigurationNDf03(3, None, 0, None, None, None, None, None, 0, sz(0), None) == S.ERR_NULLPTR
    assert L.shafftGetCommunicatorf03(None, None) == S.ERR_NULLPTR
    assert fh.value != 0
