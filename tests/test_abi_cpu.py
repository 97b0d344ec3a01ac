"""C-ABI boundary checks that need no GPU: the libraries load, export every
function include/*.h declares, and the host state machine returns the
reference's status codes (src/cpp/shafft.cpp, src/cpp/shafft_internal.cpp)."""
import ctypes
import json
import os
import re
import subprocess
import sys
import threading

import pytest

import shafft_b200 as S
from shafft_b200 import _sm100

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header):
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    names = set()
    for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(([^;{)]*)\)\s*;", text):
        name = m.group(1)
        if name in ("if", "while", "sizeof", "return", "switch", "defined"):
            continue
        pre = text[max(0, m.start() - 80):m.start()]
        if "typedef" in pre.split(";")[-1] or "#define" in pre.split("\n")[-1]:
            continue
        names.add(name)
    return names


@pytest.mark.parametrize("header,lib", [
    ("include/shafft/shafft.h", "shafft_b200/lib/libshafft.so"),
    ("include/shafft/shafft_f03.h", "shafft_b200/lib/libshafft.so"),
    ("include/shafft_sm100.h", "shafft_b200/lib/libshafft_sm100.so"),
    ("include/mpi_shim/mpi.h", "shafft_b200/lib/libshafft_mpishim.so"),
])
def test_every_declared_symbol_is_exported(header, lib):
    names = declared_functions(os.path.join(ROOT, header))
    assert len(names) > 5
    so = ctypes.CDLL(os.path.join(ROOT, lib))
    missing = [n for n in sorted(names) if not hasattr(so, n)]
    assert not missing, missing


def test_backend_and_version():
    assert S.backend_name() == "sm100"
    assert S.version_string() == "1.1.0-alpha"
    a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    S.load().shafftGetVersion(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    assert (a.value, b.value, c.value) == (1, 1, 0)


def test_nd_state_machine_without_gpu():
    p = S.FFTND()
    assert not p.is_configured()
    assert p.plan() == S.ERR_PLAN_NOT_INIT                      # plan before init
    assert p.execute(S.FORWARD) == S.ERR_PLAN_NOT_INIT          # execute before plan
    assert p.normalize() == S.ERR_PLAN_NOT_INIT                 # normalize before plan
    assert p.init([1, 1, 1], [64, 64, 32]) == 0
    assert p.is_configured() and p.is_active()
    assert p.alloc_size() == 64 * 64 * 32 and p.global_size() == 64 * 64 * 32
    assert p.init([1, 1, 1], [64, 64, 32]) == S.ERR_INVALID_STATE  # re-init
    assert p.set_buffers(0, 0) == S.ERR_NULLPTR
    rc, d, w = p.get_buffers()
    assert rc == S.ERR_NO_BUFFER and d == 0 and w == 0
    assert p.execute(S.FORWARD) == S.ERR_PLAN_NOT_INIT
    rc, sub, off = p.get_layout()
    assert rc == 0 and sub == [64, 64, 32] and off == [0, 0, 0]
    rc, ca, da = p.get_axes()
    assert rc == 0 and ca == [0, 1, 2]


@pytest.mark.parametrize("comm_dims,dims,code", [
    ([1, 1, 2], [4, 4, 4], S.ERR_INVALID_DECOMP),   # last axis distributed
    ([0, 1, 1], [4, 4, 4], S.ERR_INVALID_DECOMP),   # unresolved zeros (resolve through configurationND)
    ([2, 1, 1], [4, 4, 4], S.ERR_INVALID_DECOMP),   # grid of 2 on one rank
    ([1, 1, 1], [4, 0, 4], S.ERR_INVALID_DIM),
])
def test_nd_init_errors(comm_dims, dims, code):
    p = S.FFTND()
    assert p.init(comm_dims, dims) == code
    assert S.load().shafftLastErrorStatus() == code


def test_nd_init_bad_type_and_null():
    p = S.FFTND()
    assert p.init([1], [8], precision=7) == S.ERR_INVALID_FFTTYPE
    lib = S.load()
    assert lib.shafftNDInit(None, 1, None, None, 0, S.MPI_COMM_WORLD, 0) == S.ERR_NULLPTR
    assert lib.shafftPlan(None) == S.ERR_NULLPTR
    assert lib.shafftExecute(None, 0) == S.ERR_NULLPTR


def test_inactive_rank_plan_is_noop():
    # plan_data_base.hpp:35-58 -- inactive ranks (MPI_COMM_NULL) execute nothing
    p = S.FFTND()
    assert p.init([1, 1], [8, 8], comm=S.MPI_COMM_NULL) == 0
    assert not p.is_active() and p.alloc_size() == 0
    assert p.plan() == 0
    assert p.set_buffers(0, 0) == 0
    assert p.execute(S.FORWARD) == 0 and p.normalize() == 0


def test_fft1d_configuration_and_errors():
    rc, ln, ls, al = S.configuration_1d(1000003)
    assert (rc, ln, ls, al) == (0, 1000003, 0, 1000003)
    p = S.FFT1D()
    assert p.plan() == S.ERR_PLAN_NOT_INIT    # shafftPlan -> fft1dCreatePlans before init (shafft_internal.cpp:760-770)
    assert p.init(1 << 31) == S.ERR_SIZE_OVERFLOW
    q = S.FFT1D()
    assert q.init(0) == S.ERR_INVALID_DIM
    r = S.FFT1D()
    assert r.init(4096) == 0 and r.alloc_size() == 4096
    assert r.init(4096) == S.ERR_INVALID_STATE


def test_configuration_nd():
    rc, cd, nda, sub, off, cs = S.configuration_nd([64, 64, 32])
    assert rc == 0 and cd == [1, 1, 1] and nda == 0 and sub == [64, 64, 32] and off == [0, 0, 0] and cs == 1
    # memLimit counts data + work buffers (configuration.cpp:26-58)
    rc, *_ = S.configuration_nd([64, 64, 32], mem_limit=2 * 8 * 64 * 64 * 32)
    assert rc == 0
    rc, *_ = S.configuration_nd([64, 64, 32], mem_limit=2 * 8 * 64 * 64 * 32 - 1)
    assert rc == S.ERR_INVALID_DECOMP


def test_error_state_is_thread_local():
    lib = S.load()
    p = S.FFTND()
    assert p.init([1, 1, 2], [4, 4, 4]) == S.ERR_INVALID_DECOMP
    seen = {}

    def other():
        lib.shafftClearLastError()
        seen["status"] = lib.shafftLastErrorStatus()
    t = threading.Thread(target=other)
    t.start()
    t.join()
    assert seen["status"] == 0
    assert lib.shafftLastErrorStatus() == S.ERR_INVALID_DECOMP
    assert lib.shafftErrorSourceName(0) == b"SHAFFT"
    assert lib.shafftErrorSourceName(2) == b"CUDA"
    lib.shafftClearLastError()
    assert lib.shafftLastErrorStatus() == 0


def test_planner_fuses_exchange_block_maps():
    """Host-only planner: where a slab exchange's pack / unpack goes.  Forward
    (store map, pack along axis 1 into 2 blocks): the last step, the column
    pass of axis 1, writes the blocks.  Backward (load map): the plan starts
    with that column pass, out of place, reading the blocks, and the row pass
    of axis 2 follows in place.  Non-power-of-two maps stay separate."""
    # a 3-D slab exchange distributes the last axis: blocks of 512 / P points
    q = _sm100.plan_query_mapped([256, 512, 512], [1, 2], 0, None, (256 * 512, 512, 1, 2))
    assert q["fused"] == 2 and [s["map"] for s in q["steps"]] == [0, 2]
    q = _sm100.plan_query_mapped([256, 512, 512], [1, 2], 0, (256 * 512, 512, 1, 2), None)
    assert q["fused"] == 1 and [s["map"] for s in q["steps"]] == [1, 0]
    q = _sm100.plan_query_mapped([256, 512, 512], [1, 2], 0, None, (256, 512, 512, 2))
    assert q["fused"] == 2 and [s["map"] for s in q["steps"]] == [0, 2]
    assert q["steps"][-1]["fast"] == 1 and q["steps"][-1]["out"] == "dst"
    q = _sm100.plan_query_mapped([256, 512, 512], [1, 2], 0, (256, 512, 512, 2), None)
    assert q["fused"] == 1 and [s["map"] for s in q["steps"]] == [1, 0]
    assert [(s["in"], s["out"]) for s in q["steps"]] == [("src", "dst"), ("dst", "dst")]
    q = _sm100.plan_query_mapped([64, 64, 32], [1, 2], 1, (64, 64, 32, 4), None)
    assert q["fused"] == 1
    q = _sm100.plan_query_mapped([8, 48, 32], [1, 2], 0, None, (8, 48, 32, 2))
    assert q["fused"] == 0 and all(s["map"] == 0 for s in q["steps"])
    q = _sm100.plan_query_mapped([8, 64, 32], [1, 2], 0, None, (8, 64, 32, 3))  # uneven blocks
    assert q["fused"] == 0
    with pytest.raises(RuntimeError):
        _sm100.plan_query_mapped([8, 64, 32], [1, 2], 0, None, (8, 64, 16, 2))  # wrong element count


def test_planner_direct_dft_range():
    """Host-only planner: an axis with a prime factor above 13 is one direct
    DFT pass while L^2 <= 128 M (M the Bluestein length: every L up to 362),
    Bluestein beyond; SHAFFT_SM100_DIRECT_MAX caps the direct range."""
    def kinds(dims, prec=0):
        return [s["kind"] for s in _sm100.plan_query(list(dims), prec)["steps"]]
    for L in (17, 131, 257, 263, 331, 353, 362):
        assert kinds([L]) == ["pass"], L
    for L in (367, 383, 509, 1021):
        assert kinds([L])[0] == "bluestein_modulate", L
    assert kinds([5, 353], 1) == ["pass", "pass"]
    old = os.environ.get("SHAFFT_SM100_DIRECT_MAX")
    try:
        os.environ["SHAFFT_SM100_DIRECT_MAX"] = "128"
        assert kinds([131])[0] == "bluestein_modulate"
        assert kinds([127]) == ["pass"]
    finally:
        if old is None:
            del os.environ["SHAFFT_SM100_DIRECT_MAX"]
        else:
            os.environ["SHAFFT_SM100_DIRECT_MAX"] = old


def test_planner_pass_lists():
    """Host-only planner: pass structure of the headline and config shapes."""
    # headline: transposing X and Y passes, then the Z column pass
    q = _sm100.plan_query([512, 512, 512], 0)
    assert [s["kind"] for s in q["steps"]] == ["pass"] * 3
    assert [s["in_row"] for s in q["steps"]] == [1, 1, 0]
    assert all(s["fast"] for s in q["steps"])
    q = _sm100.plan_query([256, 256, 256], 1)
    assert [s["kind"] for s in q["steps"]] == ["pass"] * 3
    # Bluestein, M = 2^21 = 128^3: complex64 fuses the modulate into the first
    # pass's loads and the multiply / demodulate into the stores of the last
    # passes of the two convolution FFTs (bs bits 1, 2, 4); complex128 keeps
    # the element-wise steps
    q = _sm100.plan_query([1000003], 0)
    assert [s["kind"] for s in q["steps"]] == ["pass"] * 6
    assert [s["bs"] for s in q["steps"]] == [1, 0, 2, 0, 0, 4]
    assert [s["in"] for s in q["steps"]][0] == "src" and q["steps"][-1]["out"] == "dst"
    q = _sm100.plan_query([1000003], 1)
    kinds = [s["kind"] for s in q["steps"]]
    assert kinds[0] == "bluestein_modulate" and kinds[-1] == "bluestein_demodulate"
    assert q["steps"][0]["M"] == 1 << 21
    q = _sm100.plan_query([1488375], 0)
    assert all(s["kind"] == "pass" for s in q["steps"]) and len(q["steps"]) == 2
    q = _sm100.plan_query([1, 1, 1], 0)
    assert [s["kind"] for s in q["steps"]] == ["copy"]
    # the final step always writes the destination buffer
    for dims in ([63, 47, 31], [1 << 24], [4096, 3], [7, 11, 13, 17], [2, 3, 4, 5]):
        q = _sm100.plan_query(dims, 0)
        assert q["steps"][-1]["out"] == "dst", dims


def test_planner_prefetch_passes():
    """The complex64 512-point transposing passes run the prefetching kernel
    (one wave ahead by default); column passes, other lengths and
    complex128 run the plain kernel.  Run in a child process so that the
    switches are read fresh."""
    code = ("import json, sys; sys.path.insert(0, sys.argv[1]); from shafft_b200 import _sm100; "
            "print(json.dumps([[s.get('prefetch') for s in _sm100.plan_query(d, p)['steps']] "
            "for d, p in (([512, 512, 512], 0), ([512, 512, 512], 1), ([256, 256, 256], 0))]))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

    def query(**env):
        e = {k: v for k, v in os.environ.items() if not k.startswith("SHAFFT_SM100_PREFETCH")}
        e.update(env)
        r = subprocess.run([sys.executable, "-c", code, root], env=e, capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stderr
        return json.loads(r.stdout.strip().splitlines()[-1])

    assert query() == [[4, 4, 0], [0, 0, 0], [0, 0, 0]]
    assert query(SHAFFT_SM100_PREFETCH_ROW="0") == [[0, 0, 0], [0, 0, 0], [0, 0, 0]]
    assert query(SHAFFT_SM100_PREFETCH_ROW="2", SHAFFT_SM100_PREFETCH_COL="3") == \
        [[2, 2, 3], [0, 0, 0], [0, 0, 0]]


def test_planner_balanced_splits():
    """Measured-faster splits: balanced specialised factors for complex64,
    largest last factor for complex128, balanced generic pair otherwise."""
    def lens(dims, prec=0, flags=0):
        return [s["L"] for s in _sm100.plan_query(dims, prec, flags)["steps"] if s["kind"] == "pass"]
    assert lens([1 << 24]) == [256, 256, 256]
    assert lens([1 << 24], 1) == [64, 512, 512]
    assert lens([1488375]) == [1215, 1225]
    q = _sm100.plan_query([1000003], 0)
    assert [s["L"] for s in q["steps"] if s["kind"] == "pass"] == [128] * 6


def test_planner_tensor_core_modes():
    """Tensor-core planning: every pass (flag 1) or only the axes with a prime
    factor above 13 (flag 2); complex64 only; unknown flags refused."""
    TC, PRIME = _sm100.PLAN_TENSOR_CORE, _sm100.PLAN_TC_PRIME_AXES
    q = _sm100.plan_query([1 << 24], 0, TC)
    assert [s["L"] for s in q["steps"]] == [64] * 4 and all(s["tc"] for s in q["steps"])
    q = _sm100.plan_query([1488375], 0, TC)
    assert sorted(s["L"] for s in q["steps"]) == [27, 35, 35, 45]
    # hybrid: the prime axis on the tensor cores, the smooth ones plain
    q = _sm100.plan_query([4096, 61, 16], 0, PRIME)
    assert [(s["L"], s["tc"]) for s in q["steps"]] == [(16, 0), (61, 1), (64, 0), (64, 0)]
    q = _sm100.plan_query([512, 512, 512], 0, PRIME)
    assert not any(s["tc"] for s in q["steps"]) and all(s["fast"] for s in q["steps"])
    q = _sm100.plan_query([53, 59, 61], 0, PRIME)
    assert [s["L"] for s in q["steps"]] == [61, 59, 53] and all(s["tc"] for s in q["steps"])
    assert q["steps"][-1]["out"] == "dst"
    # primes above 64 keep the plain path (direct DFT or Bluestein)
    q = _sm100.plan_query([97, 64], 0, PRIME)
    assert not any(s.get("tc") for s in q["steps"])
    for bad_prec, flags in ((1, TC), (1, PRIME)):
        with pytest.raises(_sm100.Sm100Error):
            _sm100.plan_query([64], bad_prec, flags)
    with pytest.raises(_sm100.Sm100Error):
        _sm100.plan_query([64], 0, 8)


def test_measured_plan_query_uses_cached_choice(tmp_path, monkeypatch):
    """A measured plan's host-only description follows the per-shape cache
    (written by plan creation on a GPU); without an entry it is the default."""
    cache = tmp_path / "plans.txt"
    monkeypatch.setenv("SHAFFT_SM100_PLAN_CACHE", str(cache))
    M = _sm100.PLAN_MEASURE
    lens = lambda q: [s["L"] for s in q["steps"] if s["kind"] == "pass"]
    assert lens(_sm100.plan_query([1 << 24], 0, M)) == [256, 256, 256]
    # key: precision, flags without the measure bit, axis mask, dims; then
    # balanced, widen, tensor-core choice
    cache.write_text("c64:f0:m18446744073709551615:16777216 0 1 -1\n")
    assert lens(_sm100.plan_query([1 << 24], 0, M)) == [16, 1024, 1024]
    assert lens(_sm100.plan_query([1 << 24], 0)) == [256, 256, 256]


@pytest.mark.parametrize("dims,prec", [((1488375,), 0), ((1488375,), 1), ((4096, 97), 0), ((512, 45, 45), 0),
                                       ((2048, 33), 0), ((35, 27, 45), 0)])
def test_generic_pass_tile_pitch_rule(dims, prec):
    """Generic passes size their shared-memory tile [L][pitch] with pitch W
    for column input and for row input of W <= 4, and W + 1 for row input of
    W >= 8 (bank-conflict rule of generic_pitch in the kernel library)."""
    q = _sm100.plan_query(dims, prec, 0)
    es = 16 if prec else 8
    seen = 0
    for s in q["steps"]:
        if s["kind"] != "pass" or s.get("fast") or s.get("tc"):
            continue
        W = s["W"]
        want = 1 if W == 1 else (W + 1 if (s["in_row"] and W >= 8) else W)
        assert s["smem"] == s["L"] * want * es, s
        seen += 1
    assert seen


def test_nd_init_refuses_unknown_output_policy():
    """An output policy outside {REDISTRIBUTED, INITIAL} returns
    ERR_INVALID_LAYOUT (src/c/shafftc.cpp:42-56, 91-94; the reference's
    tests/integration/c/test_c_api.c "shafftNDInit(invalid_policy)")."""
    p = S.FFTND()
    assert p.init([1, 1, 1], [16, 16, 16], output_policy=2) == 12  # SHAFFT_ERR_INVALID_LAYOUT
    assert not p.is_configured()
    assert p.init([1, 1, 1], [16, 16, 16], output_policy=1) == 0


def test_real_transform_plan_refuses_odd_last_axis():
    """shafft_sm100_rplan_create checks its shape before touching a device:
    an odd last length is refused with SHAFFT_SM100_ENOTSUP."""
    import ctypes
    from shafft_b200 import _sm100
    lib = _sm100.load()
    h = ctypes.c_void_p()
    dims = (ctypes.c_int64 * 2)(3, 5)
    assert lib.shafft_sm100_rplan_create(ctypes.byref(h), 2, dims, 0) == 4
    assert b"even" in lib.shafft_sm100_last_error_message()
    dims = (ctypes.c_int64 * 1)(0)
    assert lib.shafft_sm100_rplan_create(ctypes.byref(h), 1, dims, 0) == 1
