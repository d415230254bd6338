"""Pass-specialised kernels (host side, no GPU): every register-staged pass of
the layered workload gets generated CUDA source, and NVRTC compiles it for
sm_100a. The GPU side (the same amplitudes as the interpreter and the
oracle) is tests/test_gpu_passkernels.py."""
import ctypes
import ctypes.util

import pytest

import kate_b200 as K
from kate_b200 import _lib, circuits


def plan(circ, **kw):
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.kate_plan_create(circ.handle, 12, 4, 0, ctypes.byref(h)) == 0, _lib.last_error()
    return L, h


def source(L, h, i, from_zero=0):
    size = ctypes.c_size_t()
    st = L.kate_plan_pass_source(h, i, from_zero, None, 0, ctypes.byref(size))
    if st != 0:
        return None
    buf = ctypes.create_string_buffer(size.value)
    assert L.kate_plan_pass_source(h, i, from_zero, buf, size.value, ctypes.byref(size)) == 0
    return buf.value.decode()


def nvrtc():
    for name in ("libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"):
        try:
            return ctypes.CDLL(name)
        except OSError:
            continue
    return None


def nvrtc_compile(lib, src):
    prog = ctypes.c_void_p()
    assert lib.nvrtcCreateProgram(ctypes.byref(prog), src.encode(), b"kate_pass.cu", 0, None, None) == 0
    opts = [b"--gpu-architecture=sm_100a", b"-std=c++17", b"-default-device", b"--fmad=true"]
    arr = (ctypes.c_char_p * len(opts))(*opts)
    r = lib.nvrtcCompileProgram(prog, len(opts), arr)
    n = ctypes.c_size_t()
    lib.nvrtcGetProgramLogSize(prog, ctypes.byref(n))
    log = ctypes.create_string_buffer(n.value)
    lib.nvrtcGetProgramLog(prog, log)
    cub = ctypes.c_size_t()
    if r == 0:
        lib.nvrtcGetCUBINSize(prog, ctypes.byref(cub))
    lib.nvrtcDestroyProgram(ctypes.byref(prog))
    return r, log.value.decode(errors="replace"), cub.value


def test_every_pass_of_the_layered_workload_has_a_kernel():
    n = 30
    c = K.Circuit(n, circuits.layered(n, 20, seed=1234))
    L, h = plan(c)
    try:
        np_ = ctypes.c_int()
        L.kate_plan_num_passes(h, ctypes.byref(np_))
        assert np_.value == 58
        srcs = [source(L, h, i) for i in range(np_.value)]
        assert all(s is not None for s in srcs)
        # Straight-line code: one __global__ per pass, no op dispatch.
        for s in srcs:
            assert s.count("__global__") == 1 and "switch" not in s
        z = source(L, h, 0, 1)
        assert z is not None and z != srcs[0] and "c != 0" in z
    finally:
        L.kate_plan_destroy(h)


def test_pass_without_a_program_has_no_source():
    # n < 12: generic kernel only.
    c = K.Circuit(8, circuits.layered(8, 2, seed=1))
    L, h = plan(c)
    try:
        size = ctypes.c_size_t()
        assert L.kate_plan_pass_source(h, 0, 0, None, 0, ctypes.byref(size)) != 0
        assert "register-staged" in _lib.last_error()
    finally:
        L.kate_plan_destroy(h)


def test_generated_sources_compile_for_sm100a():
    lib = nvrtc()
    if lib is None:
        pytest.skip("libnvrtc not available")
    n = 30
    c = K.Circuit(n, circuits.layered(n, 20, seed=1234))
    L, h = plan(c)
    try:
        # A two-stage pass with direct HBM I/O, a pass copied in/out through
        # shared memory, the eight-stage pass, pass 0 generating |0...0> and
        # pass 0 computing a product-state input.
        for i, fz in ((2, 0), (10, 0), (19, 0), (0, 1), (0, 2)):
            r, log, nbytes = nvrtc_compile(lib, source(L, h, i, fz))
            assert r == 0, log
            assert nbytes > 0
    finally:
        L.kate_plan_destroy(h)


def test_product_form_of_first_passes_compiles():
    """The form of pass 0 that computes a product-state input (per-qubit
    factors as a second parameter): for first passes that load straight from
    HBM and for ones that copy in through shared memory."""
    lib = nvrtc()
    if lib is None:
        pytest.skip("libnvrtc not available")
    seen = set()
    for n, gates in ((30, circuits.layered(30, 20, seed=1234)), (20, circuits.qulacs_bench(20)),
                     (16, circuits.qft(16)), (22, circuits.hea(22, 4, seed=3))):
        c = K.Circuit(n, gates)
        L, h = plan(c)
        try:
            src = source(L, h, 0, 2)
            if src is None:
                continue
            assert "ProdTab PI" in src and "ptl[" in src
            seen.add("cp.async" in source(L, h, 0, 0))
            r, log, nbytes = nvrtc_compile(lib, src)
            assert r == 0, log
        finally:
            L.kate_plan_destroy(h)
    assert seen, "no first pass had a product form"


def test_searched_headline_plan_reads_and_writes_hbm_directly():
    # With the planner's search (what 30-qubit complex128 simulators use),
    # the first stage of most passes loads straight from HBM and the last
    # stage stores straight to it (its lanes 0..3 hold the tile bits that
    # the write-back moves to physical bits 0..3), so those passes skip the
    # copy-in and write-back through the shared tile.
    n = 30
    c = K.Circuit(n, circuits.layered(n, 20, seed=1234))
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.kate_plan_create(c.handle, 12, 4, 16, ctypes.byref(h)) == 0
    npass = ctypes.c_int()
    L.kate_plan_num_passes(h, ctypes.byref(npass))
    srcs = [source(L, h, i) for i in range(npass.value)]
    L.kate_plan_destroy(h)
    assert all(s for s in srcs)
    direct_loads = sum("cp.async.cg" not in s for s in srcs)
    direct_stores = sum("cpT" not in s for s in srcs)
    assert npass.value <= 21
    assert direct_loads >= 16 and direct_stores >= 15


def test_stage_quarter_warp_lanes_lie_in_distinct_bank_groups():
    # A 16-byte shared access is served per quarter warp: the three low
    # lane bits of a stage must sit on tile bits of distinct residue mod 3
    # (distinct bank groups under the tile's swizzle), or the exchange
    # loads and stores take extra wavefronts.
    from plan_emulator import PlanView
    pv = PlanView(K.Circuit(30, circuits.layered(30, 20, seed=1234)), 12, 4, 16)
    total = good = 0
    for prog in pv.programs:
        for si in range(int(prog["nstages"])):
            total += 1
            good += len({int(t) % 3 for t in prog["stb"][si][:3]}) == 3
    assert total > 100 and good >= 0.95 * total
