"""mfd_read_integral_noalloc against mfd_read_integral, through the C ABI.

The allocation-free read stages JE and rho_end through a fixed device buffer a few z-planes
at a time; it must return exactly what mfd_read_integral returns (tolerance: bit-identical,
the same values are gathered by the same arithmetic), on two calls in a row, for grids that
fit in one chunk and grids that need several, and refuse grids whose z-plane does not fit.
It must also do what it exists for: take no device memory.  The device's default memory
pool (the one mfd_read_integral's temporary comes from) is watched through the driver API:
its high-water mark of memory in use must not rise during the reads.
"""
import ctypes as C

import numpy as np
import pytest

import cases
import maxwellfdtd_b200 as M
from maxwellfdtd_b200 import _abi

pytestmark = pytest.mark.gpu

SCRATCH = 16 << 20   # MFD_NOALLOC_SCRATCH_BYTES
WHICH = (_abi.MFD_INT_SA, _abi.MFD_INT_E2, _abi.MFD_INT_JE, _abi.MFD_INT_RHO)


def _noalloc_fn(lib):
    f = lib.lib.mfd_read_integral_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
    return f


def _read_noalloc(st, which):
    dt = np.float64 if which == _abi.MFD_INT_RHO else st.dtype
    out = np.full(st.N, np.nan, dtype=dt)   # the read must overwrite every element
    rc = _noalloc_fn(st.lib)(st.h, int(which), out.ctypes.data_as(C.c_void_p))
    return rc, out


def _plasma_box(n, dtype, nsteps=12):
    """A grid filled with an ionising medium, driven by a strong plane source at z = 0."""
    nx, ny, nz = n
    g = cases.grid3(n)
    E0 = 2e10
    src = M.SoftSource(geometry=lambda x, y, z: np.abs(z) < 26e-9, waveform=lambda x, y, z, t: E0 * np.sin(2.4e15 * t),
                       component="Ex")
    pl = M.Plasma(ionrate=M.PowerLawRate(order=8, sigma=1e-130), rho0=2.1e28, nuc=1 / 1e-15, frequency=2.4e15,
                  Uiev=9.0, mr=0.64)
    mat = M.Material(geometry=lambda x, y, z: np.abs(z) < 60e-9, eps=2.1, plasma=pl)
    dt = 0.5 / cases.C0 / np.sqrt(3 / (50e-9) ** 2)
    return M.Model(g, src, tmax=(nsteps - 0.5) * dt, pml=0, material=mat)


def _stepper(model, lib, dtype):
    b, _ = model.build_desc(dtype, None)
    st = _abi.Stepper(lib, b, dtype)
    st.run(1, model.Nt)
    return st


def _check_same(st):
    for which in WHICH:
        ref = st.read_integral(which)
        for call in range(2):   # two calls in a row
            rc, got = _read_noalloc(st, which)
            assert rc == _abi.MFD_OK, st.lib.last_error(st.h).decode()
            assert np.array_equal(ref, got), (which, call)
    return st.read_integral(_abi.MFD_INT_RHO)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_noalloc_matches_read_integral(dtype, gpu_lib):
    st = _stepper(cases.model_plasma(3, "power"), gpu_lib, dtype)
    try:
        rho = _check_same(st)
        assert rho.max() > 0, "the case must ionise"
    finally:
        st.close()


def test_noalloc_several_chunks(gpu_lib):
    """1030 x 1024 planes: rho_end (8.4 MB a plane) one plane per chunk, JE (4.2 MB) three."""
    n = (1030, 1024, 4)
    assert SCRATCH // (n[0] * n[1] * 8) == 1 and SCRATCH // (n[0] * n[1] * 4) == 3
    st = _stepper(_plasma_box(n, np.float32), gpu_lib, np.float32)
    try:
        rho = _check_same(st)
        assert rho.max() > 0
    finally:
        st.close()


def test_noalloc_refuses_planes_beyond_scratch(gpu_lib):
    """1500 x 1500 planes: rho_end (18 MB a plane) does not fit, JE (9 MB) does."""
    st = _stepper(_plasma_box((1500, 1500, 2), np.float32, nsteps=2), gpu_lib, np.float32)
    try:
        rc, _ = _read_noalloc(st, _abi.MFD_INT_RHO)
        assert rc == _abi.MFD_ERR_INVALID
        msg = st.lib.last_error(st.h).decode()
        assert "18000000" in msg and str(SCRATCH) in msg, msg
        ref = st.read_integral(_abi.MFD_INT_JE)
        rc, got = _read_noalloc(st, _abi.MFD_INT_JE)
        assert rc == _abi.MFD_OK and np.array_equal(ref, got)
    finally:
        st.close()


def test_noalloc_large_planes_without_plasma(gpu_lib):
    """A model without plasma returns zeros for JE and rho_end from both reads, even when one
    z-plane would not fit the scratch buffer (nothing is staged)."""
    g = cases.grid3((1500, 1500, 2))
    src = M.SoftSource(geometry=(0.0, 0.0, 0.0), waveform=lambda x, y, z, t: cases.pulse(t), component="Ex")
    model = M.Model(g, src, tmax=1.5 * 0.5 / cases.C0 / np.sqrt(3 / (50e-9) ** 2), pml=0)
    st = _stepper(model, gpu_lib, np.float32)
    try:
        for which in (_abi.MFD_INT_JE, _abi.MFD_INT_RHO):
            ref = st.read_integral(which)
            rc, got = _read_noalloc(st, which)
            assert rc == _abi.MFD_OK, st.lib.last_error(st.h).decode()
            assert np.array_equal(ref, got) and not got.any()
    finally:
        st.close()


CU_MEMPOOL_ATTR_USED_MEM_CURRENT, CU_MEMPOOL_ATTR_USED_MEM_HIGH = 7, 8


def _default_pool(device=0):
    """(used_now, used_high, reset_high) of the device's default memory pool (driver API)."""
    cu = C.CDLL("libcuda.so.1")
    cu.cuInit.argtypes = [C.c_uint]
    cu.cuDeviceGet.argtypes = [C.POINTER(C.c_int), C.c_int]
    cu.cuDeviceGetDefaultMemPool.argtypes = [C.POINTER(C.c_void_p), C.c_int]
    cu.cuMemPoolGetAttribute.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    cu.cuMemPoolSetAttribute.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    assert cu.cuInit(0) == 0
    dev = C.c_int()
    assert cu.cuDeviceGet(C.byref(dev), device) == 0
    pool = C.c_void_p()
    assert cu.cuDeviceGetDefaultMemPool(C.byref(pool), dev.value) == 0

    def get(attr):
        v = C.c_uint64()
        assert cu.cuMemPoolGetAttribute(pool, attr, C.byref(v)) == 0
        return v.value

    def reset_high():   # the only value the high-water mark may be set to is 0 (= current use)
        z = C.c_uint64(0)
        assert cu.cuMemPoolSetAttribute(pool, CU_MEMPOOL_ATTR_USED_MEM_HIGH, C.byref(z)) == 0

    return (lambda: get(CU_MEMPOOL_ATTR_USED_MEM_CURRENT)), (lambda: get(CU_MEMPOOL_ATTR_USED_MEM_HIGH)), reset_high


def test_noalloc_takes_no_device_memory(gpu_lib):
    st = _stepper(cases.model_plasma(3, "power"), gpu_lib, np.float32)
    try:
        used, high, reset_high = _default_pool()
        # the watch sees allocations: mfd_read_integral's grid-sized temporary raises the mark
        reset_high()
        base = used()
        st.read_integral(_abi.MFD_INT_JE)
        assert high() > base
        # the allocation-free read, every output, twice in a row: the mark stays put
        reset_high()
        base = used()
        for _ in range(2):
            for which in WHICH:
                rc, _ = _read_noalloc(st, which)
                assert rc == _abi.MFD_OK, st.lib.last_error(st.h).decode()
        assert high() == base == used()
    finally:
        st.close()
