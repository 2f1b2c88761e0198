"""The C ABI: the CUDA library loads without a GPU and exports every function declared in
include/maxwellfdtd.h; the ctypes mirror has the same struct layout as the C compiler;
mfd_create reports a clear error (no crash) when there is no device or the descriptor is bad."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import maxwellfdtd_b200 as M
from maxwellfdtd_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "maxwellfdtd.h")


def declared_functions():
    with open(HEADER) as f:
        src = f.read()
    return sorted(set(re.findall(r"MFD_API\s+[\w\s\*]+?\b(mfd_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def cuda_lib():
    from maxwellfdtd_b200 import build
    build.build()
    return C.CDLL(build.OUT)


def test_library_exports_every_declared_function(cuda_lib):
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(cuda_lib, n)]
    assert not missing, missing


def test_oracle_exports_the_same_api(oracle_lib):
    for n in declared_functions():
        short = n[len("mfd_"):]
        if short in ("set_profiling", "kernel_times", "last_run_ms", "device_bytes", "abi_version",
                     "read_integral_noalloc", "set_snapshots", "state_size", "read_state", "write_state") \
                or short.startswith(("batch_", "server_")):
            continue
        assert hasattr(oracle_lib.lib, "oracle_" + short), short


def _c_layout():
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "maxwellfdtd.h"
#define F(s, m) printf(#s "." #m " %zu\n", offsetof(s, m));
int main(void) {
  printf("mfd_pml_layer %zu\n", sizeof(mfd_pml_layer));
  printf("mfd_material %zu\n", sizeof(mfd_material));
  printf("mfd_source %zu\n", sizeof(mfd_source));
  printf("mfd_tfsf %zu\n", sizeof(mfd_tfsf));
  printf("mfd_monitor %zu\n", sizeof(mfd_monitor));
  printf("mfd_desc %zu\n", sizeof(mfd_desc));
  F(mfd_desc, dt) F(mfd_desc, nt) F(mfd_desc, bc) F(mfd_desc, pml) F(mfd_desc, Mh0) F(mfd_desc, geometry)
  F(mfd_desc, nmat) F(mfd_desc, mats) F(mfd_desc, rho_fp64) F(mfd_desc, nsrc) F(mfd_desc, srcs)
  F(mfd_desc, tfsf) F(mfd_desc, nmon) F(mfd_desc, mons) F(mfd_desc, tfsf_record) F(mfd_desc, rec_i1)
  F(mfd_desc, rec_i2) F(mfd_desc, device) F(mfd_desc, mode) F(mfd_desc, nshape) F(mfd_desc, shapes) F(mfd_desc, coords) F(mfd_desc, polarization)
  printf("mfd_shape %zu\n", sizeof(mfd_shape));
  F(mfd_shape, material) F(mfd_shape, p) F(mfd_tfsf, shape)
  F(mfd_material, nq) F(mfd_material, Aq) F(mfd_material, kerr) F(mfd_material, plasma) F(mfd_material, Rava)
  F(mfd_material, rate_kind) F(mfd_material, rate_order) F(mfd_material, rate_n) F(mfd_material, rate_y)
  F(mfd_source, coeff) F(mfd_source, npts) F(mfd_source, cells) F(mfd_source, gt)
  F(mfd_tfsf, order) F(mfd_tfsf, i1) F(mfd_tfsf, i2) F(mfd_tfsf, inc)
  F(mfd_monitor, npts) F(mfd_monitor, cells) F(mfd_monitor, nw) F(mfd_monitor, phasor)
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "lay.c")
        exe = os.path.join(d, "lay")
        with open(src, "w") as f:
            f.write(prog)
        subprocess.check_call(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), src, "-o", exe])
        out = subprocess.check_output([exe]).decode()
    return {l.split()[0]: int(l.split()[1]) for l in out.strip().splitlines()}


def test_ctypes_layout_matches_c():
    lay = _c_layout()
    types = {"mfd_pml_layer": _abi.PmlLayer, "mfd_material": _abi.Material, "mfd_source": _abi.Source,
             "mfd_tfsf": _abi.Tfsf, "mfd_monitor": _abi.Monitor, "mfd_desc": _abi.Desc, "mfd_shape": _abi.Shape}
    for k, v in lay.items():
        if "." in k:
            s, m = k.split(".")
            assert getattr(types[s], m).offset == v, k
        else:
            assert C.sizeof(types[k]) == v, k


def _tiny_model():
    g = M.Grid(zmin=0, zmax=1e-6, Nz=21)
    src = M.SoftSource(geometry=(0.5e-6,), waveform=lambda z, t: np.sin(1e15 * t), component="Ex")
    return M.Model(g, src, tmax=1e-15, pml=0.1e-6)


def test_create_without_device_or_with_bad_desc_returns_status(cuda_lib):
    lib = _abi.Library(os.path.join(ROOT, "maxwellfdtd_b200", "libmaxwellfdtd_b200.so"), "mfd_")
    b, _ = _tiny_model().build_desc(np.float32)
    b.desc.abi_version = 999
    h = C.c_void_p()
    st = lib.create(C.byref(b.desc), C.byref(h))
    assert st == _abi.MFD_ERR_INVALID
    assert "ABI" in lib.create_error().decode()
    b.desc.abi_version = _abi.ABI_VERSION
    st = lib.create(C.byref(b.desc), C.byref(h))
    assert st in (_abi.MFD_OK, _abi.MFD_ERR_NODEVICE)
    if st == _abi.MFD_OK:
        lib.destroy(h)


def test_oracle_rejects_bad_descriptors(oracle_lib):
    m = _tiny_model()
    b, _ = m.build_desc(np.float64)
    b.desc.ndim = 2    # 2-D with ny = 1 but nx = 1 is fine; make nz invalid instead
    b.desc.nz = 0
    h = C.c_void_p()
    assert oracle_lib.create(C.byref(b.desc), C.byref(h)) == _abi.MFD_ERR_INVALID
    b, _ = m.build_desc(np.float64)
    b.desc.tfsf.enabled = 1
    b.desc.tfsf.i1[2], b.desc.tfsf.i2[2] = 1, 5
    assert oracle_lib.create(C.byref(b.desc), C.byref(h)) == _abi.MFD_ERR_INVALID
    assert "TFSF box" in oracle_lib.create_error().decode()


def test_readers_fill_caller_buffers(oracle_lib):
    """read_field / read_integral / read_monitor write into a buffer the caller owns (for
    example page-locked memory) and refuse one of the wrong size or type."""
    import cases as C
    model = C.model_vacuum(2)
    mons = C.monitors(2)
    b, meta = model.build_desc(np.float32, mons)
    st = _abi.Stepper(oracle_lib, b, np.float32)
    st.run(1, model.Nt)
    buf = np.full(st.N, np.nan, np.float32)
    assert st.read_field(6, out=buf) is buf and np.array_equal(buf, st.read_field(6))
    sa = np.empty(st.N, np.float32)
    assert np.array_equal(st.read_integral(_abi.MFD_INT_SA, out=sa), st.read_integral(_abi.MFD_INT_SA))
    mm = meta["monitors"][3]
    shape = (mm["dft"].Nw, len(mm["cells"]))
    spec = np.empty(shape, np.complex128)
    assert np.array_equal(st.read_monitor(3, 6, shape, True, out=spec), st.read_monitor(3, 6, shape, True))
    with pytest.raises(ValueError):
        st.read_field(6, out=np.empty(st.N - 1, np.float32))
    with pytest.raises(ValueError):
        st.read_field(6, out=np.empty(st.N, np.float64))
    st.close()


def test_geometry_indices_follow_a_column_major_scan():
    """Monitor and source cell lists are the set cells' linear indices (x fastest), sorted:
    the same as a column-major scan of the mask, for 1-D, 2-D and 3-D masks."""
    from maxwellfdtd_b200 import geometry

    class Shape:
        def __init__(self, shape):
            self.shape, self.ndim = shape, len(shape)

    rng = np.random.default_rng(1)
    for shape in [(40,), (13, 1, 7), (9, 5, 4), (1, 6, 11)]:
        for frac in (0.0, 0.05, 0.5, 1.0):
            mask = rng.uniform(size=shape) < frac
            got = geometry.geometry2indices(mask, Shape(shape), coords=[np.arange(n) for n in shape])
            assert got.dtype == np.int64
            assert np.array_equal(got, np.flatnonzero(mask.ravel(order="F")))


def test_descriptor_inputs_in_caller_storage(oracle_lib):
    """Model.build_desc(host_alloc=...) puts the large input arrays in storage the caller
    provides (e.g. page-locked memory); the oracle's results are unchanged."""
    import cases
    g = cases.grid3((128, 128, 64))   # a material map of 1 MiB
    src = M.SoftSource(geometry=(0.0, 0.0, 0.0), waveform=lambda x, y, z, t: 1e3 * cases.pulse(t), component="Ez")
    ball = M.Material(geometry=lambda x, y, z: x * x + y * y + z * z <= (400e-9) ** 2, eps=2.25)
    model = M.Model(g, src, tmax=1e-15, pml=0, material=ball)
    got_alloc = []

    def alloc(n, dtype):
        a = np.empty(n, dtype)
        got_alloc.append(a)
        return a

    outs = []
    for host_alloc in (None, alloc):
        b, meta = model.build_desc(np.float32, None, host_alloc=host_alloc)
        st = _abi.Stepper(oracle_lib, b, np.float32)
        st.run(1, 5)
        outs.append(st.read_field(8))
        st.close()
    assert got_alloc, "no array went to the caller's storage"
    assert np.array_equal(outs[0], outs[1])


def _c_fields(src, name):
    body = re.search(r"typedef struct " + name + r" \{(.*?)\} " + name + ";", src, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        decl = re.sub(r"\[[^\]]*\]", "", decl)
        names += [re.findall(r"(\w+)\s*$", v.strip())[0] for v in decl.split(",")]   # the declarator names
    return names


def _julia_fields(src, name):
    body = re.search(r"struct " + name + r"\n(.*?)\nend", src, re.S).group(1)
    return re.findall(r"(\w+)::", body)


def test_julia_shim_mirrors_header():
    """julia/MaxwellFDTDB200.jl declares the descriptor structs with the header's fields in the
    header's order (the shim cannot run here: no Julia)."""
    with open(HEADER) as f:
        c = f.read()
    with open(os.path.join(ROOT, "julia", "MaxwellFDTDB200.jl")) as f:
        jl = f.read()
    for cname, jname in (("mfd_shape", "MfdShape"), ("mfd_pml_layer", "MfdPmlLayer"), ("mfd_material", "MfdMaterial"), ("mfd_source", "MfdSource"),
                         ("mfd_tfsf", "MfdTFSF"), ("mfd_monitor", "MfdMonitor"), ("mfd_desc", "MfdDesc")):
        assert _c_fields(c, cname) == _julia_fields(jl, jname), cname
    for fn in declared_functions():
        if fn.startswith(("mfd_batch_", "mfd_set_profiling", "mfd_kernel_times", "mfd_last_run_ms", "mfd_device_bytes",
                          "mfd_abi_version", "mfd_status", "mfd_write_field", "mfd_read_tfsf_record",
                          "mfd_tfsf_record_size", "mfd_set_snapshots", "mfd_server_poll", "mfd_server_info",
                          "mfd_server_footprint")):
            continue
        assert ":" + fn + "," in jl, fn
