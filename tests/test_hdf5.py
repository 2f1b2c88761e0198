"""The HDF5 output file (maxwellfdtd_b200/hdf5.py): the checksum is Jenkins' lookup3 (its
published test vectors), the file round-trips through the reader with every checksum
verified, its structure follows the format's fixed fields, and solve(fname="out.hdf")
writes the reference's datasets (outputs.jl, monitors.jl write_monitor) with HDF5.jl's
dimension order (the Julia shape reversed)."""
import os
import struct

import numpy as np
import pytest

import cases as C
import maxwellfdtd_b200 as M
from maxwellfdtd_b200 import hdf5


def test_lookup3_vectors():
    assert hdf5.lookup3(b"") == 0xDEADBEEF
    assert hdf5.lookup3(b"Four score and seven years ago") == 0x17770551
    assert hdf5.lookup3(b"Four score and seven years ago", 1) == 0xCD628161


def test_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    tree = {"x": rng.standard_normal(7), "pml": np.arange(6, dtype=np.int64),
            "geometry": rng.integers(0, 3, (4, 5, 6)).astype(np.int64),
            "fields": {"t": np.array([1.0, 2.0]), "Ex": rng.standard_normal((2, 3, 4, 5)).astype(np.float32)},
            "monitors": {"1": {"issum": True, "w": np.array([1.0, 2.0, 3.0]),
                               "Ex": rng.standard_normal((3, 4)) + 1j * rng.standard_normal((3, 4))}},
            "empty": np.zeros((0, 2)), "byte": np.arange(5, dtype=np.uint8)}
    p = str(tmp_path / "a.hdf")
    hdf5.write(p, tree)
    got = hdf5.read(p)

    def same(a, b):
        if isinstance(a, dict):
            assert set(a) == set(b)
            for k in a:
                same(a[k], b[k])
        else:
            a = np.asarray(a)
            a = a.astype(np.uint8) if a.dtype == np.bool_ else a
            assert a.shape == b.shape and a.dtype == b.dtype and np.array_equal(a, b)
    same(tree, got)


def test_format_fields(tmp_path):
    p = str(tmp_path / "b.h5")
    hdf5.write(p, {"v": np.arange(3, dtype=np.float64)})
    raw = open(p, "rb").read()
    assert raw[:8] == b"\x89HDF\r\n\x1a\n" and raw[8] == 2 and raw[9] == 8 and raw[10] == 8
    eof, root = struct.unpack_from("<QQ", raw, 28)
    assert eof == len(raw) and raw[root:root + 4] == b"OHDR"
    assert struct.unpack_from("<I", raw, 44)[0] == hdf5.lookup3(raw[:44])
    with pytest.raises(ValueError):
        bad = bytearray(raw)
        bad[root + 12] ^= 0xFF
        q = str(tmp_path / "c.h5")
        open(q, "wb").write(bytes(bad))
        hdf5.read(q)


def test_solve_writes_reference_layout(tmp_path, oracle_lib):
    model = C.model_materials(3)
    mons = C.monitors(3)
    fname = str(tmp_path / "out.hdf")
    sol = M.solve(model, backend=M.B200(np.float32, library=oracle_lib), monitors=mons, fname=fname, nstride=20)
    f = hdf5.read(fname)
    g = model.grid
    assert {"x", "y", "z", "t", "pml", "geometry", "Sa", "E2", "fields", "monitors"} <= set(f)
    assert f["Sa"].shape == (g.Nz, g.Ny, g.Nx) and np.array_equal(f["Sa"].T, sol.out["Sa"])
    assert f["fields"]["Ex"].shape == (len(f["fields"]["t"]), g.Nz, g.Ny, g.Nx)
    assert np.array_equal(f["fields"]["Ex"].T, sol.out["fields/Ex"])
    assert f["geometry"].dtype == np.int64 and np.array_equal(f["geometry"].T, model.geometry)
    m4 = f["monitors"]["4"]
    assert m4["Ex"].dtype == np.complex128 and np.array_equal(m4["Ex"].T, sol.out["monitors/4/Ex"])
    assert int(m4["issum"]) == 0 and np.array_equal(m4["w"], sol.out["monitors/4/w"])
    assert np.array_equal(f["monitors"]["2"]["Hy"], sol.out["monitors/2/Hy"])   # summed: a vector of Nt
