"""TFSF incident data in the compact layouts (MFD_INC_ALONG_B / ALONG_A / UNIFORM).

A plane wave along z depends on z and t only, so its face arrays are passed as [nt][b] or
[nt] values and expanded by the library.  The same model with every array in the
reference's full [nt][b][a] layout must give the same results bit for bit (oracle), on the
GPU as on the oracle, and the device must hold only the compact data.
"""
import numpy as np
import pytest

import cases as C
import maxwellfdtd_b200 as M
from maxwellfdtd_b200 import _abi, sources
from maxwellfdtd_b200 import workloads as W


def _full_layouts(monkeypatch):
    """Make the Python mirror pass every incident array in the full layout."""
    def full(r, extent):
        r = np.broadcast_to(r, (extent[0], extent[1], r.shape[2]))
        return np.ascontiguousarray(np.transpose(r, (2, 1, 0)).reshape(r.shape[2], -1)), _abi.MFD_INC_FULL
    monkeypatch.setattr(sources, "_compact", full)


def _models(nt=24, n=40):
    model3, mons3 = W.plasmonics_256(nt=nt, n=n)
    return model3, mons3


def test_layouts_chosen():
    model, _ = _models()
    shapes = model.tfsf[3]
    names = sources.TFSF_NAMES_3D
    got = dict(zip(names, shapes))
    assert got["incHy_1yz"] == _abi.MFD_INC_ALONG_B and got["incEx_x1z"] == _abi.MFD_INC_ALONG_B
    assert got["incHy_xy1"] == _abi.MFD_INC_UNIFORM and got["incEz_1yz"] == _abi.MFD_INC_UNIFORM
    arrays = dict(zip(names, model.tfsf[2]))
    assert arrays["incHy_1yz"].shape == (model.Nt, model.tfsf[1][2] - model.tfsf[0][2])   # [nt][Nzi]
    assert arrays["incHy_xy1"].shape == (model.Nt, 1)


def test_full_arrays_are_compacted(monkeypatch):
    """Data given in the full layout (as a record file holds them) with values constant
    along a face axis are passed compact."""
    model, _ = _models()
    i1, i2, arrays, shapes = model.tfsf
    d = W._plane_wave_tfsf(model.grid, i1, i2, model.t, lambda s: np.exp(-((s - 5e-15) / 2e-15) ** 2), 0.0, model.dt)
    full = {}
    (ix1, iy1, iz1), (ix2, iy2, iz2) = i1, i2
    Nxi, Nyi, Nzi = ix2 - ix1, iy2 - iy1, iz2 - iz1
    for k, name in enumerate(sources.TFSF_NAMES_3D):
        face, j = k // 4, k % 4
        a, b = ((Nyi + 1, Nzi) if j in (0, 3) else (Nyi, Nzi + 1)) if face < 2 else \
            ((Nxi + 1, Nzi) if j in (0, 3) else (Nxi, Nzi + 1)) if face < 4 else \
            ((Nxi + 1, Nyi) if j in (0, 3) else (Nxi, Nyi + 1))
        full[name] = np.ascontiguousarray(np.broadcast_to(d[name], (model.Nt, b, a)))
    for k in ("t", "box", "x", "y", "z"):
        full[k] = d[k]
    m2 = M.Model(model.grid, M.TFSFSource(data=full), tmax=model.t[-1], pml=12 * model.grid.dx)
    assert list(m2.tfsf[3]) == list(shapes)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_compact_equals_full_oracle(dtype, monkeypatch, oracle_lib):
    model, mons = _models()
    compact = C.run_all(model, oracle_lib, dtype, mons)
    _full_layouts(monkeypatch)
    model_f, mons_f = _models()
    assert all(s == _abi.MFD_INC_FULL for s in model_f.tfsf[3])
    full = C.run_all(model_f, oracle_lib, dtype, mons_f)
    assert set(compact) == set(full)
    for k in compact:
        assert np.array_equal(compact[k], full[k]), k
    assert np.abs(compact["field/Ex"]).max() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_compact_gpu_equals_full_oracle(dtype, monkeypatch, oracle_lib, gpu_lib):
    model, mons = _models()
    got = C.run_all(model, gpu_lib, dtype, mons)
    b, _ = model.build_desc(dtype, mons)
    st = _abi.Stepper(gpu_lib, b, dtype)
    small = st.device_bytes()
    st.close()
    _full_layouts(monkeypatch)
    model_f, mons_f = _models()
    ref = C.run_all(model_f, oracle_lib, dtype, mons_f)
    for k in ref:
        assert np.array_equal(ref[k], got[k]), k
    b, _ = model_f.build_desc(dtype, mons_f)
    st = _abi.Stepper(gpu_lib, b, dtype)
    big = st.device_bytes()
    st.close()
    assert big > small   # the full layout holds every face value of every step


@pytest.mark.gpu
@pytest.mark.parametrize("ndim", [2, 3])
def test_compact_record_replay_gpu(ndim, oracle_lib, gpu_lib):
    """A vacuum record run's faces (periodic in x, y) are constant along the face's
    transverse axes: the replay passes them compact and stays bit-identical to the oracle."""
    rec = C.model_tfsf_record(ndim)
    box = C.tfsf_box(ndim)
    r = C.run_all(rec, oracle_lib, np.float32, tfsf_box_=box)
    record = {k[4:]: v for k, v in r.items() if k.startswith("rec/")}
    rep = C.model_tfsf_replay(ndim, record)
    assert any(s != _abi.MFD_INC_FULL for s in rep.tfsf[3])
    ref = C.run_all(rep, oracle_lib, np.float32)
    got = C.run_all(rep, gpu_lib, np.float32)
    for k in ref:
        assert np.array_equal(ref[k], got[k]), k
