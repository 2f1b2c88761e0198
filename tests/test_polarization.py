"""The second 2-D field set (Hx, Hz, Dy, Ey; MFD_POL_EY) in the oracle.  The reference has
no such field set, so it is pinned through the reference's other code paths:

- its updates are the 3-D update_H/E kernels (models.jl:735-1162) with every y derivative
  zero: a run equals the Hx, Hz, Dy, Ey of the oracle's 3-D run of the same model on one
  periodic y cell, bit for bit (the other five components stay zero there);
- for a wave along z in an x-invariant medium it is the reference's own 2-D field set
  turned by 90 degrees: Ey equals Ex and Hx equals -Hy of the first field set, bit for bit;
- its TFSF faces leave no field outside the box in vacuum (record run, then replay).
"""
import numpy as np
import pytest

import cases
import polarization_cases as PC
import maxwellfdtd_b200 as M
from maxwellfdtd_b200 import _abi
from maxwellfdtd_b200.sources import comp_index

DTYPES = [np.float64, np.float32]
EY_FIELDS = ("Hx", "Hz", "Dy", "Ey")


def run_desc(lib, b, meta, model, dtype, fields):
    """Every output of a run straight through the ABI."""
    st = _abi.Stepper(lib, b, dtype)
    try:
        st.run(1, model.Nt)
        out = {f: st.read_field(comp_index(f)) for f in fields}
        out["Sa"] = st.read_integral(_abi.MFD_INT_SA)
        if np.any(model.geometry > 0):
            out["E2"] = st.read_integral(_abi.MFD_INT_E2)
        if model.isplasma:
            out["JE"] = st.read_integral(_abi.MFD_INT_JE)
            out["rho"] = st.read_integral(_abi.MFD_INT_RHO)
        for m, mm in enumerate(meta["monitors"]):
            npts, spectral = len(mm["cells"]), mm["kind"] == 1
            for c in ("Hx", "Hz", "Ey"):
                if spectral:
                    shape = (mm["dft"].Nw,) if mm["sum"] else (mm["dft"].Nw, npts)
                else:
                    shape = (model.Nt,) if mm["sum"] else (model.Nt, npts)
                out[f"mon{m}/{c}"] = st.read_monitor(m, comp_index(c), shape, spectral)
    finally:
        st.close()
    return out


def as_3d(b):
    """The same descriptor as a 3-D model of one periodic y cell (dy = 1: every y
    difference is 0 - 0)."""
    d = b.desc
    d.ndim, d.polarization, d.dy = 3, _abi.MFD_POL_HY, 1.0
    d.bc[_abi_face("YL")] = d.bc[_abi_face("YR")] = 1
    return b


def _abi_face(name):
    return {"XL": 0, "XR": 1, "YL": 2, "YR": 3, "ZL": 4, "ZR": 5}[name]


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("name", list(PC.CASES))
def test_ey_equals_3d_on_one_periodic_y_cell(oracle_lib, name, dtype):
    model = PC.CASES[name]()
    mons = cases.monitors(2)
    b2, meta = model.build_desc(dtype, mons, device_geometry=False)
    out2 = run_desc(oracle_lib, b2, meta, model, dtype, EY_FIELDS)
    b3, meta3 = model.build_desc(dtype, mons, device_geometry=False)
    out3 = run_desc(oracle_lib, as_3d(b3), meta3, model, dtype, EY_FIELDS + ("Hy", "Dx", "Dz", "Ex", "Ez"))
    assert np.abs(out2["Ey"]).max() > 0
    for k, v in out2.items():
        assert np.array_equal(v, out3[k]), k
    for f in ("Hy", "Dx", "Dz", "Ex", "Ez"):
        assert not np.any(out3[f]), f


def _slab_models(pol, nsteps=80):
    """A plane wave along z (source plane, x periodic, CPML in z) into Debye+Kerr and
    Lorentz+plasma slabs: x-invariant, so each field set is the other turned by 90 deg."""
    g = cases.grid2((8, 90))
    comp = "Ex" if pol == "Hy" else "Ey"
    src = M.SoftSource(geometry=cases._plane(2, -1.5e-6), waveform=lambda x, z, t: 4e9 * cases.pulse(t), component=comp)
    w0 = 2 * np.pi * M.constants.C0 / 800e-9
    pl = M.Plasma(ionrate=M.PowerLawRate(order=6, sigma=1e-100), rho0=2.1e28, nuc=1 / 1e-15, frequency=w0,
                  Uiev=9.0, mr=0.64)
    m1 = M.Material(geometry=lambda x, z: (z > -0.6e-6) & (z < 0.0), eps=2.0, mu=1.1, sigma=1e3,
                    chi=M.DebyeSusceptibility(deps=2.0, tau=1e-14), chi3=1e-19)
    m2 = M.Material(geometry=lambda x, z: z >= 0.4e-6, eps=2.1, plasma=pl,
                    chi=M.LorentzSusceptibility(deps=0.7, w0=1.6e16, delta=1e13))
    cp = M.CPML(thickness=300e-9, kmax=2.0, alpha=0.05, R0=1e-8, m=3)
    return M.Model(g, src, tmax=(nsteps - 0.5) * PC.DT2, pml=(0, 0, cp, cp), bc="periodic",
                   material=[m1, m2], polarization=pol)


@pytest.mark.parametrize("dtype", DTYPES)
def test_ey_is_the_first_field_set_turned(oracle_lib, dtype):
    a = cases.run_all(_slab_models("Hy"), oracle_lib, dtype)
    b = cases.run_all(_slab_models("Ey"), oracle_lib, dtype)
    assert np.abs(a["field/Ex"]).max() > 1e6
    assert np.array_equal(b["field/Ey"], a["field/Ex"])
    assert np.array_equal(b["field/Hx"], -a["field/Hy"])
    assert not np.any(b["field/Hz"])
    for k in ("Sa", "E2", "JE", "rho_end"):
        assert np.array_equal(b[k], a[k]), k


def ey_tfsf_leakage(lib, dtype):
    """(largest |Ey| outside the TFSF box, largest inside) after a vacuum replay.  The box's
    edges lie off the midpoints between nodes, so the record run (box indices from the T
    coordinates) and the replay (from the double coordinates) pick the same cells."""
    box = (-240e-9, 240e-9, -240e-9, 240e-9)
    r = cases.run_all(PC.ey_tfsf_record(), lib, dtype, tfsf_box_=box)
    data = {k[4:]: v for k, v in r.items() if k.startswith("rec/")}
    assert set(M.sources.TFSF_NAMES_2D_EY) <= set(data)
    model = PC.ey_tfsf_replay(data, material=False)
    out = cases.run_all(model, lib, dtype)
    g = model.grid
    X, Z = np.meshgrid(g.x, g.z, indexing="ij")
    ey = np.abs(out["field/Ey"].reshape(g.Nx, g.Nz, order="F"))
    h, d = box[1], g.dx
    inside = (np.abs(X) < h - d) & (np.abs(Z) < h - d)
    outside = (np.abs(X) > h + d) | (np.abs(Z) > h + d)
    return float(ey[outside].max()), float(ey[inside].max())


@pytest.mark.parametrize("dtype", DTYPES)
def test_ey_tfsf_leakage_in_vacuum(oracle_lib, dtype):
    out, ins = ey_tfsf_leakage(oracle_lib, dtype)
    assert ins > 1e-3
    assert out / ins < (1e-12 if dtype == np.float64 else 1e-5), (out, ins)


def test_polarization_validation(oracle_lib):
    with pytest.raises(ValueError):
        M.Model(cases.grid3(), M.SoftSource(geometry=(0.0, 0.0, 0.0), waveform=lambda x, y, z, t: 0.0,
                                            component="Ey"), tmax=1e-15, polarization="Ey")
    with pytest.raises(ValueError):   # the first field set has no Ey
        M.Model(cases.grid2(), M.SoftSource(geometry=(0.0, 0.0), waveform=lambda x, z, t: 0.0, component="Ey"),
                tmax=1e-15)
    with pytest.raises(ValueError):   # the second has no Ex
        M.Model(cases.grid2(), M.SoftSource(geometry=(0.0, 0.0), waveform=lambda x, z, t: 0.0, component="Ex"),
                tmax=1e-15, polarization="Ey")
    with pytest.raises(ValueError):
        M.Model(cases.grid2(), M.SoftSource(geometry=(0.0, 0.0), waveform=lambda x, z, t: 0.0, component="Ey"),
                tmax=1e-15, polarization="Ez")
    model = PC.ey_vacuum()
    b, _ = model.build_desc(np.float32)
    b.desc.polarization = 7
    h = _abi.C.c_void_p()
    assert oracle_lib.create(_abi.C.byref(b.desc), _abi.C.byref(h)) == _abi.MFD_ERR_INVALID
    with pytest.raises(_abi.StepperError):   # reading a component the field set lacks
        st = _abi.Stepper(oracle_lib, model.build_desc(np.float32)[0], np.float32)
        try:
            st.read_field(comp_index("Ex"))
        finally:
            st.close()
