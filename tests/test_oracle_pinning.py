"""Pins the CPU oracle beyond the reference's analytic known-answer tests.

- The reference's only data fixture, the SiO2 Keldysh rate table of its nonlinear example
  (tests/golden/SiO2_keldysh_1.03um.tf, examples/5_nonlinear_propagation), loaded and
  evaluated with the semantics of IonizationRate.jl:13-52 -- the constructor's log10 step
  and spacing check, exact knots, log-log interpolation between them, extrapolation of the
  end segments, zero for I <= 0 -- by the Python mirror and by the oracle's own functor, and
  then driving a plasma solve.
- Physics the reference tests do not check (tests/physics_cases.py): Drude and Debye
  attenuation against the susceptibility, CPML reflection with kmax = 1 and 4, energy
  conservation in a lossless periodic box, TFSF leakage in vacuum.
- Summed monitors add their points as Julia's sum does (pairwise above blocks of 1024).
"""
import ctypes as C
import os

import numpy as np
import pytest

import cases
import physics_cases as P
import maxwellfdtd_b200 as M
from maxwellfdtd_b200 import _abi
from maxwellfdtd_b200.sources import comp_index

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TF = os.path.join(GOLDEN, "SiO2_keldysh_1.03um.tf")
DTYPES = [np.float64, np.float32]


def _table():
    raw = np.loadtxt(TF)
    return raw, M.IonizationRate(TF)


def _oracle_rate(oracle_lib, rate, I, f32):
    f = oracle_lib.lib.oracle_eval_rate_table
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64]
    x = np.ascontiguousarray(rate.x, np.float64)
    y = np.ascontiguousarray(rate.y, np.float64)
    I = np.ascontiguousarray(I, np.float64)
    out = np.empty_like(I)
    rc = f(x.ctypes.data, y.ctypes.data, len(x), int(f32), I.ctypes.data, out.ctypes.data, len(I))
    assert rc == 0
    return out


def test_rate_table_fixture_constructor():
    """IonizationRate(fname): x = log10(I), y = log10(R), sorted, evenly spaced x."""
    raw, rate = _table()
    assert raw.shape == (100, 2)
    assert np.array_equal(rate.x, np.log10(raw[:, 0])) and np.array_equal(rate.y, np.log10(raw[:, 1]))
    dx = np.diff(rate.x)
    assert np.all(dx > 0) and np.allclose(dx, dx[0], rtol=np.sqrt(np.finfo(float).eps), atol=0)
    assert rate.x[0] == 13.0
    bad = raw.copy()
    bad[5, 0] *= 1.01   # uneven spacing is refused, as the reference's @assert does
    with pytest.raises(ValueError):
        M.IonizationRate(bad)


def test_rate_table_fixture_semantics(oracle_lib):
    raw, rate = _table()
    I, R = raw[:, 0], raw[:, 1]
    # knots
    got = rate(I)
    assert np.allclose(got, R, rtol=1e-12, atol=0)
    # midpoints in log10(I): log-log linear, so the geometric mean of the neighbours
    Im = np.sqrt(I[:-1] * I[1:])
    assert np.allclose(rate(Im), np.sqrt(R[:-1] * R[1:]), rtol=1e-12, atol=0)
    # below the first knot and above the last: the end segments extended
    s0 = (rate.y[1] - rate.y[0]) / (rate.x[1] - rate.x[0])
    s1 = (rate.y[-1] - rate.y[-2]) / (rate.x[-1] - rate.x[-2])
    lo, hi = I[0] / 10, I[-1] * 10
    assert np.isclose(rate(lo)[0], 10 ** (rate.y[0] - s0), rtol=1e-12)
    assert np.isclose(rate(hi)[0], 10 ** (rate.y[-1] + s1), rtol=1e-12)
    # zero and negative intensities give no ionisation (no -Inf from log10(0))
    assert np.all(rate(np.array([0.0, -1.0])) == 0)
    # the oracle's functor, in Float64 and in Float32 (the table cast as the library does)
    probe = np.concatenate([[0.0, lo, hi], I, Im, np.logspace(12.5, 16.5, 301)])
    ref = rate(probe)
    o64 = _oracle_rate(oracle_lib, rate, probe, f32=False)
    assert np.allclose(o64, ref, rtol=1e-13, atol=0)
    o32 = _oracle_rate(oracle_lib, rate, probe, f32=True)
    pos = ref > 0
    assert np.all(o32[~pos] == 0)
    assert np.max(np.abs(o32[pos] / ref[pos] - 1)) < 1e-4   # float log10 of I ~ 1e13..1e17


def plasma_fixture_model(ndim=1, nsteps=80):
    """A solid-density plasma (rho0 = 2.1e28) with the fixture's Keldysh rate in a fused-silica
    ball, driven at 1.03 um hard enough to ionise."""
    g = cases._grid(ndim)
    lam0 = 1.03e-6
    w0 = 2 * np.pi * M.C0 / lam0
    E0 = 2.0e10
    src = M.SoftSource(geometry=cases._plane(ndim, -250e-9),
                       waveform=cases._src_wave(ndim, E0, lam0), component="Ex")
    dt = 0.5 / M.C0 / np.sqrt(ndim / (50e-9) ** 2)
    pl = M.Plasma(ionrate=M.IonizationRate(TF), rho0=2.1e28, nuc=1 / 1e-15, frequency=w0, Uiev=9.0, mr=0.64)
    mat = M.Material(geometry=cases._ball(ndim, 250e-9), eps=1.45 ** 2, plasma=pl)
    return M.Model(g, src, tmax=(nsteps - 0.5) * dt, pml=150e-9, material=mat)


@pytest.mark.parametrize("dtype", DTYPES)
def test_rate_table_fixture_drives_plasma(dtype, oracle_lib):
    out = cases.run_all(plasma_fixture_model(1), oracle_lib, dtype)
    assert out["rho_end"].max() > 0 and np.all(np.isfinite(out["rho_end"]))
    assert np.all(out["rho_end"] <= 2.1e28)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("kind", ["drude", "debye"])
def test_attenuation_matches_susceptibility(kind, dtype, oracle64, oracle32):
    model, mons, check = P.case_attenuation(1, kind)
    sol = M.solve(model, backend=oracle64 if dtype == np.float64 else oracle32, monitors=mons)
    ok, err = check(sol)
    assert ok, f"{kind}: relative error {err:.4g}"


def cpml_bounds_hold(r):
    """r[(nb, kmax)]: the reflected-peak ratios of case_cpml_reflection."""
    assert r[(12, 1.0)] < 0.02 and r[(12, 4.0)] < 0.02
    assert r[(20, 1.0)] < 0.007 and r[(20, 4.0)] < 0.007
    assert r[(20, 1.0)] < r[(12, 1.0)] / 2 and r[(20, 4.0)] < r[(12, 4.0)] / 2   # thicker absorbs better
    assert r[(12, 4.0)] < r[(12, 1.0)] and r[(20, 4.0)] < r[(20, 1.0)]


@pytest.mark.parametrize("dtype", DTYPES)
def test_cpml_reflection(dtype, oracle64, oracle32):
    be = oracle64 if dtype == np.float64 else oracle32
    r = {}
    for nb in (12, 20):
        for kmax in (1.0, 4.0):
            model, mons, check = P.case_cpml_reflection(nb, kmax)
            r[(nb, kmax)] = check(M.solve(model, backend=be, monitors=mons))
    cpml_bounds_hold(r)
    model, mons, check = P.case_cpml_2d()
    assert check(M.solve(model, backend=be, monitors=mons)) < 5e-3


def energy_drift(lib, dtype):
    """Relative change of the discrete energy between steps k1, k1 + 100 and k2."""
    model, mu, k1, k2 = P.energy_box()
    b, _ = model.build_desc(dtype, None)
    st = _abi.Stepper(lib, b, dtype)
    g = model.grid
    names = ("Ex", "Ey", "Ez", "Dx", "Dy", "Dz", "Hx", "Hy", "Hz")

    def snap():
        return {c: st.read_field(comp_index(c)).reshape(g.Nx, g.Ny, g.Nz, order="F") for c in names}
    W = []
    done = 0
    try:
        for k in (k1, k1 + 100, k2):
            st.run(done + 1, k)
            f = snap()
            st.run(k + 1, k + 1)
            done = k + 1
            h = snap()
            W.append(P._energy(f, [h["Hx"], h["Hy"], h["Hz"]], mu))
    finally:
        st.close()
    assert W[0] > 0
    return max(abs(w - W[0]) / W[0] for w in W)


@pytest.mark.parametrize("dtype", DTYPES)
def test_energy_conserved_in_periodic_box(dtype, oracle_lib):
    assert energy_drift(oracle_lib, dtype) < (1e-13 if dtype == np.float64 else 2e-6)


def tfsf_leakage(lib, dtype):
    """(largest |Ex| outside the TFSF box, largest inside) after a vacuum replay."""
    rec, box, replay = P.tfsf_vacuum()
    r = cases.run_all(rec, lib, dtype, tfsf_box_=box)
    data = {k[4:]: v for k, v in r.items() if k.startswith("rec/")}
    model = replay(data)
    out = cases.run_all(model, lib, dtype)
    g = model.grid
    X, Y, Z = np.meshgrid(g.x, g.y, g.z, indexing="ij")
    ex = np.abs(out["field/Ex"].reshape(g.Nx, g.Ny, g.Nz, order="F"))
    h, d = box[1], g.dx
    inside = (np.abs(X) < h - d) & (np.abs(Y) < h - d) & (np.abs(Z) < h - d)
    outside = (np.abs(X) > h + d) | (np.abs(Y) > h + d) | (np.abs(Z) > h + d)
    return float(ex[outside].max()), float(ex[inside].max())


@pytest.mark.parametrize("dtype", DTYPES)
def test_tfsf_leakage_in_vacuum(dtype, oracle_lib):
    out, ins = tfsf_leakage(oracle_lib, dtype)
    assert ins > 1e-3
    assert out / ins < (1e-12 if dtype == np.float64 else 1e-5), (out, ins)


@pytest.mark.parametrize("dtype", DTYPES)
def test_summed_monitor_is_julia_sum(dtype, oracle_lib):
    """FieldMonitor(sum=true) over 1600 points equals Julia's pairwise sum of the same
    points' values, step by step, bit for bit."""
    g = cases.grid3((40, 40, 10))
    dt = 0.5 / M.C0 / np.sqrt(3 / (50e-9) ** 2)
    src = M.SoftSource(geometry=(0.0, 0.0, -100e-9), waveform=lambda x, y, z, t: 1e3 * cases.pulse(t), component="Ex")
    model = M.Model(g, src, tmax=(30 - 0.5) * dt, pml=0)
    plane = lambda x, y, z: np.abs(z - 75e-9) < 26e-9
    mons = [M.FieldMonitor(plane), M.FieldMonitor(plane, sum=True)]
    sol = M.solve(model, backend=M.B200(dtype, library=oracle_lib), monitors=mons)
    pts = np.asarray(sol.out["monitors/1/Ex"])
    tot = np.asarray(sol.out["monitors/2/Ex"]).ravel()
    assert pts.shape[0] == 1600 and np.abs(tot).max() > 0
    want = np.array([P.julia_sum(pts[:, k]) for k in range(pts.shape[1])], dtype=dtype)
    assert np.array_equal(tot, want)
