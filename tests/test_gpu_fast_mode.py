"""The tolerance mode (MFD_MODE_FAST) against the oracle's exact operation order.

The field updates multiply by reciprocals and fuse multiply-adds, so results are no longer
bit-identical; the tolerance bound is relative L2 <= 1e-5 in Float32 and <= 1e-12 in
Float64 for the fields, which the final fields and running sums meet against the oracle run
in the same precision.  A monitor's time series or spectrum integrates rounding over every
step at one place; where it is further than that from the same-precision oracle, the
criterion is the error against the Float64 oracle (the truth for a Float32 run): the fast
mode may be no less accurate than the exact Float32 order is, or within the bound.
Errors are measured per vector quantity (E, D, H as the concatenation of their components),
per running sum (Sa, E2) and per monitor (all its components together): a single component
that the exact order keeps at exactly zero by symmetry (Ey of an x-polarised source) would
otherwise turn rounding noise into a relative error of 1.
"""
import numpy as np
import pytest

import cases as C
import maxwellfdtd_b200 as M
import test_gpu_configs as G
from maxwellfdtd_b200 import _abi
from maxwellfdtd_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = {np.float32: 1e-5, np.float64: 1e-12}
TOL_PLASMA_STATE = {np.float32: 1e-4, np.float64: 1e-9}


def _groups(out):
    g = {}
    for k, v in out.items():
        if k.startswith("field/"):
            key = "field/" + k[6]          # E, D or H
        elif k.startswith("monitors/"):
            key = "/".join(k.split("/")[:2])
        else:
            key = k
        g.setdefault(key, []).append(np.asarray(v))
    return g


def _rel(parts_a, parts_b):
    def flat(parts):
        out = []
        for p in parts:
            if np.iscomplexobj(p):
                out += [np.real(p).ravel(), np.imag(p).ravel()]
            else:
                out.append(p.ravel())
        return np.concatenate(out).astype(np.float64)
    a, b = flat(parts_a), flat(parts_b)
    den = max(np.linalg.norm(a), np.linalg.norm(b))
    return 0.0 if den == 0 else float(np.linalg.norm(a - b) / den)


def _check(ref, got, dtype, truth=None):
    """truth(): the Float64 oracle's outputs, computed when a monitor needs them."""
    ga, gb = _groups(ref), _groups(got)
    assert set(ga) == set(gb)
    errs = {k: _rel(ga[k], gb[k]) for k in ga}
    bad = {k: e for k, e in errs.items() if k not in ("rho_end", "JE") and e > TOL[dtype]}
    fields = {k: e for k, e in bad.items() if not k.startswith("monitors/")}
    assert not fields, fields
    if bad:
        assert dtype == np.float32 and truth is not None, bad
        gt = _groups(truth())
        for k in bad:
            e_fast, e_exact = _rel(gt[k], gb[k]), _rel(gt[k], ga[k])
            assert e_fast <= max(TOL[dtype], 2 * e_exact), (k, e_fast, e_exact)
    for k in ("rho_end", "JE"):
        if k in errs:
            assert errs[k] <= TOL_PLASMA_STATE[dtype], (k, errs[k])
    return errs


CASES = {
    "vacuum": lambda n: (C.model_vacuum(n), C.monitors(n)),
    "bcs": lambda n: (C.model_bcs(n), None),
    "materials": lambda n: (C.model_materials(n), C.monitors(n)),
    "sources": lambda n: (C.model_sources(n), None),
    "poles": lambda n: (C.model_poles(n, 3, True), None),
}


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("case", sorted(CASES))
def test_fast_mode_within_tolerance(case, ndim, dtype, oracle_lib, gpu_lib):
    model, mons = CASES[case](ndim)
    ref = C.run_all(model, oracle_lib, dtype, mons)
    got = C.run_all(model, gpu_lib, dtype, mons, mode="fast")
    _check(ref, got, dtype, lambda: C.run_all(model, oracle_lib, np.float64, mons))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("case", ["wide_periodic", "wide_dirichlet", "x_overlap", "y_z_right", "midsize"])
def test_fast_mode_3d_layouts(case, dtype, oracle_lib, gpu_lib):
    """Rows across several warps, overlapping layers (the unsplit kernels), layers on some
    faces only, and the staged kernels' inner tiles."""
    import test_gpu_parity as P
    if case.startswith("wide_"):
        model = C.model_wide_rows(case[5:])
    elif case == "midsize":
        model = G._midsize_model((72, 40, 24))
    else:
        model = C.model_layers(*P.LAYER_CASES[case])
    ref = C.run_all(model, oracle_lib, dtype)
    got = C.run_all(model, gpu_lib, dtype, mode="fast")
    _check(ref, got, dtype, lambda: C.run_all(model, oracle_lib, np.float64))


def test_fast_mode_plasmonics_96(oracle_lib, gpu_lib):
    """The headline workload's configuration on a 96^3 grid, 60 steps: within 1e-5 of the
    FP32 oracle, and no further from the FP64 oracle than 1e-5 either."""
    model, mons = W.plasmonics_256(nt=60, n=96)
    got = C.run_all(model, gpu_lib, np.float32, mons, mode="fast")
    ref = C.run_all(model, oracle_lib, np.float32, mons)
    truth = C.run_all(model, oracle_lib, np.float64, mons)
    errs = _check(ref, got, np.float32, lambda: truth)
    e64 = {k: _rel(a, b) for (k, a), b in zip(_groups(truth).items(), _groups(got).values())}
    print("fast mode, plasmonics 96^3, 60 steps: vs FP32 oracle", {k: f"{v:.2e}" for k, v in errs.items()},
          "vs FP64 oracle", {k: f"{v:.2e}" for k, v in e64.items()})
    assert max(e64[k] for k in ("field/E", "field/H", "field/D")) <= 1e-5


def test_fast_mode_plasma(oracle_lib, gpu_lib):
    model = C.model_plasma(3, "power")
    ref = C.run_all(model, oracle_lib, np.float32)
    got = C.run_all(model, gpu_lib, np.float32, mode="fast")
    _check(ref, got, np.float32, lambda: C.run_all(model, oracle_lib, np.float64))


def test_batch_takes_fast_members(oracle_lib, gpu_lib):
    """Tolerance-mode members in a batch, beside exact ones: a 2-D member equals its solo run
    bit for bit (both run h2d_cell / e2d_cell); every member's fields and Sa are within the
    bound of the exact-order oracle."""
    import test_gpu_batch as TB

    def make(model, mons, mode):
        b, meta = model.build_desc(np.float32, mons, mode=mode)
        return _abi.Stepper(gpu_lib, b, np.float32), b, meta

    members = [(TB.member_model(s), "fast") for s in range(4)] + [(TB.member_model(7), "exact")] + \
              [((C.model_materials(3), None), "fast"), ((C.model_bcs(3), None), "fast")]
    solo = []
    for (m, mo), mode in members[:5]:
        st, b, meta = make(m, mo, mode)
        st.run(1, m.Nt)
        solo.append(TB.outputs_nd(st, m, meta))
        st.close()
    batch = _abi.Batch(gpu_lib)
    held = []
    for (m, mo), mode in members:
        st, b, meta = make(m, mo, mode)
        batch.add(st, m.Nt)
        held.append((st, b, meta, m))
    batch.run_all(chunk=17)
    got = [TB.outputs_nd(st, m, meta) for st, b, meta, m in held]
    for r, g in zip(solo, got[:5]):
        TB.same(r, g)
    for ((m, mo), mode), g in zip(members, got):
        b0, meta0 = m.build_desc(np.float32, mo)
        st0 = _abi.Stepper(oracle_lib, b0, np.float32)
        st0.run(1, m.Nt)
        ref = TB.outputs_nd(st0, m, meta0)
        st0.close()
        for group in ("E", "D", "H"):
            keys = [k for k in ref if k.startswith("field/" + group)]
            e = _rel([ref[k] for k in keys], [g[k] for k in keys])
            assert e <= TOL[np.float32], (group, e)
        assert _rel([ref["Sa"]], [g["Sa"]]) <= TOL[np.float32]
    batch.close()
    for st, *_ in held:
        st.close()


def test_mode_is_validated(gpu_lib):
    model = C.model_vacuum(1)
    b, _ = model.build_desc(np.float32, None)
    b.desc.mode = 7
    with pytest.raises(_abi.StepperError):
        _abi.Stepper(gpu_lib, b, np.float32)
    with pytest.raises(ValueError):
        M.B200(np.float32, mode="quick")


def test_tensor_core_fold_against_fp64_sum(gpu_lib):
    """Float32 spectral monitors in the tolerance mode are folded on the tensor cores (TF32
    high and low parts, three products per 8 staged steps, FP32 partial sums per fold of at
    most 64 steps, added to the FP64 spectra).  Checked against an FP64 sum over the same
    run's recorded time series (a field monitor on the same plane): 80 frequencies (a full
    and a partial 64-frequency tile), a plane whose point count is no multiple of the
    128-point tile, and 75 steps (a full fold and a partial one of 11 steps)."""
    from maxwellfdtd_b200.monitors import DFT
    model = C.model_vacuum(3, nsteps=75)
    plane = C._plane(3, 150e-9)
    w = np.linspace(1.0e15, 4.0e15, 80)
    mons = [M.FieldMonitor(plane), M.SpectralMonitor(plane, w=w)]
    sol = M.solve(model, backend=M.B200(np.float32, library=gpu_lib, mode="fast"), monitors=mons)
    out = sol.out
    t_T = np.asarray(out["t"], dtype=np.float32)
    assert len(t_T) == 75
    dft = DFT(t_T, np.float32, w=w)
    fac = 2.0 * (dft.phasor[..., 0] + 1j * dft.phasor[..., 1]) * float(np.float32(model.dt))   # [Nt][Nw]
    npts = out["monitors/1/Ex"].shape[0]
    assert npts % 128 != 0
    for c in ("Hx", "Hy", "Hz", "Ex", "Ey", "Ez"):
        ref = out[f"monitors/1/{c}"].astype(np.float64) @ fac      # (npts, Nw)
        got = out[f"monitors/2/{c}"]
        assert got.shape == ref.shape
        den = np.linalg.norm(ref)
        if den == 0:
            assert not np.any(got)
            continue
        rel = float(np.linalg.norm(got - ref) / den)
        assert rel <= 1e-5, (c, rel)


def test_fast_mode_widened_y_layers_with_material(oracle_lib, gpu_lib):
    """The tolerance mode widens each y-layer launch to whole tiles of 4 rows; here the
    5-row CPML layers become 8-row launches, and a Drude+Lorentz ball lies in the rows that
    move from the core launch to the layer launch and in the core rows next to them (rows
    5-9), so the layer launches run with the material map and the response runs apart."""
    g = C.grid3((40, 38, 24))
    src = M.SoftSource(geometry=C._plane(3, -250e-9), waveform=C._src_wave(3, 2e8), component="Ex")
    dt = 0.5 / C.C0 / np.sqrt(3 / (50e-9) ** 2)
    ball = C._ball(3, 120e-9, (0.0, -575e-9, 0.0))
    m = M.Material(geometry=ball, eps=3.0, chi=[M.DrudeSusceptibility(wp=1.37e16, gamma=1.07e14),
                                                M.LorentzSusceptibility(deps=1.1, w0=4.2e15, delta=5e14)])
    model = M.Model(g, src, tmax=(60 - 0.5) * dt, pml=200e-9, material=[m])
    mons = C.monitors(3)
    ref = C.run_all(model, oracle_lib, np.float32, mons)
    got = C.run_all(model, gpu_lib, np.float32, mons, mode="fast")
    _check(ref, got, np.float32, lambda: C.run_all(model, oracle_lib, np.float64, mons))
    exact = C.run_all(model, gpu_lib, np.float32, mons)   # the exact mode keeps the layer bounds
    for k in ref:
        if k.startswith("field/") or k in ("Sa", "E2"):
            assert np.array_equal(np.asarray(ref[k]), np.asarray(exact[k])), k


def test_fast_mode_thick_z_layers(oracle_lib, gpu_lib):
    """z CPML layers of 19 planes, which the tolerance mode's z-layer launches split into
    blocks of 10 and 9 planes (layers of at most 16 planes go in one march per block)."""
    g = C.grid3((24, 20, 56))
    src = M.SoftSource(geometry=C._plane(3, -250e-9), waveform=C._src_wave(3, 2e8), component="Ex")
    dt = 0.5 / C.C0 / np.sqrt(3 / (50e-9) ** 2)
    model = M.Model(g, src, tmax=(60 - 0.5) * dt, pml=(100e-9, 100e-9, 100e-9, 100e-9, 900e-9, 900e-9))
    assert model.pml[4].nb == 19 and model.pml[5].nb == 19
    mons = C.monitors(3)
    ref = C.run_all(model, oracle_lib, np.float32, mons)
    got = C.run_all(model, gpu_lib, np.float32, mons, mode="fast")
    _check(ref, got, np.float32, lambda: C.run_all(model, oracle_lib, np.float64, mons))
