"""Batches of 2-D and 3-D models (mfd_batch_*): every member's results are bit-identical to
running it alone with mfd_run, whatever the tile shape, the graph length, the join time or
the mix of sizes, dimensions, step counts, materials and sources in the batch."""
import numpy as np
import pytest

import cases as C
import maxwellfdtd_b200 as M
from maxwellfdtd_b200 import _abi
from maxwellfdtd_b200.sources import comp_index, field_components

pytestmark = pytest.mark.gpu


def member_model(seed):
    """A 2-D model of seeded size, step count, materials (dielectric, Debye, Drude, Lorentz,
    Kerr) and sources (soft point, hard point on H, soft line)."""
    rng = np.random.default_rng(seed)
    nx, nz = int(rng.integers(20, 150)), int(rng.integers(20, 150))
    nsteps = int(rng.integers(15, 70))
    g = C.grid2((nx, nz))
    dt = 0.5 / C.C0 / np.sqrt(2 / (50e-9) ** 2)
    mats = []
    for k in range(int(rng.integers(0, 4))):
        cx, cz = rng.uniform(-0.4, 0.4) * nx * 50e-9, rng.uniform(-0.4, 0.4) * nz * 50e-9
        a, b = rng.uniform(60e-9, 400e-9, size=2)
        geo = (lambda cx, cz, a, b: (lambda x, z: ((x - cx) / a) ** 2 + ((z - cz) / b) ** 2 <= 1))(cx, cz, a, b)
        kind = k % 4
        if kind == 0:
            mats.append(M.Material(geometry=geo, eps=float(rng.uniform(1, 12)), sigma=float(rng.uniform(0, 1e4))))
        elif kind == 1:
            mats.append(M.Material(geometry=geo, eps=float(rng.uniform(1, 6)),
                                   chi=M.DebyeSusceptibility(deps=float(rng.uniform(1, 5)), tau=float(10 ** rng.uniform(-15, -13)))))
        elif kind == 2:
            mats.append(M.Material(geometry=geo, eps=2.0, chi=[M.DrudeSusceptibility(wp=1.37e16, gamma=1.07e14),
                                                               M.LorentzSusceptibility(deps=1.1, w0=4.2e15, delta=5e14)]))
        else:
            mats.append(M.Material(geometry=geo, eps=2.0, mu=1.2, chi3=1e-19))
    lam = float(rng.uniform(400e-9, 1600e-9))
    srcs = [M.SoftSource(geometry=(0.0, 0.0), waveform=lambda x, z, t, lam=lam: 1e2 * C.pulse(t, lam), component="Ez")]
    if seed % 3 == 1:
        srcs.append(M.HardSource(geometry=(50e-9, -50e-9), waveform=lambda x, z, t: 1e-4 * C.pulse(t), component="Hy"))
    if seed % 3 == 2:
        srcs.append(M.SoftSource(geometry=lambda x, z: np.abs(z + 100e-9) < 26e-9,
                                 waveform=lambda x, z, t: 30.0 * C.pulse(t), component="Ex"))
    bc = ("periodic", "periodic", "dirichlet", "neumann") if seed % 2 else "periodic"
    model = M.Model(g, srcs, tmax=(nsteps - 0.5) * dt, pml=150e-9 if seed % 4 else (150e-9, 0, 100e-9, 150e-9),
                    bc=bc, material=mats or None)
    pts = [(0.0, 0.0), (100e-9, 50e-9), (-150e-9, 100e-9), (0.0, -200e-9)]
    mons = [M.FieldMonitor(p) for p in pts]
    return model, mons


def outputs(st, model, meta):
    out = {f"field/{c}": st.read_field(comp_index(c)) for c in field_components(2)}
    out["Sa"] = st.read_integral(_abi.MFD_INT_SA)
    out["E2"] = st.read_integral(_abi.MFD_INT_E2)
    for m, mm in enumerate(meta["monitors"]):
        for c in field_components(2):
            if c.startswith("D"):
                continue
            out[f"mon/{m}/{c}"] = st.read_monitor(m, comp_index(c), (model.Nt, len(mm["cells"])), False)
    out["status"] = np.array(st.status())
    return out


def make(model, mons, lib):
    b, meta = model.build_desc(np.float32, mons)
    return _abi.Stepper(lib, b, np.float32), b, meta


def alone(model, mons, lib):
    st, b, meta = make(model, mons, lib)
    st.run(1, model.Nt)
    out = outputs(st, model, meta)
    st.close()
    return out


def same(a, b):
    assert set(a) == set(b)
    bad = [k for k in a if not np.array_equal(a[k], b[k], equal_nan=True)]
    assert not bad, bad


@pytest.mark.parametrize("tile,graph,chunk", [((0, 0), 4, 1000), ((0, 0), 16, 40), ((32, 4), 8, 1000),
                                              ((128, 2), 5, 13), ((32, 16), 64, 1000)])
def test_batch_members_match_alone(tile, graph, chunk, gpu_lib):
    models = [member_model(s) for s in range(12)]
    ref = [alone(m, mo, gpu_lib) for m, mo in models]
    batch = _abi.Batch(gpu_lib)
    batch.config(*tile, graph)
    held = []
    for m, mo in models:
        st, b, meta = make(m, mo, gpu_lib)
        batch.add(st, m.Nt)
        held.append((st, b, meta, m))
    batch.run_all(chunk=chunk)      # graph replays and, for the remainders, direct launches
    for (st, b, meta, m), r in zip(held, ref):
        same(r, outputs(st, m, meta))
    info = batch.info()
    assert info["cell_updates"] == sum(m.grid.Nx * m.grid.Nz * m.Nt for m, _ in models)
    if tile != (0, 0):
        assert info["tile"] == tile
    batch.close()
    for st, *_ in held:
        st.close()


def test_batch_join_midway_and_partial_windows(gpu_lib):
    """Members join between runs, and one member runs its steps in two windows (first alone,
    then in the batch): the results equal one uninterrupted run."""
    models = [member_model(s) for s in (20, 21, 22, 23)]
    ref = [alone(m, mo, gpu_lib) for m, mo in models]
    batch = _abi.Batch(gpu_lib)
    held = []
    for i, (m, mo) in enumerate(models[:2]):
        st, b, meta = make(m, mo, gpu_lib)
        batch.add(st, m.Nt)
        held.append((st, b, meta, m))
    batch.run(9)
    m, mo = models[2]
    st, b, meta = make(m, mo, gpu_lib)
    st.run(1, 5)                   # first steps alone
    batch.add(st, m.Nt)
    held.append((st, b, meta, m))
    m, mo = models[3]
    st, b, meta = make(m, mo, gpu_lib)
    batch.add(st, 10)              # a window that ends early, then the rest alone
    held.append((st, b, meta, m))
    batch.run_all(chunk=11)
    st.run(11, m.Nt)
    for (st, b, meta, m), r in zip(held, ref):
        same(r, outputs(st, m, meta))
    batch.close()
    for st, *_ in held:
        st.close()


def test_batch_member_matches_oracle(oracle_lib, gpu_lib):
    m, mo = member_model(5)
    ref = alone(m, mo, oracle_lib)
    batch = _abi.Batch(gpu_lib)
    st, b, meta = make(m, mo, gpu_lib)
    batch.add(st, m.Nt)
    batch.run_all()
    same(ref, outputs(st, m, meta))
    batch.close()
    st.close()


def test_batch_nonfinite_member_reports_like_alone(gpu_lib):
    g = C.grid2((30, 30))
    src = M.SoftSource(geometry=(0.0, 0.0), waveform=lambda x, z, t: 1e30 * C.pulse(t), component="Ez")
    bad = M.Model(g, src, tmax=1e-13, CN=1.5, pml=0)
    st0, b0, meta0 = make(bad, None, gpu_lib)
    with pytest.raises(_abi.StepperError):
        st0.run(1, bad.Nt)
    good, mo = member_model(3)
    batch = _abi.Batch(gpu_lib)
    st, b, meta = make(bad, None, gpu_lib)
    st2, b2, meta2 = make(good, mo, gpu_lib)
    batch.add(st, bad.Nt)
    batch.add(st2, good.Nt)
    batch.run_all()
    assert st.status() == st0.status() and st.status()[1] > 0
    same(alone(good, mo, gpu_lib), outputs(st2, good, meta2))
    batch.close()
    for s in (st0, st, st2):
        s.close()


def test_batch_rejects_and_guards(gpu_lib):
    batch = _abi.Batch(gpu_lib)
    m3 = C.model_vacuum(1)
    st3, _, _ = make(m3, None, gpu_lib)
    with pytest.raises(_abi.StepperError) as ei:
        batch.add(st3, m3.Nt)
    assert ei.value.code == _abi.MFD_ERR_INVALID and "2-D or 3-D" in str(ei.value)
    m, mo = member_model(1)
    st, b, meta = make(m, mo, gpu_lib)
    with pytest.raises(_abi.StepperError):
        batch.add(st, m.Nt + 1)                  # beyond Nt
    batch.add(st, m.Nt)
    with pytest.raises(_abi.StepperError):
        st.run(1, 2)                             # stepped by the batch until it retires
    with pytest.raises(_abi.StepperError):
        batch.add(st, m.Nt)                      # already a member
    batch.run_all()
    assert st.status()[0] == m.Nt
    batch.close()
    st.close()
    st3.close()


def rich_member(seed):
    """2-D member with a plane-wave TFSF source (at a seeded position among its point
    sources), spectral monitors (per point and summed) and a summed field monitor."""
    from maxwellfdtd_b200 import workloads
    from maxwellfdtd_b200.model import time_range
    rng = np.random.default_rng(100 + seed)
    nx, nz = int(rng.integers(40, 160)), int(rng.integers(40, 160))
    nsteps = int(rng.integers(20, 150))
    g = C.grid2((nx, nz))
    dt = 0.5 / C.C0 / np.sqrt(2 / (50e-9) ** 2)
    t = time_range(dt, (nsteps - 0.5) * dt)
    m_in = 6
    i1, i2 = (m_in, 1, m_in), (nx + 1 - m_in, 1, nz + 1 - m_in)
    f = lambda s: C.pulse(s)
    data = workloads._plane_wave_tfsf_2d(g, i1, i2, t, f, g.z[i1[2] - 1], dt)
    srcs = [M.TFSFSource(data=data)]
    if seed % 2:
        srcs.insert(0, M.SoftSource(geometry=(0.0, 0.0), waveform=lambda x, z, t: 10 * C.pulse(t), component="Ez"))
    mat = M.Material(geometry=lambda x, z: x ** 2 + z ** 2 <= (300e-9) ** 2, eps=2.0,
                     chi=M.LorentzSusceptibility(deps=1.1, w0=4.2e15, delta=5e14))
    model = M.Model(g, srcs, tmax=(nsteps - 0.5) * dt, pml=100e-9, material=mat)
    line = lambda x, z: np.abs(z - 200e-9) < 26e-9
    mons = [M.SpectralMonitor(line, w=np.linspace(1e15, 4e15, int(rng.integers(8, 33)))),
            M.SpectralMonitor(line, sum=True),
            M.FieldMonitor(line, sum=True), M.FieldMonitor((0.0, 100e-9))]
    return model, mons


def outputs_rich(st, model, meta):
    out = {f"field/{c}": st.read_field(comp_index(c)) for c in field_components(2)}
    out["Sa"] = st.read_integral(_abi.MFD_INT_SA)
    for k, mm in enumerate(meta["monitors"]):
        spectral = mm["kind"] == 1
        for c in ("Hy", "Ex", "Ez"):
            if spectral:
                shape = (mm["dft"].Nw,) if mm["sum"] else (mm["dft"].Nw, len(mm["cells"]))
            else:
                shape = (model.Nt,) if mm["sum"] else (model.Nt, len(mm["cells"]))
            out[f"mon/{k}/{c}"] = st.read_monitor(k, comp_index(c), shape, spectral)
    out["status"] = np.array(st.status())
    return out


@pytest.mark.parametrize("graph", [16, 64, 3])
def test_batch_tfsf_and_staged_monitors_match_alone(graph, gpu_lib):
    models = [rich_member(s) for s in range(6)] + [member_model(s) for s in range(3)]
    ref = []
    for m, mo in models:
        st, b, meta = make(m, mo, gpu_lib)
        st.run(1, m.Nt)
        ref.append(outputs_rich(st, m, meta))
        st.close()
    batch = _abi.Batch(gpu_lib)
    batch.config(0, 0, graph)
    held = []
    for m, mo in models:
        st, b, meta = make(m, mo, gpu_lib)
        batch.add(st, m.Nt)
        held.append((st, b, meta, m))
    batch.run_all(chunk=100)
    for (st, b, meta, m), r in zip(held, ref):
        same(r, outputs_rich(st, m, meta))
    batch.close()
    for st, *_ in held:
        st.close()


def outputs_nd(st, model, meta):
    """Every output of a 2-D or 3-D member: fields, Sa, E2, each monitor's components, status."""
    nd = model.grid.ndim
    out = {f"field/{c}": st.read_field(comp_index(c)) for c in field_components(nd)}
    out["Sa"] = st.read_integral(_abi.MFD_INT_SA)
    out["E2"] = st.read_integral(_abi.MFD_INT_E2)
    for k, mm in enumerate(meta["monitors"]):
        spectral = mm["kind"] == 1
        for c in field_components(nd):
            if c.startswith("D"):
                continue
            if spectral:
                shape = (mm["dft"].Nw,) if mm["sum"] else (mm["dft"].Nw, len(mm["cells"]))
            else:
                shape = (model.Nt,) if mm["sum"] else (model.Nt, len(mm["cells"]))
            out[f"mon/{k}/{c}"] = st.read_monitor(k, comp_index(c), shape, spectral)
    out["status"] = np.array(st.status())
    return out


def members_3d(lib):
    """3-D members: mixed boundary conditions with CPML kmax != 1 on some faces, conductive and
    magnetic materials with Debye/Drude/Lorentz/Kerr, three and five poles, plasma, CPML
    layers that overlap, a TFSF replay (of a record run on lib), and every kind of monitor."""
    rec = C.run_all(C.model_tfsf_record(3), lib, np.float32, tfsf_box_=C.tfsf_box(3))
    record = {k[4:]: v for k, v in rec.items() if k.startswith("rec/")}
    return [(C.model_bcs(3), C.monitors(3)), (C.model_materials(3), C.monitors(3)),
            (C.model_poles(3, 3, True), None), (C.model_poles(3, 5, False), C.monitors(3)),
            (C.model_plasma(3), None), (C.model_layers((20, 9, 5), (1, 1, 1, 1, 1, 1)), None),
            (C.model_tfsf_replay(3, record), C.monitors(3))]


@pytest.mark.parametrize("tile,graph", [((0, 0), 16), ((32, 4), 7), ((64, 8), 64)])
def test_batch_3d_members_match_alone(tile, graph, gpu_lib):
    """3-D members mixed with 2-D members equal their solo runs bit for bit."""
    models = members_3d(gpu_lib) + [member_model(s) for s in range(4)] + [rich_member(s) for s in range(2)]
    ref = []
    for m, mo in models:
        st, b, meta = make(m, mo, gpu_lib)
        st.run(1, m.Nt)
        ref.append(outputs_nd(st, m, meta))
        st.close()
    batch = _abi.Batch(gpu_lib)
    batch.config(*tile, graph)
    held = []
    for m, mo in models:
        st, b, meta = make(m, mo, gpu_lib)
        batch.add(st, m.Nt)
        held.append((st, b, meta, m))
    batch.run_all(chunk=23)
    for (st, b, meta, m), r in zip(held, ref):
        same(r, outputs_nd(st, m, meta))
    info = batch.info()
    assert info["cell_updates"] == sum(m.grid.Nx * m.grid.Ny * m.grid.Nz * m.Nt for m, _ in models)
    batch.close()
    for st, *_ in held:
        st.close()


def test_batch_3d_member_matches_oracle(oracle_lib, gpu_lib):
    """A batched 3-D member (materials, monitors) against the CPU oracle: bit for bit, the
    summed monitors (another summation order) within relative L2 1e-5."""
    m, mo = C.model_materials(3), C.monitors(3)
    st0, b0, meta0 = make(m, mo, oracle_lib)
    st0.run(1, m.Nt)
    ref = outputs_nd(st0, m, meta0)
    st0.close()
    batch = _abi.Batch(gpu_lib)
    st, b, meta = make(m, mo, gpu_lib)
    batch.add(st, m.Nt)
    batch.run_all()
    got = outputs_nd(st, m, meta)
    for k in ref:
        if k.startswith("mon/1/") or k.startswith("mon/4/"):
            a, b = np.asarray(ref[k], dtype=np.complex128), np.asarray(got[k], dtype=np.complex128)
            den = max(np.linalg.norm(a), np.linalg.norm(b))
            assert den == 0 or np.linalg.norm(a - b) / den <= 1e-5, k
        else:
            assert np.array_equal(got[k], ref[k], equal_nan=True), k
    batch.close()
    st.close()
