"""The serving loop's host logic on the CPU, through the oracle library (solo lanes only):
admission in arrival order within the memory budget and the slot limits, every request
completed with the results it has alone, latency statistics."""
import numpy as np
import pytest

import cases as C
import maxwellfdtd_b200 as M
from maxwellfdtd_b200 import serve


def small_requests(n=8, seed=0):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        nd = 2 if i % 2 else 1
        if nd == 2:
            g = C.grid2((int(rng.integers(12, 30)), int(rng.integers(12, 30))))
            src = M.SoftSource(geometry=(0.0, 0.0), waveform=lambda x, z, t: C.pulse(t), component="Ez")
            mons = [M.FieldMonitor((0.0, 0.0)), M.SpectralMonitor((50e-9, 0.0), w=np.linspace(1e15, 3e15, 5))]
        else:
            g = C.grid1(int(rng.integers(30, 80)))
            src = M.SoftSource(geometry=(0.0,), waveform=lambda z, t: C.pulse(t), component="Ex")
            mons = [M.FieldMonitor((0.0,))]
        dt = 0.5 / C.C0 / np.sqrt(nd / (50e-9) ** 2)
        model = M.Model(g, src, tmax=(int(rng.integers(10, 30)) - 0.5) * dt, pml=100e-9)
        reqs.append(serve.Request(i, model, mons, arrival=0.002 * i))
    return reqs


def test_serve_completes_in_order_within_budget(oracle_lib):
    reqs = small_requests()
    budget = 2.5 * max(r.bytes for r in reqs)
    srv = serve.Server(oracle_lib, budget_bytes=budget, max_active=3, max_solo=2, use_batch=False, read_fields=True)
    st = srv.run(reqs)
    assert st["requests"] == len(reqs) and st["errors"] == 0
    assert srv.admitted == [r.id for r in sorted(reqs, key=lambda r: r.arrival)]   # FIFO
    assert srv.peak_used <= budget and srv.peak_active <= 2
    assert st["latency_p99_s"] >= st["latency_p50_s"] > 0
    for r in reqs:
        assert r.t_submit <= r.t_admit <= r.t_done
        ref, status, _ = serve.solve_alone(oracle_lib, r)
        assert set(ref) == set(r.out)
        for k in ref:
            assert np.array_equal(ref[k], r.out[k]), (r.id, k)


def test_serve_rejects_request_beyond_budget(oracle_lib):
    reqs = small_requests(2)
    srv = serve.Server(oracle_lib, budget_bytes=min(r.bytes for r in reqs) - 1, use_batch=False)
    with pytest.raises(ValueError):
        srv.run(reqs)


def test_native_footprint_without_gpu():
    """The library's admission estimate (mfd_server_footprint) is host code: it runs without a
    device and agrees with the Python estimate within 10 %."""
    from maxwellfdtd_b200 import _abi
    import ctypes
    lib = M.load_library()
    for r in small_requests(6) + [serve.Request(9, C.model_materials(3), C.monitors(3), 0.0)]:
        est = lib.server_footprint(ctypes.byref(r.builder.desc))
        assert est > 0
        assert abs(est - r.bytes) <= 0.1 * r.bytes + (1 << 16), (est, r.bytes)
