"""The serving loop on the GPU: each request's results in the mix (batched 2-D and small 3-D
members, solo lanes, admitted as memory frees up) equal its results alone, bit for bit; the
admission footprint bounds what mfd_create allocates."""
import numpy as np
import pytest

import cases as C
import maxwellfdtd_b200 as M
from maxwellfdtd_b200 import _abi, serve, workloads

pytestmark = pytest.mark.gpu


def footprint_models():
    out = [(C.model_materials(3), C.monitors(3)), (C.model_materials(2), C.monitors(2)),
           (C.model_plasma(3, "table"), None), (C.model_bcs(1), C.monitors(1))]
    out += [(m, mo) for _, m, mo in workloads.served(n=6, steps_scale=0.02, n2=(64, 160), n3=(24, 48), seed=7)]
    out += workloads.batch2d(n=3, steps_scale=0.01, nmin=64, nmax=128)
    return out


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_footprint_bounds_device_bytes(dtype, gpu_lib):
    for model, mons in footprint_models():
        b, meta = model.build_desc(dtype, mons)
        est = serve.footprint(b, model, dtype)
        st = _abi.Stepper(gpu_lib, b, dtype)
        got = st.device_bytes()
        st.close()
        assert got <= est <= 1.1 * got + (1 << 20), (model.grid.ndim, got, est)


def test_serve_mix_matches_alone(gpu_lib):
    reqs = [serve.Request(i, m, mo, a) for i, (a, m, mo) in
            enumerate(workloads.served(n=10, steps_scale=0.02, n2=(64, 160), n3=(24, 48), seed=3))]
    k = len(reqs)
    for j, (m, mo) in enumerate(workloads.batch2d(n=6, steps_scale=0.01, nmin=64, nmax=160, seed=4)):
        reqs.append(serve.Request(k + j, m, mo, 0.004 * j))
    k = len(reqs)
    reqs.append(serve.Request(k, C.model_materials(3), C.monitors(3), 0.01, dtype=np.float64))   # a solo lane
    assert any(r.batchable and r.model.grid.ndim == 3 for r in reqs)
    assert any(r.batchable and r.model.grid.ndim == 2 for r in reqs) and any(not r.batchable for r in reqs)
    budget = 3 * max(r.bytes for r in reqs)
    srv = serve.Server(gpu_lib, budget_bytes=budget, max_active=6, max_solo=3, chunk=16, read_fields=True)
    st = srv.run(reqs)
    assert st["errors"] == 0 and st["requests"] == len(reqs)
    assert srv.peak_used <= budget
    for r in reqs:
        ref, status, _ = serve.solve_alone(gpu_lib, r)
        assert tuple(r.status) == tuple(status)
        bad = [key for key in ref if not np.array_equal(ref[key], r.out[key], equal_nan=True)]
        assert not bad, (r.id, r.batchable, bad)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_native_footprint_bounds_device_bytes(dtype, gpu_lib):
    """mfd_server_footprint, the admission estimate the native server uses."""
    for model, mons in footprint_models():
        b, meta = model.build_desc(dtype, mons)
        est = gpu_lib.server_footprint(C_byref(b))
        st = _abi.Stepper(gpu_lib, b, dtype)
        got = st.device_bytes()
        st.close()
        assert got <= est <= 1.1 * got + (1 << 20), (model.grid.ndim, got, est)


def C_byref(builder):
    import ctypes
    return ctypes.byref(builder.desc)


def test_native_server_api(gpu_lib):
    """Submit, wait, read through the request's handle, release; a request larger than the
    budget is refused at submission; unknown ids are refused."""
    models = [(C.model_materials(3), C.monitors(3)), (C.model_materials(2), C.monitors(2)),
              (C.model_bcs(1), None)]
    builders = [m.build_desc(np.float32, mo) for m, mo in models]
    budget = 4 * max(gpu_lib.server_footprint(C_byref(b)) for b, _ in builders)
    srv = _abi.Server(gpu_lib, budget_bytes=budget, max_active=2, max_solo=1)
    try:
        ids = [srv.submit(b) for b, _ in builders]
        for rid, (b, meta), (model, mons) in zip(ids, builders, models):
            assert srv.wait(rid, 300.0) == _abi.MFD_REQ_DONE
            state, times, nbytes, code = srv.poll(rid)
            assert state == _abi.MFD_REQ_DONE and code == _abi.MFD_OK and nbytes > 0
            assert times[0] <= times[1] <= times[2] <= times[3]
            h = srv.handle(rid, np.float32)
            got = h.read_field(6)
            alone = _abi.Stepper(gpu_lib, b, np.float32)
            alone.run(1, model.Nt)
            assert np.array_equal(got, alone.read_field(6))
            alone.close()
            assert h.status()[0] == model.Nt
            srv.release(rid)
        info = srv.info()
        assert info["done"] == len(ids) and info["failed"] == 0 and info["used_bytes"] == 0
        assert info["peak_used_bytes"] <= budget and info["peak_active"] <= 2
        big, _ = C.model_materials(3).build_desc(np.float32, C.monitors(3))
        small_srv = _abi.Server(gpu_lib, budget_bytes=1e5, max_active=1, max_solo=1)
        with pytest.raises(_abi.StepperError) as ei:
            small_srv.submit(big)
        assert ei.value.code == _abi.MFD_ERR_ADMISSION
        small_srv.close()
        with pytest.raises(_abi.StepperError):
            srv.poll(12345)
    finally:
        srv.close()
