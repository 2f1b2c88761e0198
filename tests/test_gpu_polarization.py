"""The second 2-D field set (Hx, Hz, Dy, Ey; MFD_POL_EY) on the GPU against the oracle:
bit for bit in the exact mode (summed monitors and plasma within the tolerances of the
first field set's tests), within 1e-5 / 1e-12 in the tolerance mode, TFSF record and
replay, state images, and the batch's refusal."""
import ctypes as Cc

import numpy as np
import pytest

import cases as C
import polarization_cases as PC
from maxwellfdtd_b200 import _abi
from maxwellfdtd_b200.sources import comp_index
from test_gpu_parity import SUMMED, TOL, TOL_PLASMA_STATE, _compare, _rel

pytestmark = pytest.mark.gpu

DTYPES = [np.float64, np.float32]


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("name", ["vacuum", "bcs", "materials", "poles", "sources"])
def test_ey_parity_exact(name, dtype, oracle_lib, gpu_lib):
    model = PC.CASES[name]()
    mons = C.monitors(2) if name in ("vacuum", "materials") else None
    ref = C.run_all(model, oracle_lib, dtype, mons)
    got = C.run_all(model, gpu_lib, dtype, mons)
    _compare(ref, got, dtype, exact=True, loose=SUMMED)
    assert np.abs(got["field/Ey"]).max() > 0


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("rate", ["power", "table"])
def test_ey_parity_plasma(rate, dtype, oracle_lib, gpu_lib):
    model = PC.ey_plasma(rate)
    ref = C.run_all(model, oracle_lib, dtype)
    got = C.run_all(model, gpu_lib, dtype)
    assert np.max(ref["rho_end"]) > 0, "the case must ionise"
    state = ("rho_end", "JE")
    _compare({k: v for k, v in ref.items() if k not in state}, {k: v for k, v in got.items() if k not in state},
             dtype, exact=False)
    truth = ref if dtype == np.float64 else C.run_all(model, oracle_lib, np.float64)
    for k in state:
        if dtype == np.float64:
            assert _rel(ref[k], got[k]) <= TOL_PLASMA_STATE[dtype], (k, _rel(ref[k], got[k]))
        else:
            e_gpu, e_cpu = _rel(got[k], truth[k]), _rel(ref[k], truth[k])
            assert e_gpu <= max(2 * e_cpu, TOL_PLASMA_STATE[dtype]), (k, e_gpu, e_cpu)


@pytest.mark.parametrize("dtype", DTYPES)
def test_ey_tfsf_record_replay(dtype, oracle_lib, gpu_lib):
    box = (-240e-9, 240e-9, -240e-9, 240e-9)
    rec = PC.ey_tfsf_record()
    ref = C.run_all(rec, oracle_lib, dtype, tfsf_box_=box)
    got = C.run_all(rec, gpu_lib, dtype, tfsf_box_=box)
    _compare(ref, got, dtype, exact=True)
    record = {k[4:]: v for k, v in ref.items() if k.startswith("rec/")}
    rep = PC.ey_tfsf_replay(record)
    ref2 = C.run_all(rep, oracle_lib, dtype, C.monitors(2))
    got2 = C.run_all(rep, gpu_lib, dtype, C.monitors(2))
    _compare(ref2, got2, dtype, exact=True, loose=SUMMED)
    assert np.abs(got2["field/Ey"]).max() > 0


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("name", ["bcs", "materials"])
def test_ey_fast_mode(name, dtype, oracle_lib, gpu_lib):
    """The tolerance mode: fields, Sa and E2 within relative L2 1e-5 (FP32) / 1e-12 (FP64)
    of the exact order."""
    model = PC.CASES[name]()
    ref = C.run_all(model, oracle_lib, dtype)
    got = C.run_all(model, gpu_lib, dtype, mode="fast")
    for k in ref:
        assert _rel(ref[k], got[k]) <= TOL[dtype], (k, _rel(ref[k], got[k]))


def test_ey_state_image_resumes_bit_for_bit(gpu_lib):
    model = PC.ey_materials()
    n = model.Nt // 2
    b, _ = model.build_desc(np.float32)
    st = _abi.Stepper(gpu_lib, b, np.float32)
    st.run(1, n)
    img = st.read_state()
    st.run(n + 1, model.Nt)
    want = {c: st.read_field(comp_index(c)) for c in ("Hx", "Hz", "Dy", "Ey")}
    want["Sa"] = st.read_integral(_abi.MFD_INT_SA)
    st.close()
    b2, _ = model.build_desc(np.float32)
    st2 = _abi.Stepper(gpu_lib, b2, np.float32)
    st2.write_state(img)
    st2.run(n + 1, model.Nt)
    for c in ("Hx", "Hz", "Dy", "Ey"):
        assert np.array_equal(st2.read_field(comp_index(c)), want[c]), c
    assert np.array_equal(st2.read_integral(_abi.MFD_INT_SA), want["Sa"])
    st2.close()


def test_batch_refuses_the_second_field_set(gpu_lib):
    model = PC.ey_vacuum()
    b, _ = model.build_desc(np.float32)
    st = _abi.Stepper(gpu_lib, b, np.float32)
    bt = _abi.Batch(gpu_lib)
    try:
        with pytest.raises(_abi.StepperError, match="field set"):
            bt.add(st, model.Nt)
    finally:
        bt.close()
        st.close()
