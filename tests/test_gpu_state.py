"""Model state images (mfd_read_state / mfd_write_state) through the C ABI.

A run that is stopped, saved, loaded into a fresh handle made from the same descriptor and
continued there gives the same results, bit for bit, as the run that was never stopped:
fields, running sums, CPML psi, ADE and plasma state, monitor records and DFT accumulators
all travel in the image.  Images of another model's layout are refused.
"""
import numpy as np
import pytest

import cases as C
from maxwellfdtd_b200 import _abi
from maxwellfdtd_b200.sources import comp_index, field_components

pytestmark = pytest.mark.gpu


def _outputs(st, model, meta):
    nd = model.grid.ndim
    out = {c: st.read_field(comp_index(c)) for c in field_components(nd)}
    for w in (_abi.MFD_INT_SA, _abi.MFD_INT_E2, _abi.MFD_INT_JE, _abi.MFD_INT_RHO):
        out[f"int{w}"] = st.read_integral(w)
    comps = {3: ("Hx", "Hy", "Hz", "Ex", "Ey", "Ez"), 2: ("Hy", "Ex", "Ez"), 1: ("Hy", "Ex")}[nd]
    for k, mm in enumerate(meta["monitors"]):
        spectral = mm["kind"] == 1
        npts = len(mm["cells"])
        for c in comps:
            if spectral:
                shape = (mm["dft"].Nw,) if mm["sum"] else (mm["dft"].Nw, npts)
            else:
                shape = (model.Nt,) if mm["sum"] else (model.Nt, npts)
            out[f"m{k}/{c}"] = st.read_monitor(k, comp_index(c), shape, spectral)
    out["status"] = np.array(st.status())
    return out


BUILDERS = {
    "materials": lambda n: (C.model_materials(n), C.monitors(n)),
    "plasma": lambda n: (C.model_plasma(n, "table"), None),
    "bcs": lambda n: (C.model_bcs(n), None),
}


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("ndim", [1, 2, 3])
@pytest.mark.parametrize("case", sorted(BUILDERS))
def test_save_restore_continue(case, ndim, dtype, gpu_lib):
    model, mons = BUILDERS[case](ndim)
    b, meta = model.build_desc(dtype, mons)
    whole = _abi.Stepper(gpu_lib, b, dtype)
    whole.run(1, model.Nt)
    ref = _outputs(whole, model, meta)
    whole.close()

    cut = model.Nt // 2 - 1
    first = _abi.Stepper(gpu_lib, b, dtype)
    first.run(1, cut)
    image = first.read_state()
    assert image.size == gpu_lib.state_size(first.h)
    first.close()
    second = _abi.Stepper(gpu_lib, b, dtype)
    second.write_state(image)
    assert second.status()[0] == cut
    second.run(cut + 1, model.Nt)
    got = _outputs(second, model, meta)
    second.close()
    for k in ref:
        assert np.array_equal(ref[k], got[k], equal_nan=True), k


def test_state_of_another_model_is_refused(gpu_lib):
    m1 = C.model_vacuum(3)
    m2 = C.model_materials(3)
    b1, _ = m1.build_desc(np.float32, None)
    b2, _ = m2.build_desc(np.float32, None)
    s1 = _abi.Stepper(gpu_lib, b1, np.float32)
    s2 = _abi.Stepper(gpu_lib, b2, np.float32)
    try:
        s1.run(1, 5)
        img = s1.read_state()
        with pytest.raises(_abi.StepperError) as ei:
            s2.write_state(img)
        assert ei.value.code == _abi.MFD_ERR_INVALID and "layout" in str(ei.value)
        with pytest.raises(_abi.StepperError):
            s1.write_state(img[:100])              # truncated
        bad = img.copy()
        bad[:8] = 0
        with pytest.raises(_abi.StepperError):
            s1.write_state(bad)                    # not an image
        s1.write_state(img)                        # its own image loads
    finally:
        s1.close()
        s2.close()


def test_state_moves_a_run_back(gpu_lib):
    """Loading an earlier image into the same handle rewinds it: the steps after it are
    recomputed with the same result."""
    model, mons = C.model_materials(3), C.monitors(3)
    b, meta = model.build_desc(np.float32, mons)
    st = _abi.Stepper(gpu_lib, b, np.float32)
    try:
        st.run(1, 20)
        img = st.read_state()
        st.run(21, model.Nt)
        a = _outputs(st, model, meta)
        st.write_state(img)
        st.run(21, model.Nt)
        b2 = _outputs(st, model, meta)
        for k in a:
            assert np.array_equal(a[k], b2[k]), k
    finally:
        st.close()
