"""The reference's own known-answer tests (test/*.jl) run on the CUDA library, with the
reference's tolerances, in Float32 (its GPU() default) and Float64."""
import numpy as np
import pytest

import maxwellfdtd_b200 as M
from reference_cases import CASES

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_reference_known_answer_gpu(name, dtype, gpu_lib):
    model, check = CASES[name]()
    sol = M.solve(model, backend=M.B200(np.dtype(dtype)))
    ok, err = check(sol)
    assert ok, f"{name} {dtype}: relative error {err:.4g}"
