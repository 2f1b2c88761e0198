"""Pins the CPU oracle to the reference: its own known-answer tests (test/*.jl), same grids,
sources, analytic solutions and tolerances, in Float64 (the reference's CPU() default) and
Float32 (its GPU() default)."""
import numpy as np
import pytest

import maxwellfdtd_b200 as M
from reference_cases import CASES


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_reference_known_answer(name, dtype, oracle_lib):
    model, check = CASES[name]()
    sol = M.solve(model, backend=M.B200(np.dtype(dtype), library=oracle_lib))
    ok, err = check(sol)
    assert ok, f"{name} {dtype}: relative error {err:.4g}"
