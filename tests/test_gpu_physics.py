"""The physics checks of tests/test_oracle_pinning.py on the CUDA library, and the
reference's Keldysh rate table (tests/golden/SiO2_keldysh_1.03um.tf) driving the device's
table lookup, against the oracle."""
import numpy as np
import pytest

import cases
import physics_cases as P
import maxwellfdtd_b200 as M
import test_oracle_pinning as T

pytestmark = pytest.mark.gpu

DTYPES = [np.float64, np.float32]


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("ndim,kind", [(1, "drude"), (1, "debye"), (3, "drude")])
def test_attenuation_matches_susceptibility_gpu(ndim, kind, dtype, gpu_lib):
    """The 3-D grid is that of test/3d_test_losses.jl (11 x 11 cells of 5 um across, dz =
    67 nm); the weak Debye medium's attenuation is only resolved within 1e-2 on the 1-D
    grid (3-D: 2-4 % on the oracle as well), so it is checked there."""
    model, mons, check = P.case_attenuation(ndim, kind)
    sol = M.solve(model, backend=M.B200(dtype, library=gpu_lib), monitors=mons)
    ok, err = check(sol)
    assert ok, f"{kind} {ndim}-D: relative error {err:.4g}"


@pytest.mark.parametrize("dtype", DTYPES)
def test_cpml_reflection_gpu(dtype, gpu_lib):
    be = M.B200(dtype, library=gpu_lib)
    r = {}
    for nb in (12, 20):
        for kmax in (1.0, 4.0):
            model, mons, check = P.case_cpml_reflection(nb, kmax)
            r[(nb, kmax)] = check(M.solve(model, backend=be, monitors=mons))
    T.cpml_bounds_hold(r)
    model, mons, check = P.case_cpml_2d()
    assert check(M.solve(model, backend=be, monitors=mons)) < 5e-3


@pytest.mark.parametrize("dtype", DTYPES)
def test_energy_conserved_in_periodic_box_gpu(dtype, gpu_lib):
    assert T.energy_drift(gpu_lib, dtype) < (1e-13 if dtype == np.float64 else 2e-6)


@pytest.mark.parametrize("dtype", DTYPES)
def test_tfsf_leakage_in_vacuum_gpu(dtype, gpu_lib):
    out, ins = T.tfsf_leakage(gpu_lib, dtype)
    assert ins > 1e-3
    assert out / ins < (1e-12 if dtype == np.float64 else 1e-5), (out, ins)


@pytest.mark.parametrize("dtype,rho_fp64", [(np.float64, True), (np.float32, True), (np.float32, False)])
@pytest.mark.parametrize("ndim", [1, 2, 3])
def test_rate_table_fixture_gpu(ndim, dtype, rho_fp64, oracle_lib, gpu_lib):
    """Fields within the tolerance bound (relative L2 1e-5 in Float32, 1e-12 in Float64) of
    the same-precision oracle; the plasma density and delivered energy no further from the
    FP64 oracle than twice the FP32 oracle's own distance (or 1e-4): both sides evaluate
    log10/pow with their own libm."""
    model = T.plasma_fixture_model(ndim)
    ref = cases.run_all(model, oracle_lib, dtype, rho_fp64=rho_fp64)
    got = cases.run_all(model, gpu_lib, dtype, rho_fp64=rho_fp64)
    assert ref["rho_end"].max() > 0
    tol = 1e-12 if dtype == np.float64 else 1e-5
    state = ("rho_end", "JE")
    rel = lambda a, b: float(np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64)) /
                             max(np.linalg.norm(np.asarray(a, np.float64)), np.linalg.norm(np.asarray(b, np.float64)), 1e-300))
    bad = [(k, rel(ref[k], got[k])) for k in ref if k not in state and rel(ref[k], got[k]) > tol]
    assert not bad, bad
    if dtype == np.float64:
        for k in state:
            assert rel(ref[k], got[k]) <= 1e-9, k
    else:
        truth = cases.run_all(model, oracle_lib, np.float64)
        for k in state:
            e_gpu, e_cpu = rel(got[k], truth[k]), rel(ref[k], truth[k])
            assert e_gpu <= max(2 * e_cpu, 1e-4), (k, e_gpu, e_cpu)
