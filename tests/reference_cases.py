"""The reference's known-answer tests (test/*.jl) as model builders.

Each builder returns (model, check) where check(solution) -> (ok, detail) applies the
reference's own criterion with its own tolerance.  The same cases run on the CPU oracle
(tests/test_oracle_reference.py) and on the GPU (tests/test_gpu_reference.py).
"""
import numpy as np

import maxwellfdtd_b200 as M
from maxwellfdtd_b200 import C0, EPS0


def _isapprox(a, b, rtol):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    err = np.linalg.norm(a - b) / max(np.linalg.norm(a), np.linalg.norm(b))
    return err <= rtol, float(err)


def _pulse(t):
    lam0 = 2e-6
    tau0 = 20e-15
    dt0 = 3 * tau0
    w0 = 2 * np.pi * C0 / lam0
    return np.exp(-(t - dt0) ** 2 / tau0 ** 2) * np.cos(w0 * (t - dt0))


# test/1d_test.jl:1-30 ---------------------------------------------------------------------
def case_1d():
    grid = M.Grid(zmin=-5e-6, zmax=55e-6, Nz=2001)

    def waveform(z, t):
        return _pulse(t)

    src = M.HardSource(geometry=lambda z: abs(z) < grid.dz / 2, waveform=waveform, component="Ex")
    model = M.Model(grid, src, tmax=150e-15, pml=4e-6)
    Eth = waveform(grid.z, model.t[-1] - grid.z / C0)
    return model, lambda sol: _isapprox(sol.field.Ex, Eth, 1e-2)


# test/2d_test.jl:1-37 ---------------------------------------------------------------------
def case_2d():
    grid = M.Grid(xmin=-55e-6, xmax=55e-6, Nx=11, zmin=-5e-6, zmax=55e-6, Nz=1101)
    a0 = 10e-6

    def waveform(x, z, t):
        return np.exp(-0.5 * (x / a0) ** 2) * _pulse(t)

    src = M.HardSource(geometry=lambda x, z: abs(z) < grid.dz / 2, waveform=waveform, component="Ex")
    model = M.Model(grid, src, tmax=150e-15, pml=4e-6)
    X, Z = np.meshgrid(grid.x, grid.z, indexing="ij")
    Eth = waveform(X, Z, model.t[-1] - Z / C0)
    return model, lambda sol: _isapprox(sol.field.Ex, Eth, 5e-2)


# test/3d_test.jl:1-39 ---------------------------------------------------------------------
def case_3d():
    grid = M.Grid(xmin=-55e-6, xmax=55e-6, Nx=11, ymin=-55e-6, ymax=55e-6, Ny=11,
                  zmin=-5e-6, zmax=55e-6, Nz=801)
    a0 = 10e-6

    def waveform(x, y, z, t):
        return np.exp(-0.5 * (np.sqrt(x ** 2 + y ** 2) / a0) ** 2) * _pulse(t)

    src = M.HardSource(geometry=lambda x, y, z: abs(z) < grid.dz / 2, waveform=waveform, component="Ex")
    model = M.Model(grid, src, tmax=150e-15, pml=4e-6)
    X, Y, Z = np.meshgrid(grid.x, grid.y, grid.z, indexing="ij")
    Eth = waveform(X, Y, Z, model.t[-1] - Z / C0)
    return model, lambda sol: _isapprox(sol.field.Ex, Eth, 1e-1)


# test/{1,2,3}d_test_losses.jl ---------------------------------------------------------------
def _losses_check(z, ki, ndim):
    def check(sol):
        Sa = np.asarray(sol.out["Sa"], dtype=np.float64)
        mask = (z < 0) | (z > 20e-6)
        shape = [1] * Sa.ndim
        shape[-1] = len(z)
        m = np.broadcast_to(mask.reshape(shape), Sa.shape)
        Sa = np.where(m, 0.0, Sa)
        Sa = Sa / Sa.max()
        I = np.where(m, 0.0, np.broadcast_to(np.exp(-2 * ki * z).reshape(shape), Sa.shape))
        return _isapprox(Sa, I, 1e-2)
    return check


def case_losses(ndim, kind):
    """kind: 'sigma' (conductivity, eps=2.25, sigma=300) or 'lorentz' (deps=2, w0=2pi c/1um)."""
    if ndim == 1:
        grid = M.Grid(zmin=-15e-6, zmax=25e-6, Nz=2001)
        geo_src = lambda z: abs(z - -10e-6) <= grid.dz / 2
        geo_mat = lambda z: z >= 0
        wf = lambda z, t: _pulse(t)
    elif ndim == 2:
        grid = M.Grid(xmin=-25e-6, xmax=25e-6, Nx=61, zmin=-15e-6, zmax=25e-6, Nz=601)
        geo_src = lambda x, z: abs(z - -10e-6) <= grid.dz / 2
        geo_mat = lambda x, z: z >= 0
        wf = lambda x, z, t: _pulse(t)
    else:
        grid = M.Grid(xmin=-25e-6, xmax=25e-6, Nx=11, ymin=-25e-6, ymax=25e-6, Ny=11,
                      zmin=-15e-6, zmax=25e-6, Nz=601)
        geo_src = lambda x, y, z: abs(z - -10e-6) <= grid.dz / 2
        geo_mat = lambda x, y, z: z >= 0
        wf = lambda x, y, z, t: _pulse(t)
    src = M.SoftSource(geometry=geo_src, waveform=wf, component="Ex")
    lam0 = 2e-6
    w0 = 2 * np.pi * C0 / lam0
    if kind == "sigma":
        sigma = 300
        er = 1.5 ** 2
        ei = sigma / (EPS0 * w0)
        ni = np.sqrt((np.sqrt(er ** 2 + ei ** 2) - er) / 2)
        ki = ni * w0 / C0
        mat = M.Material(geometry=geo_mat, eps=er, sigma=sigma)
        tmax = 300e-15
    else:
        chi = M.LorentzSusceptibility(deps=2, w0=2 * np.pi * C0 / 1e-6, delta=0.01 * 2 * np.pi * C0 / 1e-6)
        n0 = np.sqrt(1 + M.susceptibility(chi, w0))
        ki = n0.imag * w0 / C0
        mat = M.Material(geometry=geo_mat, chi=chi)
        tmax = 600e-15
    model = M.Model(grid, src, tmax=tmax, pml=5e-6, material=mat)
    return model, _losses_check(grid.z, ki, ndim)


CASES = {
    "1d": case_1d, "2d": case_2d, "3d": case_3d,
    "1d_sigma": lambda: case_losses(1, "sigma"), "1d_lorentz": lambda: case_losses(1, "lorentz"),
    "2d_sigma": lambda: case_losses(2, "sigma"), "2d_lorentz": lambda: case_losses(2, "lorentz"),
    "3d_sigma": lambda: case_losses(3, "sigma"), "3d_lorentz": lambda: case_losses(3, "lorentz"),
}
