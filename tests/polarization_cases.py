"""Models of the second 2-D field set (Hx, Hz, Dy, Ey; Model(..., polarization="Ey")) for
the oracle and GPU tests: the same media, boundaries and sources as the first field set's
cases, driven through Ey, Hx and Hz."""
import numpy as np

import maxwellfdtd_b200 as M
from maxwellfdtd_b200.constants import C0, EPS0

from cases import _ball, _plane, _src_wave, grid2, pulse

DT2 = 0.5 / C0 / np.sqrt(2 / (50e-9) ** 2)


def _model(src, nsteps, **kw):
    return M.Model(grid2(), src, tmax=(nsteps - 0.5) * DT2, polarization="Ey", **kw)


def ey_vacuum(nsteps=60):
    src = M.SoftSource(geometry=_plane(2, -200e-9), waveform=_src_wave(2), component="Ey")
    return _model(src, nsteps, pml=150e-9)


def ey_bcs(nsteps=60):
    """Mixed boundary conditions, CPML with kmax != 1 on two faces, a point source."""
    src = M.SoftSource(geometry=(50e-9, -100e-9), waveform=_src_wave(2, 3.0), component="Ey")
    cp = M.CPML(thickness=150e-9, kmax=4.0, alpha=0.05, R0=1e-8, m=4)
    return _model(src, nsteps, pml=(0, cp, cp, 0), bc=("dirichlet", "neumann", "periodic", "neumann"))


def ey_materials(nsteps=70):
    """Conductive dielectric with mu != 1, Drude+Lorentz ball, Debye+Kerr slab."""
    src = M.SoftSource(geometry=_plane(2, -250e-9), waveform=_src_wave(2, 2e8), component="Ey")
    m1 = M.Material(geometry=lambda x, z: x > 0, eps=2.25, mu=1.3, sigma=2e4)
    m2 = M.Material(geometry=_ball(2, 160e-9), eps=3.0,
                    chi=[M.DrudeSusceptibility(wp=1.37e16, gamma=1.07e14),
                         M.LorentzSusceptibility(deps=1.1, w0=4.2e15, delta=5e14)])
    m3 = M.Material(geometry=lambda x, z: z >= 150e-9, eps=2.0, chi=M.DebyeSusceptibility(deps=2.0, tau=1e-14),
                    chi3=1e-19)
    return _model(src, nsteps, pml=150e-9, material=[m1, m2, m3])


def ey_poles(nsteps=50):
    """Five poles and Kerr in a ball over a one-pole slab."""
    src = M.SoftSource(geometry=_plane(2, -250e-9), waveform=_src_wave(2, 3e8), component="Ey")
    kinds = [lambda i: M.LorentzSusceptibility(deps=0.5 + 0.2 * i, w0=(3 + i) * 1e15, delta=(1 + i) * 1e14),
             lambda i: M.DrudeSusceptibility(wp=(1 + 0.1 * i) * 1e16, gamma=1.07e14),
             lambda i: M.DebyeSusceptibility(deps=1.0 + i, tau=(1 + i) * 1e-14)]
    m1 = M.Material(geometry=_ball(2, 200e-9), eps=2.0, chi=[kinds[i % 3](i) for i in range(5)], chi3=1e-19)
    m2 = M.Material(geometry=lambda x, z: z >= 200e-9, eps=1.5,
                    chi=M.LorentzSusceptibility(deps=0.7, w0=5e15, delta=2e14))
    return _model(src, nsteps, pml=150e-9, material=[m1, m2])


def ey_plasma(rate="power", nsteps=60):
    E0 = 1.3e10
    src = M.SoftSource(geometry=_plane(2, -250e-9), waveform=_src_wave(2, E0), component="Ey")
    w0 = 2 * np.pi * C0 / 800e-9
    if rate == "power":
        ionrate = M.PowerLawRate(order=8, sigma=1e-130)
    else:
        I = np.logspace(12, 20, 81)
        ionrate = M.IonizationRate(np.stack([I, 1e-130 * I ** 8], axis=1))
    pl = M.Plasma(ionrate=ionrate, rho0=2.1e28, nuc=1 / 1e-15, frequency=w0, Uiev=9.0, mr=0.64)
    chi3 = 4 / 3 * 1.45 ** 2 * EPS0 * C0 * 2.5e-20
    mat = M.Material(geometry=_ball(2, 250e-9), eps=1.45 ** 2, chi3=chi3, plasma=pl,
                     chi=M.LorentzSusceptibility(deps=0.7, w0=1.6e16, delta=1e13))
    return _model(src, nsteps, pml=150e-9, material=mat)


def ey_sources(nsteps=50):
    """Hard sources on Hx and Hz, an explicit soft source on Ey, a soft source on Dy."""
    s1 = M.HardSource(geometry=(0.0, -150e-9), waveform=_src_wave(2, 1e-3), component="Hx")
    s2 = M.SoftSource(geometry=_plane(2, 100e-9), waveform=_src_wave(2, 0.7), component="Ey", explicit=True)
    s3 = M.HardSource(geometry=(100e-9, 0.0), waveform=_src_wave(2, 2e-3), component="Hz")
    s4 = M.SoftSource(geometry=_plane(2, 100e-9), waveform=_src_wave(2, 0.3), component="Ey")
    return _model([s1, s2, s3, s4], nsteps, pml=100e-9)


CASES = {"vacuum": ey_vacuum, "bcs": ey_bcs, "materials": ey_materials, "poles": ey_poles,
         "plasma_power": lambda: ey_plasma("power"), "plasma_table": lambda: ey_plasma("table"),
         "sources": ey_sources}


def ey_tfsf_record(nsteps=60):
    """Vacuum record run of the second field set: an Ey plane source, periodic in x,
    absorbing in z."""
    src = M.SoftSource(geometry=_plane(2, -400e-9), waveform=lambda x, z, t: pulse(t), component="Ey")
    return _model(src, nsteps, pml=(0, 0, 100e-9, 100e-9))


def ey_tfsf_replay(record, nsteps=60, material=True):
    mat = M.Material(geometry=_ball(2, 120e-9), eps=2.25) if material else None
    return _model(M.TFSFSource(data=record), nsteps, pml=100e-9, material=mat)
