"""Materials and their update coefficients (reference src/materials.jl)."""
import math
from dataclasses import dataclass, field
from typing import Any, Callable, Optional

import numpy as np

from .constants import C0, EPS0, HBAR, ME, MU0, QE


# ----------------------------------------------------------------------------------------
# Susceptibilities (materials.jl:486-587)
# ----------------------------------------------------------------------------------------
class Susceptibility:
    pass


@dataclass
class DebyeSusceptibility(Susceptibility):
    deps: float
    tau: float

    def chi(self, w):
        return self.deps / (1 - 1j * w * self.tau)

    def ade_coefficients(self, dt):
        aq = 1 / self.tau
        bq = EPS0 * self.deps / self.tau
        return 1 - aq * dt, 0.0, bq * dt


@dataclass
class DrudeSusceptibility(Susceptibility):
    wp: float
    gamma: float

    def chi(self, w):
        return -(self.wp * self.wp) / (w * w + 1j * w * self.gamma)

    def ade_coefficients(self, dt):
        aq = self.gamma
        bq = EPS0 * (self.wp * self.wp)
        Aq = 2 / (aq * dt / 2 + 1)
        Bq = (aq * dt / 2 - 1) / (aq * dt / 2 + 1)
        Cq = bq * (dt * dt) / (aq * dt / 2 + 1)
        return Aq, Bq, Cq


@dataclass
class LorentzSusceptibility(Susceptibility):
    deps: float
    w0: float
    delta: float

    def chi(self, w):
        return self.deps * (self.w0 * self.w0) / (self.w0 * self.w0 - w * w - 2j * w * self.delta)

    def ade_coefficients(self, dt):
        aq = 2 * self.delta
        bq = self.w0 * self.w0
        cq = EPS0 * self.deps * (self.w0 * self.w0)
        Aq = (2 - bq * (dt * dt)) / (aq * dt / 2 + 1)
        Bq = (aq * dt / 2 - 1) / (aq * dt / 2 + 1)
        Cq = cq * (dt * dt) / (aq * dt / 2 + 1)
        return Aq, Bq, Cq


def susceptibility(chi, w):
    """``susceptibility(chi, w)`` for one susceptibility or a list of them (materials.jl:581-587)."""
    if isinstance(chi, (list, tuple)):
        tot = 0j
        for c in chi:
            tot += c.chi(w)
        return tot
    return chi.chi(w)


# ----------------------------------------------------------------------------------------
# Ionisation-rate closures.  The reference's plasma kernel calls a user Julia function
# ionrate(I) (models.jl:1117); a C ABI cannot call a closure, so the forms the reference
# ships are passed as parameters.
# ----------------------------------------------------------------------------------------
@dataclass
class PowerLawRate:
    """MPI rate ``10^(order*log10(I) + log10(sigma))`` (3D_plasma.jl:67)."""
    order: float
    sigma: float = None
    log10c: float = None

    def __post_init__(self):
        if self.log10c is None:
            self.log10c = math.log10(self.sigma)

    def __call__(self, I):
        I = np.asarray(I, dtype=np.float64)
        with np.errstate(divide="ignore"):
            return 10.0 ** (self.order * np.log10(I) + self.log10c)


class IonizationRate:
    """Log-log table of (intensity, rate) with equally spaced log10 intensities
    (examples/5_nonlinear_propagation/IonizationRate.jl:13-52)."""

    def __init__(self, source):
        if isinstance(source, str):
            data = np.loadtxt(source)
        else:
            data = np.asarray(source, dtype=np.float64)
        x = np.log10(data[:, 0])
        y = np.log10(data[:, 1])
        dx = np.diff(x)
        if not np.all(np.diff(x) > 0):
            raise ValueError("IonizationRate: intensities must be sorted")
        if not np.allclose(dx, dx[0], rtol=np.sqrt(np.finfo(float).eps), atol=0):
            raise ValueError("IonizationRate: log10 intensities must be evenly spaced")
        self.x = x
        self.y = y

    def __call__(self, I):
        I = np.atleast_1d(np.asarray(I, dtype=np.float64))
        out = np.zeros_like(I)
        pos = I > 0
        xi = np.log10(I[pos])
        n = len(self.x)
        i = np.searchsorted(self.x, xi, side="left") - 1
        i = np.where(xi <= self.x[0], 0, np.where(xi >= self.x[-1], n - 2, i))
        dydx = (self.y[i + 1] - self.y[i]) / (self.x[i + 1] - self.x[i])
        out[pos] = 10.0 ** (self.y[i] + dydx * (xi - self.x[i]))
        return out


def sampled_rate(fn, Imin=1e8, Imax=1e22, n=2001):
    """Any other closure: sampled on an even log10(I) grid and interpolated log-log on the
    device.  The interpolation error is that of linear interpolation in log-log space on
    this grid."""
    I = np.logspace(math.log10(Imin), math.log10(Imax), n)
    R = np.asarray([fn(v) for v in I], dtype=np.float64)
    R = np.maximum(R, np.finfo(float).tiny)
    return IonizationRate(np.stack([I, R], axis=1))


@dataclass
class Plasma:
    """``Plasma(; ionrate, rho0, nuc, frequency, Uiev, mr=1)`` (materials.jl:48-61)."""
    ionrate: Any
    rho0: float
    nuc: float
    frequency: float
    Uiev: float
    mr: float = 1.0


def ade_plasma_coefficients(nuc, mr, dt):
    """materials.jl:64-69"""
    Ap = 2 / (nuc * dt / 2 + 1)
    Bp = (nuc * dt / 2 - 1) / (nuc * dt / 2 + 1)
    Cp = (QE * QE) / (ME * mr) * (dt * dt) / (nuc * dt / 2 + 1)
    return Ap, Bp, Cp


@dataclass
class Material:
    """``Material(; geometry, eps=1, mu=1, sigma=0, chi, chi2, chi3, plasma)`` (materials.jl:1-44).
    geometry: a function of the grid coordinates or a boolean array of the grid's shape."""
    geometry: Any
    eps: float = 1.0
    mu: float = 1.0
    sigma: float = 0.0
    chi: Any = None
    chi2: Optional[float] = None
    chi3: Optional[float] = None
    plasma: Optional[Plasma] = None

    def __post_init__(self):
        if self.eps < 0:
            raise ValueError(
                f"You specified negative eps={self.eps}. Negative, frequency-independent "
                "permittivities lead to exponentially growing solutions. To model a material with "
                "negative permittivity, use frequency-dependent susceptibility chi.")


@dataclass
class MaterialStruct:
    """Update coefficients of one material (materials.jl:115-196, 247-331, 389-483)."""
    Mh: float
    Me: float
    Md1: float
    Md2: float
    Aq: np.ndarray
    Bq: np.ndarray
    Cq: np.ndarray
    iskerr: bool
    Mk2: float
    Mk3: float
    isplasma: bool
    Rava: float = 0.0
    ksi: float = 0.0
    rho0: float = 0.0
    Ap: float = 0.0
    Bp: float = 0.0
    Cp: float = 0.0
    Ma: float = 0.0
    rate: Any = None

    @property
    def nq(self):
        return len(self.Aq)


def material_struct(material, dt):
    eps, mu = float(material.eps), float(material.mu)
    sigma = float(material.sigma)
    sigmaD = sigma / (EPS0 * eps)
    Mh = dt / (MU0 * mu)
    Me = 1 / (EPS0 * eps)
    Md1 = (1 - sigmaD * dt / 2) / (1 + sigmaD * dt / 2)
    Md2 = dt / (1 + sigmaD * dt / 2)
    chi = material.chi
    if chi is None:
        Aq = Bq = Cq = np.zeros(0)
    else:
        chis = list(chi) if isinstance(chi, (list, tuple)) else [chi]
        coefs = [c.ade_coefficients(dt) for c in chis]
        Aq = np.array([c[0] for c in coefs], dtype=np.float64)
        Bq = np.array([c[1] for c in coefs], dtype=np.float64)
        Cq = np.array([c[2] for c in coefs], dtype=np.float64)
    if material.chi2 is None and material.chi3 is None:
        iskerr, Mk2, Mk3 = False, 0.0, 0.0
    else:
        iskerr = True
        Mk2 = 0.0 if material.chi2 is None else EPS0 * material.chi2
        Mk3 = 0.0 if material.chi3 is None else EPS0 * material.chi3
    ms = MaterialStruct(Mh, Me, Md1, Md2, Aq, Bq, Cq, iskerr, Mk2, Mk3, False)
    pl = material.plasma
    if pl is not None:
        ms.isplasma = True
        chi0 = susceptibility(chi, pl.frequency) if chi is not None else 0
        n = math.sqrt((eps + complex(chi0).real) * mu)
        ms.ksi = n * EPS0 * C0 / 2
        ms.Ap, ms.Bp, ms.Cp = ade_plasma_coefficients(pl.nuc, pl.mr, dt)
        Ui = pl.Uiev * QE
        Wph = HBAR * pl.frequency
        K = math.ceil(Ui / Wph)
        sigmaB = (QE * QE) / (ME * pl.mr) * pl.nuc / (pl.nuc * pl.nuc + pl.frequency * pl.frequency)
        ms.Rava = sigmaB / Ui
        ms.Ma = K * Wph * dt
        ms.rho0 = pl.rho0
        rate = pl.ionrate
        if not isinstance(rate, (PowerLawRate, IonizationRate)):
            rate = sampled_rate(rate)
        ms.rate = rate
    return ms
