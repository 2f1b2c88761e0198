"""Monitors and the DFT (reference src/monitors.jl, src/dft.jl)."""
from dataclasses import dataclass
from typing import Any, Optional

import numpy as np

from .geometry import geometry2indices


@dataclass
class FieldMonitor:
    """``FieldMonitor(geometry; sum=false)`` (monitors.jl:7-30)."""
    geometry: Any
    sum: bool = False


@dataclass
class SpectralMonitor:
    """``SpectralMonitor(geometry; wmin, wmax, sum=false)`` (monitors.jl:198-223).

    The reference accumulates on the FFT bins 2*pi*k/(Nt*dt) between wmin and wmax.  ``w``
    (an extension) gives an explicit list of angular frequencies instead."""
    geometry: Any
    wmin: Optional[float] = None
    wmax: Optional[float] = None
    sum: bool = False
    w: Optional[Any] = None


class DFT:
    """``DFT(t; wmin, wmax, sum)`` (dft.jl:1-24), evaluated with the element-type-T time
    range the reference's monitors see after adapt()."""

    def __init__(self, t_T, dtype, wmin=None, wmax=None, w=None):
        T = np.dtype(dtype).type
        Nt = len(t_T)
        dt = T(T(t_T[1]) - T(t_T[0]))
        tshift = T(Nt // 2) * dt if Nt % 2 == 0 else T((Nt + 1) // 2) * dt
        self.dt = dt
        self.tshift = T(tshift)
        if w is None:
            Nw = Nt // 2 + 1
            dtNt = float(T(dt * T(Nt)))
            ws = np.array([2 * np.pi * (iw - 1) / dtNt for iw in range(1, Nw + 1)])
            iwmin = 1 if wmin is None else int(np.argmin(np.abs(ws - wmin))) + 1
            iwmax = Nw if wmax is None else int(np.argmin(np.abs(ws - wmax))) + 1
            ws = ws[iwmin - 1:iwmax]
        else:
            ws = np.asarray(w, dtype=np.float64).ravel()
        self.w = ws
        self.Nw = len(ws)
        # phase exp(-1im*w*(t - tshift)) (dft.jl:40, 44): (t - tshift) in T, times -w in double
        d = (np.asarray(t_T, dtype=T) - T(tshift)).astype(np.float64)
        theta = (-ws)[None, :] * d[:, None]
        ph = np.empty((Nt, self.Nw, 2))
        ph[:, :, 0] = np.cos(theta)
        ph[:, :, 1] = np.sin(theta)
        self.phasor = ph


def monitor_struct(monitor, grid, coords_T, t_T, dtype):
    cells = geometry2indices(monitor.geometry, grid, coords_T)
    if len(cells) == 0:
        raise ValueError("I did not find any grid points which satisfy your monitor geometry.")
    if isinstance(monitor, FieldMonitor):
        return {"kind": 0, "sum": bool(monitor.sum), "cells": cells}
    dft = DFT(t_T, dtype, monitor.wmin, monitor.wmax, monitor.w)
    return {"kind": 1, "sum": bool(monitor.sum), "cells": cells, "dft": dft}
