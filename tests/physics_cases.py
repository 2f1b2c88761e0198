"""Physics checks that pin paths the reference's own known-answer tests do not reach.

The reference tests (test/*.jl) check vacuum propagation and the attenuation of a pulse in a
conductive and in a Lorentz medium.  These cases extend the same kind of analytic check to
the other dispersive models and to properties any correct Yee/CPML/TFSF implementation has:

- attenuation of Sa in a Drude and in a Debye medium against exp(-2 ki z), ki from the
  model's own susceptibility (materials.jl:503-587), by the criterion and tolerance of
  test/1d_test_losses.jl;
- CPML absorption, kmax = 1 and kmax != 1: the pulse a layer sends back (1-D, normal
  incidence) and what a point source leaves outside the layers (2-D, every angle);
- conservation of the discrete electromagnetic energy in a lossless periodic box
  W_k = 1/2 sum(E_k . D_k) + 1/2 sum(mu0 mu H_k . H_{k+1}), which the Yee scheme with
  periodic faces keeps exactly up to rounding;
- TFSF replay of a vacuum record run in vacuum: the scattered field outside the box.

The attenuation and CPML builders return (model, monitors, check); check(solution) gives
(ok, detail) or the measured ratio.
"""
import numpy as np

import maxwellfdtd_b200 as M
from maxwellfdtd_b200 import C0, EPS0, MU0


def _isapprox(a, b, rtol):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    err = np.linalg.norm(a - b) / max(np.linalg.norm(a), np.linalg.norm(b))
    return err <= rtol, float(err)


def _pulse(t, lam0=2e-6, tau0=20e-15):
    t0 = 3 * tau0
    w0 = 2 * np.pi * C0 / lam0
    return np.exp(-(t - t0) ** 2 / tau0 ** 2) * np.cos(w0 * (t - t0))


def case_attenuation(ndim, kind, deps=0.05):
    """test/{1,3}d_test_losses.jl with a Drude or a Debye medium in z >= 0.  Drude: eps = 2.25,
    wp = 0.55 w0, gamma = 10 w0 (a conductor-like regime: ki varies slowly across the
    pulse's band).  Debye: deps = 0.05, tau = 1/w0 (the loss peak, flat in frequency)."""
    lam0 = 2e-6
    w0 = 2 * np.pi * C0 / lam0
    if ndim == 1:
        grid = M.Grid(zmin=-15e-6, zmax=25e-6, Nz=2001)
        geo_src = lambda z: abs(z - -10e-6) <= grid.dz / 2
        geo_mat = lambda z: z >= 0
        wf = lambda z, t: _pulse(t)
    else:
        grid = M.Grid(xmin=-25e-6, xmax=25e-6, Nx=11, ymin=-25e-6, ymax=25e-6, Ny=11,
                      zmin=-15e-6, zmax=25e-6, Nz=601)
        geo_src = lambda x, y, z: abs(z - -10e-6) <= grid.dz / 2
        geo_mat = lambda x, y, z: z >= 0
        wf = lambda x, y, z, t: _pulse(t)
    src = M.SoftSource(geometry=geo_src, waveform=wf, component="Ex")
    if kind == "drude":
        chi = M.DrudeSusceptibility(wp=0.55 * w0, gamma=10 * w0)
        eps = 2.25
    else:
        chi = M.DebyeSusceptibility(deps=deps, tau=1 / w0)
        eps = 1.0
    n = np.sqrt(eps + M.susceptibility(chi, w0))
    ki = abs(n.imag) * w0 / C0
    mat = M.Material(geometry=geo_mat, eps=eps, chi=chi)
    model = M.Model(grid, src, tmax=400e-15, pml=5e-6, material=mat)
    z = grid.z

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
    # the attenuation over the checked depth must be substantial for the check to mean much
    assert 2 * ki * 20e-6 > 0.5, (kind, 2 * ki * 20e-6)
    return model, None, check


def case_cpml_reflection(nb, kmax):
    """1-D: a pulse (600 nm, 2 fs) from a soft source runs past a monitor into an nb-cell CPML
    (kmax, alpha = 0.05, R0 = 1e-8, m = 3) 150 cells further on.  The monitor sees the
    incident pulse, then, 300 cells of travel later, what the layer sent back; check(sol)
    returns the ratio of the two peaks.  The reference evaluates kappa, sigma and the
    recursion coefficients at the integer grid points for the E and the H psi alike
    (pml.jl:57-121), so a thin layer at this resolution reflects about 1 %."""
    d = 20e-9
    g = 150
    n = 2 * (nb + 2 * g) + 1
    grid = M.Grid(zmin=-(n - 1) * d / 2, zmax=(n - 1) * d / 2, Nz=n)
    cp = M.CPML(thickness=nb * d, kmax=kmax, alpha=0.05, R0=1e-8, m=3)
    lam0, tau0 = 600e-9, 2e-15
    src = M.SoftSource(geometry=(-g * d,), waveform=lambda z, t: _pulse(t, lam0, tau0), component="Ex")
    model = M.Model(grid, src, tmax=8 * tau0 + (4 * g + 20) * d / C0, pml=cp, bc="dirichlet")
    mon = M.FieldMonitor((g * d,))
    half = int(g * d / (C0 * model.dt))   # steps for 150 cells: half the round trip to the layer

    def check(sol):
        tr = np.abs(np.asarray(sol.out["monitors/1/Ex"], dtype=np.float64)).ravel()
        i = int(np.argmax(tr))
        assert i + half < len(tr), "the run must cover the reflected pulse"
        return float(tr[i + half:].max() / tr[i])
    return model, [mon], check


def case_cpml_2d(kmax=4.0):
    """2-D: a point source at the centre of a 161 x 161 grid with 12-cell CPML on every face
    (every angle of incidence).  After the wave has run into the layers, the largest field
    left outside them, relative to the largest field at the source, is returned."""
    d = 20e-9
    nb = 12
    cp = M.CPML(thickness=nb * d, kmax=kmax, alpha=0.05, R0=1e-8, m=3)
    n = 161
    L = (n - 1) * d / 2
    grid = M.Grid(xmin=-L, xmax=L, Nx=n, zmin=-L, zmax=L, Nz=n)
    lam0, tau0 = 400e-9, 1.5e-15
    src = M.SoftSource(geometry=(0.0, 0.0), waveform=lambda x, z, t: _pulse(t, lam0, tau0), component="Ez")
    mon = M.FieldMonitor((2 * d, 0.0))
    model = M.Model(grid, src, tmax=6 * tau0 + 2.5 * (n / 2) * d / C0, pml=(cp, cp, cp, cp))

    def check(sol):
        peak = float(np.abs(np.asarray(sol.out["monitors/1/Ez"], dtype=np.float64)).max())
        f = np.abs(np.asarray(sol.field["Ez"], dtype=np.float64)).reshape(n, n, order="F")
        inner = f[nb + 2:n - nb - 2, nb + 2:n - nb - 2]
        return float(inner.max() / peak)
    return model, [mon], check


def _energy(fields, H_next, mu_map):
    E = [np.asarray(fields[c], dtype=np.float64) for c in ("Ex", "Ey", "Ez")]
    D = [np.asarray(fields[c], dtype=np.float64) for c in ("Dx", "Dy", "Dz")]
    H = [np.asarray(fields[c], dtype=np.float64) for c in ("Hx", "Hy", "Hz")]
    we = 0.5 * sum(float(np.sum(e * dd)) for e, dd in zip(E, D))
    wh = 0.5 * sum(float(np.sum(MU0 * mu_map * h * hn)) for h, hn in zip(H, H_next))
    return we + wh


def energy_box(n=16, d=50e-9, k1=80, k2=400):
    """Lossless periodic box (every face periodic, no CPML): vacuum with a dielectric,
    magnetic block (eps 2.25, mu 1.3) and a soft source whose pulse has ended before step k1.
    Returns (model, mu_map, k1, k2)."""
    L = (n - 1) * d / 2
    grid = M.Grid(xmin=-L, xmax=L, Nx=n, ymin=-L, ymax=L, Ny=n, zmin=-L, zmax=L, Nz=n)
    dt = 0.5 / C0 / np.sqrt(3 / d ** 2)
    tau0 = 4 * dt
    src = M.SoftSource(geometry=(0.0, 0.0, -0.2e-6),
                       waveform=lambda x, y, z, t: np.exp(-((t - 20 * dt) / tau0) ** 2), component="Ex")
    blk = lambda x, y, z: (np.abs(x) < 0.15e-6) & (np.abs(y - 0.05e-6) < 0.2e-6) & (z > 0)
    mat = M.Material(geometry=blk, eps=2.25, mu=1.3)
    model = M.Model(grid, src, tmax=(k2 + 1 - 0.5) * dt, pml=0, bc="periodic", material=mat)
    X, Y, Z = np.meshgrid(grid.x, grid.y, grid.z, indexing="ij")
    mu_map = np.where(blk(X, Y, Z), 1.3, 1.0)
    return model, mu_map, k1, k2


def tfsf_vacuum(n=(24, 22, 26), d=50e-9, nsteps=400):
    """(record model, box, replay builder): the reference's record run (a soft Ex plane
    source, periodic in x and y, CPML in z) and its replay in vacuum with CPML on every face."""
    nx, ny, nz = n
    g = M.Grid(xmin=-(nx - 1) * d / 2, xmax=(nx - 1) * d / 2, Nx=nx, ymin=-(ny - 1) * d / 2, ymax=(ny - 1) * d / 2,
               Ny=ny, zmin=-(nz - 1) * d / 2, zmax=(nz - 1) * d / 2, Nz=nz)
    dt = 0.5 / C0 / np.sqrt(3 / d ** 2)
    src = M.SoftSource(geometry=lambda x, y, z: np.abs(z + 450e-9) < 26e-9,
                       waveform=lambda x, y, z, t: _pulse(t, 1e-6, 4e-15), component="Ex")
    rec = M.Model(g, src, tmax=(nsteps - 0.5) * dt, pml=(0, 0, 0, 0, 150e-9, 150e-9))
    h = 300e-9
    box = (-h, h, -h, h, -h, h)

    def replay(data):
        return M.Model(g, M.TFSFSource(data=data), tmax=(nsteps - 0.5) * dt, pml=150e-9)
    return rec, box, replay


def julia_sum(v):
    """Julia's sum of a vector (Base.mapreduce_impl with pairwise_blocksize 1024, leaf blocks
    added left to right), in the vector's own element type."""
    v = np.asarray(v)
    n = len(v)
    if n <= 1024:
        s = v[0]
        for x in v[1:]:
            s = s + x
        return s
    mid = (n - 1) // 2 + 1
    return julia_sum(v[:mid]) + julia_sum(v[mid:])
