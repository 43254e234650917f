"""Seeded synthetic marine OBS models shaped like the reference's example
experiments (water layer over a sinusoidal seafloor, a gradient crust with a
checkerboard perturbation, a sediment base and an undulating Moho).

The reference only ever runs on script-generated checkerboards
(run_vel_checkerboard.py:223-330 writes the smesh, the Moho and the sediment
base; :373-420 writes the shot geometry).  This module produces the same kind
of arrays directly, in the layout `read_smesh` returns
(read_tomo2d.f90:8-81): node x positions, seafloor depth, depth relative to
the seafloor, and velocity(ix, iz_rel).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class SmeshModel:
    xpos: np.ndarray          # (nx,) km
    topo: np.ndarray          # (nx,) seafloor depth, km
    zrel: np.ndarray          # (nzs,) depth below the seafloor, km
    vel: np.ndarray           # (nzs, nx) km/s; row iz holds depth zrel[iz]
    vwater: float
    sed_z: np.ndarray         # (nx,) sediment base depth, km
    moho_z: np.ndarray        # (nx,) Moho depth, km
    obs_x: np.ndarray         # OBS (source) x positions, km
    picks: np.ndarray = field(default_factory=lambda: np.zeros((0, 4)))
    # picks columns: source index (0-based), phase id (1..5), shot x, shot z
    name: str = ""

    @property
    def nx(self) -> int:
        return int(self.xpos.size)

    @property
    def dx(self) -> float:
        return float(self.xpos[1] - self.xpos[0])

    def pgrid_nz(self) -> int:
        """Propagation-grid rows, invert2d_main.f90:242-246."""
        zmax = self.zrel[-1] + self.topo.max() + 5.0
        return int(np.floor(zmax / self.dx + 0.5)) + 1


def _crust_velocity(zrel, z_abs, moho_abs, lower_crust, x, cb, lc_thick=8.0):
    """1-D gradient (4.5 -> 7.5 km/s over 25 km below the seafloor), optional
    lower crust 6.5 -> 7.2 km/s above the Moho, 8.0 km/s mantle, and a
    sin x sin checkerboard of relative amplitude cb['amp']."""
    v = 4.5 + (7.5 - 4.5) * np.clip(zrel / 25.0, 0.0, 1.0)
    if lower_crust:
        top_lc = moho_abs - lc_thick
        in_lc = (z_abs >= top_lc) & (z_abs < moho_abs)
        frac = np.clip((z_abs - top_lc) / lc_thick, 0.0, 1.0)
        v = np.where(in_lc, 6.5 + 0.7 * frac, v)
        v = np.where(z_abs >= moho_abs, 8.0, v)
    if cb is not None and cb["amp"] > 0:
        pert = np.sin(2 * np.pi * x / (2 * cb["dx"])) * np.sin(2 * np.pi * z_abs / (2 * cb["dz"]))
        v = v * (1.0 + cb["amp"] * pert * (zrel > 0.01))
    return v


def checkerboard_model(nx: int, dx: float, zrel_max: float, nzs: int, *, n_obs: int,
                       obs_spacing: float, shot_spacing: float, lower_crust: bool,
                       moho_base: float = 20.0, moho_amp: float = 1.0,
                       moho_wavelength: float = 40.0, cb_dx: float = 10.0,
                       cb_dz: float = 5.0, cb_amp: float = 0.05, seed: int = 0,
                       max_offset: float = 60.0, phases=(1,), name: str = "",
                       lc_thick: float = 8.0) -> SmeshModel:
    rng = np.random.default_rng(seed)
    x0 = 0.0
    xpos = x0 + dx * np.arange(nx, dtype=np.float64)
    topo = 3.0 + 0.5 * np.sin(2 * np.pi * xpos / 50.0)
    zrel = np.linspace(0.0, zrel_max, nzs)
    moho = moho_base + moho_amp * np.sin(2 * np.pi * xpos / moho_wavelength)
    sed = topo + 1.5 + 0.3 * np.sin(2 * np.pi * xpos / 25.0 + 1.0)
    X, ZR = np.meshgrid(xpos, zrel)                       # (nzs, nx)
    zabs = ZR + topo[None, :]
    vel = _crust_velocity(ZR, zabs, moho[None, :], lower_crust, X,
                          dict(amp=cb_amp, dx=cb_dx, dz=cb_dz), lc_thick)
    xmax = xpos[-1]
    first = 0.5 * (xmax - obs_spacing * (n_obs - 1))
    obs_x = np.round((first + obs_spacing * np.arange(n_obs)) / dx) * dx
    obs_x = np.clip(obs_x, xpos[1], xpos[-2])
    shots = np.arange(0.5, xmax - 0.5 + 1e-9, shot_spacing)
    picks = []
    for s, ox in enumerate(obs_x):
        for ph in phases:
            lo = 0.0 if ph == 1 else 5.0
            for rx in shots:
                off = abs(rx - ox)
                if lo <= off <= max_offset:
                    picks.append((s, ph, rx, 0.005))
    picks = np.array(picks, dtype=np.float64).reshape(-1, 4)
    del rng
    return SmeshModel(xpos=xpos, topo=topo, zrel=zrel, vel=vel, vwater=1.5, sed_z=sed,
                      moho_z=moho, obs_x=obs_x, picks=picks, name=name)


def config(k: int, cb_amp: float | None = None) -> SmeshModel:
    """The benchmark configurations (sizes of the reference experiments
    scaled up to the 2001x401 and 4001x601 grids) and small test models.
    cb_amp overrides the checkerboard amplitude (0: the smooth model)."""
    cb = {} if cb_amp is None else {"cb_amp": float(cb_amp)}
    if k == 0:   # 401x121 at 0.25 km, 10 OBS, 200 shots, Pg
        return checkerboard_model(401, 0.25, 21.5, 87, n_obs=10, obs_spacing=10.0,
                                  shot_spacing=0.5, lower_crust=False, seed=0,
                                  phases=(1,), name="pg-401x121", **cb)
    if k == 1:   # 2001x401 at 0.1 km, 30 OBS, 1000 shots, Pg + PmP
        return checkerboard_model(2001, 0.1, 31.5, 127, n_obs=30, obs_spacing=6.5,
                                  shot_spacing=0.2, lower_crust=True, seed=1,
                                  phases=(1, 3), name="pg-pmp-2001x401", **cb)
    if k == 4:   # 4001x601 at 0.1 km, 100 OBS, 4000 shots, all phases
        return checkerboard_model(4001, 0.1, 51.5, 207, n_obs=100, obs_spacing=4.0,
                                  shot_spacing=0.1, lower_crust=True, seed=4,
                                  moho_base=18.0, moho_amp=2.0, cb_dx=20.0, cb_dz=6.0,
                                  phases=(1, 2, 3, 4, 5), name="joint-4001x601", **cb)
    raise ValueError(f"unknown config {k}")


def start_model(k: int) -> SmeshModel:
    """Starting model of the inversion benchmark on configuration k: the
    smooth model (no checkerboard) with a flat Moho at the true Moho's mean
    depth; the true model is config(k)."""
    import dataclasses
    m = config(k, cb_amp=0.0)
    return dataclasses.replace(m, moho_z=np.full_like(m.moho_z, float(m.moho_z.mean())))


def small_model(nx: int = 121, dx: float = 0.25, zrel_max: float = 8.0, nzs: int = 33,
                n_obs: int = 2, seed: int = 7, phases=(1, 3), cb_amp: float = 0.05,
                max_offset: float = 25.0) -> SmeshModel:
    """A few-thousand-node model the oracle solves in milliseconds."""
    return checkerboard_model(nx, dx, zrel_max, nzs, n_obs=n_obs,
                              obs_spacing=(nx - 1) * dx / (n_obs + 1), shot_spacing=0.5,
                              lower_crust=True, moho_base=8.5, moho_amp=0.5,
                              moho_wavelength=15.0, cb_dx=5.0, cb_dz=2.5, cb_amp=cb_amp,
                              seed=seed, phases=phases, max_offset=max_offset, name="small",
                              lc_thick=3.0)


def _grf(rng, nz: int, nx: int, dz: float, dx: float, corr: float) -> np.ndarray:
    """Gaussian random field on an nz x nx grid with a Gaussian correlation of
    length corr (km), unit standard deviation (spectral filtering of white
    noise)."""
    w = rng.standard_normal((nz, nx))
    kz = np.fft.fftfreq(nz, d=dz)[:, None]
    kx = np.fft.fftfreq(nx, d=dx)[None, :]
    filt = np.exp(-(np.pi * corr) ** 2 * (kx * kx + kz * kz))
    f = np.real(np.fft.ifft2(np.fft.fft2(w) * filt))
    s = f.std()
    return f / s if s > 0 else f


def uneven_model(k: int, max_obs: int = 40) -> SmeshModel:
    """Model k of the uneven-size multi-model batch (seed 100 + k): grid sizes
    drawn uniformly from 401x121 to 2001x401 at 0.1 to 0.25 km spacing; a
    random 1-D velocity gradient with a 3 to 8% Gaussian-random-field
    perturbation (correlation length 5 km); a sediment layer 1 to 3 km thick
    below the seafloor at 1.8 to 3.0 km/s; a Moho at 14 to 22 km; 10 to
    max_obs OBS.  Every phase can be traced (water, sediment and Moho are all
    present)."""
    rng = np.random.default_rng(100 + k)
    dx = float(rng.uniform(0.1, 0.25))
    nx = int(rng.integers(401, 2002))
    nz_target = int(rng.integers(121, 402))
    topo_mean = float(rng.uniform(2.0, 3.5))
    xpos = dx * np.arange(nx, dtype=np.float64)
    topo = topo_mean + 0.5 * np.sin(2 * np.pi * xpos / float(rng.uniform(30.0, 80.0)))
    zmax = (nz_target - 1) * dx
    zrel_max = max(8.0, zmax - topo.max() - 5.0)
    nzs = max(16, int(zrel_max / 0.25) + 1)
    zrel = np.linspace(0.0, zrel_max, nzs)
    X, ZR = np.meshgrid(xpos, zrel)
    sed_th = float(rng.uniform(1.0, 3.0))
    v_sed = float(rng.uniform(1.8, 3.0))
    v0, grad = float(rng.uniform(4.2, 5.2)), float(rng.uniform(0.08, 0.14))
    vel = np.minimum(v0 + grad * ZR, 7.6)
    amp = float(rng.uniform(0.03, 0.08))
    vel = vel * (1.0 + amp * np.clip(_grf(rng, nzs, nx, zrel[1] - zrel[0], dx, 5.0), -3, 3) / 3)
    vel = np.where(ZR < sed_th, v_sed + (ZR / sed_th) * 0.3, vel)
    moho_base = min(float(rng.uniform(14.0, 22.0)), topo.max() + zrel_max - 2.0)
    moho = moho_base + float(rng.uniform(0.3, 1.5)) * np.sin(2 * np.pi * xpos / 40.0)
    zabs = ZR + topo[None, :]
    vel = np.where(zabs >= moho[None, :], 8.0, vel)
    sed = topo + sed_th
    n_obs = int(rng.integers(10, max_obs + 1))
    width = xpos[-1]
    obs_x = np.round(np.linspace(0.05 * width, 0.95 * width, n_obs) / dx) * dx
    obs_x = np.clip(obs_x, xpos[1], xpos[-2])
    return SmeshModel(xpos=xpos, topo=topo, zrel=zrel, vel=vel, vwater=1.5, sed_z=sed,
                      moho_z=moho, obs_x=obs_x, name=f"uneven-{k}")
