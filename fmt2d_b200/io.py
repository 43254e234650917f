"""The reference's files for this library: readers of its input files
(read_tomo2d.f90; fmt2d_read_smesh / fmt2d_read_refl / fmt2d_read_geom,
Fortran list-directed rules), writers of the same formats, `model_from_files`,
which turns a velocity mesh, the sediment-base and Moho files and a geometry
file into the model descriptor and picks that `Fmt2d.upload` /
`Fmt2d.forward` / `Fmt2d.trace` take, and writers of the inversion's output
files (write_model2d's smesh / refl / model_iter files, write_residuals2d)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .synth import SmeshModel


def _err(rc: int, what: str):
    if rc != 0:
        buf = C.create_string_buffer(512)
        N.lib().fmt2d_io_last_error(buf, 512)
        raise N.Fmt2dError(f"{what} failed ({rc}): {buf.value.decode()}")


def read_smesh(path: str) -> dict:
    """read_smesh (read_tomo2d.f90:8-81): xpos, topo, zpos_rel and vel as
    (nz, nx) (row iz at depth zpos_rel[iz] below the seafloor)."""
    L = N.lib()
    nx, nz, vw, va = C.c_int(), C.c_int(), C.c_double(), C.c_double()
    p = str(path).encode()
    _err(L.fmt2d_read_smesh(p, C.byref(nx), C.byref(nz), C.byref(vw), C.byref(va), None, None,
                            None, None), "fmt2d_read_smesh")
    x, t, z = np.zeros(nx.value), np.zeros(nx.value), np.zeros(nz.value)
    v = np.zeros(nx.value * nz.value)
    _err(L.fmt2d_read_smesh(p, C.byref(nx), C.byref(nz), C.byref(vw), C.byref(va), N.ptr(x),
                            N.ptr(t), N.ptr(z), N.ptr(v)), "fmt2d_read_smesh")
    return dict(xpos=x, topo=t, zrel=z, vel=v.reshape(nz.value, nx.value), vwater=vw.value,
                vair=va.value)


def read_refl(path: str):
    """read_refl (read_tomo2d.f90:83-139): the (x, z) nodes of an interface."""
    L = N.lib()
    n = C.c_int()
    p = str(path).encode()
    _err(L.fmt2d_read_refl(p, C.byref(n), None, None), "fmt2d_read_refl")
    x, z = np.zeros(n.value), np.zeros(n.value)
    _err(L.fmt2d_read_refl(p, C.byref(n), N.ptr(x), N.ptr(z)), "fmt2d_read_refl")
    return x, z


def read_geom(path: str) -> dict:
    """read_geom (read_tomo2d.f90:141-248): OBS positions and, per receiver
    (shot), its position, 1-based OBS id, phase, observed time and
    uncertainty."""
    L = N.lib()
    no, nr = C.c_int(), C.c_int()
    p = str(path).encode()
    _err(L.fmt2d_read_geom(p, C.byref(no), C.byref(nr), *([None] * 8)), "fmt2d_read_geom")
    ox, oz = np.zeros(no.value), np.zeros(no.value)
    rx, rz, to, un = (np.zeros(nr.value) for _ in range(4))
    oid, ph = np.zeros(nr.value, np.int32), np.zeros(nr.value, np.int32)
    _err(L.fmt2d_read_geom(p, C.byref(no), C.byref(nr), N.ptr(ox), N.ptr(oz), N.ptr(rx),
                           N.ptr(rz), N.ptr(oid), N.ptr(ph), N.ptr(to), N.ptr(un)),
         "fmt2d_read_geom")
    return dict(obs_x=ox, obs_z=oz, rec_x=rx, rec_z=rz, obs_id=oid, phase=ph, t_obs=to, unc=un)


def write_smesh(path: str, xpos, topo, zrel, vel, vwater: float, vair: float = 0.33):
    """A velocity mesh in read_smesh's format; vel is (nz, nx)."""
    vel = np.asarray(vel, dtype=np.float64)
    with open(path, "w") as f:
        f.write(f"{len(xpos)} {len(zrel)} {float(vwater)!r} {float(vair)!r}\n")
        for a in (xpos, topo, zrel):
            f.write(" ".join(repr(float(v)) for v in a) + "\n")
        for ix in range(vel.shape[1]):
            f.write(" ".join(repr(float(v)) for v in vel[:, ix]) + "\n")


def write_refl(path: str, x, z):
    """An interface in read_refl's format."""
    with open(path, "w") as f:
        for a, b in zip(x, z):
            f.write(f"{float(a)!r} {float(b)!r}\n")


def write_geom(path: str, obs_x, obs_z, picks, t_obs=None, unc=None):
    """Shot geometry and picks in read_geom's format; picks columns: source
    index (0-based), phase, shot x, shot z (a negative t_obs marks a pick
    without an observation)."""
    picks = np.asarray(picks, dtype=np.float64).reshape(-1, 4)
    t_obs = np.full(len(picks), -1.0) if t_obs is None else np.asarray(t_obs, dtype=np.float64)
    unc = np.full(len(picks), 0.05) if unc is None else np.asarray(unc, dtype=np.float64)
    with open(path, "w") as f:
        f.write(f"{len(obs_x)}\n")
        for s, (ox, oz) in enumerate(zip(obs_x, obs_z)):
            k = np.where(picks[:, 0] == s)[0]
            f.write(f"s {float(ox)!r} {float(oz)!r} {len(k)}\n")
            for i in k:
                f.write(f"r {float(picks[i, 2])!r} {float(picks[i, 3])!r} {int(picks[i, 1])} "
                        f"{float(t_obs[i])!r} {float(unc[i])!r}\n")


def iface_on_grid(x_nodes, z_nodes, xpos) -> np.ndarray:
    """Depths of an interface at the grid's x: linear between its nodes,
    clamped at its ends, with the node spacing x(2) - x(1) as
    interpolate_iface_z_inv reads it (src/inversion2d.f90)."""
    xn, zn = np.asarray(x_nodes, dtype=np.float64), np.asarray(z_nodes, dtype=np.float64)
    out = np.empty(len(xpos))
    if xn.size < 2:
        out[:] = zn[0]
        return out
    dx = xn[1] - xn[0]
    for k, px in enumerate(np.asarray(xpos, dtype=np.float64)):
        i = int(np.floor((px - xn[0]) / dx)) + 1
        if i < 1:
            out[k] = zn[0]
        elif i >= xn.size:
            out[k] = zn[-1]
        else:
            w = min(1.0, max(0.0, (px - xn[i - 1]) / dx))
            out[k] = (1.0 - w) * zn[i - 1] + w * zn[i]
    return out


def model_from_files(smesh: str, sed: str, moho: str, geom: str | None = None,
                     name: str = "") -> tuple[SmeshModel, dict | None]:
    """The model descriptor (and picks) from the reference's input files:
    the velocity mesh, the sediment base and the Moho (each interpolated onto
    the mesh's x) and, optionally, the geometry file (picks = OBS index,
    phase, shot x, shot z; the geometry dict carries t_obs and uncertainty)."""
    sm = read_smesh(smesh)
    xs, zs = read_refl(sed)
    xm, zm = read_refl(moho)
    g = read_geom(geom) if geom else None
    obs_x = g["obs_x"] if g else np.zeros(0)
    picks = (np.stack([g["obs_id"] - 1, g["phase"], g["rec_x"], g["rec_z"]], axis=1)
             .astype(np.float64) if g else np.zeros((0, 4)))
    m = SmeshModel(xpos=sm["xpos"], topo=sm["topo"], zrel=sm["zrel"], vel=sm["vel"],
                   vwater=sm["vwater"], sed_z=iface_on_grid(xs, zs, sm["xpos"]),
                   moho_z=iface_on_grid(xm, zm, sm["xpos"]), obs_x=obs_x, picks=picks, name=name)
    return m, g


# ---------------------------------------------------------------- output files
def _rows(values, per_line: int, fmt: str) -> str:
    """Fortran '(nFw.d)' output: per_line values a record."""
    v = list(values)
    return "".join("".join(format(x, fmt) for x in v[i:i + per_line]) + "\n"
                   for i in range(0, len(v), per_line)) if v else "\n"


def smesh_from_grid(xpos, seafloor, zrel, zgrid, vel_grid, active):
    """The velocity of the inversion grid sampled back onto the smesh layout
    (depth zrel below the seafloor), write_model2d's rule
    (src/inversion2d.f90:3866-3901): at z = seafloor + zrel, linear between
    the bracketing grid rows, taking the lower row alone when the upper one is
    inactive or slower than 2 km/s (no interpolation across the seafloor);
    clamped to the first / last row outside the grid.  vel_grid, active:
    (nz, nx).  Returns (nzs, nx)."""
    xpos = np.asarray(xpos, dtype=np.float64)
    zrel = np.asarray(zrel, dtype=np.float64)
    zg = np.asarray(zgrid, dtype=np.float64)
    V = np.asarray(vel_grid, dtype=np.float64)
    A = np.asarray(active, dtype=bool)
    nz = zg.size
    out = np.zeros((zrel.size, xpos.size))
    for ix in range(xpos.size):
        for iz, zr in enumerate(zrel):
            z = seafloor[ix] + zr
            lo, hi = 0, nz - 1
            for k in range(nz - 1):
                if zg[k] <= z <= zg[k + 1]:
                    lo, hi = k, k + 1
                    break
            if z <= zg[0]:
                v = V[0, ix]
            elif z >= zg[nz - 1]:
                v = V[nz - 1, ix]
            else:
                w = (z - zg[lo]) / (zg[hi] - zg[lo])
                if A[lo, ix] and V[lo, ix] >= 2.0:
                    v = (1.0 - w) * V[lo, ix] + w * V[hi, ix]
                else:
                    v = V[hi, ix]
            out[iz, ix] = v
    return out


def write_model(directory: str, g, iteration: int, zrel, vwater: float, vair: float = 0.33):
    """write_model2d (src/inversion2d.f90:3842-3962) for a context's current
    model: vgrid_1_vtype1.smesh (the velocity back on the input smesh's
    relative depths), iface_<k>.refl of the inverted interface, and
    model_iter<iteration>.dat (the grid velocity by column and the interface
    depths).  These files restart an inversion (`model_from_files`)."""
    import os
    inv, nvp, npar = g.inv_index()
    vel = g.velocity()                         # (nz, nx)
    nz, nx = vel.shape
    xpos = np.asarray(g.model.xpos, dtype=np.float64)
    seafloor = g.interface(2)
    zgrid = np.arange(nz) * g.dx
    zrel = np.asarray(zrel, dtype=np.float64)
    sm = smesh_from_grid(xpos, seafloor, zrel, zgrid, vel, inv > 0)
    with open(os.path.join(directory, "vgrid_1_vtype1.smesh"), "w") as f:
        f.write(f"{nx:6d}{zrel.size:6d}{vwater:10.3f}{vair:10.3f}\n")
        f.write(_rows(xpos, 10, "12.4f"))
        f.write(_rows(seafloor, 10, "12.4f"))
        f.write(_rows(zrel, 10, "12.4f"))
        for ix in range(nx):
            f.write("".join(format(v, "10.4f") for v in sm[:, ix]) + "\n")
    k = int(getattr(g, "iface_inv", 4))
    zi = g.interface(k) if npar > nvp else None
    if zi is not None:
        with open(os.path.join(directory, f"iface_{k}.refl"), "w") as f:
            for x, z in zip(xpos, zi):
                f.write(f"{x:12.3f}{z:12.3f}\n")
    with open(os.path.join(directory, f"model_iter{int(iteration)}.dat"), "w") as f:
        f.write(f"Iteration {int(iteration)}\n")
        f.write("vgrid 1 vtype 1\n")
        for ix in range(nx):
            f.write(_rows(vel[:, ix], 10, "10.4f"))
        if zi is not None:
            f.write(f"iface {k}\n")
            f.write(_rows(zi, 10, "12.4f"))


def write_residuals(path: str, src, rcv_x, rcv_z, phase, obs, t_calc, valid):
    """write_residuals2d (src/inversion2d.f90:3342-3377): one line per valid
    pick with an observation (src_id is 1-based, as the reference numbers its
    sources)."""
    keep = np.asarray(valid, dtype=bool) & (np.asarray(obs) >= 0.0)
    with open(path, "w") as f:
        f.write("# src_id  rcv_x  rcv_z  phase_id  obs_time  calc_time  residual\n")
        for i in np.flatnonzero(keep):
            o, c = float(obs[i]), float(t_calc[i])
            f.write(f"{int(src[i]) + 1:6d}{float(rcv_x[i]):12.3f}{float(rcv_z[i]):10.3f}"
                    f"{int(phase[i]):4d}{o:12.6f}{c:12.6f}{_es14_6(o - c)}\n")
    return int(keep.sum())


def _es14_6(x: float) -> str:
    """Fortran ES14.6: d.dddddde+xx right-justified in 14 columns."""
    m, e = f"{x:.6e}".split("e")
    return f"{m}E{int(e):+03d}".rjust(14)


def write_arrivals(arrivals_path: str, obs_path: str, entry_path: str, ircv, src, phase,
                   t_calc, valid, water_time, entry_x, entry_z):
    """write_arrivals2d (fmt2d_main.f90:1655-1719): the arrivals file (every
    ray: receiver, source, phase, arrival time, time without the water leg,
    water time; -1 for an invalid ray), the observed-times file (the valid
    rays, their count first) and entry_points.dat (the valid rays' seafloor
    entry points and water times, their count first).  Receivers and sources
    are written 1-based; ircv is the pick's receiver (shot) index, 0-based.
    The reference writes one entry point per receiver and phase (the last
    source's); this writes each ray's own."""
    valid = np.asarray(valid, dtype=bool)
    n = int(valid.sum())
    with open(arrivals_path, "w") as fa, open(obs_path, "w") as fo, open(entry_path, "w") as fe:
        fo.write(f"{n}\n")
        fe.write(f"{n}\n")
        for i in range(len(valid)):
            head = f"{int(ircv[i]) + 1:8d}{int(src[i]) + 1:8d}{int(phase[i]):8d}"
            w = float(water_time[i])
            if valid[i]:
                t = float(t_calc[i])
                fa.write(f"{head}{t:15.6f}{t - w:15.6f}{w:12.6f}\n")
                fo.write(f"{head}{t:15.6f}\n")
                fe.write(f"{head}{float(entry_x[i]):15.6f}{float(entry_z[i]):15.6f}{w:12.6f}\n")
            else:
                fa.write(f"{head}{-1.0:15.6f}{-1.0:15.6f}{w:12.6f}\n")
    return n
