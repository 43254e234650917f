"""Damping choice around LSQR: the call pattern of lsqr_inversion2d
(src/inversion2d.f90:533-739), host control flow over a solver that returns
the model update for given velocity and interface damping weights.

With a fixed damping weight it is one solve.  Otherwise (tomo2d's auto
damping) it solves without damping, then searches the interface damping
weight and then the velocity damping weight with the reference's
secant/bisection iteration until the RMS model change is within 30% of its
target, and finishes with one solve at the chosen weights: at most
1 + 12 + 12 + 1 solves.

`Fmt2d.lsqr_damped` runs it on the device LSQR (fmt2d_lsqr); any other
solver with the same meaning can be passed to `damping_search`.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable

import numpy as np


def avg_dmv(dm, gtg_diag, eps_min: float, n_vel_parms: int) -> float:
    """RMS of the velocity part of dm over the columns the data constrain
    (gtg >= 0.01 eps_min); calc_avg_dmv, src/inversion2d.f90:6523-6543."""
    dm = np.asarray(dm, dtype=np.float64)[:n_vel_parms]
    act = np.asarray(gtg_diag, dtype=np.float64)[:n_vel_parms] >= eps_min * 0.01
    n = int(act.sum())
    return float(np.sqrt(np.sum(dm[act] ** 2) / n)) if n else 0.0


def avg_dmd(dm, mvscale, n_vel_parms: int) -> float:
    """RMS depth change of the interface parameters (mvscale * dm);
    calc_avg_dmd, src/inversion2d.f90:6549-6567."""
    dz = (np.asarray(mvscale, dtype=np.float64)[n_vel_parms:]
          * np.asarray(dm, dtype=np.float64)[n_vel_parms:])
    return float(np.sqrt(np.sum(dz ** 2) / dz.size)) if dz.size else 0.0


@dataclass
class DampingResult:
    dm: np.ndarray            # model update of the final solve
    wdv: float                # velocity damping weight used
    wdv_iface: float          # interface damping weight used
    avg_dmv: float            # RMS velocity change of dm + dm_sum
    avg_dmd: float            # RMS depth change of dm + dm_sum
    solves: list              # (wdv, wdv_iface) of every solve, in order


def _secant(f: Callable[[float], float], target: float) -> float:
    """The reference's secant/bisection search on f(w) = avg(w) - target
    (src/inversion2d.f90:575-637 and :652-715): start from w = 1 and 100,
    keep the point with the smaller |f| as the iterate, step by the secant,
    halve towards 0 or 1e7 when the step leaves (0, 1e7], at most 10 steps,
    stop above 1e7 or once |f| < 0.3 target."""
    ddm = target * 0.3
    wd1, wd2 = np.float64(1.0), np.float64(100.0)
    fl = np.float64(f(float(wd1)))
    f_val = np.float64(f(float(wd2)))
    if abs(fl) < abs(f_val):
        wd_rts, wd_xl = wd1, wd2
        fl, f_val = f_val, fl
    else:
        wd_xl, wd_rts = wd1, wd2
    with np.errstate(divide="ignore", invalid="ignore"):
        for _ in range(10):
            dx = (wd_xl - wd_rts) * f_val / (f_val - fl)
            if wd_rts + dx <= 0.0:
                wd_xl, fl = wd_rts, f_val
                wd_rts = wd_rts * 0.5
            elif wd_rts + dx > 1.0e7:
                wd_xl, fl = wd_rts, f_val
                wd_rts = wd_rts + (1.0e7 - wd_rts) * 0.5
            else:
                wd_xl, fl = wd_rts, f_val
                wd_rts = wd_rts + dx
            f_val = np.float64(f(float(wd_rts)))
            if wd_rts > 1.0e7 or abs(f_val) < ddm:
                break
    return float(wd_rts)


def damping_search(solve: Callable[[float, float], np.ndarray], dm_sum, gtg_diag, mvscale,
                   eps_min: float, n_vel_parms: int, *, lam_damp: float = 0.0,
                   lam_damp_iface: float = 0.0, target_dv: float = 0.0,
                   target_dd: float = 0.0) -> DampingResult:
    """Choose the damping weights and solve (src/inversion2d.f90:533-739).

    solve(wdv, wdv_iface) returns the model update dm (nparm) of run_lsqr
    with those damping weights and the caller's smoothing; dm_sum is the
    model change accumulated by earlier outer iterations, gtg_diag the column
    norms of G, mvscale the column scaling, n_vel_parms the number of velocity
    parameters (the rest are interface parameters).  lam_damp > 0 fixes the
    velocity weight (and the interface weight: lam_damp_iface if > 0, else
    lam_damp); otherwise target_dv (fraction) and target_dd (km) are the RMS
    changes the auto damping aims for."""
    dm_sum = np.zeros_like(np.asarray(gtg_diag, dtype=np.float64)) if dm_sum is None \
        else np.asarray(dm_sum, dtype=np.float64)
    nparm = dm_sum.size
    n_iface = nparm - n_vel_parms
    solves = []

    def run(wdv: float, wdi: float) -> np.ndarray:
        solves.append((float(wdv), float(wdi)))
        return np.asarray(solve(float(wdv), float(wdi)), dtype=np.float64)

    def avgs(dm):
        t = dm + dm_sum
        return (avg_dmv(t, gtg_diag, eps_min, n_vel_parms),
                avg_dmd(t, mvscale, n_vel_parms) if n_iface > 0 else 0.0)

    if lam_damp > 0.0:
        wdi = lam_damp_iface if (n_iface > 0 and lam_damp_iface > 0.0) else lam_damp
        dm = run(lam_damp, wdi)
        v, d = avgs(dm)
        return DampingResult(dm, float(lam_damp), float(wdi), v, d, solves)

    # step 1: no damping
    dm = run(0.0, 0.0)
    v0, d0 = avgs(dm)
    # step 2: interface damping (velocity weight 0 meanwhile)
    wd_iface = 0.0
    if n_iface > 0 and d0 > target_dd:
        wd_iface = _secant(lambda w: avgs(run(0.0, w))[1] - target_dd, target_dd)
    # step 3: velocity damping at the chosen interface weight
    wd = 0.0
    if v0 > target_dv:
        wd = _secant(lambda w: avgs(run(w, wd_iface))[0] - target_dv, target_dv)
    dm = run(wd, wd_iface)
    v, d = avgs(dm)
    return DampingResult(dm, wd, wd_iface, v, d, solves)
