"""One outer iteration of FMT2D's joint velocity + interface inversion on the
device path: the loop body of lsqr_inversion2d (src/inversion2d.f90:256-937).

Per iteration:

1. the alternating mode (:261-277: joint, velocity only, interface only, or
   every 4th iteration interface-only under the automatic schedule);
2. the forward (every source's time fields, fmt2d_forward), the ray
   backtrace and Frechet rows of every pick (fmt2d_trace, run_forward2d
   :4145-4545);
3. the pick selection, residuals, phase weights and column scaling with the
   parameters the mode fixes scaled to zero (fmt2d_select_data,
   read_frechet_data2d :3965-4052 and :334-379);
4. gtg, eps_min = max(1e-6, 1e-4 max gtg) (:466-486), the Gaussian smoothing
   matrices for smooth_type 2 and 3 (:516-522), and the damping choice over
   the device LSQR (fixed damping or tomo2d's auto damping, :533-739), the
   LSQR's right-hand side jumping to the accumulated model change;
5. the update: masked columns and fixed parameters zeroed, the velocity part
   capped at max_rel_pert (:743-773);
6. the line search (:829-868): step lengths 1, 0.75, 0.5, 0.25, 0.125,
   0.0625 from the one accepted last time, each a model step
   (apply_model_step :7173-7237, fmt2d_update_model) and a forward with the
   ray backtrace, until the RMS residual drops below the iteration's starting
   RMS; the best step is kept (or the model restored) and added to the
   accumulated change (:870-903).

Everything that touches a field, a ray or the LSQR runs in the CUDA library;
the host does the O(nparm) vector arithmetic of steps 5 and 6 with numpy.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from .api import Fmt2d, select_data

LADDER = (1.0, 0.75, 0.5, 0.25, 0.125, 0.0625)   # inversion2d.f90:839-851


@dataclass
class InversionParams:
    """The arguments of lsqr_inversion2d that shape one iteration
    (src/inversion2d.f90:112-117), with the reference's defaults where it
    has them."""
    phases: tuple = (1, 3)
    lam_damp: float = 0.0            # > 0: fixed damping, else auto damping
    lam_damp_iface: float = 0.0
    lam_smooth: float = 10.0
    lam_smooth_iface: float = 10.0
    smooth_type: int = 1             # 1 Laplacian, 2 Gaussian, 3 hybrid
    corr_x: float = 0.0              # Gaussian correlation lengths (km)
    corr_z: float = 0.0
    corr_x_iface: float = 0.0
    crit_chi: float = 1.0            # inv_crit_chi (s)
    lsqr_max_iter: int = 2000
    target_dv: float = 0.03          # auto damping targets (:495-499)
    target_dd: float = 0.5
    refl_weight: float = 1.0         # column scaling of interface parameters
    wt_psed: float = 1.0
    wt_pmp: float = 1.0
    wt_pgss: float = 1.0
    iface_step_ratio: float = 1.0
    max_rel_pert: float = 0.3
    alt_inv_mode: int = -1           # -1 automatic, 0 joint, 1 velocity, 2 interface


@dataclass
class IterationResult:
    iteration: int
    mode: int
    ndata: int
    rms_orig: float
    rms_new: float
    step: float
    wdv: float
    wdv_iface: float
    avg_dmv: float
    avg_dmd: float
    lsqr_solves: int
    forwards: int
    seconds: float
    phases_s: dict = field(default_factory=dict)


class Inversion:
    """State of an inversion on one context: the sources, the picks with their
    observed times, the initial velocity (the reference of the column scaling
    and of the 70-130% velocity bounds), the accumulated model change and the
    line-search ladder position.

    picks: (npick, 4) array of (source index, phase 1..5, receiver x, z) as in
    synth.SmeshModel.picks; obs: observed times (s), < 0 for none."""

    def __init__(self, g: Fmt2d, src_x, picks, obs, params: InversionParams | None = None):
        self.g = g
        self.p = params or InversionParams()
        self.src_x = np.ascontiguousarray(src_x, dtype=np.float64)
        P = np.asarray(picks, dtype=np.float64)
        self.src = np.ascontiguousarray(P[:, 0], dtype=np.int32)
        self.phase = np.ascontiguousarray(P[:, 1], dtype=np.int32)
        self.rx = np.ascontiguousarray(P[:, 2])
        self.rz = np.ascontiguousarray(P[:, 3])
        self.obs = np.ascontiguousarray(obs, dtype=np.float64)
        if self.obs.size != self.src.size:
            raise ValueError("one observed time per pick")
        self.inv, self.nvp, self.npar = g.inv_index()
        self.v_init = g.velocity().copy()
        self.vel_nodes = self.inv > 0                      # (nz, nx)
        self.vel_ids = self.inv[self.vel_nodes] - 1        # parameter of each such node
        self.n_iface = self.npar - self.nvp
        mv = np.ones(self.npar)
        mv[self.vel_ids] = 1.0 / np.maximum(self.v_init[self.vel_nodes], 1.0)   # :185-194
        mv[self.nvp:] = self.p.refl_weight                                        # :195-204
        self.mvscale = mv
        self.dm_sum = np.zeros(self.npar)
        self.ls_prev = 0
        self.iter = 0
        self.forwards = 0
        self.iface = getattr(g, "iface_inv", 4)

    # ---------------------------------------------------------------- pieces
    def _mode(self) -> int:
        if self.n_iface <= 0:
            return 0
        if self.p.alt_inv_mode == -1:
            return 2 if self.iter % 4 == 0 else 1
        return self.p.alt_inv_mode

    def forward_and_trace(self, rows: bool = True):
        """Forward of every source and the ray backtrace of every pick on the
        current model (with the Frechet rows, or times only for the line
        search); returns (t_calc, valid)."""
        self.g.forward(self.src_x, self.p.phases)
        if rows:
            t, valid, _ = self.g.trace(self.src, self.phase, self.rx, self.rz)
        else:
            t, valid = self.g.trace_times(self.src, self.phase, self.rx, self.rz)
        self.forwards += 1
        return t, valid

    def rms(self, t, valid) -> float:
        """RMS residual over the valid picks with an observation within
        crit_chi (compute_rms_after_forward, src/inversion2d.f90:3298-3339)."""
        r = self.obs - t
        keep = valid & (self.obs >= 0.0) & (np.abs(r) <= self.p.crit_chi)
        n = int(keep.sum())
        return float(np.sqrt(np.sum(r[keep] ** 2) / n)) if n else 1.0e20

    def apply_step(self, vel0, z0, dm, step, step_iface):
        """apply_model_step (src/inversion2d.f90:7173-7237) from the saved
        model (vel0, z0): slowness + step * mvscale * dm, bounded to 2..10
        km/s and to 70-130% of the initial velocity; interface depth +
        step_iface * mvscale * dm, each node's move capped at 0.5 km."""
        vel = vel0.copy()
        if step > 0.0:
            cur = vel0[self.vel_nodes]
            trial_s = 1.0 / cur + step * self.mvscale[self.vel_ids] * dm[self.vel_ids]
            safe = np.where(trial_s > 0.0, trial_s, 1.0)
            tv = np.where(trial_s > 0.0, 1.0 / safe, 2.0)
            tv = np.clip(tv, 2.0, 10.0)
            init = self.v_init[self.vel_nodes]
            bounded = init >= 2.0
            tv = np.where(bounded & (tv > init * 1.30), init * 1.30, tv)
            tv = np.where(bounded & (tv < init * 0.70), init * 0.70, tv)
            vel[self.vel_nodes] = tv
        z = None                                  # the saved interface, restored
        if self.n_iface > 0 and z0 is not None:
            z = z0.copy()
            if step_iface > 0.0:
                z = z0 + np.clip(step_iface * self.mvscale[self.nvp:] * dm[self.nvp:], -0.5, 0.5)
        self.g.update_model(vel=vel, iface_z=z)

    # ---------------------------------------------------------------- iteration
    def iteration(self) -> IterationResult:
        """One outer iteration (src/inversion2d.f90:256-937)."""
        p, g = self.p, self.g
        self.iter += 1
        mode = self._mode()
        t0 = time.perf_counter()
        ph = {}
        f0 = self.forwards
        # forward, rays and Frechet rows
        t, valid = self.forward_and_trace()
        rp, gi, gv = g.frechet_rows()
        ph["forward_trace"] = time.perf_counter() - t0
        # selection, weights, column scaling with the fixed parameters at 0
        mv = self.mvscale.copy()
        if mode == 1:
            mv[self.nvp:] = 0.0
        elif mode == 2:
            mv[:self.nvp] = 0.0
        srp, sgi, sgv, res, wt, pick = select_data(
            self.phase, self.obs, t, valid.astype(np.int32), rp, gi, gv, mv,
            crit_chi=p.crit_chi, wt_psed=p.wt_psed, wt_pmp=p.wt_pmp, wt_pgss=p.wt_pgss)
        nd = srp.size - 1
        if nd == 0:
            raise RuntimeError(f"iteration {self.iter}: no valid data")
        r_raw = self.obs[pick] - t[pick]
        rms_orig = float(np.sqrt(np.sum(r_raw * r_raw) / nd))      # compute_rms2d
        t1 = time.perf_counter()
        g.set_frechet(nd, self.npar, srp, sgi, sgv)
        gtg = g.gtg_diag()
        eps_min = max(1.0e-6, 1.0e-4 * float(gtg.max()))
        if p.smooth_type in (2, 3):
            g.set_smoothing(mv, p.corr_x if p.smooth_type == 2 else 0.0,
                            p.corr_z if p.smooth_type == 2 else 0.0, p.corr_x_iface)
        dres = g.lsqr_damped(res, self.dm_sum, gtg, mv, lam_damp=p.lam_damp,
                             lam_damp_iface=p.lam_damp_iface, target_dv=p.target_dv,
                             target_dd=p.target_dd, w_smooth=p.lam_smooth,
                             w_smooth_iface=p.lam_smooth_iface, eps_min=eps_min,
                             max_iter=min(p.lsqr_max_iter, 2000), smooth_type=p.smooth_type)
        ph["lsqr"] = time.perf_counter() - t1
        # the update: masked columns and fixed parameters zeroed, velocity cap
        dm = dres.dm.copy()
        dm[:self.nvp][gtg[:self.nvp] < eps_min * 0.01] = 0.0
        if mode == 1:
            dm[self.nvp:] = 0.0
        elif mode == 2:
            dm[:self.nvp] = 0.0
        dv = dm[:self.nvp]
        dm[:self.nvp] = np.where(np.abs(dv) > p.max_rel_pert,
                                 np.copysign(p.max_rel_pert, dv), dv)
        # line search from the step accepted last time
        t2 = time.perf_counter()
        vel0 = g.velocity().copy()
        z0 = g.interface(self.iface).copy() if self.n_iface > 0 else None
        rms_best, step_len, ok = rms_orig, 0.0, self.ls_prev
        for k in range(self.ls_prev, len(LADDER)):
            s = LADDER[k]
            self.apply_step(vel0, z0, dm, s, s * p.iface_step_ratio)
            rms_try = self.rms(*self.forward_and_trace(rows=False))
            if rms_try < rms_best:
                rms_best, step_len, ok = rms_try, s, k
            if rms_try < rms_orig:
                break
        if step_len > 0.0:
            self.ls_prev = ok
            if step_len != LADDER[k]:      # the last model tried is not the best
                self.apply_step(vel0, z0, dm, step_len, step_len * p.iface_step_ratio)
            rms_new = rms_best
        else:
            g.update_model(vel=vel0, iface_z=z0)
            rms_new = rms_orig
        ph["line_search"] = time.perf_counter() - t2
        step_iface = step_len * p.iface_step_ratio if self.n_iface > 0 else 0.0
        scaled = dm.copy()
        scaled[:self.nvp] *= step_len
        scaled[self.nvp:] *= step_iface
        self.dm_sum += scaled
        return IterationResult(
            iteration=self.iter, mode=mode, ndata=nd, rms_orig=rms_orig, rms_new=rms_new,
            step=step_len, wdv=dres.wdv, wdv_iface=dres.wdv_iface, avg_dmv=dres.avg_dmv,
            avg_dmd=dres.avg_dmd,
            lsqr_solves=len(dres.solves), forwards=self.forwards - f0,
            seconds=time.perf_counter() - t0, phases_s=ph)
