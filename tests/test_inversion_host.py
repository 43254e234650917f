"""Host pieces of the inversion iteration (fmt2d_b200/inversion.py), CPU:
the model step against a loop restatement of apply_model_step
(src/inversion2d.f90:7173-7237), the RMS rule of compute_rms_after_forward
(:3298-3339) and the alternating schedule (:261-277)."""
import numpy as np

from fmt2d_b200 import synth
from fmt2d_b200.api import Fmt2d
from fmt2d_b200.inversion import Inversion, InversionParams


def _inv(params=None):
    m = synth.small_model()
    g = Fmt2d(-1).upload(m)
    obs = np.full(m.picks.shape[0], 1.0)
    return m, g, Inversion(g, m.obs_x, m.picks, obs, params)


def _loop_step(inv, vel0, z0, dm, step, step_iface):
    vel = vel0.copy()
    nz, nx = vel.shape
    for iz in range(nz):
        for ix in range(nx):
            idx = inv.inv[iz, ix]
            if idx <= 0 or step <= 0.0:
                continue
            cur = 1.0 / vel0[iz, ix]
            ts = cur + step * inv.mvscale[idx - 1] * dm[idx - 1]
            tv = 2.0
            if ts > 0.0:
                tv = 1.0 / ts
            tv = min(max(tv, 2.0), 10.0)
            v0 = inv.v_init[iz, ix]
            if v0 >= 2.0:
                tv = min(tv, v0 * 1.30)
                tv = max(tv, v0 * 0.70)
            vel[iz, ix] = tv
    z = z0.copy()
    if step_iface > 0.0:
        for ix in range(nx):
            idx = inv.nvp + ix
            dz = step_iface * inv.mvscale[idx] * dm[idx]
            z[ix] += min(max(dz, -0.5), 0.5)
    return vel, z


def test_model_step_matches_loop():
    m, g, inv = _inv(InversionParams(refl_weight=0.8))
    rng = np.random.default_rng(3)
    dm = rng.normal(0.0, 0.05, inv.npar)
    dm[inv.nvp:] = rng.normal(0.0, 0.6, inv.npar - inv.nvp)
    dm[:5] = [-2.0, 2.0, 5.0, -5.0, 0.4]          # bounds and the negative-slowness branch
    vel0, z0 = g.velocity().copy(), g.interface(4).copy()
    for step, si in ((1.0, 1.0), (0.25, 0.5), (0.0, 1.0), (0.5, 0.0)):
        inv.apply_step(vel0, z0, dm, step, si)
        ev, ez = _loop_step(inv, vel0, z0, dm, step, si)
        assert np.array_equal(g.velocity(), ev)
        assert np.array_equal(g.interface(4), ez if si > 0.0 else z0)
    assert inv.mvscale[inv.nvp] == 0.8
    vel_ok = inv.vel_nodes
    assert np.array_equal(inv.mvscale[inv.vel_ids], 1.0 / np.maximum(inv.v_init[vel_ok], 1.0))


def test_rms_rule_and_schedule():
    m, g, inv = _inv(InversionParams(crit_chi=0.5))
    n = inv.obs.size
    t = np.full(n, 0.9)
    t[0] = 0.2                                      # |res| 0.8 > crit_chi: dropped
    valid = np.ones(n, bool)
    valid[1] = False
    inv.obs[2] = -1.0
    keep = np.ones(n, bool)
    keep[[0, 1, 2]] = False
    assert abs(inv.rms(t, valid) - np.sqrt(np.mean((inv.obs[keep] - t[keep]) ** 2))) < 1e-15
    modes = []
    for it in range(1, 9):
        inv.iter = it
        modes.append(inv._mode())
    assert modes == [1, 1, 1, 2, 1, 1, 1, 2]
