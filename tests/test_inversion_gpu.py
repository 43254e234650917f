"""The inversion iteration on the device path (fmt2d_b200/inversion.py,
lsqr_inversion2d's loop body, src/inversion2d.f90:256-937) on the small
model: observed times from the checkerboard model, the inversion started
from the smooth model.  Each iteration must lower the RMS residual (or keep
the model when no step does), the next iteration's starting RMS must be the
accepted RMS (the same model forwarded again), and the model steps must stay
inside the reference's bounds."""
import dataclasses

import numpy as np
import pytest

from fmt2d_b200 import synth
from fmt2d_b200.api import Fmt2d
from fmt2d_b200.inversion import Inversion, InversionParams

pytestmark = pytest.mark.gpu


def _observed(m, phases):
    g = Fmt2d(0).upload(m)
    g.forward(m.obs_x, phases)
    P = m.picks
    t, valid, _ = g.trace(P[:, 0].astype(np.int32), P[:, 1].astype(np.int32), P[:, 2], P[:, 3])
    rng = np.random.default_rng(9)
    obs = np.where(valid, t + rng.normal(0.0, 0.005, t.size), -1.0)
    g.close()
    return obs


@pytest.mark.parametrize("params", [
    InversionParams(phases=(1, 3), lam_damp=1.0, lam_smooth=10.0, lam_smooth_iface=10.0,
                    alt_inv_mode=0),
    InversionParams(phases=(1, 3), lam_damp=0.0, lam_smooth=5.0, lam_smooth_iface=5.0,
                    smooth_type=3, corr_x_iface=2.0, alt_inv_mode=-1, lsqr_max_iter=300),
])
def test_iterations_lower_rms(params):
    true = synth.small_model()
    start = dataclasses.replace(synth.small_model(cb_amp=0.0),
                                moho_z=true.moho_z + 0.15)
    obs = _observed(true, params.phases)
    g = Fmt2d(0).upload(start)
    inv = Inversion(g, start.obs_x, start.picks, obs, params)
    v_init = inv.v_init.copy()
    prev = None
    for _ in range(2):
        r = inv.iteration()
        assert r.ndata > 0 and r.forwards >= 2 and r.lsqr_solves >= 1
        assert r.rms_new <= r.rms_orig
        if r.step > 0.0:
            assert r.rms_new < r.rms_orig
        if prev is not None:
            assert abs(r.rms_orig - prev.rms_new) <= 1e-9 * prev.rms_new
        prev = r
        v = g.velocity()
        vn = inv.vel_nodes
        assert np.all(v[vn] >= 2.0 - 1e-12) and np.all(v[vn] <= 10.0 + 1e-12)
        big = v_init[vn] >= 2.0
        assert np.all(v[vn][big] <= v_init[vn][big] * 1.30 * (1 + 1e-12))
        assert np.all(v[vn][big] >= v_init[vn][big] * 0.70 * (1 - 1e-12))
        assert np.array_equal(v[~vn], v_init[~vn])
