"""The oracle's Frechet rows against finite differences of its own forward
solve and ray backtrace: the identity the reference checks in
fd_verify_frechet (src/inversion2d.f90:5668-5833, avg(dt_pred / dt_fd) over
picks), here along a smooth velocity perturbation instead of one node.

The 401x121 model is perturbed by 0.1% inside a Gaussian blob in the middle
of the crust, away from the seafloor (whose water-side cell corners carry no
parameters); Pg picks of three sources with receivers on the seafloor (no
water leg) are traced on both models.  dt_pred = sum_j G_ij ds_j with ds the
change of the propagation-grid slowness at parameter j, dt_fd = t' - t."""
import dataclasses

import numpy as np

from fmt2d_b200 import synth
from fmt2d_b200.api import phase_mask


def test_frechet_rows_match_finite_differences(oracle_lib):
    m = synth.config(0)
    X, ZR = np.meshgrid(m.xpos, m.zrel)
    xc, zc = 0.5 * (m.xpos[0] + m.xpos[-1]), 0.45 * m.zrel[-1]
    blob = np.exp(-((X - xc) / (0.15 * (m.xpos[-1] - m.xpos[0]))) ** 2
                  - ((ZR - zc) / (0.2 * m.zrel[-1])) ** 2)
    m2 = dataclasses.replace(m, vel=m.vel * (1.0 + 1.0e-3 * blob))
    o1, o2 = oracle_lib.Oracle(m), oracle_lib.Oracle(m2)
    inv, nvp, npar = o1.inv_idx()
    ok = inv > 0
    ds = np.zeros(npar + 1)
    ds[inv[ok]] = 1.0 / o2.pgrid_velocity()[ok] - 1.0 / o1.pgrid_velocity()[ok]
    pred, fd = [], []
    for s in range(3):
        o1.forward(s, m.obs_x[s], phase_mask((1,)))
        o2.forward(s, m.obs_x[s], phase_mask((1,)))
        for rx in np.arange(m.xpos[1] + 0.5, m.xpos[-2], 2.5):
            if abs(rx - m.obs_x[s]) < 2.0:
                continue
            zsf = np.interp(rx, m.xpos, m.topo)
            a, b = o1.trace(s, 1, rx, zsf + 1e-6), o2.trace(s, 1, rx, zsf + 1e-6)
            if not (a["valid"] and b["valid"]):
                continue
            assert a["idx"].size and a["idx"].max() <= nvp   # Pg rows: velocity parameters only
            pred.append(float(np.sum(a["val"] * ds[a["idx"]])))
            fd.append(b["t"] - a["t"])
    pred, fd = np.array(pred), np.array(fd)
    assert pred.size >= 80
    big = np.abs(fd) > 0.2 * np.abs(fd).max()      # rays that cross the blob
    assert big.sum() >= 20
    ratio = pred[big] / fd[big]
    assert abs(ratio.mean() - 1.0) < 0.03, ratio.mean()
    assert ratio.min() > 0.85 and ratio.max() < 1.15, (ratio.min(), ratio.max())
    assert np.corrcoef(pred, fd)[0, 1] > 0.999
