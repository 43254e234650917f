"""Committed golden vectors (tests/golden/small_model.npz, written by
tests/golden/make_golden.py from the oracle): the oracle must reproduce them
exactly (CPU), and the device path must match them within the tolerances of
the other parity tests (GPU): traveltimes within 0.5 ms with identical
reached sets, receiver times within 0.5 ms where both are valid with valid
flags agreeing on at least 93% of picks (coincident-seed ties, see
test_rays_gpu), LSQR iterates within 1e-6 of max|dm| after 40 iterations."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
GOLD = os.path.join(HERE, "golden", "small_model.npz")


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def test_oracle_reproduces_golden(gold, oracle_lib):
    import make_golden
    now = make_golden.generate()
    assert set(now) == set(gold)
    for k, v in now.items():
        a, b = np.asarray(v), gold[k]
        assert a.shape == b.shape and a.dtype == b.dtype, k
        if a.dtype.kind == "f":
            assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), k   # bit for bit
        else:
            assert np.array_equal(a, b), k


@pytest.mark.gpu
def test_device_against_golden(gold):
    import make_golden
    from fmt2d_b200 import synth
    from fmt2d_b200.api import Fmt2d
    m = synth.small_model()
    g = Fmt2d(0).upload(m).forward(m.obs_x, make_golden.PHASES)
    for s in range(len(m.obs_x)):
        for tf in make_golden.TFS:
            To, Tg = gold[f"T_{s}_{tf}"], g.field(s, tf)[0]
            ro, rg = To < 1e19, Tg < 1e19
            assert (ro == rg).all(), (s, tf)
            assert np.abs(To[ro] - Tg[ro]).max() <= 0.5e-3, (s, tf)
    t, valid, nnz = g.trace(gold["pick_src"], gold["pick_phase"], gold["pick_x"], gold["pick_z"])
    gv = gold["pick_valid"]
    assert np.mean(valid == gv) >= 0.93
    both = valid & gv
    assert np.abs(t[both] - gold["pick_t"][both]).max() <= 0.5e-3
    npar = int(gold["ls_nparm"])
    rp = gold["ls_row_ptr"]
    g.set_frechet(rp.size - 1, npar, rp, gold["ls_gindx"], gold["ls_gval"])
    kw = {k: v for k, v in make_golden.LSQR.items()}
    dm, iters, rnorm, bnorm, t2 = g.lsqr(gold["ls_residual"], gold["ls_dm_sum"], gold["ls_gtg"],
                                         eps_min=float(gold["ls_eps_min"]), **kw)
    assert iters == int(gold["ls_iters"])
    assert np.abs(dm - gold["ls_dm"]).max() <= 1e-6 * np.abs(gold["ls_dm"]).max()
