"""The data of an LSQR solve from traced picks (fmt2d_select_data):
read_frechet_data2d's selection (src/inversion2d.f90:3965-4052) and
lsqr_inversion2d's weighting (:334-379), against a loop restatement of the
reference on the oracle's rays of the small model (CPU)."""
import numpy as np
import pytest

from fmt2d_b200 import synth


def _restated(phase, obs, t, valid, rp, gi, gv, mv, crit, w):
    rows, res, wts, pk = [], [], [], []
    for p in range(phase.size):
        if not valid[p] or obs[p] < 0.0:
            continue
        r = obs[p] - t[p]
        if abs(r) > crit:
            continue
        wt = 1.0
        if phase[p] == 2:
            wt = wt * w[0]
        elif phase[p] == 3:
            wt = wt * w[1]
        elif phase[p] in (4, 5):
            wt = wt * w[2]
        idx = gi[rp[p] - 1: rp[p + 1] - 1]
        val = gv[rp[p] - 1: rp[p + 1] - 1].copy()
        for k, j in enumerate(idx):
            if 1 <= j <= mv.size:
                val[k] = val[k] * mv[j - 1] * wt
        rows.append((idx, val))
        res.append(r * wt)
        wts.append(wt)
        pk.append(p)
    orp = np.concatenate([[1], 1 + np.cumsum([a.size for a, _ in rows])]).astype(np.int32)
    cat = lambda k, dt: (np.concatenate([r[k] for r in rows]).astype(dt) if rows
                         else np.zeros(0, dt))
    return orp, cat(0, np.int32), cat(1, np.float64), np.array(res), np.array(wts), np.array(pk)


@pytest.fixture(scope="module")
def traced(oracle_lib):
    from fmt2d_b200.api import phase_mask
    m = synth.small_model(phases=(1, 2, 3, 4, 5))
    o = oracle_lib.Oracle(m)
    for s, sx in enumerate(m.obs_x):
        o.forward(s, sx, phase_mask((1, 2, 3, 4, 5)))
    pk = m.picks
    rs = [o.trace(int(p[0]), int(p[1]), p[2], p[3]) for p in pk]
    valid = np.array([r["valid"] for r in rs], np.int32)
    t = np.array([r["t"] for r in rs])
    sizes = [r["idx"].size if r["valid"] else 0 for r in rs]
    rp = np.concatenate([[1], 1 + np.cumsum(sizes)]).astype(np.int32)
    gi = np.concatenate([r["idx"] for r, v in zip(rs, valid) if v]).astype(np.int32)
    gv = np.concatenate([r["val"] for r, v in zip(rs, valid) if v])
    _, _, npar = o.inv_idx()
    rng = np.random.default_rng(4)
    obs = t + rng.normal(0.0, 0.05, t.size)
    obs[rng.random(t.size) < 0.1] = -1.0                      # picks without an observation
    return pk[:, 1].astype(np.int32), obs, t, valid, rp, gi, gv, npar


@pytest.mark.parametrize("crit,w", [(0.1, (1.0, 1.0, 1.0)), (0.06, (0.5, 2.0, 0.25)),
                                    (1e9, (1.0, 0.0, 3.0))])
def test_matches_restatement(traced, crit, w):
    from fmt2d_b200.api import select_data
    phase, obs, t, valid, rp, gi, gv, npar = traced
    mv = 0.1 + np.random.default_rng(9).random(npar)
    got = select_data(phase, obs, t, valid, rp, gi, gv, mv, crit_chi=crit, wt_psed=w[0],
                      wt_pmp=w[1], wt_pgss=w[2])
    ref = _restated(phase, obs, t, valid, rp, gi, gv, mv, crit, w)
    for a, b in zip(got, ref):
        assert np.array_equal(np.asarray(a), np.asarray(b))
    assert got[5].size > 0 and (got[5].size < phase.size)


def test_empty_and_bad_arguments(traced):
    from fmt2d_b200 import _native as N
    from fmt2d_b200.api import select_data
    phase, obs, t, valid, rp, gi, gv, npar = traced
    out = select_data(phase, obs, t, np.zeros_like(valid), rp, gi, gv, np.ones(npar),
                      crit_chi=1.0)
    assert out[0].tolist() == [1] and out[1].size == 0 and out[3].size == 0
    bad = rp.copy()
    bad[1] = bad[2] + 1                                       # decreasing row pointers
    with pytest.raises(N.Fmt2dError):
        select_data(phase, obs, t, valid, bad, gi, gv, np.ones(npar), crit_chi=1.0)
