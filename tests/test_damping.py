"""The damping choice around LSQR (lsqr_inversion2d's call pattern,
src/inversion2d.f90:533-739) on the host: with an analytic solver whose RMS
changes are known in closed form, and with the oracle's LSQR on a G traced
on the small model (CPU)."""
import numpy as np
import pytest

from fmt2d_b200 import synth
from fmt2d_b200.damping import avg_dmd, avg_dmv, damping_search
from _cases import oracle_G


def _analytic(nvp=50, nif=10, seed=3):
    rng = np.random.default_rng(seed)
    a, b = 0.05 * rng.standard_normal(nvp), 0.5 * rng.standard_normal(nif)
    solve = lambda wdv, wdi: np.concatenate([a / (1.0 + wdv), b / (1.0 + wdi)])
    return a, b, solve, np.ones(nvp + nif), np.ones(nvp + nif)


def test_averages():
    dm = np.array([3.0, 4.0, 100.0, 1.0, 2.0])
    gtg = np.array([1.0, 1.0, 1e-9, 0.0, 0.0])
    assert avg_dmv(dm, gtg, 1.0, 3) == pytest.approx(np.sqrt(12.5))   # third column masked
    assert avg_dmd(dm, np.array([1, 1, 1, 2.0, 0.5]), 3) == pytest.approx(np.sqrt(2.5))
    assert avg_dmd(dm, np.ones(5), 5) == 0.0


def test_fixed_damping_is_one_solve():
    a, b, solve, gtg, mv = _analytic()
    r = damping_search(solve, None, gtg, mv, 1.0, a.size, lam_damp=2.0)
    assert r.solves == [(2.0, 2.0)]
    r = damping_search(solve, None, gtg, mv, 1.0, a.size, lam_damp=2.0, lam_damp_iface=5.0)
    assert r.solves == [(2.0, 5.0)] and r.wdv_iface == 5.0
    # no interface parameters: the interface weight follows the velocity weight
    r = damping_search(lambda w, wi: a / (1 + w), None, np.ones(a.size), np.ones(a.size), 1.0,
                       a.size, lam_damp=2.0, lam_damp_iface=5.0)
    assert r.solves == [(2.0, 2.0)]


def test_no_search_below_targets():
    a, b, solve, gtg, mv = _analytic()
    r = damping_search(solve, None, gtg, mv, 1.0, a.size, target_dv=1.0, target_dd=10.0)
    assert r.solves == [(0.0, 0.0), (0.0, 0.0)] and r.wdv == 0.0 and r.wdv_iface == 0.0


def test_auto_damping_reaches_targets():
    a, b, solve, gtg, mv = _analytic()
    rv, rd = np.sqrt(np.mean(a ** 2)), np.sqrt(np.mean(b ** 2))
    tv, td = rv / 10.0, rd / 4.0
    r = damping_search(solve, None, gtg, mv, 1.0, a.size, target_dv=tv, target_dd=td)
    assert abs(r.avg_dmv - tv) < 0.3 * tv and abs(r.avg_dmd - td) < 0.3 * td
    assert len(r.solves) <= 26
    # order: undamped, interface search from weights 1 and 100 (velocity weight
    # 0), velocity search from 1 and 100 at the chosen interface weight, final
    assert r.solves[0] == (0.0, 0.0)
    assert r.solves[1] == (0.0, 1.0) and r.solves[2] == (0.0, 100.0)
    # first secant step of the interface search, written out
    f1, f2 = rd / 2.0 - td, rd / 101.0 - td
    wd_rts, wd_xl, fl, fv = (1.0, 100.0, f2, f1) if abs(f1) < abs(f2) else (100.0, 1.0, f1, f2)
    step = (wd_xl - wd_rts) * fv / (fv - fl)
    expect = wd_rts + step if 0.0 < wd_rts + step <= 1e7 else None
    if expect is not None:
        assert r.solves[3][1] == pytest.approx(expect, rel=1e-12)
    k = next(i for i, s in enumerate(r.solves) if s[0] == 1.0)
    assert r.solves[k] == (1.0, r.wdv_iface) and r.solves[k + 1] == (100.0, r.wdv_iface)
    assert r.solves[-1] == (r.wdv, r.wdv_iface)
    np.testing.assert_allclose(r.dm, solve(r.wdv, r.wdv_iface))


def test_with_oracle_lsqr(oracle_lib):
    m = synth.small_model()
    o = oracle_lib.Oracle(m)
    nd, npar, rp, gi, gv, tc, used = oracle_G(o, m)
    inv, nvp, _ = o.inv_idx()
    assert npar > nvp                                   # interface parameters present
    rows = np.repeat(np.arange(nd), np.diff(rp))
    gtg = np.bincount(gi - 1, weights=gv ** 2, minlength=npar)
    rng = np.random.default_rng(0)
    dm_true = np.concatenate([0.02 * rng.standard_normal(nvp), 0.3 * rng.standard_normal(npar - nvp)])
    residual = np.bincount(rows, weights=gv * dm_true[gi - 1], minlength=nd)
    eps_min = 1e-6 * gtg.max()

    def solve(wdv, wdi):
        return o.lsqr(nd, npar, gi, gv, rp, residual, gtg, np.zeros(npar), eps_min, wdv, wdi,
                      1.0, 1.0, 300)[0]

    r0 = damping_search(solve, None, gtg, np.ones(npar), eps_min, nvp, target_dv=10.0,
                        target_dd=10.0)
    assert len(r0.solves) == 2
    tv, td = 0.5 * r0.avg_dmv, 0.5 * r0.avg_dmd
    r = damping_search(solve, None, gtg, np.ones(npar), eps_min, nvp, target_dv=tv, target_dd=td)
    assert r.wdv > 0.0 and r.wdv_iface > 0.0 and len(r.solves) <= 26
    assert abs(r.avg_dmv - tv) < 0.3 * tv, (r.avg_dmv, tv)
    assert r.avg_dmd < r0.avg_dmd


def test_api_wrapper_plumbing(oracle_lib):
    """Fmt2d.lsqr_damped passes the weights, smoothing and limits to each
    LSQR solve and takes n_vel_parms from the model (host-only context, the
    device solve replaced by the oracle's)."""
    from fmt2d_b200.api import Fmt2d
    m = synth.small_model()
    o = oracle_lib.Oracle(m)
    nd, npar, rp, gi, gv, tc, used = oracle_G(o, m)
    gtg = np.bincount(gi - 1, weights=gv ** 2, minlength=npar)
    residual = np.ones(nd) * 1e-3
    g = Fmt2d(-1).upload(m)
    g.nparm = npar
    seen = []

    def fake_lsqr(res, dm_sum, gtg_diag, **kw):
        seen.append(kw)
        s = np.zeros(npar) if dm_sum is None else dm_sum
        dm = o.lsqr(nd, npar, gi, gv, rp, res, gtg_diag, s, kw["eps_min"], kw["wdv"],
                    kw["wdv_iface"], kw["w_smooth"], kw["w_smooth_iface"], kw["max_iter"])[0]
        return dm, 0, 0.0, 0.0, 0.0

    g.lsqr = fake_lsqr
    r = g.lsqr_damped(residual, None, gtg, lam_damp=3.0, lam_damp_iface=0.5, w_smooth=2.0,
                      w_smooth_iface=1.5, eps_min=1e-9, max_iter=50)
    assert len(seen) == 1
    assert seen[0] == dict(wdv=3.0, wdv_iface=0.5, w_smooth=2.0, w_smooth_iface=1.5,
                           eps_min=1e-9, max_iter=50, smooth_type=1)
    assert r.dm.shape == (npar,) and r.wdv == 3.0 and r.wdv_iface == 0.5
