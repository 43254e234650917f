"""The oracle's LSQR restatement (run_lsqr, src/inversion2d.f90:6578-7167)
pinned against SciPy's independent LSQR (CPU).

SciPy is driven by the same operator pair the reference applies: the
augmented matrix [G; w_s L; w_d I] with masked velocity columns, whose
"transpose" the reference forms as [G^T, diag(w_s) L, diag(w_d)] (it treats
the weighted Laplacian as symmetric).  Both implement Golub-Kahan
bidiagonalisation with the same updates, so after the same number of
iterations the solutions agree to rounding.
"""
import numpy as np
import pytest
from scipy.sparse.linalg import lsqr

from fmt2d_b200 import synth
from _cases import oracle_G, csr_to_scipy, ref_ops as _ref_ops


@pytest.fixture(scope="module")
def case(oracle_lib):
    m = synth.small_model()
    o = oracle_lib.Oracle(m)
    nd, npar, rp, gi, gv, tc, used = oracle_G(o, m)
    inv, nvp, npar2 = o.inv_idx()
    assert npar == npar2
    return m, o, nd, npar, nvp, rp, gi, gv


@pytest.mark.parametrize("ws_v,ws_i,wd_v,wd_i", [(0.0, 0.0, 1.0, 1.0), (3.0, 3.0, 0.5, 0.5),
                                                 (10.0, 2.0, 1.0, 0.3)])
@pytest.mark.parametrize("max_iter", [8, 40, 2000])
def test_oracle_lsqr_matches_scipy(oracle_lib, case, ws_v, ws_i, wd_v, wd_i, max_iter):
    """Same iterates as SciPy while rounding differences stay small.  Without
    reorthogonalisation both amplify them (by about 1.3x per iteration on this
    model), so runs to convergence are compared by misfit, not iterate."""
    m, o, nd, npar, nvp, rp, gi, gv = case
    G = csr_to_scipy(nd, npar, rp, gi, gv)
    rng = np.random.default_rng(11)
    r = rng.normal(0.0, 0.05, nd)
    dm_sum = rng.normal(0.0, 0.01, npar)
    gtg = np.asarray(G.multiply(G).sum(axis=0)).ravel()
    eps_min = max(1e-6, 1e-4 * gtg.max())
    mask = gtg[:nvp] < 0.01 * eps_min
    dm, iters, rnorm, t2 = o.lsqr(nd, npar, gi, gv, rp, r, gtg, dm_sum, eps_min, wd_v, wd_i, ws_v,
                                  ws_i, max_iter)
    assert 1 <= iters <= max_iter + 1
    if iters <= max_iter:
        assert t2 < 1e-4
    A, ws, wd = _ref_ops(o, G, nvp, mask, ws_v, ws_i, wd_v, wd_i)
    L = o.laplacian(npar, dm_sum)
    b = np.concatenate([r, -(ws * L), -(wd * dm_sum)])
    x = lsqr(A, b, damp=0.0, atol=0.0, btol=0.0, conlim=0.0, iter_lim=min(iters, max_iter))[0]
    res_o, res_s = np.linalg.norm(A @ dm - b), np.linalg.norm(A @ x - b)
    assert abs(rnorm - res_o) <= 1e-6 * np.linalg.norm(b)
    if max_iter <= 40:
        scale = np.abs(x).max()
        assert np.abs(dm - x).max() <= 1e-6 * scale, np.abs(dm - x).max() / scale
    else:
        assert abs(res_o - res_s) <= 1e-4 * res_s


def test_oracle_products(oracle_lib, case):
    m, o, nd, npar, nvp, rp, gi, gv = case
    G = csr_to_scipy(nd, npar, rp, gi, gv)
    rng = np.random.default_rng(3)
    x, y = rng.normal(size=npar), rng.normal(size=nd)
    np.testing.assert_allclose(oracle_lib.spmv(nd, npar, gi, gv, rp, x), G @ x, rtol=1e-12,
                               atol=1e-12)
    np.testing.assert_allclose(oracle_lib.spmv(nd, npar, gi, gv, rp, y, transpose=True), G.T @ y,
                               rtol=1e-12, atol=1e-12)


def test_oracle_zero_rhs(oracle_lib, case):
    m, o, nd, npar, nvp, rp, gi, gv = case
    dm, iters, rnorm, t2 = o.lsqr(nd, npar, gi, gv, rp, np.zeros(nd), np.ones(npar),
                                  np.zeros(npar), 1e-6, 1.0, 1.0, 1.0, 1.0, 100)
    assert iters == 0 and not dm.any()
