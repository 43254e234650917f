"""The oracle's run_lsqr for the Gaussian (smooth_type 2) and hybrid
(smooth_type 3) layouts, src/inversion2d.f90:507-511 and 6578-7167, pinned
against SciPy's independent LSQR driven by the operator pair the reference
applies (CPU):

  2: [G; w_s R_h; w_s R_v; w_d I] with the interface Gaussian R_i in the R_h
     block's interface rows; adjoint R_h^T, R_v^T and R_i itself;
  3: [G; w_s L (velocity rows) + w_si R_i (interface rows); w_d I]; adjoint
     L and R_i themselves;

masked velocity columns (gtg < 0.01 eps_min) zeroed in every block.  The
general routine also reproduces the Laplacian layout (smooth_type 1) bit for
bit."""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.linalg import LinearOperator, lsqr

from fmt2d_b200 import synth
from _cases import oracle_G, csr_to_scipy

CX, CZ, CI = 2.0, 1.0, 3.0


@pytest.fixture(scope="module")
def case(oracle_lib):
    m = synth.small_model()
    o = oracle_lib.Oracle(m)
    nd, npar, rp, gi, gv, tc, used = oracle_G(o, m)
    inv, nvp, _ = o.inv_idx()
    G = csr_to_scipy(nd, npar, rp, gi, gv)
    rng = np.random.default_rng(5)
    # velocity columns scaled per node; the interface columns by one weight,
    # as the reference assumes when it applies R_i as its own adjoint
    mv = 0.2 + rng.random(npar)
    mv[nvp:] = 0.7
    mats = {}
    for which in (0, 1, 2):
        r, c, v = o.gauss_smooth(which, mv, CX, CZ, CI)
        mats[which] = sp.csr_matrix((v, c - 1, r - 1), shape=(npar, npar))
    return o, nd, npar, nvp, rp, gi, gv, G, mv, mats


def _ops(o, G, nvp, keep, st, ws, wsi, wdv, wdi, mats):
    nd, npar = G.shape
    vel = np.arange(npar) < nvp
    wd = np.where(vel, np.where(keep, wdv, 0.0), wdi)
    Rh, Rv, Ri = mats[0], mats[1], mats[2]
    nsm = 2 * npar if st == 2 else npar

    def smooth(x):
        if st == 2:
            h, v = ws * (Rh @ x), ws * (Rv @ x)
            h[~keep], v[~keep] = 0.0, 0.0
            h[nvp:] = wsi * (Ri @ x)[nvp:]
            return np.concatenate([h, v])
        lap = o.laplacian(npar, x)
        out = np.where(keep, ws * lap, 0.0)
        out[nvp:] = wsi * (Ri @ x)[nvp:]
        return out

    def smooth_T(y):
        if st == 2:
            h, v = Rh.T @ y[:npar], Rv.T @ y[npar:]
            h[~keep], v[~keep] = 0.0, 0.0
            out = ws * h + ws * v
            out[nvp:] += wsi * (Ri @ y[:npar])[nvp:]
            return out
        lap = o.laplacian(npar, y)
        out = np.where(keep, ws * lap, 0.0)
        out[nvp:] = wsi * (Ri @ y)[nvp:]
        return out

    def mv(x):
        x = np.where(keep, x.ravel(), 0.0)
        return np.concatenate([G @ x, smooth(x), wd * x])

    def rmv(u):
        u = u.ravel()
        y = G.T @ u[:nd] + smooth_T(u[nd:nd + nsm]) + wd * u[nd + nsm:]
        return np.where(keep, y, 0.0)

    A = LinearOperator((nd + nsm + npar, npar), matvec=mv, rmatvec=rmv, dtype=np.float64)
    return A, smooth, wd


@pytest.mark.parametrize("st", [2, 3])
@pytest.mark.parametrize("ws,wsi,wdv,wdi", [(1.0, 1.0, 0.5, 0.5), (5.0, 2.0, 1.0, 0.3),
                                            (0.0, 3.0, 0.0, 1.0)])
def test_matches_scipy(case, st, ws, wsi, wdv, wdi):
    o, nd, npar, nvp, rp, gi, gv, G, mv, mats = case
    rng = np.random.default_rng(11)
    r = rng.normal(0.0, 0.05, nd)
    dm_sum = rng.normal(0.0, 0.01, npar)
    gtg = np.asarray(G.multiply(G).sum(axis=0)).ravel()
    eps_min = max(1e-6, 1e-4 * gtg.max())
    keep = np.concatenate([gtg[:nvp] >= 0.01 * eps_min, np.ones(npar - nvp, bool)])
    n_it = 25
    dm, iters, rnorm, t2 = o.lsqr_smooth(st, nd, npar, gi, gv, rp, r, gtg, dm_sum, mv, CX, CZ, CI,
                                         eps_min, wdv, wdi, ws, wsi, n_it)
    A, smooth, wd = _ops(o, G, nvp, keep, st, ws, wsi, wdv, wdi, mats)
    b = np.concatenate([r, -smooth(dm_sum), -(wd * dm_sum)])
    x = lsqr(A, b, damp=0.0, atol=0.0, btol=0.0, conlim=0.0, iter_lim=min(iters, n_it))[0]
    assert abs(rnorm - np.linalg.norm(A @ dm - b)) <= 1e-6 * np.linalg.norm(b)
    scale = np.abs(x).max()
    assert np.abs(dm - x).max() <= 1e-6 * scale, np.abs(dm - x).max() / scale


@pytest.mark.parametrize("ws,wsi,wdv,wdi", [(0.0, 0.0, 1.0, 1.0), (3.0, 3.0, 0.5, 0.5)])
def test_type1_identical_to_laplacian_routine(case, ws, wsi, wdv, wdi):
    o, nd, npar, nvp, rp, gi, gv, G, mv, mats = case
    rng = np.random.default_rng(2)
    r = rng.normal(0.0, 0.05, nd)
    dm_sum = rng.normal(0.0, 0.01, npar)
    gtg = np.asarray(G.multiply(G).sum(axis=0)).ravel()
    eps_min = max(1e-6, 1e-4 * gtg.max())
    a = o.lsqr(nd, npar, gi, gv, rp, r, gtg, dm_sum, eps_min, wdv, wdi, ws, wsi, 60)
    b = o.lsqr_smooth(1, nd, npar, gi, gv, rp, r, gtg, dm_sum, mv, CX, CZ, CI, eps_min, wdv, wdi,
                      ws, wsi, 60)
    assert np.array_equal(a[0], b[0]) and a[1] == b[1] and a[2] == b[2] and a[3] == b[3]
