"""Coarse inversion grids (fmt2d_projection / fmt2d_project_rows): the
projection P from coarse parameters onto the model's and the rows of G P,
which the reference does not have (it inverts on the propagation grid, P = I)
and which the benchmark configurations use (2 x 1 km on the 0.25 km grid,
2 x 0.5 km on the 0.1 km grid, interface nodes every 2 km).  Checked on the
CPU by the identities that define them: P = I at ratio 1, rows of P are
interpolation weights that sum to 1, (G P) x = G (P x), and P against a
numpy restatement of the bilinear weights."""
import numpy as np
import pytest
import scipy.sparse as sp

from fmt2d_b200 import synth
from _cases import oracle_G


@pytest.fixture(scope="module")
def small(oracle_lib):
    from fmt2d_b200.api import Fmt2d
    m = synth.small_model()
    g = Fmt2d(-1).upload(m)
    o = oracle_lib.Oracle(m)
    nd, npar, rp, gi, gv, _, _ = oracle_G(o, m)
    return m, g, (nd, npar, rp, gi, gv)


def _csr(rp, col, val, ncol):
    return sp.csr_matrix((val, col - 1, rp - 1), shape=(rp.size - 1, ncol))


def test_ratio_one_is_identity(small):
    from fmt2d_b200.api import project_rows
    m, g, (nd, npar, rp, gi, gv) = small
    pr = g.projection(1, 1, 1)
    prp, pcol, pval = pr["P"]
    assert pr["npar"] == npar and pr["nvp"] == g.inv_index()[1]
    np.testing.assert_array_equal(prp, np.arange(1, npar + 2))
    np.testing.assert_array_equal(pcol, np.arange(1, npar + 1))
    assert (pval == 1.0).all()
    orp, ogi, ogv = project_rows(rp, gi, gv, npar, prp, pcol, pval)
    np.testing.assert_array_equal(orp, rp)
    np.testing.assert_array_equal(ogi, gi)
    assert np.array_equal(ogv.view(np.uint64), gv.view(np.uint64))   # bit for bit


@pytest.mark.parametrize("kx,kz,ki", [(8, 4, 8), (3, 5, 4), (20, 2, 7)])
def test_interpolation_and_product(small, kx, kz, ki):
    from fmt2d_b200.api import project_rows
    m, g, (nd, npar, rp, gi, gv) = small
    pr = g.projection(kx, kz, ki)
    prp, pcol, pval = pr["P"]
    nvp, npc = g.inv_index()[1], pr["npar"]
    P = _csr(prp, pcol, pval, npc)
    # interpolation weights: non-negative, summing to one per fine parameter
    assert (pval > 0).all()
    np.testing.assert_allclose(np.asarray(P.sum(axis=1)).ravel(), 1.0, rtol=0, atol=1e-15)
    # every coarse parameter is used; velocity and interface blocks stay apart
    assert (np.asarray((P != 0).sum(axis=0)).ravel() > 0).all()
    assert P[:nvp, pr["nvp"]:].nnz == 0 and P[nvp:, :pr["nvp"]].nnz == 0
    # bilinear weights, restated
    inv = g.inv_index()[0]
    cidx = pr["coarse_idx"]
    iz, ix = np.nonzero(inv > 0)
    order = np.argsort(inv[iz, ix])
    iz, ix = iz[order], ix[order]
    a, b = (ix % kx) / kx, (iz % kz) / kz
    i, j = ix // kx, iz // kz
    D = np.zeros((nvp, pr["nvp"]))
    for (di, dj, w) in ((0, 0, (1 - a) * (1 - b)), (1, 0, a * (1 - b)), (0, 1, (1 - a) * b),
                        (1, 1, a * b)):
        ok = w != 0
        np.add.at(D, (np.arange(nvp)[ok], cidx[j[ok] + dj, i[ok] + di] - 1), w[ok])
    np.testing.assert_allclose(P[:nvp, :pr["nvp"]].toarray(), D, rtol=0, atol=1e-15)
    # (G P) x = G (P x)
    G = _csr(rp, gi, gv, npar)
    orp, ogi, ogv = project_rows(rp, gi, gv, npar, prp, pcol, pval)
    GP = _csr(orp, ogi, ogv, npc)
    assert all((np.diff(ogi[orp[k] - 1: orp[k + 1] - 1]) > 0).all() for k in range(nd))
    x = np.random.default_rng(kx).normal(size=npc)
    np.testing.assert_allclose(GP @ x, G @ (P @ x), rtol=1e-12, atol=1e-12 * np.abs(G @ (P @ x)).max())


def test_benchmark_grid_sizes():
    """The 4001x601 model on 2 km x 0.5 km with interface nodes every 2 km:
    about 24 k velocity parameters plus 201 interface parameters."""
    from fmt2d_b200.api import Fmt2d
    m = synth.config(4)
    g = Fmt2d(-1).upload(m)
    pr = g.projection(20, 5, 20)
    assert pr["npar"] - pr["nvp"] == 201
    assert 15000 < pr["nvp"] <= 201 * 121
    assert pr["coarse_idx"].shape == (121, 201)


def test_errors(small):
    from fmt2d_b200 import _native as N
    from fmt2d_b200.api import project_rows
    m, g, (nd, npar, rp, gi, gv) = small
    with pytest.raises(N.Fmt2dError):
        g.projection(0, 1, 1)
    bad = rp.copy()
    bad[0] = 0
    with pytest.raises(N.Fmt2dError):
        project_rows(bad, gi, gv, npar, *g.projection(1, 1, 1)["P"])


def test_lsqr_on_coarse_grid(small, oracle_lib):
    """LSQR with the Laplacian on the coarse parameter grid (the oracle's
    run_lsqr with an explicit geometry): at ratio 1 it is the model-grid solve
    bit for bit; on a coarse grid it fits data made by a coarse model."""
    from fmt2d_b200.api import project_rows
    m, g, (nd, npar, rp, gi, gv) = small
    o = oracle_lib.Oracle(m)
    rng = np.random.default_rng(21)
    r = rng.normal(0.0, 0.05, nd)
    G = _csr(rp, gi, gv, npar)
    gtg = np.asarray(G.multiply(G).sum(axis=0)).ravel()
    eps_min = max(1e-6, 1e-4 * gtg.max())
    inv, nvp, _ = g.inv_index()
    a = o.lsqr(nd, npar, gi, gv, rp, r, gtg, np.zeros(npar), eps_min, 0.5, 0.5, 3.0, 3.0, 60)
    b = oracle_lib.lsqr_geom(inv, nvp, npar - nvp, nd, npar, gi, gv, rp, r, gtg, np.zeros(npar),
                             eps_min, 0.5, 0.5, 3.0, 3.0, 60)
    assert np.array_equal(a[0], b[0]) and a[1:] == b[1:]
    pr = g.projection(4, 2, 4)
    prp, pcol, pval = pr["P"]
    npc, nvpc = pr["npar"], pr["nvp"]
    crp, cgi, cgv = project_rows(rp, gi, gv, npar, prp, pcol, pval)
    Gc = _csr(crp, cgi, cgv, npc)
    x_true = np.concatenate([0.01 * rng.standard_normal(nvpc), 0.2 * rng.standard_normal(npc - nvpc)])
    d = Gc @ x_true
    gtgc = np.asarray(Gc.multiply(Gc).sum(axis=0)).ravel()
    dm, it, rn, t2 = oracle_lib.lsqr_geom(pr["coarse_idx"], nvpc, npc - nvpc, nd, npc, cgi, cgv,
                                          crp, d, gtgc, np.zeros(npc), 1e-12 * gtgc.max(), 0.0,
                                          0.0, 0.0, 0.0, 400)
    assert np.linalg.norm(Gc @ dm - d) < 0.05 * np.linalg.norm(d)
