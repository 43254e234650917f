"""Gaussian smoothing matrices of run_lsqr's smooth_type 2/3 layouts
(build_gauss_smooth_matrix and build_iface_gauss_smooth_matrix,
src/inversion2d.f90:1252-1616): the library's host build
(fmt2d_gauss_smooth) against the oracle's restatement, bit for bit, and the
properties the construction guarantees (CPU)."""
import numpy as np
import pytest

from fmt2d_b200 import synth


@pytest.fixture(scope="module", params=["small", "cfg0"])
def pair(request, oracle_lib):
    from fmt2d_b200.api import Fmt2d
    m = synth.small_model() if request.param == "small" else synth.config(0)
    o = oracle_lib.Oracle(m)
    g = Fmt2d(-1).upload(m)
    inv, nvp, npar = g.inv_index()
    return m, o, g, nvp, npar


@pytest.mark.parametrize("which,cx,cz,ci", [(0, 1.0, 0.5, 0.0), (1, 1.0, 0.5, 0.0),
                                            (0, 3.3, 1.7, 0.0), (1, 3.3, 1.7, 0.0),
                                            (2, 0.0, 0.0, 2.0), (2, 0.0, 0.0, 7.5)])
def test_library_matches_oracle(pair, which, cx, cz, ci):
    m, o, g, nvp, npar = pair
    mv = 0.1 + np.random.default_rng(which).random(npar)
    rp, col, val = g.gauss_smooth(which, mv, cx, cz, ci)
    orp, ocol, oval = o.gauss_smooth(which, mv, cx, cz, ci)
    np.testing.assert_array_equal(rp, orp)
    np.testing.assert_array_equal(col, ocol)
    assert np.array_equal(val.view(np.uint64), oval.view(np.uint64))   # bit for bit


def test_structure(pair):
    m, o, g, nvp, npar = pair
    one = np.ones(npar)
    for which, args in ((0, (1.5, 0.0, 0.0)), (1, (0.0, 0.8, 0.0)), (2, (0.0, 0.0, 2.0))):
        rp, col, val = g.gauss_smooth(which, one, *args)
        counts = np.diff(rp)
        covered = np.arange(npar) < nvp if which < 2 else np.arange(npar) >= nvp
        assert (counts[covered] >= 1).all() and (counts[~covered] == 0).all()
        rows = np.repeat(np.arange(npar), counts)
        # the diagonal closes each row and the row sums vanish (R 1 = 0)
        assert (col[rp[1:][covered] - 2] == np.arange(1, npar + 1)[covered]).all()
        assert np.abs(np.bincount(rows, weights=val, minlength=npar)).max() < 1e-12
        # uniform mvscale: the pattern and values are symmetric
        A = np.zeros((npar, npar)) if npar < 3000 else None
        if A is not None:
            A[rows, col - 1] = val
            np.testing.assert_allclose(A, A.T, atol=1e-15)


def test_mvscale_is_a_column_scaling(pair):
    m, o, g, nvp, npar = pair
    mv = 0.5 + np.random.default_rng(7).random(npar)
    rp1, col1, val1 = g.gauss_smooth(0, np.ones(npar), 2.0)
    rpm, colm, valm = g.gauss_smooth(0, mv, 2.0)
    np.testing.assert_array_equal(col1, colm)
    np.testing.assert_allclose(valm, val1 * mv[col1 - 1], rtol=1e-15)


def test_errors(pair):
    from fmt2d_b200 import _native as N
    m, o, g, nvp, npar = pair
    with pytest.raises(ValueError):
        g.gauss_smooth(0, np.ones(npar - 1), 1.0)
    with pytest.raises(N.Fmt2dError, match="corr_x"):
        g.gauss_smooth(0, np.ones(npar), 0.0)
    with pytest.raises(N.Fmt2dError):
        g.gauss_smooth(3, np.ones(npar), 1.0)
    rp, col, val = g.gauss_smooth(2, np.ones(npar), 0.0, 0.0, 0.0)   # no interface smoothing
    assert col.size == 0 and (rp == 1).all()
