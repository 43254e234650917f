"""Host logic of Fmt2d.gradient_on_params (no GPU): the adjoint gradient
placed on the inversion parameters (velocity parameters by inv_idx, then the
inverted interface's nodes) and projected with P^T onto a coarse grid,
checked against a dense restatement."""
import numpy as np
import pytest

from fmt2d_b200.api import Fmt2d


class _Stub:
    """Just what gradient_on_params reads from a context."""

    def __init__(self, inv, nvp, npar, iface_inv):
        self._inv, self._nvp, self._npar, self.iface_inv = inv, nvp, npar, iface_inv

    def inv_index(self):
        return self._inv, self._nvp, self._npar


def _case(seed=0, nz=7, nx=9):
    rng = np.random.default_rng(seed)
    inv = np.zeros((nz, nx), np.int32)
    active = np.arange(nz)[:, None] >= 2                 # below the "seafloor" row
    active = np.broadcast_to(active, (nz, nx))
    inv[active] = np.arange(1, active.sum() + 1)
    nvp = int(active.sum())
    npar = nvp + nx
    grad = {"grad_slow": rng.normal(size=(nz, nx)), "grad_iface": rng.normal(size=(5, nx))}
    return _Stub(inv, nvp, npar, 4), grad


def test_gradient_on_fine_parameters():
    g, grad = _case()
    out = Fmt2d.gradient_on_params(g, grad)
    inv, nvp, npar = g.inv_index()
    ref = np.zeros(npar)
    for iz in range(inv.shape[0]):
        for ix in range(inv.shape[1]):
            if inv[iz, ix] > 0:
                ref[inv[iz, ix] - 1] = grad["grad_slow"][iz, ix]
    ref[nvp:] = grad["grad_iface"][g.iface_inv - 1]
    assert np.array_equal(out, ref)


def test_gradient_projected_with_pt():
    g, grad = _case(seed=1)
    _, nvp, npar = g.inv_index()
    rng = np.random.default_rng(2)
    ncoarse = 11
    # a random P (1-based CSR, one row per fine parameter)
    P = (rng.random((npar, ncoarse)) < 0.3) * rng.uniform(0.1, 1.0, (npar, ncoarse))
    rp = np.concatenate([[1], 1 + np.cumsum((P != 0).sum(axis=1))]).astype(np.int32)
    col = (np.nonzero(P)[1] + 1).astype(np.int32)
    val = P[P != 0]
    proj = {"P": (rp, col, val), "npar": ncoarse, "nvp": 5}
    out = Fmt2d.gradient_on_params(g, grad, proj)
    fine = Fmt2d.gradient_on_params(g, grad)
    np.testing.assert_allclose(out, P.T @ fine, rtol=1e-13, atol=1e-13)


def test_gradient_needs_interface_part():
    g, grad = _case()
    with pytest.raises(ValueError):
        Fmt2d.gradient_on_params(g, {"grad_slow": grad["grad_slow"]})
