"""fmt2d_lsqr_noalloc: the LSQR solve for callers that cannot allocate device
memory while they solve (a driver overlapping the solve with other streams,
where cudaMalloc / cudaFree would synchronise the device, or a program whose
device memory is reserved up front by its own pool).  Called through the C
ABI with caller-owned device buffers, it must give what fmt2d_lsqr gives, on
two calls in a row (the shared scratch array keeps the previous call's
contents, so each call has to clear what starts at zero).

Tolerance: that of the fixed-iteration LSQR tests, 1e-6 of max|dm|, the same
stopping iteration, rnorm within 1e-9 of the right-hand-side norm.
"""
import ctypes as C

import numpy as np
import pytest

from fmt2d_b200 import synth
from _cases import oracle_G

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda:0")


def _noalloc(g, r, dm_sum, gtg, **kw):
    import torch
    from fmt2d_b200 import _native as N
    p = N.LsqrParams(1, int(kw["max_iter"]), float(kw["wdv"]), float(kw["wdv_iface"]),
                     float(kw["w_smooth"]), float(kw["w_smooth_iface"]), float(kw["eps_min"]))
    dr = _dev(r)
    ds = None if dm_sum is None else _dev(dm_sum)
    dg = None if gtg is None else _dev(gtg)
    dm = torch.full((g.nparm,), np.nan, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    it, rn, bn, t2 = C.c_int(), C.c_double(), C.c_double(), C.c_double()
    ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
    rc = g.L.fmt2d_lsqr_noalloc(g.h, C.byref(p), ptr(dr), ptr(dg), ptr(ds), ptr(dm),
                                C.byref(it), C.byref(rn), C.byref(bn), C.byref(t2))
    g._check(rc, "fmt2d_lsqr_noalloc")
    torch.cuda.synchronize()
    return dm.cpu().numpy(), it.value, rn.value, bn.value, t2.value


def test_noalloc_matches_lsqr_on_two_calls(oracle_lib):
    from fmt2d_b200.api import Fmt2d
    m = synth.small_model()
    o = oracle_lib.Oracle(m)
    nd, npar, rp, gi, gv, _, _ = oracle_G(o, m)
    g = Fmt2d(0).upload(m)
    g.set_frechet(nd, npar, rp, gi, gv)
    rng = np.random.default_rng(21)
    gtg = g.gtg_diag()
    eps_min = max(1e-6, 1e-4 * gtg.max())
    calls = [
        (rng.normal(0, 0.05, nd), rng.normal(0, 0.01, npar), gtg,
         dict(wdv=1.0, wdv_iface=0.3, w_smooth=10.0, w_smooth_iface=2.0, max_iter=40)),
        (rng.normal(0, 0.02, nd), None, None,
         dict(wdv=0.5, wdv_iface=0.5, w_smooth=3.0, w_smooth_iface=3.0, max_iter=2000)),
    ]
    for r, dm_sum, gg, kw in calls:
        kw["eps_min"] = eps_min
        ref = g.lsqr(r, dm_sum, gg, **kw)
        out = _noalloc(g, r, dm_sum, gg, **kw)
        assert out[1] == ref[1]
        assert np.abs(out[0] - ref[0]).max() <= 1e-6 * np.abs(ref[0]).max()
        assert abs(out[2] - ref[2]) <= 1e-9 * ref[3]
        assert abs(out[3] - ref[3]) <= 1e-12 * ref[3]


def test_noalloc_rejects_oversize(oracle_lib):
    """A 2001x401-grid parameterisation (about 0.74 M parameters) needs more
    than the fixed scratch array holds: a clear error, no work."""
    from fmt2d_b200 import _native as N
    from fmt2d_b200.api import Fmt2d
    m = synth.config(1)
    g = Fmt2d(0).upload(m)
    _, _, npar = g.inv_index()
    rp = np.array([1, 3], np.int32)
    g.set_frechet(1, npar, rp, np.array([1, 2], np.int32), np.array([0.1, 0.2]))
    with pytest.raises(N.Fmt2dError, match="too large for the no-alloc scratch"):
        _noalloc(g, np.ones(1), None, None, wdv=1.0, wdv_iface=1.0, w_smooth=1.0,
                 w_smooth_iface=1.0, eps_min=1e-6, max_iter=10)
