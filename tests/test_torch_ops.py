"""The PyTorch operators (torch.ops.fmt2d.*) on the C ABI.

CPU: the operator library loads and registers every operator with its
schema.  GPU: each operator called with CUDA tensors matches the ctypes path
bit for bit (forward + field, trace + Frechet rows, LSQR)."""
import numpy as np
import pytest
import torch

from fmt2d_b200 import synth
from fmt2d_b200 import torch_ops


def test_ops_registered():
    ops = torch_ops.load()
    for name in torch_ops.OPS:
        op = getattr(ops, name)
        assert op.default._schema.name == f"fmt2d::{name}"


@pytest.mark.gpu
def test_ops_match_ctypes_path():
    from fmt2d_b200.api import Fmt2d, phase_mask
    ops = torch_ops.load()
    m = synth.small_model()
    phases = (1, 2, 3, 4, 5)
    a, b = Fmt2d(0).upload(m), Fmt2d(0).upload(m)
    src = np.asarray(m.obs_x, dtype=np.float64)
    a.forward(src, phases)
    ops.forward(torch_ops.handle(b), torch.tensor(src, device="cuda"), phase_mask(phases))
    for s in range(src.size):
        for tf in range(1, 13):
            T, gx, gz = a.field(s, tf)
            Tt, gxt, gzt = ops.field(torch_ops.handle(b), s, tf)
            assert Tt.is_cuda and Tt.dtype == torch.float64
            assert np.array_equal(Tt.cpu().numpy(), T)
            assert np.array_equal(gxt.cpu().numpy(), gx, equal_nan=True)
            assert np.array_equal(gzt.cpu().numpy(), gz, equal_nan=True)
    P = m.picks
    si, ph = P[:, 0].astype(np.int32), P[:, 1].astype(np.int32)
    t, v, nnz = a.trace(si, ph, P[:, 2], P[:, 3])
    rp, gi, gv = a.frechet_rows()
    dev = lambda x: torch.tensor(x, device="cuda")
    tt, vt, nnzt = ops.trace(torch_ops.handle(b), dev(si), dev(ph), dev(P[:, 2]), dev(P[:, 3]))
    assert tt.is_cuda and nnzt == nnz
    assert np.array_equal(tt.cpu().numpy(), t) and np.array_equal(vt.cpu().numpy() != 0, v)
    rpt, git, gvt = ops.frechet_rows(torch_ops.handle(b), si.size, nnzt, 1)
    assert np.array_equal(rpt.numpy(), rp) and np.array_equal(git.numpy(), gi)
    assert np.array_equal(gvt.numpy(), gv)
    # LSQR on the valid rows
    keep = np.flatnonzero(v)
    rows = [(gi[rp[k] - 1:rp[k + 1] - 1], gv[rp[k] - 1:rp[k + 1] - 1]) for k in keep]
    srp = np.concatenate([[1], 1 + np.cumsum([r[0].size for r in rows])]).astype(np.int32)
    sgi = np.concatenate([r[0] for r in rows]).astype(np.int32)
    sgv = np.concatenate([r[1] for r in rows])
    _, nvp, npar = a.inv_index()
    for g in (a, b):
        g.set_frechet(keep.size, npar, srp, sgi, sgv)
    res = np.random.default_rng(4).normal(0.0, 0.05, keep.size)
    dm, it, rn, bn, t2 = a.lsqr(res, wdv=1.0, wdv_iface=1.0, w_smooth=3.0, w_smooth_iface=3.0,
                                eps_min=1e-6, max_iter=50)
    empty = torch.empty(0, dtype=torch.float64, device="cuda")
    dmt, itt, rnt, bnt, t2t = ops.lsqr(torch_ops.handle(b), dev(res), empty, empty, 1, 50, 1.0,
                                       1.0, 3.0, 3.0, 1e-6)
    assert dmt.is_cuda and itt == it and rnt == rn and bnt == bn and t2t == t2
    assert np.array_equal(dmt.cpu().numpy(), dm)
