"""Row-partitioned LSQR over several processes (smooth_type 1 layout).

The augmented system of run_lsqr (src/inversion2d.f90:6578-7167) with the
Laplacian smoothing and damping rows,

    [G; w_s L; w_d I] dm = [r; -w_s L dm_sum; -w_d dm_sum],

with G's rows split across the ranks by pick (each rank holds the Frechet
rows of its own sources, as the sources are shared out in multi-GPU runs)
and everything over the parameters (v, w, dm and the smoothing and damping
rows) replicated.  Each Golub-Kahan step needs G_r v on the local rows and
sum_r G_r^T u_r; the latter, together with each rank's |u_r|^2, is the one
all_reduce(SUM) of nparm + 1 values per iteration.  Because the norm of u is
known only after that reduction, u is scaled after G^T u is formed
((G^T u) / beta where run_lsqr forms G^T (u / beta)), so the iterates agree
with the single-process solve to rounding, not bit for bit.

The recurrences, the masking of inactive velocity columns (gtg < 0.01
eps_min), the test2 stopping rule (atol 1e-4) and the iteration count
follow run_lsqr (src/inversion2d.f90:6608-7157).  The products are passed
in: the local rows as two callables (G_r x, G_r^T y) and the Laplacian as one
(the reference applies the same operator for both products); laplacian_csr
builds that Laplacian (apply_laplacian_smooth_2d, :1161-1249) as a sparse
matrix.  Vectors are host arrays; the collective runs on the process group
given (gloo or NCCL via CPU tensors).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class DistLsqrResult:
    dm: np.ndarray
    iters: int
    rnorm: float
    bnorm: float
    test2: float


def laplacian_csr(inv_idx: np.ndarray, nparm: int, iface_start: int, iface_nx: int):
    """The smoothing operator of apply_laplacian_smooth_2d
    (src/inversion2d.f90:1161-1249) as a scipy CSR matrix: the 5-point
    Laplacian over the active velocity nodes of inv_idx ((nz, nx), 1-based
    parameter ids, 0 inactive) with -k on the diagonal for k active
    neighbours, plus the 1-D interface Laplacian over parameters
    iface_start+1 .. iface_start+iface_nx (one-sided at the ends)."""
    import scipy.sparse as sp
    inv = np.asarray(inv_idx)
    nz, nx = inv.shape
    rows, cols, vals = [], [], []
    nb = np.zeros((nz, nx))
    # neighbour pairs along x and along z: +1 both ways, each counted once
    for a, b in ((inv[:, :-1], inv[:, 1:]), (inv[:-1, :], inv[1:, :])):
        both = (a > 0) & (b > 0)
        i, j = a[both] - 1, b[both] - 1
        rows += [i, j]
        cols += [j, i]
        vals += [np.ones(i.size), np.ones(i.size)]
    act = inv > 0
    nb[:, :-1] += act[:, 1:]
    nb[:, 1:] += act[:, :-1]
    nb[:-1, :] += act[1:, :]
    nb[1:, :] += act[:-1, :]
    d = inv[act] - 1
    rows.append(d)
    cols.append(d)
    vals.append(-nb[act])
    # the interface nodes: one-sided at the ends, centred inside
    st, nxi = iface_start, iface_nx
    ix = np.arange(1, nxi + 1)
    idx = st + ix
    ok = (idx >= 1) & (idx <= nparm)
    first, last, mid = ok & (ix == 1), ok & (ix == nxi) & (ix != 1), ok & (ix > 1) & (ix < nxi)
    first &= st + 2 <= nparm
    for sel, offs, w in ((first, (1,), -1.0), (last, (-1,), -1.0), (mid, (-1, 1), -2.0)):
        r = idx[sel] - 1
        for o in offs:
            rows.append(r)
            cols.append(r + o)
            vals.append(np.ones(r.size))
        rows.append(r)
        cols.append(r)
        vals.append(np.full(r.size, w))
    rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    return sp.csr_matrix((vals, (rows, cols)), shape=(nparm, nparm))


def _allreduce_sum(vec: np.ndarray, group) -> np.ndarray:
    if group is None:
        return vec
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(vec))
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.numpy()


def lsqr_rows(g_local, gt_local, residual_local, nparm: int, n_vel_parms: int, lap,
              gtg_diag, dm_sum, *, eps_min: float, wdv: float, wdv_iface: float,
              w_smooth: float, w_smooth_iface: float, max_iter: int, group=None,
              atol: float = 1.0e-4) -> DistLsqrResult:
    """Solve the augmented system with this rank's rows of G.

    g_local(x) -> G_r x (this rank's rows), gt_local(y) -> G_r^T y, lap(v) ->
    L v; residual_local: this rank's rows of r; gtg_diag, dm_sum: replicated
    (nparm).  Every rank returns the same dm."""
    npm, nvp = int(nparm), int(n_vel_parms)
    gtg = np.asarray(gtg_diag, dtype=np.float64)
    dms = np.asarray(dm_sum, dtype=np.float64)
    masked = np.zeros(npm, bool)
    masked[:nvp] = gtg[:nvp] < eps_min * 0.01
    smooth = w_smooth > 0.0 or w_smooth_iface > 0.0
    damp = wdv > 0.0 or wdv_iface > 0.0

    def scale_s(o):
        o = o.copy()
        o[:nvp] = np.where(masked[:nvp], 0.0, w_smooth * o[:nvp])
        o[nvp:] = w_smooth_iface * o[nvp:]
        return o

    def damp_rows(x):
        o = np.zeros(npm)
        if damp:
            o[:nvp] = np.where(masked[:nvp], 0.0, wdv * x[:nvp])
            o[nvp:] = wdv_iface * x[nvp:]
        return o

    uG = np.asarray(residual_local, dtype=np.float64).copy()
    uL = -scale_s(lap(dms)) if smooth else np.zeros(npm)
    uD = -damp_rows(dms)

    def reduce_gt(u_g):
        """sum over ranks of [G_r^T u_g, |u_g|^2]: the iteration's one collective"""
        packed = np.empty(npm + 1)
        packed[:npm] = gt_local(u_g) if u_g.size else 0.0
        packed[npm] = float(np.dot(u_g, u_g))
        out = _allreduce_sum(packed, group)
        return out[:npm], out[npm]

    def at_rest(gtu, u_l, u_d):
        out = gtu.copy()
        if smooth:
            out = out + scale_s(lap(u_l))
        if damp:
            out[:nvp] = out[:nvp] + np.where(masked[:nvp], 0.0, wdv * u_d[:nvp])
            out[nvp:] = out[nvp:] + wdv_iface * u_d[nvp:]
        return out

    gt, ssq = reduce_gt(uG)
    bnorm = float(np.sqrt(ssq + np.dot(uL, uL) + np.dot(uD, uD)))
    dm = np.zeros(npm)
    if bnorm < 1.0e-30:
        return DistLsqrResult(dm, 0, 0.0, bnorm, 0.0)
    beta = bnorm
    uG, uL, uD = uG / beta, uL / beta, uD / beta
    v = at_rest(gt / beta, uL, uD)
    v[masked] = 0.0
    alpha = float(np.sqrt(np.dot(v, v)))
    if alpha < 1.0e-30:
        return DistLsqrResult(dm, 0, bnorm, bnorm, 0.0)
    v = v / alpha
    w = v.copy()
    phibar, rhobar, anorm2 = beta, alpha, alpha * alpha + beta * beta
    rnorm, test2 = 0.0, 0.0
    it = 1
    while it <= max_iter:
        v[masked] = 0.0
        uG = g_local(v) - alpha * uG
        uL = (scale_s(lap(v)) if smooth else np.zeros(npm)) - alpha * uL
        uD = damp_rows(v) - alpha * uD
        gt, ssq = reduce_gt(uG)
        beta = float(np.sqrt(ssq + np.dot(uL, uL) + np.dot(uD, uD)))
        if beta > 0.0:
            uG, uL, uD, gt = uG / beta, uL / beta, uD / beta, gt / beta
        v = at_rest(gt, uL, uD) - beta * v
        v[masked] = 0.0
        alpha = float(np.sqrt(np.dot(v, v)))
        if alpha > 0.0:
            v = v / alpha
        anorm2 = anorm2 + alpha * alpha + beta * beta
        rho = float(np.sqrt(rhobar * rhobar + beta * beta))
        c, s = rhobar / rho, beta / rho
        theta = s * alpha
        rhobar = -c * alpha
        phi = c * phibar
        phibar = s * phibar
        z = w.copy()
        z[masked] = 0.0
        w = v - (theta / rho) * w
        w[masked] = 0.0
        dm = dm + (phi / rho) * z
        rnorm = abs(phibar)
        arnorm = phibar * alpha * abs(c)
        test2 = arnorm / (np.sqrt(anorm2) * rnorm + 1.0e-30)
        if test2 < atol or 1.0 + test2 <= 1.0:
            break
        it += 1
    return DistLsqrResult(dm, it, rnorm, bnorm, float(test2))
