"""Shared inputs of the tests: a sensitivity matrix G built from the oracle's
own ray rows (compute_frechet_for_ray2d restated) on a small model, so the
products and LSQR run on the sparsity pattern the reference produces."""
from __future__ import annotations

import numpy as np


def oracle_G(o, m, max_rows=None, phases=(1, 3)):
    """Trace the model's picks with the oracle and stack the valid rows as a
    1-based CSR (read_frechet_data2d's layout).  Returns
    (ndata, nparm, row_ptr, gindx, gval, t_calc, picks_used)."""
    from fmt2d_b200.api import phase_mask
    _, _, nparm = o.inv_idx()
    mask = phase_mask(phases)
    rows, tcal, used = [], [], []
    for s, sx in enumerate(m.obs_x):
        o.forward(s, sx, mask)
    for p in m.picks:
        s, ph, rx, rz = int(p[0]), int(p[1]), float(p[2]), float(p[3])
        if ph not in phases:
            continue
        r = o.trace(s, ph, rx, rz)
        if not r["valid"] or r["idx"].size == 0:
            continue
        rows.append((r["idx"], r["val"]))
        tcal.append(r["t"])
        used.append(p)
        if max_rows and len(rows) >= max_rows:
            break
    rp = np.zeros(len(rows) + 1, np.int32)
    rp[0] = 1
    for i, (ix, _) in enumerate(rows):
        rp[i + 1] = rp[i] + ix.size
    gindx = np.concatenate([ix for ix, _ in rows]).astype(np.int32)
    gval = np.concatenate([v for _, v in rows])
    return len(rows), nparm, rp, gindx, gval, np.array(tcal), np.array(used)


def random_G(ndata, nparm, nnz_row, seed):
    """Ray-like random rows: runs of neighbouring columns with positive
    lengths (1-based CSR)."""
    rng = np.random.default_rng(seed)
    rp = np.ones(ndata + 1, np.int32)
    idx, val = [], []
    for i in range(ndata):
        k = max(1, int(rng.integers(nnz_row // 2, 3 * nnz_row // 2 + 1)))
        start = int(rng.integers(0, max(1, nparm - 4 * k)))
        cols = np.unique(start + np.cumsum(rng.integers(1, 5, size=k))) % nparm
        cols = np.unique(cols)
        idx.append(cols + 1)
        val.append(rng.uniform(0.01, 0.3, size=cols.size))
        rp[i + 1] = rp[i] + cols.size
    return ndata, nparm, rp, np.concatenate(idx).astype(np.int32), np.concatenate(val)


def csr_to_scipy(ndata, nparm, rp, gindx, gval):
    import scipy.sparse as sp
    return sp.csr_matrix((gval, gindx - 1, rp - 1), shape=(ndata, nparm))


def ref_ops(o, G, nvp, mask, ws_v, ws_i, wd_v, wd_i):
    """The reference's augmented operator pair as a SciPy LinearOperator plus
    the smoothing and damping weights per parameter."""
    from scipy.sparse.linalg import LinearOperator
    nd, npar = G.shape
    m_all = np.concatenate([mask, np.zeros(npar - nvp, bool)])
    vel = np.arange(npar) < nvp
    ws = np.where(vel, np.where(m_all, 0.0, ws_v), ws_i)
    wd = np.where(vel, np.where(m_all, 0.0, wd_v), wd_i)
    keep = ~m_all

    def mv(x):
        x = np.where(keep, x.ravel(), 0.0)
        return np.concatenate([G @ x, ws * o.laplacian(npar, x), wd * x])

    def rmv(u):
        u = u.ravel()
        y = G.T @ u[:nd] + ws * o.laplacian(npar, u[nd:nd + npar]) + wd * u[nd + npar:]
        return np.where(keep, y, 0.0)

    return LinearOperator((nd + 2 * npar, npar), matvec=mv, rmatvec=rmv, dtype=np.float64), ws, wd


def lsqr_problem(pyoracle, seed=5):
    """A damped, smoothed LSQR problem on the small model for the partitioned
    solver's tests: the oracle's rays give G (rows tagged with their source),
    seeded residuals and dm_sum, gtg = the column sums of G^2."""
    from fmt2d_b200 import synth
    m = synth.small_model()
    o = pyoracle.Oracle(m)
    nd, npar, rp, gi, gv, _, used = oracle_G(o, m)
    inv, nvp, _ = o.inv_idx()
    rng = np.random.default_rng(seed)
    G = csr_to_scipy(nd, npar, rp, gi, gv)
    gtg = np.asarray(G.multiply(G).sum(axis=0)).ravel()
    return dict(o=o, nd=nd, npar=npar, nvp=nvp, inv=inv, rp=rp, gi=gi, gv=gv,
                src=used[:, 0].astype(int), res=rng.normal(0.0, 0.05, nd),
                dm_sum=rng.normal(0.0, 1e-3, npar), gtg=gtg,
                weights=dict(eps_min=1e-4 * float(gtg.max()), wdv=1.0, wdv_iface=0.5,
                             w_smooth=10.0, w_smooth_iface=3.0))
