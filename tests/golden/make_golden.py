"""Golden vectors for the small test model, written by the oracle (the FP64
restatement of the reference path in oracle/).  The reference is Fortran and
no Fortran compiler exists where this build runs, so these vectors come from
the oracle, not from the reference binary: they pin the oracle against
drift and give the device tests fixed expected values.

    python tests/golden/make_golden.py      # rewrites tests/golden/small_model.npz

Contents (synth.small_model(), both OBS, Pg + PmP):
  T_<s>_<tf>        traveltimes of time fields 1, 4, 5 (region node order)
  pick_*            picks (source, phase, x, z) and their t_calc / valid
  row_ptr, gindx, gval   their Frechet rows (1-based CSR, invalid picks empty)
  ls_*              an LSQR solve on the rows of the first 40 valid picks
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)

OUT = os.path.join(HERE, "small_model.npz")
PHASES = (1, 3)
TFS = (1, 4, 5)
LSQR = dict(wdv=0.5, wdv_iface=0.5, w_smooth=3.0, w_smooth_iface=3.0, max_iter=40)


def generate() -> dict:
    import pyoracle
    from fmt2d_b200 import synth
    from fmt2d_b200.api import phase_mask
    from _cases import oracle_G, csr_to_scipy
    pyoracle.build()
    m = synth.small_model()
    o = pyoracle.Oracle(m)
    mask = phase_mask(PHASES)
    out = {}
    for s, sx in enumerate(m.obs_x):
        o.forward(s, sx, mask)
        for tf in TFS:
            out[f"T_{s}_{tf}"] = o.field(s, tf)[0]
    pk = m.picks[np.isin(m.picks[:, 1], PHASES)]
    t, valid, idx, val = [], [], [], []
    for p in pk:
        r = o.trace(int(p[0]), int(p[1]), float(p[2]), float(p[3]))
        t.append(r["t"] if r["valid"] else 0.0)
        valid.append(r["valid"])
        idx.append(r["idx"] if r["valid"] else np.zeros(0, np.int32))
        val.append(r["val"] if r["valid"] else np.zeros(0))
    rp = np.concatenate([[1], 1 + np.cumsum([a.size for a in idx])]).astype(np.int32)
    out.update(pick_src=pk[:, 0].astype(np.int32), pick_phase=pk[:, 1].astype(np.int32),
               pick_x=pk[:, 2], pick_z=pk[:, 3], pick_t=np.array(t), pick_valid=np.array(valid),
               row_ptr=rp, gindx=np.concatenate(idx).astype(np.int32), gval=np.concatenate(val))
    nd, npar, lrp, lgi, lgv, _, _ = oracle_G(o, m, max_rows=40, phases=PHASES)
    G = csr_to_scipy(nd, npar, lrp, lgi, lgv)
    rng = np.random.default_rng(11)
    r = rng.normal(0.0, 0.05, nd)
    dm_sum = rng.normal(0.0, 0.01, npar)
    gtg = np.asarray(G.multiply(G).sum(axis=0)).ravel()
    eps_min = max(1e-6, 1e-4 * gtg.max())
    dm, it, rn, t2 = o.lsqr(nd, npar, lgi, lgv, lrp, r, gtg, dm_sum, eps_min, LSQR["wdv"],
                            LSQR["wdv_iface"], LSQR["w_smooth"], LSQR["w_smooth_iface"],
                            LSQR["max_iter"])
    out.update(ls_nparm=np.int64(npar), ls_row_ptr=lrp, ls_gindx=lgi, ls_gval=lgv, ls_residual=r,
               ls_dm_sum=dm_sum, ls_gtg=gtg, ls_eps_min=np.float64(eps_min), ls_dm=dm,
               ls_iters=np.int64(it), ls_rnorm=np.float64(rn))
    return out


if __name__ == "__main__":
    d = generate()
    np.savez_compressed(OUT, **d)
    print(f"wrote {OUT}: {len(d)} arrays, {os.path.getsize(OUT) / 1024:.0f} KiB")
