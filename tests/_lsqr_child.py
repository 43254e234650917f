"""One rank of the world-size-2 row-partitioned LSQR test (launched by
torch.distributed.run on gloo): every rank builds the same sensitivity rows
from the oracle's rays on the small model, keeps the rows of its own sources
(source index modulo the world size) and solves with
fmt2d_b200.dist_lsqr.lsqr_rows; each rank writes its result to
argv[1]/lsqr_rank<r>.npz."""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402
import torch.distributed as dist  # noqa: E402

import bench  # noqa: E402
import pyoracle  # noqa: E402
from _cases import csr_to_scipy, lsqr_problem  # noqa: E402
from fmt2d_b200.dist_lsqr import laplacian_csr, lsqr_rows  # noqa: E402

world, rank, _ = bench.dist_setup(2)
P = lsqr_problem(pyoracle)
G = csr_to_scipy(P["nd"], P["npar"], P["rp"], P["gi"], P["gv"])
mine = np.flatnonzero(P["src"] % world == rank)
Gr = G[mine]
L = laplacian_csr(P["inv"], P["npar"], P["nvp"], P["npar"] - P["nvp"])
out = {}
for max_iter in (40, 2000):
    r = lsqr_rows(lambda x: Gr @ x, lambda y: Gr.T @ y, P["res"][mine], P["npar"], P["nvp"],
                  lambda v: L @ v, P["gtg"], P["dm_sum"], max_iter=max_iter,
                  group=dist.group.WORLD, **P["weights"])
    out[f"dm{max_iter}"] = r.dm
    out[f"it{max_iter}"] = r.iters
    out[f"rn{max_iter}"] = r.rnorm
np.savez(os.path.join(sys.argv[1], f"lsqr_rank{rank}.npz"), rows=mine.size, **out)
dist.destroy_process_group()
