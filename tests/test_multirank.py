"""The multi-process path of bench.py on the host: two ranks launched by
torch.distributed.run (as for `bench.py --gpus 2`), the process group on
gloo, the step time reduced as the max over ranks, the sources shared out
(each rank its own 30), and the reference arm printing its one JSON line
from rank 0 only."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _torchrun(args, timeout):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={_port()}"] + args
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True,
                          timeout=timeout)


def _json_lines(out: str):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


def test_max_over_ranks_gloo(tmp_path):
    r = _torchrun([os.path.join("tests", "_rank_child.py"), str(tmp_path)], timeout=240)
    assert r.returncode == 0, r.stderr[-2000:]
    rows = [json.load(open(tmp_path / f"rank{k}.json")) for k in range(2)]
    assert [d["rank"] for d in rows] == [0, 1]
    assert all(d["world"] == 2 and d["backend"] == "gloo" for d in rows)
    assert all(d["max_ms"] == 15.0 for d in rows)
    # each rank solves its own sources: 30 per rank, 60 distinct in all
    a, b = (set(round(x, 6) for x in d["src"]) for d in rows)
    assert len(a) == len(b) == 30 and not (a & b)


def test_reference_arm_two_ranks():
    r = _torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
                   "--warmup", "0"], timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    rows = _json_lines(r.stdout)
    assert len(rows) == 1, r.stdout
    d = rows[0]
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"


# rounding of the differently ordered sums grows over the iterations: 40
# iterations agree to 1e-8 of max|dm|, a converged solve (~200 iterations, the
# same count) to 1e-5
TOL = {40: 1e-8, 2000: 1e-5}


def _oracle_lsqr(P, max_iter):
    w = P["weights"]
    return P["o"].lsqr(P["nd"], P["npar"], P["gi"], P["gv"], P["rp"], P["res"], P["gtg"],
                       P["dm_sum"], w["eps_min"], w["wdv"], w["wdv_iface"], w["w_smooth"],
                       w["w_smooth_iface"], max_iter)


def test_partitioned_lsqr_one_process(oracle_lib):
    """fmt2d_b200.dist_lsqr on one process (all rows, no collective): its
    Laplacian is apply_laplacian_smooth_2d's, and its iterates are run_lsqr's
    (the oracle's restatement) to rounding."""
    import numpy as np
    from _cases import csr_to_scipy, lsqr_problem
    from fmt2d_b200.dist_lsqr import laplacian_csr, lsqr_rows
    P = lsqr_problem(oracle_lib)
    L = laplacian_csr(P["inv"], P["npar"], P["nvp"], P["npar"] - P["nvp"])
    v = np.random.default_rng(2).normal(size=P["npar"])
    ref = P["o"].laplacian(P["npar"], v)
    assert np.max(np.abs(L @ v - ref)) <= 1e-12 * np.max(np.abs(ref))
    G = csr_to_scipy(P["nd"], P["npar"], P["rp"], P["gi"], P["gv"])
    for max_iter in (40, 2000):
        r = lsqr_rows(lambda x: G @ x, lambda y: G.T @ y, P["res"], P["npar"], P["nvp"],
                      lambda x: L @ x, P["gtg"], P["dm_sum"], max_iter=max_iter, **P["weights"])
        dm, it, rn, _ = _oracle_lsqr(P, max_iter)
        assert r.iters == it
        assert np.max(np.abs(r.dm - dm)) <= TOL[max_iter] * np.max(np.abs(dm))
        assert abs(r.rnorm - rn) <= TOL[max_iter] * rn


def test_partitioned_lsqr_two_ranks(oracle_lib, tmp_path):
    """Two gloo ranks, each with the rows of its own sources and one
    all_reduce of [G_r^T u_r, |u_r|^2] per iteration: both ranks return the
    same dm, equal to the single-process run_lsqr's to rounding."""
    import numpy as np
    from _cases import lsqr_problem
    r = _torchrun([os.path.join("tests", "_lsqr_child.py"), str(tmp_path)], timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    a, b = (np.load(tmp_path / f"lsqr_rank{k}.npz") for k in range(2))
    P = lsqr_problem(oracle_lib)
    assert int(a["rows"]) > 0 and int(b["rows"]) > 0 and int(a["rows"]) + int(b["rows"]) == P["nd"]
    for max_iter in (40, 2000):
        k = f"dm{max_iter}"
        assert np.array_equal(a[k], b[k])
        dm, it, rn, _ = _oracle_lsqr(P, max_iter)
        assert int(a[f"it{max_iter}"]) == it
        assert np.max(np.abs(a[k] - dm)) <= TOL[max_iter] * np.max(np.abs(dm))
