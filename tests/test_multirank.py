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
