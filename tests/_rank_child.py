"""One rank of the world-size-2 host test (launched by torch.distributed.run):
sets up the process group the way bench.py does, reduces a per-rank time
with max-over-ranks, takes its share of the sources and writes rank<r>.json
into the folder given as argv[1]."""
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import torch  # noqa: E402

import bench  # noqa: E402

world, rank, local = bench.dist_setup(2)
ms = bench.max_over_ranks(10.0 + 5.0 * rank, world, torch.device("cpu"))
from fmt2d_b200 import synth  # noqa: E402

src = bench.source_set(synth.config(1), rank, world)
bench.barrier(world)
import torch.distributed as dist  # noqa: E402

backend = dist.get_backend()
dist.destroy_process_group()
with open(os.path.join(sys.argv[1], f"rank{rank}.json"), "w") as f:
    json.dump({"rank": rank, "world": world, "local": local, "max_ms": ms,
               "backend": backend, "src": src.tolist()}, f)
