"""Run under torch.distributed.run with 2 CPU ranks (gloo): the benchmark's
replica plumbing (process group, barrier, max over ranks) without a GPU."""
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402

rank, world, local, pg = bench.dist_setup(2)
bench.barrier(pg)
worst = bench.dist_max(pg, 1.5 + rank)
bench.barrier(pg)
if rank == 0:
    print(json.dumps({"world": world, "max": worst}), flush=True)
pg.destroy_process_group()
