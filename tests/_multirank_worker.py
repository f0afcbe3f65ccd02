"""Worker for test_multirank.py (run under torch.distributed.run with gloo on
CPU): the replica plumbing of bench.py -- per-rank streams and the
max-over-ranks timing -- with two ranks."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "torch-admp_b200")):
    sys.path.insert(0, p)

import torch.distributed as dist  # noqa: E402

import bench  # noqa: E402


def main():
    dist.init_process_group("gloo")
    rank, world, _ = bench.rank_info()
    local_ms = 10.0 * (rank + 1)            # rank r "took" 10 (r + 1) ms
    worst = bench.max_over_ranks(local_ms)
    stream = bench.rank_stream(8, rank)
    first = [int(r.natoms) for r in stream[:4]]
    gathered = [None] * world
    dist.all_gather_object(gathered, first)
    # one file per rank: the ranks share stdout, where their lines may interleave
    with open(os.path.join(sys.argv[1], f"rank{rank}.json"), "w") as f:
        json.dump({"rank": rank, "world": world, "max_ms": worst, "streams": gathered}, f)
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
