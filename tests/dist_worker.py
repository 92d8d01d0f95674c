"""Worker of tests/test_multirank_cpu.py, launched by torch.distributed.run with the gloo backend:
runs the bench's multi-rank helpers (rank setup, max-over-ranks timing, whole-job rate) and prints
one JSON line per rank."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def main():
    rank, world, local = bench.dist_setup(2, backend="gloo")
    slowest = bench.max_over_ranks(1.0 + 0.5 * rank, world, local)
    bench.barrier(world)
    rate = bench.whole_job_rate(world, 1000, 10, slowest)
    print(json.dumps({"rank": rank, "world": world, "max_seconds": slowest, "rate": rate}), flush=True)
    import torch.distributed as dist
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
