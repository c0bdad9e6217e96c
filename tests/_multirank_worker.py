"""One rank of the world-size-2 test of bench.py's multi-rank plumbing (launched by
tests/test_multirank.py through torch.distributed.run, gloo on CPU)."""
import datetime
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import torch.distributed as dist  # noqa: E402

import bench  # noqa: E402


def main():
    rank, local_rank, world = bench.dist_env()
    assert world == 2 and rank == local_rank
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    # the slowest replica defines the job's time
    assert bench.reduce_max(1.5 + rank, world, "cpu") == 2.5
    bench.barrier(world)
    # every rank times the precision rank 0 chose
    assert bench.broadcast_choice("bf16x3" if rank == 0 else "fp32", world) == "bf16x3"
    bench.barrier(world)
    dist.destroy_process_group()
    print(f"rank {rank} ok")


if __name__ == "__main__":
    main()
