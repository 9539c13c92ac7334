"""One rank of the CPU multi-process test (gloo): the bench's process-group
plumbing and its dealing of independent units to ranks.  Prints one JSON
line."""
import json
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), ".."))
import bench  # noqa: E402


def main():
    ws, rank, local = bench.dist_init()
    import torch.distributed as dist
    mine = bench.rank_share(int(sys.argv[1]), ws, rank)
    gathered = [None] * ws
    dist.all_gather_object(gathered, mine)
    bench.barrier(ws)
    out = {"rank": rank, "ws": ws, "max": bench.allmax(ws, float(rank + 1)),
           "sum": bench.allsum(ws, float(10 * (rank + 1))), "units": gathered}
    dist.destroy_process_group()
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
