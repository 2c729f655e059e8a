"""One rank of the multi-rank bench checks, launched by torch.distributed.run
with the gloo backend on CPU (tests/test_multirank.py).

Each rank renders nothing: it feeds its own stand-in step times through the
bench's reduction helpers and writes what it saw to <out_dir>/rank<k>.json.
"""
import datetime
import json
import os
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import torch.distributed as dist  # noqa: E402

import bench  # noqa: E402


def main():
    out_dir = Path(sys.argv[1])
    rank, world, local = bench._dist_env()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    # rank k "took" 1.0 + k seconds; the slowest rank sets the job time
    dev_s = bench.max_over_ranks(1.0 + rank, dist, "cpu")
    # a second reduction in the same order on every rank (the e2e leg)
    e2e_s = bench.max_over_ranks(0.25 * (world - rank), dist, "cpu")
    value = bench.whole_job_rate(2_000_000, world, dev_s)
    dist.barrier()
    (out_dir / f"rank{rank}.json").write_text(json.dumps(
        {"rank": rank, "world": world, "local": local, "dev_s": dev_s, "e2e_s": e2e_s, "value": value}))
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
