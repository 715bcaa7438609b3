"""Multi-rank host logic on CPU (gloo, world size 2): bench.py runs one
replica volume per GPU with no collective on the data path; the ranks meet
only for the barrier and the max-over-ranks timing, checked here with the
same helper over gloo."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as tmp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, outdir):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    # each replica reports its own time; all must see the slowest
    got = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
    dist.barrier()
    with open(os.path.join(outdir, f"r{rank}"), "w") as f:
        f.write(repr(got))
    dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks(tmp_path):
    port = _free_port()
    tmp.spawn(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    vals = [float(open(tmp_path / f"r{r}").read()) for r in range(2)]
    assert vals == [15.0, 15.0]


def test_single_rank_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
