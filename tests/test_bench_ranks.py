"""bench.py's multi-rank plumbing on CPU: two gloo ranks through dist_setup,
barrier, max_over_ranks and sum_over_ranks (the replica runs of
`bench.py --gpus N` time each rank on its own data and report
sum(rows) / max(time))."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist

    r, w, local = bench.dist_setup()
    assert (r, w, local) == (rank, world, rank)
    assert dist.get_backend() == "gloo"
    bench.barrier(w)
    mx = bench.max_over_ranks(1.5 + 2.0 * rank, w)     # per-rank "times"
    sm = bench.sum_over_ranks(1000 * (rank + 1), w)    # per-rank "rows"
    with open(os.path.join(out_dir, "rank%d.txt" % rank), "w") as f:
        f.write("%r %r\n" % (mx, sm))
    dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    for rank in range(world):
        mx, sm = open(tmp_path / ("rank%d.txt" % rank)).read().split()
        assert float(mx) == 1.5 + 2.0 * (world - 1)
        assert float(sm) == 1000 * sum(range(1, world + 1))


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.25, 1) == 3.25
    assert bench.sum_over_ranks(7, 1) == 7
