"""The multi-rank path of the bench on CPU: two gloo ranks (replicas, no
collective on the data path) agree on the job's time as the maximum over
ranks and count the units of every rank."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import sys

    import torch
    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        local = [100.0 + 50.0 * rank, 10.0 * (rank + 1)]  # ms: rank 1 is the slower one in both arms
        rates, mx = bench.job_rates(local, 1_000_000, 10)
        out[rank] = (rates, mx)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_job_rates_max_over_two_gloo_ranks():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    assert res[0] == res[1]
    rates, mx = res[0]
    assert mx == [150.0, 20.0]
    assert rates[0] == pytest.approx(2 * 1e6 * 10 / 0.150 / 1e6)
    assert rates[1] == pytest.approx(2 * 1e6 * 10 / 0.020 / 1e6)


def test_job_rates_single_process():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    rates, mx = bench.job_rates([200.0], 500_000, 4)
    assert mx == [200.0] and rates[0] == pytest.approx(500_000 * 4 / 0.2 / 1e6)
