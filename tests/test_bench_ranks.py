"""The bench's multi-GPU bookkeeping (replicas, max over ranks, whole-job rate)
on two gloo ranks on CPU; the GPU part is one independent replica per rank."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    # rank r pretends its timed region took (r+1) * 10 ms and its e2e loop (r+1) s
    total_ms, e2e_s = bench.max_over_ranks(dist, [10.0 * (rank + 1), 1.0 * (rank + 1)])
    ms, value, e2e = bench.whole_job_rates(world, 5, total_ms, 4, e2e_s)
    a, b = bench.inputs(1 + rank)
    out[rank] = (total_ms, e2e_s, ms, value, e2e, int(a[0]), int(b[0]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_and_whole_job_rate():
    import bench

    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][:5] == res[1][:5], "ranks must report identical aggregated numbers"
    total_ms, e2e_s, ms, value, e2e = res[0][:5]
    assert total_ms == 20.0 and e2e_s == 2.0          # the slowest rank
    assert ms == pytest.approx(4.0)
    assert value == pytest.approx(2 * bench.N_OUT / 4e-3 / 1e6)   # both replicas' output over the max time
    assert e2e == pytest.approx(2 * bench.N_OUT * 4 / 2.0 / 1e6)
    assert res[0][5:] != res[1][5:], "each rank works on its own replica inputs"
