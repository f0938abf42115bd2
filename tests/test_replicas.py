"""Replica bookkeeping of bench runs with N > 1 (max over ranks, whole-job rate),
run as two gloo ranks on the CPU."""
import os
import socket

import torch.multiprocessing as mp

from rqcopt_hpc_b200.replicas import whole_job_rate


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from rqcopt_hpc_b200.replicas import max_over_ranks, world_size
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    # rank r took 100 + 50 r ms device time and 200 - 10 r ms end to end
    m = max_over_ranks([100.0 + 50 * rank, 200.0 - 10 * rank])
    out[rank] = (world_size(), m[0], m[1])
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    assert res[0] == res[1] == (2, 150.0, 200.0)
    # whole-job throughput: 2 ranks x 3 steps over the slowest rank's 150 ms
    assert abs(whole_job_rate(2, 3, 150.0) - 40.0) < 1e-12


def test_single_rank_is_identity():
    from rqcopt_hpc_b200.replicas import max_over_ranks, world_size
    assert world_size() == 1
    assert max_over_ranks([1.5, 2.5]) == [1.5, 2.5]
