"""The multi-rank plumbing of the benchmark on CPU: two gloo ranks over 127.0.0.1.  The
job's time is the maximum over ranks, and the batched workload gives every rank its own
batch (the ranks partition the job; no collective touches the data)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    from datetime import timedelta

    import torch.distributed as dist

    import bench
    from jkogb_b200 import gen
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    t = bench.max_over_ranks(10.0 * rank + 1.0)
    b = gen.batch(3, 16, 32, seed=bench.rank_batch_seed(rank))
    out[rank] = (t, float(np.sum(b[0][0])))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_time_and_partition():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 11.0      # the slowest rank's time on every rank
    assert res[0][1] != res[1][1]              # different batches on different ranks


def test_single_process_max_is_identity():
    import bench
    assert bench.max_over_ranks(3.5) == 3.5


def test_clock_summary_parses_samples():
    import bench

    class _Done:
        def terminate(self):
            pass

        def wait(self, t):
            pass

    import tempfile
    fd, name = tempfile.mkstemp(suffix=".csv")
    os.close(fd)
    f = open(name, "w")
    f.write("0, 1965, 1965, 500.0, 0x0, Not Active, Not Active, Not Active, Active\n")
    f.write("0, 1900, 1965, 900.0, 0x4, Not Active, Active, Not Active, Not Active\n")
    c = bench._clock_summary(_Done(), f)
    assert c["sm_mhz"] == 1932.5 and c["sm_max_mhz"] == 1965.0
    assert c["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
