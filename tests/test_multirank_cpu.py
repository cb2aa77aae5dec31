"""The multi-rank paths on CPU: gloo ranks over 127.0.0.1.  The job's time is the maximum
over ranks; one batch of matrices is partitioned over the ranks by estimated cost (the
longest-processing-time rule on N^4), each rank solves its share and rank 0 gathers the
per-matrix results back into the batch's order.  The ranks solve with the oracle here,
so the test needs no GPU."""
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


def _oracle_solve(mats, Js):
    import oracle
    out = []
    for Y, J in zip(mats, Js):
        r = oracle.step_loop(Y, J, nt=1)
        out.append((int(r["info"]), r["sigma"].copy()))
    return out


def _rank(rank, world, port, out):
    from datetime import timedelta

    import torch.distributed as dist

    import bench
    from jkogb_b200 import gen, partition
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    t = bench.max_over_ranks(10.0 * rank + 1.0)
    b = gen.batch(9, 8, 24, seed=11)
    res, share = partition.solve_partitioned([Y for Y, _ in b], [J for _, J in b], _oracle_solve)
    out[rank] = (t, [int(i) for i in share], res)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_partitioned_batch():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 11.0            # the slowest rank's time on every rank
    s0, s1 = set(res[0][1]), set(res[1][1])
    assert s0 and s1 and not (s0 & s1) and (s0 | s1) == set(range(9))  # disjoint shares, the whole batch
    assert res[1][2] is None                         # only rank 0 gathers
    from jkogb_b200 import gen
    b = gen.batch(9, 8, 24, seed=11)
    direct = _oracle_solve([Y for Y, _ in b], [J for _, J in b])
    got = res[0][2]
    assert len(got) == 9
    for (i1, s1_), (i2, s2_) in zip(got, direct):   # the batch's order, the results of solving each alone
        assert i1 == i2 and np.array_equal(s1_, s2_)


def test_partition_balance_on_the_batch_workload():
    from jkogb_b200 import gen, partition
    ns = [Y.shape[0] for Y, _ in gen.batch(4096, 16, 128, seed=4)]
    for world in (1, 2, 4, 8):
        shares = partition.partition(ns, world)
        allidx = np.concatenate(shares)
        assert np.array_equal(np.sort(allidx), np.arange(len(ns)))   # every matrix exactly once
        assert partition.imbalance(shares, ns) < 1.002                # estimated costs within 0.2%


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
