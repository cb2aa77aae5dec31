"""Host-side helpers that need no GPU: the packed layout of the batched solver and the
workload generators' documented properties."""
import numpy as np

import jkogb_b200 as jk
from jkogb_b200 import gen


def test_batch_pack_round_trip_and_offsets():
    b = gen.batch(7, 16, 40, seed=3)
    mats = [Y for Y, _ in b]
    Js = [J for _, J in b]
    A, J, n, off = jk.batch_pack(mats, Js)
    assert off[0] == 0 and all(off[m + 1] - off[m] == n[m] ** 2 for m in range(len(n)))
    assert A.size == off[-1] and J.size == int(np.sum(n)) and J.dtype == np.int32
    for Y, Z in zip(mats, jk.batch_unpack(A, n, off)):
        assert np.array_equal(Y, Z)


def test_batch_generator_properties():
    b = gen.batch(64, 16, 128, seed=4)
    ns = np.array([Y.shape[0] for Y, _ in b])
    assert np.all(ns % 2 == 0) and ns.min() >= 16 and ns.max() <= 128
    for Y, J in b:
        assert set(np.unique(J)) <= {-1, 1}
        assert Y.flags.f_contiguous


def test_graded_generator_scales():
    Y, J = gen.graded(64, 1e-6, seed=2)
    norms = np.linalg.norm(Y, axis=0)
    assert norms.max() / norms.min() > 1e3
    assert int(np.sum(J == 1)) == 32 and int(np.sum(J == -1)) == 32


def test_bench_recorded_traffic():
    """bench.py's roofline takes the weight kernel's DRAM bytes per launch from the committed ncu
    captures: the cold-cache figure and the one with the cache as a build leaves it."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    cold, warm = bench._recorded_traffic("djk_n2048_graded")
    assert cold is not None and warm is not None and 0 < warm < cold
    assert bench._recorded_traffic("no_such_workload") == (None, None)
