"""Bit parity with the oracle at the benchmark configurations, on bounded prefixes of the
solve: the N = 2048 graded matrix (J 1024/1024 in a seeded permutation, N_2 = 1024), the
complex N = 1024 matrix (J 512/512, N_2 = 512) and the N = 4096 graded matrix with
column scales down to 1e-10 (J 2048/2048, N_2 = 2048).  The GPU stops at the step limit
(max_steps = K, INFO JK_ERR_MAX_STEPS) exactly where the oracle stops after K steps
(stop_after = K); A, U, Z, SIGMA and every step's pivot list must agree bit for bit.
The full solves take 10^4 steps and more, far beyond what the oracle can run here."""
import os

import numpy as np
import pytest

import oracle
from jkogb_b200 import gen

pytestmark = pytest.mark.gpu

NT = os.cpu_count() or 1


def _jk():
    import jkogb_b200 as jk
    jk.lib()
    return jk


def _same(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    if a.shape != b.shape:
        return False
    fa, fb = a.view(np.float64), b.view(np.float64)
    na, nb = np.isnan(fa), np.isnan(fb)
    return np.array_equal(na, nb) and np.array_equal(np.where(na, 0.0, fa).view(np.uint64),
                                                      np.where(nb, 0.0, fb).view(np.uint64))


PREFIXES = [
    # (name, generator, N_2, steps K)
    ("djk_n2048_graded", lambda: gen.graded(2048, 1e-6, seed=2), 1024, 12),
    ("zjk_n1024", lambda: gen.complex_gaussian(1024, seed=3), 512, 3),
    ("djk_n4096_graded", lambda: gen.graded(4096, 1e-10, seed=5, random_signs=False), 2048, 2),
]


@pytest.mark.parametrize("name,make,n_2,k", PREFIXES, ids=[p[0] for p in PREFIXES])
def test_headline_prefix_bitexact(name, make, n_2, k):
    jk = _jk()
    Y, J = make()
    g = jk.step_loop(Y, J, n_2=n_2, max_steps=k, trace=True, trace_steps=k + 2, trace_piv=(k + 2) * n_2)
    o = oracle.step_loop(Y, J, n_2=n_2, nt=NT, stop_after=k, trace=True, max_steps=k + 2,
                         max_piv=(k + 2) * n_2)
    assert o["info"] == k and g["info"] == -24
    tg, to = g["trace"], o["trace"]
    assert np.array_equal(tg["sl"], to["sl"]) and np.array_equal(tg["nl"], to["nl"])
    assert np.array_equal(tg["piv"], to["piv"])
    for key in ("A", "U", "Z", "sigma"):
        assert _same(g[key], o[key]), key


def test_complex_weights_n1024_bitexact():
    """The complex weights at the complex workload's order, through k_absmat and the
    pipelined sign-class tiles of k_hyp_z_pm (the production path at N = 1024), on the
    input and after a few steps."""
    jk = _jk()
    Y, J = gen.complex_gaussian(1024, seed=3)
    A = jk.step_loop(Y, J, n_2=512, max_steps=2)["A"]
    for X in (Y, A):
        W = jk.weights(X, J)
        w, P, Q, tt = oracle.weights(X, J, id_tru=1, nt=NT)
        got = W[P - 1, Q - 1]
        assert np.array_equal(np.isnan(got), np.isnan(w))
        m = ~np.isnan(w)
        assert _same(got[m], w[m])


def test_complex_weights_partial_tiles_bitexact():
    """The pipelined complex tiles with partial tiles in both directions and both pair
    orientations: N = 700 with 300 "+" signs in a seeded permutation, and a column scaled
    down so that rotated entries leave the range of the multiplication-scaled hypot."""
    jk = _jk()
    Y, J = gen.complex_gaussian(700, seed=4, n_plus=300)
    J = J[np.random.default_rng(6).permutation(700)]
    Y[:, 5] *= 1e-305
    Y[:, 9] *= 1e300
    W = jk.weights(Y, J)
    w, P, Q, tt = oracle.weights(Y, J, id_tru=1, nt=NT)
    got = W[P - 1, Q - 1]
    assert np.array_equal(np.isnan(got), np.isnan(w))
    m = ~np.isnan(w)
    assert _same(got[m], w[m])
