"""The accuracy oracle (oracle/jk_accuracy.c, one-sided hyperbolic Jacobi in __float128 and
long double) on the CPU: the two precisions agree, the FP64 restatement of the reference's
loop reaches the extended-precision values to 1e-12 relative per J sign class, and the
committed fixture agrees with a fresh computation."""
import os

import numpy as np
import pytest

import oracle
from jkogb_b200 import gen

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sigma_ref.npz")


@pytest.mark.parametrize("kind,n,seed", [("g", 16, 1), ("g", 48, 2), ("r", 40, 3), ("z", 24, 4), ("z", 40, 5)])
def test_fp64_loop_within_1e12_of_quad(kind, n, seed):
    if kind == "g":
        Y, J = gen.graded(n, 1e-6, seed=seed)
    elif kind == "r":
        Y, J = gen.gaussian(n, seed=seed)
    else:
        Y, J = gen.complex_gaussian(n, seed=seed)
    sq, _ = oracle.accurate_sigma(Y, J, "q")
    sl, _ = oracle.accurate_sigma(Y, J, "ld")
    assert oracle.sigma_rel_err(sl, sq, J) < 1e-15
    o = oracle.step_loop(Y, J, nt=1)
    assert o["info"] > 0
    assert oracle.sigma_rel_err(o["sigma"], sq, J) < 1e-12


def test_quad_recovers_prescribed_values():
    """On a small prescribed matrix (moderate grading) the oracle returns the prescribed
    values up to the rounding of the matrix's construction."""
    sig, J = gen.prescribed_graded_sigma(32, 1e-3, seed=9)
    Y, _ = gen.prescribed_graded(32, 1e-3, seed=9)
    s, _ = oracle.accurate_sigma(Y, J, "q")
    assert oracle.sigma_rel_err(s, sig, J) < 1e-11


def test_fixture_reproduces():
    ref = np.load(GOLD)
    Y, J = gen.gaussian(256, seed=1, n_plus=192)
    s, _ = oracle.accurate_sigma(Y, J, "ld")
    assert str(ref["djk_n256__precision"]) == "q"
    assert oracle.sigma_rel_err(s, ref["djk_n256"], J) < 1e-15
