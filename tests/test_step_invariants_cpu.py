"""The oracle's row and column transformations (BA / AB of DSTEP_TRANSF, src/D/dstep.F90:301-346,
src/Z/zstep.F90) against what they must preserve, after every prefix of a solve.  The loop
keeps Y = U A Z^-1 with U unitary and Z J-unitary (U accumulates the left 2x2 factors, Z the
right ones); a loop stopped after K steps is returned in the finished form (SIGMA the
diagonal, the diagonal of A zeroed, Z := J Z^H J as JZTJ / JZHJ do), so
Y = U (A + diag(SIGMA)) Z, U^H U = I and Z^H J Z = J.  Checked after 1, 2, 5 and 20 steps on
real and complex inputs, to a few units of roundoff (the full solves are checked the same way
at the end, and against the accuracy oracle's sigma, in the accuracy tests)."""
import numpy as np
import pytest

import oracle
from jkogb_b200 import gen


@pytest.mark.parametrize("kind", ["d", "z"])
def test_prefix_reconstruction_and_factors(kind):
    if kind == "d":
        Y, J = gen.graded(26, 1e-4, seed=51)
    else:
        Y, J = gen.complex_gaussian(20, seed=52, n_plus=8)
        J = J[np.random.default_rng(4).permutation(20)]
    n = Y.shape[0]
    Jm = np.diag(J.astype(np.float64))
    ny = np.linalg.norm(Y)
    for k in (1, 2, 5, 20):
        o = oracle.step_loop(Y, J, nt=1, stop_after=k)
        assert o["info"] == k
        A, U, Z, s = o["A"], o["U"], o["Z"], o["sigma"]
        assert np.all(np.diag(A) == 0)
        Af = A.copy()
        np.fill_diagonal(Af, s)
        assert np.linalg.norm(Y - U @ Af @ Z) <= 64 * n * np.finfo(float).eps * ny, k
        assert np.linalg.norm(U.conj().T @ U - np.eye(n)) <= 64 * n * np.finfo(float).eps, k
        zn = np.linalg.norm(Z) ** 2
        assert np.linalg.norm(Z.conj().T @ Jm @ Z - Jm) <= 64 * n * np.finfo(float).eps * zn, k
