"""Accuracy of the GPU solve against the accuracy oracle (extended-precision one-sided
hyperbolic Jacobi, fixtures in tests/golden/sigma_ref.npz made by make_sigma.py): the
max relative error of the hyperbolic singular values per J sign class, the reconstruction
residual, the orthogonality of U and the J-unitarity of Z, per result."""
import os

import numpy as np
import pytest

import oracle
from jkogb_b200 import gen

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sigma_ref.npz")

# The bound per input: 1e-12 for iid Gaussian inputs; on column-graded inputs (scales down
# to 1e-6) the reference's own FP64 method, to which the GPU is bit-identical, reaches
# 1.4e-12 (graded, N = 512) and 1.1e-11 (prescribed spectrum, N = 512) against the
# extended-precision values, measured on a B200, so the bound there is 5e-11.
CASES = [
    ("djk_n256", lambda: gen.gaussian(256, seed=1, n_plus=192), 128, 1e-12),
    ("graded512", lambda: gen.graded(512, 1e-6, seed=3), 0, 5e-11),
    ("prescribed512", lambda: gen.prescribed_graded(512, 1e-6, seed=8), 0, 5e-11),
    ("complex384", lambda: gen.complex_gaussian(384, seed=3), 0, 1e-12),
]


def invariants(Y, J, r):
    """(reconstruction residual, orthogonality of U, J-unitarity of Z) of one result."""
    n = Y.shape[0]
    U, Z, s = r["U"], r["Z"], r["sigma"]
    res = np.linalg.norm(Y - U @ np.diag(s) @ Z) / np.linalg.norm(Y)
    orth = np.linalg.norm(U.conj().T @ U - np.eye(n))
    Jd = np.diag(np.asarray(J, float))
    Zi = Jd @ Z.conj().T @ Jd  # the accumulated right transformation
    junit = np.linalg.norm(Zi.conj().T @ Jd @ Zi - Jd) / np.linalg.norm(Zi) ** 2
    return res, orth, junit


@pytest.mark.parametrize("name,make,n_2,tol", CASES, ids=[c[0] for c in CASES])
def test_sigma_accuracy(name, make, n_2, tol):
    import jkogb_b200 as jk
    ref = np.load(GOLD)[name]
    Y, J = make()
    r = jk.step_loop(Y, J, n_2=n_2)
    assert r["info"] > 0
    err = oracle.sigma_rel_err(r["sigma"], ref, J)
    assert err <= tol, err
    res, orth, junit = invariants(Y, J, r)
    assert res < 1e-12 and orth < 1e-11 and junit < 1e-12, (res, orth, junit)
