"""CUDA path against the oracle, bit for bit (integer, index and floating-point bits alike).

Every comparison here is exact: the kernels restate the reference's operation sequence
(fused FMADs, IEEE division and sqrt), so any differing bit is a failure.
"""
import numpy as np
import pytest

import oracle
from jkogb_b200 import gen

pytestmark = pytest.mark.gpu


def _jk():
    import jkogb_b200 as jk
    jk.lib()
    return jk


def _same(a, b):
    """Bit-identical arrays, except that any two NaNs compare equal (payloads may differ)."""
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype.kind not in "fc":
        return a.dtype == b.dtype and np.array_equal(a, b)
    fa, fb = a.view(np.float64), b.view(np.float64)
    na, nb = np.isnan(fa), np.isnan(fb)
    if not np.array_equal(na, nb):
        return False
    return np.array_equal(np.where(na, 0.0, fa).view(np.uint64), np.where(nb, 0.0, fb).view(np.uint64))


def _rand_2x2(rng, cnt, cplx):
    B = rng.standard_normal((cnt, 2, 2)) * np.exp(rng.uniform(-30, 30, (cnt, 2, 2)))
    if cplx:
        B = B + 1j * rng.standard_normal((cnt, 2, 2)) * np.exp(rng.uniform(-30, 30, (cnt, 2, 2)))
    # structured cases: zeros, triangles, diagonals, tiny and huge entries, ties
    B[::7, 1, 0] = 0.0
    B[::11, 0, 1] = 0.0
    B[::13, 0, 0] = 0.0
    B[::17] = np.where(np.eye(2, dtype=bool), B[::17], 0.0)
    B[::19, 0, 0] = B[::19, 1, 1]
    B[::23] *= 1e-300
    B[::29] *= 1e300
    B[::31, 1, 1] = -B[::31, 1, 1]
    J = np.where(rng.uniform(size=(cnt, 2)) < 0.5, 1, -1).astype(np.int32)
    # equal columns with J = (-1, 1): no hyperbolic transformation, INFO -10 / -11 mostly
    B[3::37, :, 1] = B[3::37, :, 0]
    J[3::37] = (-1, 1)
    return B, J


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("th1", [0.75, 1.0])
def test_hsvd2_batch_bitexact(cplx, th1):
    jk = _jk()
    rng = np.random.Generator(np.random.PCG64(100 + int(cplx)))
    B, J = _rand_2x2(rng, 3000, cplx)
    B[5] = np.nan
    B[6, 0, 1] = np.inf
    if not cplx:
        # blocks whose hyperbolic tangent rounds to 1 or beyond (src/shared/ktransf.F90:76-79, 133-136)
        h = float.fromhex
        B[7] = [[h("-0x1.4a1f253355902p+0"), h("-0x1.4a1f253355902p+0")],
                [h("-0x1.e177757c5cfd8p-3"), h("-0x1.e177757c5cfd8p-3")]]
        B[8] = [[h("-0x1.66ac4cd29aad3p+0"), h("-0x1.66ac4cd29aad4p+0")],
                [h("0x1.410e13af8d388p-4"), h("0x1.410e13af8d389p-4")]]
        J[7] = J[8] = (-1, 1)
    A, U, Z, info = jk.hsvd2_batch(B, J, th1)
    codes = set()
    for k in range(len(B)):
        a, u, z, inf = oracle.hsvd2(B[k], J[k], th1)
        assert inf == info[k], (k, inf, info[k])
        codes.add(int(inf))
        if inf >= 0:
            assert _same(a, A[k]) and _same(u, U[k]) and _same(z, Z[k]), k
    if not cplx:
        assert {-10, -11} <= codes


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("n", [3, 5, 17, 64, 97])
def test_weights_bitexact(cplx, n):
    jk = _jk()
    rng = np.random.Generator(np.random.PCG64(n))
    for trial in range(3):
        Y = rng.standard_normal((n, n))
        if cplx:
            Y = Y + 1j * rng.standard_normal((n, n))
        if trial == 1:  # a partly diagonal matrix: NaN weights ("no transformation") appear
            Y[np.triu_indices(n, 3)] = 0.0
            Y[np.tril_indices(n, -3)] = 0.0
        if trial == 2:
            Y *= np.exp(rng.uniform(-40, 40, (1, n)))
        J = np.where(rng.uniform(size=n) < 0.6, 1, -1).astype(np.int32)
        W = jk.weights(Y, J)
        w, P, Q, tt = oracle.weights(Y, J, id_tru=1)
        got = W[P - 1, Q - 1]
        assert _same(np.isnan(got), np.isnan(w))
        m = ~np.isnan(w)
        assert _same(got[m], w[m])
        assert _same(W, W.T) or np.array_equal(np.isnan(W), np.isnan(W.T))


def test_select_matches_reference_fixture(golden):
    jk = _jk()
    g = golden
    for c in range(len(g["g_n"])):
        n, n2 = int(g["g_n"][c]), int(g["g_n2"][c])
        a, b = g["g_off"][c], g["g_off"][c + 1]
        w, P, Q = g["g_w"][a:b], g["g_p"][a:b], g["g_q"][a:b]
        W = np.full((n, n), np.nan)
        W[P - 1, Q - 1] = w
        W[Q - 1, P - 1] = w
        want = g["g_sel"][g["g_soff"][c]:g["g_soff"][c + 1]]
        assert np.array_equal(jk.select(W, n2), want), c


@pytest.mark.parametrize("n", [4, 9, 33, 120, 300])
def test_select_random_ties(n):
    jk = _jk()
    rng = np.random.Generator(np.random.PCG64(7 * n))
    for trial in range(4):
        P, Q, _ = oracle.pairs(n, np.ones(n, np.int32), 1)
        w = rng.integers(0, 4 + 20 * trial, len(P)).astype(np.float64) - (trial == 3) * 5
        w[rng.uniform(size=len(P)) < 0.1 * trial] = np.nan
        if trial == 2:
            w[::3] = -0.0
        W = np.full((n, n), np.nan)
        W[P - 1, Q - 1] = w
        W[Q - 1, P - 1] = w
        for n2 in (1, n // 3, n // 2):
            n2 = max(n2, 1)
            assert np.array_equal(jk.select(W, n2), oracle.select(n, w, P, Q, n2, id_ncp=2, nt=1)), (trial, n2)


@pytest.mark.parametrize("n", [40, 300, 1000, 2100])
def test_select_near_equal_weights(n):
    """Weights that agree in the top 48 bits of their order key and differ only in the low
    bits, mixed with exact ties and zeros: the partner ranking reorders those runs by the
    full key (a second sort) and the selection equals the oracle's (orders of 512 and more
    use the cluster matching; above 2048 the ranking holds sixteen keys per thread)."""
    jk = _jk()
    rng = np.random.Generator(np.random.PCG64(11 * n))
    for trial in range(3):
        P, Q, _ = oracle.pairs(n, np.ones(n, np.int32), 1)
        base = np.array([1.0, 2.5, 0.0, 3.75])[rng.integers(0, 4, len(P))]
        ulp = rng.integers(0, 2 ** 14, len(P)) * (trial > 0)   # low bits only (an order key's last 16)
        w = (base.view(np.int64) + ulp).view(np.float64)
        w[base == 0.0] = 0.0
        if trial == 2:
            w[rng.uniform(size=len(P)) < 0.3] = np.nan
        W = np.full((n, n), np.nan)
        W[P - 1, Q - 1] = w
        W[Q - 1, P - 1] = w
        for n2 in (n // 3, n // 2):
            assert np.array_equal(jk.select(W, n2), oracle.select(n, w, P, Q, n2, id_ncp=2, nt=8)), (trial, n2)


CASES = [
    # (kind, n, n_plus, n_2, seed)
    ("d", 3, 2, 0, 1), ("d", 4, 4, 0, 2), ("d", 5, 0, 0, 3), ("d", 8, 5, 0, 4), ("d", 16, 12, 3, 5),
    ("d", 31, 20, 0, 6), ("d", 64, 48, 0, 7), ("d", 64, 32, 1, 8), ("d", 100, 37, 17, 9),
    ("z", 3, 1, 0, 11), ("z", 8, 4, 0, 12), ("z", 21, 15, 0, 13), ("z", 48, 24, 0, 14), ("z", 40, 40, 7, 15),
]


@pytest.mark.parametrize("kind,n,n_plus,n_2,seed", CASES)
def test_solve_bitexact(kind, n, n_plus, n_2, seed):
    jk = _jk()
    rng = np.random.Generator(np.random.PCG64(seed))
    Y = rng.standard_normal((n, n))
    if kind == "z":
        Y = Y + 1j * rng.standard_normal((n, n))
    J = np.concatenate([np.ones(n_plus, np.int32), -np.ones(n - n_plus, np.int32)])
    rng.shuffle(J)
    g = jk.step_loop(Y, J, n_2=n_2, trace=True)
    o = oracle.step_loop(Y, J, n_2=n_2, nt=1, trace=True)
    assert g["info"] == o["info"]
    tg, to = g["trace"], o["trace"]
    assert tg["n_steps"] == to["n_steps"]
    assert np.array_equal(tg["sl"], to["sl"]) and np.array_equal(tg["nl"], to["nl"])
    assert np.array_equal(tg["piv"], to["piv"])
    assert np.array_equal(tg["trig"], to["trig"]) and np.array_equal(tg["hyp"], to["hyp"])
    assert _same(tg["tw"], to["tw"])
    for k in ("A", "U", "Z", "sigma"):
        assert _same(g[k], o[k]), k


def test_solve_n256_config_bitexact():
    """The 256 x 256 workload (J: 192 x +1 then 64 x -1, N_2 = 128) against the oracle."""
    jk = _jk()
    Y, J = gen.gaussian(256, seed=1, n_plus=192)
    g = jk.step_loop(Y, J, n_2=128, trace=True)
    o = oracle.step_loop(Y, J, n_2=128, nt=8, trace=True)
    assert g["info"] == o["info"] > 0
    assert np.array_equal(g["trace"]["piv"], o["trace"]["piv"])
    for k in ("A", "U", "Z", "sigma"):
        assert _same(g[k], o[k]), k


@pytest.mark.parametrize("n,cplx", [(512, False), (384, True)])
def test_invariants_larger(n, cplx):
    jk = _jk()
    Y, J = (gen.complex_gaussian if cplx else gen.graded)(n, seed=3) if cplx else gen.graded(n, 1e-6, seed=3)
    r = jk.step_loop(Y, J)
    U, Z, s = r["U"], r["Z"], r["sigma"]
    assert r["info"] > 0
    assert np.linalg.norm(Y - U @ np.diag(s) @ Z) / np.linalg.norm(Y) < 1e-12
    assert np.linalg.norm(U.conj().T @ U - np.eye(n)) < 1e-11
    Jd = np.diag(J.astype(float))
    Zi = Jd @ Z.conj().T @ Jd  # the accumulated right transformation
    assert np.linalg.norm(Zi.conj().T @ Jd @ Zi - Jd) / np.linalg.norm(Zi) ** 2 < 1e-12


def test_nonfinite_input_info():
    jk = _jk()
    for cplx in (False, True):
        Y, J = (gen.complex_gaussian if cplx else gen.gaussian)(12, seed=4)
        Y[3, 7] = np.inf
        o = oracle.step_loop(Y, J, nt=1)
        try:
            g = jk.step_loop(Y, J)
            ginfo = g["info"]
        except jk.JkError as e:
            ginfo = e.info
        assert ginfo == o["info"]


def test_device_pointer_entry():
    import torch
    jk = _jk()
    n = 48
    Y, J = gen.gaussian(n, seed=12)
    A = torch.from_numpy(np.ascontiguousarray(Y.T)).cuda().t()
    U = torch.empty((n, n), dtype=torch.float64, device="cuda").t()
    Z = torch.empty((n, n), dtype=torch.float64, device="cuda").t()
    s = torch.empty(n, dtype=torch.float64, device="cuda")
    info = jk.step_loop_dev(A, U, Z, s, J)
    o = oracle.step_loop(Y, J, nt=1)
    assert info == o["info"]
    assert _same(U.cpu().numpy(), o["U"]) and _same(s.cpu().numpy(), o["sigma"])


@pytest.mark.parametrize("case", ["sorted", "graded", "unbalanced"])
def test_weights_bitexact_large_tiles(case):
    """Orders large enough for the two-kernel real hyperbolic path (setup + pipelined scan):
    J sorted (every pair of a warp has its "+" vertex as p: the shared-column scan), J in a
    seeded permutation (tiles near the diagonal mix the two orientations), and an odd order
    with 700 "+" signs in a permutation (partial tiles in both directions, warps with fewer
    than four pairs per thread)."""
    jk = _jk()
    if case == "sorted":
        Y, J = gen.gaussian(800, seed=21, n_plus=400)
    elif case == "graded":
        Y, J = gen.graded(800, 1e-6, seed=21)
    else:
        Y, J = gen.gaussian(1811, seed=9, n_plus=700)
        J = J[np.random.default_rng(5).permutation(1811)]
    W = jk.weights(Y, J)
    w, P, Q, tt = oracle.weights(Y, J, id_tru=1, nt=8)
    got = W[P - 1, Q - 1]
    assert _same(np.isnan(got), np.isnan(w))
    m = ~np.isnan(w)
    assert _same(got[m], w[m])
