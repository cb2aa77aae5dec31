"""The oracle against fixtures produced by the reference's own C sources (tests/golden)."""
import numpy as np
import pytest

import oracle


def test_greedy_selection_matches_reference(golden):
    g = golden
    for c in range(len(g["g_n"])):
        n, n2 = int(g["g_n"][c]), int(g["g_n2"][c])
        a, b = g["g_off"][c], g["g_off"][c + 1]
        w, P, Q = g["g_w"][a:b], g["g_p"][a:b], g["g_q"][a:b]
        want = g["g_sel"][g["g_soff"][c]:g["g_soff"][c + 1]]
        for ncp, nt in ((1, 1), (1, 4), (2, 1)):
            got = oracle.select(n, w, P, Q, n2, id_ncp=ncp, nt=nt)
            assert np.array_equal(got, want), (c, ncp, nt)


def test_row_cyclic_pairs_match_reference(golden):
    g = golden
    off = 0
    po = 0
    for c in range(len(g["p_n"])):
        n = int(g["p_n"][c])
        J = g["p_j"][off:off + n]
        nn = n * (n - 1) // 2
        P, Q, tt = oracle.pairs(n, J, 2)
        assert tt == g["p_nt"][c]
        assert np.array_equal(P, g["p_p"][po:po + nn]) and np.array_equal(Q, g["p_q"][po:po + nn])
        off += n
        po += nn


@pytest.mark.parametrize("kind", ["d", "z"])
def test_2x2_hsvd_against_reference_80bit(golden, kind):
    # sigma of the double-precision oracle within 1e-12 (relative) of the 80-bit reference kernel
    B, J, S, I = golden[f"{kind}2_b"], golden[f"{kind}2_j"], golden[f"{kind}2_s"], golden[f"{kind}2_info"]
    for k in range(len(B)):
        A, U, Z, info = oracle.hsvd2(B[k], J[k], th1=1.0)
        assert (info < 0) == (I[k] < 0)
        if info < 0:
            continue
        s = np.array([A[0, 0].real, A[1, 1].real])
        np.testing.assert_allclose(s, S[k], rtol=1e-12, atol=0)


@pytest.mark.parametrize("kind", ["d", "z"])
def test_2x2_dtest_residual(kind):
    # the dtest/ztest recipe (src/D/dtest.F90:38-73): E = B - U^H diag(A) (J Z^H J), in extended precision
    rng = np.random.Generator(np.random.PCG64(7))
    worst = 0.0
    for _ in range(500):
        B = rng.standard_normal((2, 2)) * np.exp(rng.uniform(-8, 8, (2, 2)))
        if kind == "z":
            B = B + 1j * rng.standard_normal((2, 2))
        J2 = [int(rng.choice([-1, 1])), int(rng.choice([-1, 1]))]
        A, U, Z, info = oracle.hsvd2(B, J2, th1=1.0)
        assert info >= 0
        Jd = np.diag(np.array(J2, float))
        lt = np.clongdouble if kind == "z" else np.longdouble
        E = B.astype(lt) - U.conj().T.astype(lt) @ np.diag(np.diag(A)).astype(lt) @ (Jd @ Z.conj().T @ Jd).astype(lt)
        worst = max(worst, float(np.max(np.abs(E)) / np.max(np.abs(B))))
    assert worst < 1e-14


def test_scale_exponent_hypot():
    L = oracle.lib()
    assert L.jo_exponent(1.0) == 1 and L.jo_exponent(0.5) == 0 and L.jo_exponent(5e-324) == -1073
    assert L.jo_scale(5e-324, 1074) == 1.0
    assert L.jo_scale(1.0, -1075) == 0.0 and L.jo_scale(1.5, -1074) == 5e-324 * 2  # ties to even
    assert L.jo_scale(3.0, -1075) == 5e-324 * 2
    rng = np.random.Generator(np.random.PCG64(3))
    x = rng.standard_normal(2000) * np.exp(rng.uniform(-600, 600, 2000))
    y = rng.standard_normal(2000) * np.exp(rng.uniform(-600, 600, 2000))
    h = np.array([L.jo_hypot(a, b) for a, b in zip(x, y)])
    ref = np.hypot(x.astype(np.longdouble), y.astype(np.longdouble))
    assert np.max(np.abs(h - ref) / ref) < 1.2e-16


def test_small_solve_invariants():
    from jkogb_b200 import gen
    for cplx in (False, True):
        Y, J = (gen.complex_gaussian if cplx else gen.gaussian)(24, seed=11)
        r = oracle.step_loop(Y, J, n_2=0, nt=2)
        assert r["info"] > 0
        U, Z, s = r["U"], r["Z"], r["sigma"]
        assert np.linalg.norm(Y - U @ np.diag(s) @ Z) / np.linalg.norm(Y) < 1e-13
        assert np.linalg.norm(U.conj().T @ U - np.eye(24)) < 1e-12
        ev = np.sort(np.linalg.eigvalsh(Y @ np.diag(J.astype(float)) @ Y.conj().T))
        assert np.max(np.abs(ev - np.sort(J * s * s))) / np.max(np.abs(ev)) < 1e-13


def test_thread_count_determinism():
    from jkogb_b200 import gen
    Y, J = gen.gaussian(40, seed=5)
    a = oracle.step_loop(Y, J, nt=1, trace=True)
    b = oracle.step_loop(Y, J, nt=4, trace=True)
    assert a["info"] == b["info"]
    assert np.array_equal(a["trace"]["piv"], b["trace"]["piv"])
    for k in ("U", "Z", "sigma"):
        assert np.array_equal(a[k], b[k])


def test_pair_order_and_ncp_strategies_equivalent():
    # TRU1 and TRU2 list the pairs differently, but the record sort is a total order, so the
    # loop's results do not depend on it; NCP1 and NCP2 take the same greedy set
    import numpy as np
    import oracle
    from jkogb_b200 import gen
    Y, J = gen.graded(20, 1e-3, seed=12)
    base = oracle.step_loop(Y, J, id_ncp=2, id_tru=1, nt=1, trace=True)
    for ncp, tru, nt in ((1, 1, 3), (2, 2, 1), (1, 2, 2)):
        r = oracle.step_loop(Y, J, id_ncp=ncp, id_tru=tru, nt=nt, trace=True)
        assert r["info"] == base["info"]
        assert np.array_equal(r["trace"]["piv"], base["trace"]["piv"])
        for k in ("A", "U", "Z", "sigma"):
            assert np.array_equal(np.ascontiguousarray(r[k]).view(np.uint8), np.ascontiguousarray(base[k]).view(np.uint8))


def test_ncp3_takes_the_best_walk():
    # AW_NCP3's pick is the walk of largest value among all start offsets; it is one of
    # the walks, and its value is at least the plain walk's (start offset 1)
    import numpy as np
    import oracle
    from jkogb_b200 import gen
    Y, J = gen.graded(14, 1e-2, seed=13)
    w, P, Q, _ = oracle.weights(Y, J)
    p2 = oracle.select(14, w, P, Q, 7, id_ncp=2)
    p3 = oracle.select(14, w, P, Q, 7, id_ncp=3)
    W = {(int(a), int(b)): x for a, b, x in zip(P, Q, w)}

    def value(piv):
        ws = [W[(int(a), int(b))] for a, b in piv]
        last = max([k for k, x in enumerate(ws) if x > 0], default=-1)
        wp = 0.0
        for k in range(last, -1, -1):
            wp += ws[k]
        wn = 0.0
        for k in range(last + 1, len(ws)):
            wn += ws[k]
        return wp + wn

    assert value(p3) >= value(p2)
    used = set()
    for a, b in p3:
        assert a not in used and b not in used
        used |= {int(a), int(b)}


def test_trig_weight_against_reference_extended(golden):
    """DASUM2 / DASUM4 of the oracle (the trigonometric pair weight of DMAGF2T / ZMAGF2T,
    src/D/dtransf.F90:12-38, src/Z/ztransf.F90:18-75) against the reference's own
    extended-precision statement of that weight, src/alt/tweight.c:82-92 (dtw, ztw), on
    seeded entries spanning 1e-130 .. 1e130 with zeros: within two units in the last place
    (4.5e-16 relative; 98% agree exactly, none differs by more than one unit), and "no
    transformation" (NaN there, 0 here) exactly when both entries are zero.  The defunct
    real dfn2 (src/alt/tweight.c:3-22) returns the smaller entry squared, 0, when one entry
    is zero, so the real comparison excludes the rows with exactly one zero entry."""
    L = oracle.lib()
    for kind in ("d", "z"):
        X, W = golden[f"tw{kind}_x"], golden[f"tw{kind}_w"]
        n_cmp = 0
        for (a, b), w in zip(X, W):
            if kind == "d":
                got = L.jo_dasum2(float(a.real), float(b.real))
                zero_a, zero_b = a == 0.0, b == 0.0
                if zero_a != zero_b:
                    continue  # the defect above
            else:
                got = L.jo_dasum4(float(a.real), float(a.imag), float(b.real), float(b.imag))
                zero_a = zero_b = (a == 0.0 and b == 0.0)
            if zero_a and zero_b:
                assert np.isnan(w) and got == 0.0
                continue
            assert np.isfinite(w) and got > 0.0
            assert abs(got - w) <= 4.5e-16 * w, (kind, a, b, got, w)
            n_cmp += 1
        assert n_cmp > 1200


def test_hypot_and_dasum_against_reference_x87(golden):
    """The project-own HYPOT (jo_hypot: exact power-of-two scaling, one Newton step from
    error-free products; the GPU kernels restate it) against the reference's x87
    extended-precision HYPOTwX87, and the oracle's DASUM2 / DASUM4 against the extended
    forms of src/var/shared/cutils.c:82-95, on seeded operands over the whole exponent range
    (subnormals, zeros, close magnitudes, gaps beyond 54 binades): the hypot bit for bit,
    DASUM2 / DASUM4 within one unit in the last place (both infinite where the squares
    overflow)."""
    L = oracle.lib()
    H = golden["hx_x"]
    refs = (("hypot", golden["hx_hypot"], lambda r: L.jo_hypot(r[0], r[1]), 0),
            ("dasum2", golden["hx_dasum2"], lambda r: L.jo_dasum2(r[0], r[1]), 1),
            ("dasum4", golden["hx_dasum4"], lambda r: L.jo_dasum4(r[0], r[1], r[2], r[3]), 1))
    for name, want, f, ulps in refs:
        n_fin = 0
        for r, w in zip(H, want):
            g = f([float(x) for x in r])
            if not np.isfinite(w):
                assert g == w, (name, r, g, w)
                continue
            assert abs(g - w) <= ulps * np.spacing(abs(w)), (name, r, g, w)
            n_fin += 1
        assert n_fin > 1000


def test_2x2_hyperbolic_tangent_at_one_fails():
    """A 2x2 block with two (nearly) equal columns and J = diag(-1, 1) has no hyperbolic
    transformation: KHSVD2U / KHSVD2L find |tanh| >= 1 and return INFO -10 / -11
    (src/shared/ktransf.F90:76-79, 133-136), which DHSVD2 passes on; the weight phase turns
    such a pair into "no transformation" (NaN)."""
    h = float.fromhex
    cases = [([[h("-0x1.4a1f253355902p+0"), h("-0x1.4a1f253355902p+0")],
               [h("-0x1.e177757c5cfd8p-3"), h("-0x1.e177757c5cfd8p-3")]], -10),
             ([[h("-0x1.66ac4cd29aad3p+0"), h("-0x1.66ac4cd29aad4p+0")],
               [h("0x1.410e13af8d388p-4"), h("0x1.410e13af8d389p-4")]], -11)]
    for B, want in cases:
        A, U, Z, info = oracle.hsvd2(np.array(B), [-1, 1], th1=1.0)
        assert info == want
        A, U, Z, info = oracle.hsvd2(np.array(B), [-1, 1], th1=0.75)
        assert info == want
    # exactly equal columns: most seeded blocks fail with -10 (the rest pass by rounding)
    rng = np.random.default_rng(7)
    fails = 0
    for _ in range(400):
        B = rng.standard_normal((2, 2))
        B[:, 1] = B[:, 0]
        A, U, Z, info = oracle.hsvd2(B, [-1, 1], th1=1.0)
        assert info in (-10, 7)
        fails += info == -10
    assert fails > 200
