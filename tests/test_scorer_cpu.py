"""The learned ranking's host-side pieces that need no GPU: the numpy oracle's BF16
rounding, gradient and Gram features, and the training target."""
import numpy as np
import pytest

import oracle.mlp as om


def test_bf16_rounding_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -3.1415926, 0.0], np.float32)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: to even (1.0); 1 + 1.5 * 2^-8 rounds up
    assert om.bf16(x).tolist()[:4] == [1.0, 1.0, 1.0078125, 1.0078125]
    assert om.bf16(x)[4] == -3.140625 and om.bf16(x)[5] == 0.0


def test_oracle_gradient_against_finite_differences():
    # with weights that are already BF16 values, the loss is smooth in the biases that
    # follow the last rounding and its gradient there is the float64 one
    r = np.random.default_rng(1)
    P = (r.standard_normal(om.H * om.NF + om.H + om.H * om.H + om.H + om.H + 1) * 0.3).astype(np.float32)
    P = om.bf16(P).astype(np.float32)
    X = r.standard_normal((50, om.NF)).astype(np.float32)
    T = r.standard_normal(50).astype(np.float32)
    _, g = om.loss_grad(X, T, P)
    # the second bias block and b3 enter after every rounding: exact finite differences
    b2 = om.H * om.NF + om.H + om.H * om.H
    for k in (b2, b2 + 5, len(P) - 1):
        h = 1e-3
        Pp, Pm = P.astype(np.float64).copy(), P.astype(np.float64).copy()
        Pp[k] += h
        Pm[k] -= h
        lp, _ = om.loss_grad(X, T, Pp.astype(np.float32))
        lm, _ = om.loss_grad(X, T, Pm.astype(np.float32))
        assert abs((lp - lm) / (2 * h) - g[k]) < 1e-3 * max(1.0, abs(g[k]))


def test_target_is_the_clamped_log_ratio():
    from jkogb_b200.scorer import target_of
    w = np.array([1.0, 2.0, 1.0, -4.0, 1.0, 0.0, -1.0])
    wg = np.array([1.0, 1.0, 2.0 ** 0.0625, -2.0 ** 1.9, 4.0, 1.0, 1.0])
    t = target_of(w, wg)
    assert np.allclose(t, [0.0, 1.0, -0.5, 0.8, -1.0, 0.0, 0.0])


@pytest.mark.parametrize("case", ["real", "complex"])
def test_oracle_gram_form_equals_the_exact_weights(case):
    """w_gram of the numpy oracle against the C oracle's exact weights (the same reduction
    summed in another order): 1e-10 relative on graded real input and on complex Gaussian
    input with an unbalanced J (ZMAGF2H's weights, whose scan sums |.|^2 of complex
    entries)."""
    import oracle
    from jkogb_b200 import gen
    Y, J = gen.graded(24, 1e-4, seed=8) if case == "real" else gen.complex_gaussian(27, seed=4, n_plus=17)
    X, Wg = om.features(Y, J, 3)
    w, P, Q, tt = oracle.weights(Y, J, id_tru=1, nt=1)
    ex = {(int(p) - 1, int(q) - 1): v for p, q, v in zip(P, Q, w)}
    plus, minus = np.nonzero(J == 1)[0], np.nonzero(J == -1)[0]
    k, checked = 0, 0
    for a in plus:
        for b in minus:
            if np.isfinite(Wg[k]):
                e = ex[(min(a, b), max(a, b))]
                assert abs(Wg[k] - e) <= 1e-10 * abs(e)
                checked += 1
            k += 1
    assert checked > 20
