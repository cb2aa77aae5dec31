"""The learned ranking's host-side pieces that need no GPU: the numpy oracle's BF16
rounding and gradient, and the training target map."""
import numpy as np

import oracle.mlp as om


def test_bf16_rounding_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -3.1415926, 0.0], np.float32)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: to even (1.0); 1 + 1.5 * 2^-8 rounds up
    assert om.bf16(x).tolist()[:4] == [1.0, 1.0, 1.0078125, 1.0078125]
    assert om.bf16(x)[4] == -3.140625 and om.bf16(x)[5] == 0.0


def test_oracle_gradient_against_finite_differences():
    # with weights that are already BF16 values, the loss is smooth in the biases and,
    # through the straight-through rule, its gradient is the float64 one
    r = np.random.default_rng(1)
    P = (r.standard_normal(om.H * om.NF + om.H + om.H * om.H + om.H + om.H + 1) * 0.3).astype(np.float32)
    P = om.bf16(P).astype(np.float32)
    X = r.standard_normal((50, om.NF)).astype(np.float32)
    T = r.standard_normal(50).astype(np.float32)
    _, g = om.loss_grad(X, T, P)
    b1 = om.H * om.NF  # the first bias block: exact finite differences (no rounding)
    for k in (b1, b1 + 5, len(P) - 1):
        h = 1e-3
        Pp, Pm = P.astype(np.float64).copy(), P.astype(np.float64).copy()
        Pp[k] += h
        Pm[k] -= h
        lp, _ = om.loss_grad(X, T, Pp.astype(np.float32))
        lm, _ = om.loss_grad(X, T, Pm.astype(np.float32))
        assert abs((lp - lm) / (2 * h) - g[k]) < 1e-3 * max(1.0, abs(g[k]))


def test_target_map_is_monotone():
    from jkogb_b200.scorer import g_of
    w = np.array([-1e10, -1.0, -1e-300, -5e-324, 0.0, 5e-324, 1e-300, 1e-20, 1.0, 1e10])
    g = g_of(w)
    assert np.all(np.diff(g) > 0)
