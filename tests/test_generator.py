"""The prescribed-spectrum generator: the oracle recovers the hyperbolic singular values
it was given (relative error 1e-13), each attached to its J entry."""
import numpy as np

import oracle
from jkogb_b200 import gen


def _class_err(s, sig, J):
    e = 0.0
    for g in (1, -1):
        m = np.asarray(J) == g
        if m.any():
            e = max(e, float(np.max(np.abs(np.sort(s[m]) - np.sort(sig[m])) / np.sort(sig[m]))))
    return e


def test_prescribed_spectrum_recovered_by_oracle():
    r = np.random.default_rng(1)
    for n, npl, seed in ((32, 20, 3), (24, 12, 4), (17, 16, 5)):
        J = np.array([1] * npl + [-1] * (n - npl))
        r.shuffle(J)
        sig = np.exp(r.uniform(-3, 3, n))
        Y = gen.prescribed(sig, J, seed=seed)
        res = oracle.step_loop(Y, J, nt=2)
        assert res["info"] > 0
        assert np.all(res["sigma"] > 0)
        assert _class_err(res["sigma"], sig, J) < 1e-13
