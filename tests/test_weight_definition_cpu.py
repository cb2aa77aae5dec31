"""The oracle's pair weights against their definition, evaluated independently in extended
precision.  ABODNDF2 / ABODNZF2 (src/D/dtransf.F90:246-348, src/Z/ztransf.F90:452-637) state
the weight of a hyperbolic pair (p, q) as ||old X old Y||_F^2 - ||new X new Y||_F^2 over the
rows i != p, q of the columns X = A(:,p), Y = A(:,q) transformed by the pair's 2x2 right
factor Z (X' = Z11 X + Z21 Y, Y' = Z12 X + Z22 Y), plus the change of the two off-diagonal
entries of the 2x2 block (nonzero new values only with INFO bit 8).  The oracle restates the
reference's sequential, branch-specific fma chains; this test sums the definition in
numpy long double from the oracle's own 2x2 HSVD (DHSVD2 / ZHSVD2 with TH1FIX) and asks for
agreement to 4 eps of the sum of the magnitudes that enter it (measured: at most one eps).  Trigonometric pairs
weigh |A(q,p)|^2 + |A(p,q)|^2 (DASUM2 / DASUM4)."""
import numpy as np
import pytest

import oracle
from jkogb_b200 import gen

LD = np.longdouble


def _definition(A, J, p, q):
    n = A.shape[0]
    cplx = np.iscomplexobj(A)
    app, apq, aqp, aqq = A[p, p], A[p, q], A[q, p], A[q, q]
    if J[p] == J[q]:
        if cplx:
            return LD(abs(aqp.real)) ** 2 + LD(abs(aqp.imag)) ** 2 + LD(abs(apq.real)) ** 2 + LD(abs(apq.imag)) ** 2, None
        return LD(aqp) ** 2 + LD(apq) ** 2, None
    # no record ("no transformation") without off-diagonal entries and with real, non-negative
    # diagonal entries (DMAGF2H, src/D/dstep.F90:49-50; ZMAGF2H, src/Z/zstep.F90:51-52)
    c_app, c_aqq = complex(app), complex(aqq)
    if (aqp == 0 and apq == 0 and c_app.imag == 0 and c_aqq.imag == 0 and not np.signbit(c_app.real)
            and not np.signbit(c_aqq.real)):
        return None, "nan"
    B, U, Z, info = oracle.hsvd2(np.array([[app, apq], [aqp, aqq]]), [int(J[p]), int(J[q])], 0.75)
    if info < 0:
        return None, "nan"
    if not (info & 1):
        return LD(0.0), None
    if not (info & 4):
        return (_sq(aqp) + _sq(apq)), None
    a1 = B[1, 0] if (info & 8) else 0.0
    a2 = B[0, 1] if (info & 8) else 0.0
    rows = [i for i in range(n) if i != p and i != q]
    s = _sq(aqp) - _sq(a1) + _sq(apq) - _sq(a2)
    scale = _sq(aqp) + _sq(a1) + _sq(apq) + _sq(a2)
    z11, z21, z12, z22 = (_ld(Z[0, 0]), _ld(Z[1, 0]), _ld(Z[0, 1]), _ld(Z[1, 1]))
    for i in rows:
        x, y = _ld(A[i, p]), _ld(A[i, q])
        xn = _tuple_add(_mul(z11, x), _mul(z21, y)) if cplx else z11 * x + z21 * y
        yn = _tuple_add(_mul(z12, x), _mul(z22, y)) if cplx else z12 * x + z22 * y
        t = _abs2(x) + _abs2(y)
        u = _abs2(xn) + _abs2(yn)
        s += t - u
        scale += t + u
    return s, scale


def _ld(z):
    return (LD(z.real), LD(z.imag)) if np.iscomplexobj(z) else LD(z)


def _mul(a, b):
    return (a[0] * b[0] - a[1] * b[1], a[0] * b[1] + a[1] * b[0])


def _abs2(z):
    return z[0] * z[0] + z[1] * z[1] if isinstance(z, tuple) else z * z


def _sq(z):
    z = complex(z)
    return LD(z.real) ** 2 + LD(z.imag) ** 2


def _tuple_add(a, b):
    return (a[0] + b[0], a[1] + b[1])


@pytest.mark.parametrize("kind,steps", [("d", 0), ("d", 3), ("z", 0), ("z", 2)])
def test_weights_equal_their_definition(kind, steps):
    if kind == "d":
        Y, J = gen.graded(28, 1e-3, seed=31)
    else:
        Y, J = gen.complex_gaussian(20, seed=32, n_plus=9)
        J = J[np.random.default_rng(3).permutation(20)]
    A = oracle.step_loop(Y, J, nt=1, stop_after=steps)["A"] if steps else Y
    n = A.shape[0]
    w, P, Q, _ = oracle.weights(A, J, id_tru=1)
    eps = np.finfo(np.float64).eps
    checked = 0
    for k in range(len(w)):
        p, q = int(P[k]) - 1, int(Q[k]) - 1
        d, scale = _definition(A, J, p, q)
        if scale == "nan":
            assert np.isnan(w[k])
            continue
        if scale is None:
            if d == 0.0 and J[p] == J[q]:
                continue  # "no transformation" depends on the diagonal too (DMAGF2T)
            assert abs(LD(w[k]) - d) <= 4 * eps * abs(d), (k, p, q, w[k], d)
            continue
        assert abs(LD(w[k]) - d) <= 4 * eps * scale, (k, p, q, w[k], d, scale)
        checked += 1
    assert checked >= 8  # pairs compared through the column sum
