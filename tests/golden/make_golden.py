"""Regenerates tests/golden/ref_pins.npz from the reference's own C sources.

Run where the reference checkout exists (it compiles src/alt/wpqb.c, src/alt/j2apq.c,
src/var/qtransf.c and src/var/xtransf.c through oracle/ref.mk):

    python tests/golden/make_golden.py

The fixture holds, for seeded inputs, the reference C outputs of
  * the greedy non-colliding selection (src/alt/wpqb.c:196-223),
  * the row-cyclic pair list with trigonometric pairs first (src/alt/j2apq.c:3-52),
  * the 80-bit real and complex 2x2 HSVDs (src/var/qtransf.c:322, src/var/xtransf.c:426),
  * the extended-precision trigonometric pair weight (src/alt/tweight.c:82-92),
  * the x87 extended-precision HYPOT, DASUM2 and DASUM4 (src/var/shared/cutils.c:82-95).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import pairs, ref  # noqa: E402


def main():
    assert ref.available(), "the reference checkout is needed to regenerate the fixture"
    rng = np.random.Generator(np.random.PCG64(20240611))
    out = {}
    # greedy selection cases: small integer weights (many ties), NaNs, negatives, +-0
    g = []
    for t in range(48):
        n = int(rng.integers(3, 25))
        J = np.where(rng.uniform(size=n) < rng.uniform(0.2, 0.8), 1, -1)
        P, Q, _ = pairs(n, J, 1 + (t % 2))
        nn = len(P)
        w = rng.integers(0, 5, nn).astype(np.float64) * rng.choice([0.25, 1.0, 3.0])
        w[rng.uniform(size=nn) < rng.uniform(0.0, 0.5)] = np.nan
        if t % 3 == 0:
            w[rng.uniform(size=nn) < 0.3] *= -1.0
        if t % 5 == 0:
            w = w + rng.standard_normal(nn) * 1e-3
        n2 = int(rng.integers(1, n // 2 + 1))
        sel = ref.wpqb_select(n, w, P.astype(np.int64), Q.astype(np.int64), n2)
        g.append((n, n2, w, P, Q, sel))
    out["g_n"] = np.array([c[0] for c in g], np.int32)
    out["g_n2"] = np.array([c[1] for c in g], np.int32)
    out["g_off"] = np.cumsum([0] + [len(c[2]) for c in g]).astype(np.int64)
    out["g_w"] = np.concatenate([c[2] for c in g])
    out["g_p"] = np.concatenate([c[3] for c in g]).astype(np.int32)
    out["g_q"] = np.concatenate([c[4] for c in g]).astype(np.int32)
    out["g_soff"] = np.cumsum([0] + [len(c[5]) for c in g]).astype(np.int64)
    out["g_sel"] = np.concatenate([c[5] for c in g]).astype(np.int32).reshape(-1, 2)
    # pair lists
    pj, pp, pq, pnt, pn = [], [], [], [], []
    for t in range(16):
        n = int(rng.integers(2, 40))
        J = np.where(rng.uniform(size=n) < 0.5, 1, -1).astype(np.int32)
        P, Q, nt = ref.apq_pairs(n, J)
        pj.append(J); pp.append(P); pq.append(Q); pnt.append(nt); pn.append(n)
    out["p_n"] = np.array(pn, np.int32)
    out["p_nt"] = np.array(pnt, np.int32)
    out["p_j"] = np.concatenate(pj)
    out["p_p"] = np.concatenate(pp).astype(np.int32)
    out["p_q"] = np.concatenate(pq).astype(np.int32)
    # 2x2 HSVDs (TH1 = 1: no partial hyperbolic transform, as src/D/dtest.F90:35)
    for kind in ("d", "z"):
        Bs, Js, S, I = [], [], [], []
        for t in range(400):
            B = rng.standard_normal((2, 2)) * np.exp(rng.uniform(-12, 12, (2, 2)))
            if kind == "z":
                B = B + 1j * rng.standard_normal((2, 2)) * np.exp(rng.uniform(-12, 12, (2, 2)))
            if t % 7 == 0:
                B[rng.integers(0, 2), rng.integers(0, 2)] = 0.0
            J2 = np.array([rng.choice([-1, 1]), rng.choice([-1, 1])], np.int64)
            A, U, Z, info = (ref.ref_zhsvd2 if kind == "z" else ref.ref_dhsvd2)(B, J2)
            Bs.append(B); Js.append(J2); S.append([A[0, 0].real, A[1, 1].real]); I.append(info)
        out[f"{kind}2_b"] = np.array(Bs)
        out[f"{kind}2_j"] = np.array(Js, np.int32)
        out[f"{kind}2_s"] = np.array(S)
        out[f"{kind}2_info"] = np.array(I, np.int32)
    # trigonometric pair weights: a_qp, a_pq over wide exponent ranges, with zeros (a separate
    # generator, so that the cases above keep their values)
    rt = np.random.Generator(np.random.PCG64(20261204))
    for kind in ("d", "z"):
        m = 2000
        X = rt.standard_normal((m, 2)) * np.exp(rt.uniform(-300, 300, (m, 2)))
        if kind == "z":
            X = X + 1j * rt.standard_normal((m, 2)) * np.exp(rt.uniform(-300, 300, (m, 2)))
            X[::11, 0] = X[::11, 0].real  # purely real entries
        X[::7, 0] = 0.0
        X[::13, 1] = 0.0
        X[::91, :] = 0.0  # both zero: no transformation
        f = ref.ref_ztw if kind == "z" else ref.ref_dtw
        out[f"tw{kind}_x"] = X
        out[f"tw{kind}_w"] = np.array([f(a, b) for a, b in X])
    # HYPOT, DASUM2, DASUM4 in x87 extended precision: operands over the whole exponent range,
    # subnormals, zeros, equal magnitudes and wide gaps (again a generator of its own)
    rh = np.random.Generator(np.random.PCG64(20261205))
    m = 3000
    H = rh.standard_normal((m, 4)) * np.exp2(rh.integers(-1070, 1020, (m, 4)).astype(np.float64))
    H[::5, 1] = H[::5, 0] * rh.uniform(0.5, 2.0, len(H[::5]))  # close magnitudes
    H[::9, 1] = H[::9, 0] * 2.0 ** -60                             # gaps beyond 54 binades
    H[::17, 1] = 0.0
    H[::23, :2] = np.ldexp(rh.uniform(1, 2, (len(H[::23]), 2)), -1060)  # subnormal operands
    out["hx_x"] = H
    out["hx_hypot"] = np.array([ref.ref_hypot_x87(a, b) for a, b, _, _ in H])
    out["hx_dasum2"] = np.array([ref.ref_dasum2(a, b) for a, b, _, _ in H])
    out["hx_dasum4"] = np.array([ref.ref_dasum4(a, b, c, d) for a, b, c, d in H])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_pins.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
