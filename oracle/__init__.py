"""TEST INFRASTRUCTURE ONLY: ctypes front end of the C oracle (jk_oracle.c, jk_oracle_z.c).

The oracle is a CPU restatement of venovako/JKogb's step loop (src/D/dstep.F90,
src/Z/zstep.F90 and the 2x2 kernels they call).  Only tests/, the smoke check
and the benchmark's CPU-baseline leg import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libjkoracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with the system gcc (make -C oracle)."""
    if force or not os.path.exists(_SO):
        env = dict(os.environ)
        env.pop("CC", None)
        subprocess.run(["make", "-s", "-C", _HERE], check=True, env=env)
    return _SO


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_SO)
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.jo_dstep_loop.restype = C.c_int
        L.jo_dstep_loop.argtypes = [C.c_int, dp, C.c_int, dp, C.c_int, dp, C.c_int, ip, dp,
                                    C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.jo_zstep_loop.restype = C.c_int
        L.jo_zstep_loop.argtypes = [C.c_int, dp, C.c_int, dp, C.c_int, dp, C.c_int, ip, dp,
                                    C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.jo_dhsvd2.argtypes = [dp, ip, dp, dp, C.c_double, ip]
        L.jo_hypot_identity_check.restype = C.c_longlong
        L.jo_hypot_identity_check.argtypes = [C.c_longlong, C.c_ulonglong]
        L.jo_zhsvd2.argtypes = [dp, ip, dp, dp, C.c_double, ip]
        L.jo_dweights.restype = C.c_int
        L.jo_dweights.argtypes = [C.c_int, dp, C.c_int, ip, C.c_int, C.c_int, dp, ip, ip]
        L.jo_zweights.restype = C.c_int
        L.jo_zweights.argtypes = [C.c_int, dp, C.c_int, ip, C.c_int, C.c_int, dp, ip, ip]
        L.jo_select.restype = C.c_int
        L.jo_select.argtypes = [C.c_int, C.c_int, dp, ip, ip, C.c_int, C.c_int, C.c_int, ip]
        L.jo_hypot.restype = C.c_double
        L.jo_hypot.argtypes = [C.c_double, C.c_double]
        L.jo_scale.restype = C.c_double
        L.jo_scale.argtypes = [C.c_double, C.c_int]
        L.jo_exponent.restype = C.c_int
        L.jo_exponent.argtypes = [C.c_double]
        L.jo_dasum2.restype = C.c_double
        L.jo_dasum2.argtypes = [C.c_double, C.c_double]
        L.jo_dasum4.restype = C.c_double
        L.jo_dasum4.argtypes = [C.c_double] * 4
        L.jo_tru1.restype = C.c_int
        L.jo_tru1.argtypes = [C.c_int, ip, C.c_int, ip, ip, ip]
        L.jo_tru2.restype = C.c_int
        L.jo_tru2.argtypes = [C.c_int, ip, C.c_int, ip, ip, ip]
        L.jo_jstep_len.restype = C.c_int
        L.jo_jstep_len.argtypes = [C.c_int, C.c_int]
        for nm in ("jq_dsigma_q", "jq_dsigma_ld", "jq_zsigma_q", "jq_zsigma_ld"):
            f = getattr(L, nm)
            f.restype = C.c_int
            f.argtypes = [C.c_int, dp, C.c_int, ip, dp, C.c_int, C.c_int]
        L.jo_set_zba_quirk.argtypes = [C.c_int]
        L.jo_set_max_steps.argtypes = [C.c_int]
        _lib = L
    return _lib


class _Trace(C.Structure):
    _fields_ = [("max_steps", C.c_int), ("sl", C.POINTER(C.c_int)), ("nl", C.POINTER(C.c_int)),
                ("trig", C.POINTER(C.c_int)), ("hyp", C.POINTER(C.c_int)), ("tw", C.POINTER(C.c_double)),
                ("max_piv", C.c_longlong), ("piv", C.POINTER(C.c_int)), ("n_piv", C.c_longlong),
                ("n_steps", C.c_int)]


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _new_trace(max_steps, max_piv):
    tr = _Trace()
    bufs = dict(sl=np.zeros(max_steps, np.int32), nl=np.zeros(max_steps, np.int32),
                trig=np.zeros(max_steps, np.int32), hyp=np.zeros(max_steps, np.int32),
                tw=np.zeros(max_steps, np.float64), piv=np.zeros(2 * max_piv, np.int32))
    tr.max_steps = max_steps
    tr.max_piv = max_piv
    for k in ("sl", "nl", "trig", "hyp", "piv"):
        setattr(tr, k, _ip(bufs[k]))
    tr.tw = _dp(bufs["tw"])
    return tr, bufs


def _collect(tr, bufs):
    s = tr.n_steps
    m = min(s, len(bufs["sl"]))
    return dict(n_steps=s, sl=bufs["sl"][:m].copy(), nl=bufs["nl"][:m].copy(),
                trig=bufs["trig"][:m].copy(), hyp=bufs["hyp"][:m].copy(), tw=bufs["tw"][:m].copy(),
                piv=bufs["piv"][:2 * tr.n_piv].reshape(-1, 2).copy())


def step_loop(Y, J, n_2=0, id_ncp=0, id_tru=0, nt=1, trace=False, max_steps=1 << 16, max_piv=1 << 24, stop_after=0):
    """Run the oracle's DSTEP_LOOP / ZSTEP_LOOP on a copy of Y (real or complex, n x n).

    Returns a dict with info, A (the matrix after the loop, diagonal zeroed as the
    reference leaves it), U, Z (already J Z^T J / J Z^H J), sigma and, if asked, the trace.
    """
    Y = np.asarray(Y)
    n = Y.shape[0]
    cplx = np.iscomplexobj(Y)
    dt = np.complex128 if cplx else np.float64
    A = np.asfortranarray(Y.astype(dt, copy=True))
    U = np.zeros((n, n), dt, order="F")
    Z = np.zeros((n, n), dt, order="F")
    s = np.zeros(n, np.float64)
    Jc = np.ascontiguousarray(np.asarray(J).astype(np.int32))
    L = lib()
    trp, bufs = (None, None)
    if trace:
        trp, bufs = _new_trace(max_steps, max_piv)
    fn = L.jo_zstep_loop if cplx else L.jo_dstep_loop
    L.jo_set_max_steps(int(stop_after))
    info = fn(n, _dp(U), n, _dp(A), n, _dp(Z), n, _ip(Jc), _dp(s), int(n_2), int(id_ncp), int(id_tru), int(nt),
              C.byref(trp) if trace else None)
    L.jo_set_max_steps(0)
    out = dict(info=info, A=A, U=U, Z=Z, sigma=s)
    if trace:
        out["trace"] = _collect(trp, bufs)
    return out


def accurate_sigma(Y, J, precision="q", nt=None, max_sweeps=60):
    """The accuracy oracle (jk_accuracy.c): the hyperbolic singular values of Y with
    signature J by one-sided hyperbolic Jacobi in __float128 ("q") or long double ("ld"),
    rounded to float64; sigma[i] is attached to J[i] (compare within each sign class,
    sorted).  Returns (sigma, sweeps)."""
    Y = np.asarray(Y)
    n = Y.shape[0]
    cplx = np.iscomplexobj(Y)
    A = np.asfortranarray(Y.astype(np.complex128 if cplx else np.float64))
    Jc = np.ascontiguousarray(np.asarray(J).astype(np.int32))
    s = np.zeros(n, np.float64)
    nt = nt or (os.cpu_count() or 1)
    fn = getattr(lib(), f"jq_{'z' if cplx else 'd'}sigma_{precision}")
    sw = fn(n, _dp(A), n, _ip(Jc), _dp(s), int(nt), int(max_sweeps))
    if sw < 0:
        raise RuntimeError(f"the accuracy oracle did not converge ({sw})")
    return s, sw


def sigma_rel_err(sigma, ref, J):
    """Max relative error of sigma against ref, within each J sign class (both sorted)."""
    J = np.asarray(J)
    err = 0.0
    for c in (1, -1):
        m = J == c
        if m.any():
            a, b = np.sort(np.asarray(sigma)[m]), np.sort(np.asarray(ref)[m])
            err = max(err, float(np.max(np.abs(a - b) / np.abs(b))))
    return err


def hsvd2(A2, J2, th1=0.75):
    """One 2x2 HSVD (DHSVD2 / ZHSVD2). A2 is 2x2 (real or complex); returns (A, U, Z, info)."""
    A2 = np.asarray(A2)
    cplx = np.iscomplexobj(A2)
    dt = np.complex128 if cplx else np.float64
    A = np.asfortranarray(A2.astype(dt, copy=True))
    U = np.zeros((2, 2), dt, order="F")
    Z = np.zeros((2, 2), dt, order="F")
    Jc = np.ascontiguousarray(np.asarray(J2, np.int32))
    info = C.c_int(0)
    fn = lib().jo_zhsvd2 if cplx else lib().jo_dhsvd2
    fn(_dp(A), _ip(Jc), _dp(U), _dp(Z), float(th1), C.byref(info))
    return A, U, Z, info.value


def weights(A, J, id_tru=0, nt=1):
    """Weights of all pairs of one build in the reference's record order; returns (w, P, Q, TT)."""
    A = np.asarray(A)
    n = A.shape[0]
    cplx = np.iscomplexobj(A)
    Af = np.asfortranarray(A.astype(np.complex128 if cplx else np.float64))
    nn = n * (n - 1) // 2
    w = np.zeros(nn, np.float64)
    P = np.zeros(nn, np.int32)
    Q = np.zeros(nn, np.int32)
    Jc = np.ascontiguousarray(np.asarray(J, np.int32))
    fn = lib().jo_zweights if cplx else lib().jo_dweights
    tt = fn(n, _dp(Af), n, _ip(Jc), int(id_tru), int(nt), _dp(w), _ip(P), _ip(Q))
    return w, P, Q, tt


def select(n, w, P, Q, n_2, id_ncp=2, nt=1):
    """Sort + greedy selection from given pair weights; returns the (SL, 2) pivots, 1-based."""
    w = np.ascontiguousarray(w, np.float64)
    P = np.ascontiguousarray(P, np.int32)
    Q = np.ascontiguousarray(Q, np.int32)
    piv = np.zeros(2 * max(n_2, 1), np.int32)
    sl = lib().jo_select(int(n), len(w), _dp(w), _ip(P), _ip(Q), int(n_2), int(id_ncp), int(nt), _ip(piv))
    if sl < 0:
        raise RuntimeError(f"jo_select failed: {sl}")
    return piv[:2 * sl].reshape(-1, 2).copy()


def pairs(n, J, id_tru=1):
    """TRU1 / TRU2 pair enumeration; returns (P, Q, TT)."""
    nn = n * (n - 1) // 2
    P = np.zeros(nn, np.int32)
    Q = np.zeros(nn, np.int32)
    pn = np.zeros(2, np.int32)
    Jc = np.ascontiguousarray(np.asarray(J, np.int32))
    fn = lib().jo_tru2 if id_tru == 2 else lib().jo_tru1
    tt = fn(n, _ip(Jc), nn, _ip(P), _ip(Q), _ip(pn))
    return P, Q, tt
