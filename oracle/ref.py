"""TEST INFRASTRUCTURE ONLY: ctypes access to reference C sources compiled by oracle/ref.mk.

  wpqb_select(...)  -- src/alt/wpqb.c:196-223 (sort by wpqb_cmp, then greedy selection)
  apq_pairs(...)    -- src/alt/j2apq.c:3-52 (row-cyclic pair list, trigonometric first)
  ref_dhsvd2(...)   -- src/var/qtransf.c:322 (80-bit 2x2 HSVD)
  ref_zhsvd2(...)   -- src/var/xtransf.c:426 (80-bit complex 2x2 HSVD)
  ref_dtw(...), ref_ztw(...) -- src/alt/tweight.c:82-92 (extended-precision trigonometric
                       pair weight, rounded to double; NaN when it is zero)
  ref_hypot_x87(...), ref_dasum2(...), ref_dasum4(...) -- src/var/shared/cutils.c:79-95
                       (x87 extended-precision HYPOT, DASUM2, DASUM4, rounded to double)

The libraries exist only where the reference checkout was present at build time;
available() says whether they can be used.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ALT = os.path.join(_HERE, "_ref", "libjkref_alt.so")
_VAR = os.path.join(_HERE, "_ref", "libjkref_var.so")
_CUT = os.path.join(_HERE, "_ref", "libjkref_cutils.so")
# the reference checkout: $JKOGB_REFERENCE, else the repository's sibling directory `reference`
REF_ROOT = os.environ.get("JKOGB_REFERENCE", os.path.normpath(os.path.join(_HERE, "..", "..", "reference")))


def build() -> bool:
    if not (os.path.exists(_ALT) and os.path.exists(_VAR) and os.path.exists(_CUT)):
        if not os.path.isdir(os.path.join(REF_ROOT, "src")):
            return False
        env = dict(os.environ)
        env.pop("CC", None)
        subprocess.run(["make", "-s", "-C", _HERE, "-f", "ref.mk", f"REF={REF_ROOT}"], check=True, env=env)
    return os.path.exists(_ALT) and os.path.exists(_VAR) and os.path.exists(_CUT)


def available() -> bool:
    try:
        return build()
    except Exception:
        return False


class _Apq(C.Structure):
    _fields_ = [("n_a", C.c_uint32), ("n_t", C.c_uint32), ("a", C.c_void_p),
                ("p", C.POINTER(C.c_uint16)), ("q", C.POINTER(C.c_uint16))]


def _alt():
    L = C.CDLL(_ALT)
    L.wpqb_ncp.argtypes = [C.c_uint16, C.c_uint32, C.c_void_p, C.c_uint16, C.c_void_p, C.c_void_p]
    L.apq_create.restype = C.POINTER(_Apq)
    L.apq_create.argtypes = [C.c_uint16, C.c_void_p]
    L.apq_free.argtypes = [C.POINTER(_Apq)]
    L.apq_free.restype = C.c_void_p
    L.jkref_dtw.restype = C.c_double
    L.jkref_dtw.argtypes = [C.c_double, C.c_double]
    L.jkref_ztw.restype = C.c_double
    L.jkref_ztw.argtypes = [C.c_double] * 4
    return L


def ref_dtw(aqp: float, apq: float) -> float:
    """src/alt/tweight.c dtw: aqp^2 + apq^2 in extended precision (NaN if 0), rounded to double."""
    return _alt().jkref_dtw(float(aqp), float(apq))


def ref_ztw(aqp: complex, apq: complex) -> float:
    """src/alt/tweight.c ztw: |aqp|^2 + |apq|^2 in extended precision (NaN if 0), rounded to double."""
    return _alt().jkref_ztw(aqp.real, aqp.imag, apq.real, apq.imag)


def wpqb_select(n: int, w: np.ndarray, P: np.ndarray, Q: np.ndarray, n_s: int) -> np.ndarray:
    """Reference greedy selection of src/alt/wpqb.c on weights w of pairs (P,Q) (1-based).

    Records are the 16-byte wpqb unions: an x87 80-bit weight followed by uint16
    band, p, q (0-based).  Returns the selected (p, q), 1-based, in selection order.
    """
    assert np.dtype(np.longdouble).itemsize == 16
    m = len(w)
    rec = np.zeros((m, 16), np.uint8)
    rec[:, :10] = np.asarray(w, np.longdouble).view(np.uint8).reshape(m, 16)[:, :10]
    rec[:, 10:16] = np.stack([(Q - P), P - 1, Q - 1], axis=1).astype(np.uint16).view(np.uint8).reshape(m, 6)
    rec = np.ascontiguousarray(rec)
    s = np.zeros(max(n_s, 1), np.uint32)
    info = np.zeros(16, np.uint8)
    _alt().wpqb_ncp(n, m, rec.ctypes.data, n_s, s.ctypes.data, info.ctypes.data)
    sl = int(info[10:12].view(np.uint16)[0])
    pq = rec[:, 12:16].copy().view(np.uint16).reshape(m, 2).astype(np.int64) + 1
    return pq[s[:sl]]


def apq_pairs(n: int, J: np.ndarray) -> tuple[np.ndarray, np.ndarray, int]:
    """Reference row-cyclic pair list of src/alt/j2apq.c; returns 1-based (P, Q, n_t)."""
    L = _alt()
    j = np.ascontiguousarray(np.asarray(J, np.int32))
    o = L.apq_create(n, j.ctypes.data)
    na, nt = o.contents.n_a, o.contents.n_t
    P = np.ctypeslib.as_array(o.contents.p, shape=(na,)).astype(np.int64) + 1
    Q = np.ctypeslib.as_array(o.contents.q, shape=(na,)).astype(np.int64) + 1
    L.apq_free(o)
    return P, Q, int(nt)


def _var():
    L = C.CDLL(_VAR)
    for f in (L.dhsvd2_, L.zhsvd2_):
        f.argtypes = [C.c_void_p] * 5
    return L


def ref_dhsvd2(A2: np.ndarray, J2) -> tuple[np.ndarray, np.ndarray, np.ndarray, int]:
    """src/var/qtransf.c dhsvd2_ on a 2x2 (column-major like the Fortran caller)."""
    A = np.asfortranarray(np.array(A2, np.float64))
    U = np.zeros((2, 2), np.float64, order="F")
    Z = np.zeros((2, 2), np.float64, order="F")
    j = np.ascontiguousarray(np.asarray(J2, np.int64))
    info = np.zeros(1, np.int64)
    _var().dhsvd2_(A.ctypes.data, j.ctypes.data, U.ctypes.data, Z.ctypes.data, info.ctypes.data)
    return A, U, Z, int(info[0])


def ref_zhsvd2(A2: np.ndarray, J2) -> tuple[np.ndarray, np.ndarray, np.ndarray, int]:
    """src/var/xtransf.c zhsvd2_ on a complex 2x2."""
    A = np.asfortranarray(np.array(A2, np.complex128))
    U = np.zeros((2, 2), np.complex128, order="F")
    Z = np.zeros((2, 2), np.complex128, order="F")
    j = np.ascontiguousarray(np.asarray(J2, np.int64))
    info = np.zeros(1, np.int64)
    _var().zhsvd2_(A.ctypes.data, j.ctypes.data, U.ctypes.data, Z.ctypes.data, info.ctypes.data)
    return A, U, Z, int(info[0])


def _cut():
    L = C.CDLL(_CUT)
    for nm, k in (("HYPOTwX87", 2), ("DASUM2", 2), ("DASUM4", 4)):
        f = getattr(L, nm)
        f.restype = C.c_double
        f.argtypes = [C.c_double] * k
    return L


def ref_hypot_x87(a: float, b: float) -> float:
    """src/var/shared/cutils.c HYPOTwX87: sqrt(a^2 + b^2) in x87 extended precision."""
    return _cut().HYPOTwX87(float(a), float(b))


def ref_dasum2(a: float, b: float) -> float:
    """src/var/shared/cutils.c DASUM2: a^2 + b^2 in x87 extended precision."""
    return _cut().DASUM2(float(a), float(b))


def ref_dasum4(a: float, b: float, c: float, d: float) -> float:
    """src/var/shared/cutils.c DASUM4: the four squares summed from the smallest, extended precision."""
    return _cut().DASUM4(float(a), float(b), float(c), float(d))
