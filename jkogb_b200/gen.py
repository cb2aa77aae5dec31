"""Seeded synthetic inputs for the J-Kogbetliantz HSVD workloads.

Each generator returns (Y, J): Y column-major (numpy Fortran order) float64 or
complex128, J int64 signs (+1/-1), the in-memory form of the FN.Y / FN.J files
that djk / zjk read (reference README.md:53-56).
"""
from __future__ import annotations

import numpy as np


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(int(seed)))


def gaussian(n: int, seed: int = 1, n_plus: int | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Y iid N(0,1); J = n_plus entries +1 then the rest -1 (default 3n/4 +1)."""
    r = _rng(seed)
    Y = np.asfortranarray(r.standard_normal((n, n)))
    n_plus = (3 * n) // 4 if n_plus is None else n_plus
    J = np.concatenate([np.ones(n_plus, np.int64), -np.ones(n - n_plus, np.int64)])
    return Y, J


def graded(n: int, lo: float, seed: int = 2, random_signs: bool = True) -> tuple[np.ndarray, np.ndarray]:
    """Y = G*D, G iid N(0,1), D column scales log-uniform in [lo, 1]; J has n/2 of each sign,
    a seeded permutation when random_signs, else +1 first."""
    r = _rng(seed)
    G = r.standard_normal((n, n))
    d = np.exp(r.uniform(np.log(lo), 0.0, n))
    Y = np.asfortranarray(G * d[None, :])
    J = np.concatenate([np.ones(n // 2, np.int64), -np.ones(n - n // 2, np.int64)])
    if random_signs:
        J = J[r.permutation(n)]
    return Y, J


def complex_gaussian(n: int, seed: int = 3, n_plus: int | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Y complex with Re, Im iid N(0, 1/2); J = n_plus (+1) then (-1), default n/2."""
    r = _rng(seed)
    s = np.sqrt(0.5)
    Y = np.asfortranarray(r.standard_normal((n, n)) * s + 1j * (r.standard_normal((n, n)) * s))
    n_plus = n // 2 if n_plus is None else n_plus
    J = np.concatenate([np.ones(n_plus, np.int64), -np.ones(n - n_plus, np.int64)])
    return Y, J


def batch(count: int, nmin: int = 16, nmax: int = 128, seed: int = 4):
    """count real matrices of even order uniform in [nmin, nmax]; J iid +-1 with
    P(+1) ~ U[0.2, 0.8] per matrix. Returns a list of (Y, J)."""
    r = _rng(seed)
    out = []
    for _ in range(count):
        n = 2 * int(r.integers(nmin // 2, nmax // 2 + 1))
        Y = np.asfortranarray(r.standard_normal((n, n)))
        p = r.uniform(0.2, 0.8)
        J = np.where(r.uniform(size=n) < p, 1, -1).astype(np.int64)
        out.append((Y, J))
    return out


def prescribed(sigma, J, seed: int = 6, rotations: int | None = None, t_max: float = 0.5) -> np.ndarray:
    """A matrix with the prescribed hyperbolic singular values: Y = Q diag(sigma) H with Q
    orthogonal (Haar) and H J-orthogonal (H^T J H = J), a product of random hyperbolic
    rotations between a J = +1 and a J = -1 index (|tanh| <= tanh(t_max)) and plane rotations
    within a sign class.  The hyperbolic singular values of Y are sigma, each attached to its
    J entry, the known answer of the indefinite matrix Y J Y^T with eigenvalues J_i sigma_i^2
    (the construction of the reference's data generator, src/var/old/jkdatgen/, from a
    prescribed spectrum)."""
    sigma = np.asarray(sigma, np.float64)
    J = np.asarray(J)
    n = sigma.size
    r = _rng(seed)
    Q, R = np.linalg.qr(r.standard_normal((n, n)))
    Q *= np.sign(np.diag(R))
    H = np.eye(n)
    plus = np.nonzero(J == 1)[0]
    minus = np.nonzero(J == -1)[0]
    for _ in range(3 * n if rotations is None else rotations):
        if plus.size and minus.size and r.uniform() < 0.5:
            i, k = int(r.choice(plus)), int(r.choice(minus))
            t = r.uniform(-t_max, t_max)
            c, s = np.cosh(t), np.sinh(t)
        else:
            cls = plus if (plus.size > 1 and (minus.size < 2 or r.uniform() < 0.5)) else minus
            if cls.size < 2:
                continue
            i, k = (int(x) for x in r.choice(cls, 2, replace=False))
            t = r.uniform(0.0, 2.0 * np.pi)
            c, s = np.cos(t), np.sin(t)
            s = -s  # a plane rotation [[c, -s], [s, c]] on rows i, k
            hi, hk = H[i].copy(), H[k].copy()
            H[i], H[k] = c * hi + s * hk, -s * hi + c * hk
            continue
        hi, hk = H[i].copy(), H[k].copy()
        H[i], H[k] = c * hi + s * hk, s * hi + c * hk
    return np.asfortranarray(Q @ (sigma[:, None] * H))


def prescribed_graded(n: int, lo: float, seed: int = 8) -> tuple[np.ndarray, np.ndarray]:
    """A matrix with prescribed hyperbolic singular values log-uniform in [lo, 1] (the
    grading of the graded workloads), J with n/2 entries of each sign in a seeded
    permutation; built by prescribed().  Returns (Y, J); the prescribed values are
    prescribed_graded_sigma(n, lo, seed)."""
    sig, J = prescribed_graded_sigma(n, lo, seed)
    return prescribed(sig, J, seed=seed + 1000), J


def prescribed_graded_sigma(n: int, lo: float, seed: int = 8) -> tuple[np.ndarray, np.ndarray]:
    """The prescribed values and J of prescribed_graded."""
    r = _rng(seed)
    sig = np.exp(r.uniform(np.log(lo), 0.0, n))
    J = np.concatenate([np.ones(n // 2, np.int64), -np.ones(n - n // 2, np.int64)])[r.permutation(n)]
    return sig, J


# The five workloads of the benchmark plan, by name.
WORKLOADS = {
    "djk_n256": dict(kind="real", n=256, n_2=128, make=lambda: gaussian(256, seed=1, n_plus=192)),
    "djk_n2048_graded": dict(kind="real", n=2048, n_2=1024, make=lambda: graded(2048, 1e-6, seed=2)),
    "zjk_n1024": dict(kind="complex", n=1024, n_2=512, make=lambda: complex_gaussian(1024, seed=3)),
    "djk_n4096_graded": dict(kind="real", n=4096, n_2=2048,
                             make=lambda: graded(4096, 1e-10, seed=5, random_signs=False)),
}
