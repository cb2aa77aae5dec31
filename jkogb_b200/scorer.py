"""The learned ranking: training data from the exact method's trajectories, training
with the library's own forward/backward/Adam kernels, and the scored solve.

In a scored step the hyperbolic pairs that need the column scan are ranked by
w_gram * 2^(clamp(y, -1, 1) / 8): w_gram is the off-norm reduction written through the
Gram matrix of the columns without their diagonal (equal to the exact weight of DMAGF2H,
src/D/dstep.F90:41-72, up to rounding) and y the output of a network 8 -> 64 -> 64 -> 1
(ReLU, BF16 weights and inputs, FP32 biases and accumulation; tensor cores) trained to
predict clamp(8 log2(w / w_gram), -1, 1) from the pair's Gram features.  Device memory here
is torch's; all arithmetic runs in the library's kernels (jk_mlp_*).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import JkError, Handle, Opts, _opts, lib

NF = 8
HIDDEN = 64


def nparams() -> int:
    return int(lib().jk_mlp_nparams(NF))


def target_of(w, wg):
    """The training target of a scanned pair: clamp(8 log2(w / w_gram), -1, 1), 0 where the
    signs differ or either is zero."""
    w = np.asarray(w, np.float64)
    wg = np.asarray(wg, np.float64)
    ok = (w != 0) & (wg != 0) & (np.sign(w) == np.sign(wg))
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(ok, 8.0 * np.log2(np.abs(np.where(ok, w, 1.0)) / np.abs(np.where(ok, wg, 1.0))), 0.0)
    return np.clip(r, -1.0, 1.0)


def init_params(seed=0) -> np.ndarray:
    """He-initialised FP32 parameters in the library's layout (W1, b1, W2, b2, W3, b3)."""
    r = np.random.Generator(np.random.PCG64(seed))
    w1 = r.standard_normal((HIDDEN, NF)) * np.sqrt(2.0 / NF)
    w2 = r.standard_normal((HIDDEN, HIDDEN)) * np.sqrt(2.0 / HIDDEN)
    w3 = r.standard_normal(HIDDEN) * np.sqrt(1.0 / HIDDEN)
    p = np.concatenate([w1.ravel(), np.zeros(HIDDEN), w2.ravel(), np.zeros(HIDDEN), w3, [0.0]]).astype(np.float32)
    assert p.size == nparams()
    return p


def _vp(t):
    return C.c_void_p(t.data_ptr())


def _stream(torch, dev):
    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def features(dA, J, step):
    """Features of every hyperbolic pair of the column-major device matrix dA (torch, float64
    or complex128), (+ index, - index) order; returns (X (count, 8) float32 on the device,
    w_gram (count) float64 on the device, NaN for the pairs that need no scan, plus, minus)."""
    import torch
    n = dA.shape[0]
    Jc = np.ascontiguousarray(np.asarray(J, np.int32))
    plus = np.nonzero(Jc == 1)[0]
    minus = np.nonzero(Jc == -1)[0]
    m = max(len(plus) * len(minus), 1)
    X = torch.empty((m, NF), dtype=torch.float32, device=dA.device)
    Wg = torch.empty(m, dtype=torch.float64, device=dA.device)
    f = lib().jk_zmlp_features if dA.dtype == torch.complex128 else lib().jk_mlp_features
    cnt = f(n, _vp(dA), Jc.ctypes.data_as(C.POINTER(C.c_int)), int(step), _vp(X), _vp(Wg), _stream(torch, dA.device))
    if cnt < 0:
        raise JkError(int(cnt), "features: ")
    return X[:cnt], Wg[:cnt], plus, minus


def forward(X, params):
    """The network (the inference arithmetic) on device features X (count, 8); params a device
    float32 tensor of master parameters."""
    import torch
    Y = torch.empty(X.shape[0], dtype=torch.float32, device=X.device)
    rc = lib().jk_mlp_forward(NF, X.shape[0], _vp(X.contiguous()), _vp(params), _vp(Y), _stream(torch, X.device))
    if rc < 0:
        raise JkError(rc, "mlp forward: ")
    return Y


def grad(X, T, params):
    """(loss, gradient) of the mean squared error, by the library's backward kernels."""
    import torch
    cnt = X.shape[0]
    ws = int(lib().jk_mlp_grad_workspace(NF, cnt))
    work = torch.empty(ws, dtype=torch.float32, device=X.device)
    G = torch.empty_like(params)
    loss = torch.empty(1, dtype=torch.float32, device=X.device)
    rc = lib().jk_mlp_grad(NF, cnt, _vp(X.contiguous()), _vp(T.contiguous()), _vp(params), _vp(G), _vp(loss), _vp(work),
                           _stream(torch, X.device))
    if rc < 0:
        raise JkError(rc, "mlp grad: ")
    return loss, G


def training_data(mats, Js, every=4, max_pairs=4096, seed=0):
    """Features and targets along the exact method's trajectories: every `every`-th step of
    each solve, up to max_pairs scanned hyperbolic pairs with a finite weight per sampled
    step.  Returns (X, T) as device tensors."""
    import torch
    import jkogb_b200 as jk
    r = np.random.Generator(np.random.PCG64(seed))
    dev = torch.device("cuda", 0)
    xs, ts = [], []
    for Y, J in zip(mats, Js):
        n = Y.shape[0]
        A = torch.from_numpy(np.ascontiguousarray(np.asarray(Y).T)).to(dev).t().contiguous().t()
        U = torch.empty_like(A)
        Z = torch.empty_like(A)
        s = torch.empty(n, dtype=torch.float64, device=dev)
        W = torch.empty((n, n), dtype=torch.float64, device=dev).t()
        h = Handle(n, J)
        step = 0
        while True:
            X, Wg, plus, minus = features(A, J, step)
            h.weights(A.data_ptr(), W.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
            w = W[torch.from_numpy(plus).to(dev)][:, torch.from_numpy(minus).to(dev)].reshape(-1)
            ok = torch.isfinite(w) & torch.isfinite(Wg)
            idx = torch.nonzero(ok).reshape(-1)
            if idx.numel() > max_pairs:
                idx = idx[torch.from_numpy(r.choice(idx.numel(), max_pairs, replace=False)).to(dev)]
            if idx.numel():
                xs.append(X[idx].clone())
                t = target_of(w[idx].cpu().numpy(), Wg[idx].cpu().numpy())
                ts.append(torch.from_numpy(t.astype(np.float32)).to(dev))
            info = jk.step_loop_dev(A, U, Z, s, J, max_steps=every)
            if info != -24:
                break
            A.diagonal().copy_(s)  # the loop leaves the diagonal in SIGMA
            step += every
        h.close()
    return torch.cat(xs), torch.cat(ts)


def train(X, T, params=None, iters=2000, batch=8192, lr=2e-3, seed=0, log=None):
    """Adam on the mean squared error with the library's kernels; returns the FP32
    parameters (numpy) and the loss history."""
    import torch
    dev = X.device
    P = torch.from_numpy(init_params(seed) if params is None else np.asarray(params, np.float32)).to(dev)
    M = torch.zeros_like(P)
    V = torch.zeros_like(P)
    g = torch.Generator(device="cpu").manual_seed(seed)
    hist = []
    cnt = X.shape[0]
    L = lib()
    st = _stream(torch, dev)
    for it in range(1, iters + 1):
        sel = torch.randint(0, cnt, (min(batch, cnt),), generator=g).to(dev)
        xb, tb = X[sel].contiguous(), T[sel].contiguous()
        loss, G = grad(xb, tb, P)
        rc = L.jk_mlp_adam(P.numel(), _vp(P), _vp(G), _vp(M), _vp(V), it, lr, 0.9, 0.999, 1e-8, st)
        if rc < 0:
            raise JkError(rc, "adam: ")
        if it % 100 == 0 or it == iters:
            hist.append((it, float(loss.item())))
            if log:
                log(it, hist[-1][1])
    return P.cpu().numpy(), hist


class Scorer:
    """A ranking for the scored solve (jk_scorer_create): a trained network (params), or,
    with params None, the Gram-guided ranking (the scanned weights from the Gram matrix
    of the off-diagonal columns, no network)."""

    def __init__(self, params=None, stall_k=8):
        info = C.c_int(0)
        if params is None:
            self._s = lib().jk_scorer_create(0, None, int(stall_k), C.byref(info))
        else:
            p = np.ascontiguousarray(np.asarray(params, np.float32))
            if p.size != nparams():
                raise ValueError(f"expected {nparams()} parameters")
            self._s = lib().jk_scorer_create(NF, p.ctypes.data_as(C.POINTER(C.c_float)), int(stall_k), C.byref(info))
        if not self._s:
            raise JkError(info.value, "scorer: ")

    def step_loop_dev(self, A, U, Z, sigma, J, n_2=0, stream=None, max_steps=0):
        """jk_dstep_loop_dev_scored (float64) or jk_zstep_loop_dev_scored (complex128) on
        column-major torch tensors; returns (INFO, exact steps)."""
        import torch
        n = A.shape[0]
        assert A.dtype in (torch.float64, torch.complex128)
        for t in (A, U, Z):
            assert t.is_cuda and t.dtype == A.dtype and t.shape == (n, n) and t.stride() == (1, n)
        Jc = np.ascontiguousarray(np.asarray(J).astype(np.int32))
        o = _opts(max_steps, 0, 0, A.device.index or 0)
        st = stream if stream is not None else torch.cuda.current_stream(A.device)
        ex = C.c_int(0)
        f = lib().jk_zstep_loop_dev_scored if A.dtype == torch.complex128 else lib().jk_dstep_loop_dev_scored
        info = f(n, U.data_ptr(), A.data_ptr(), Z.data_ptr(), Jc.ctypes.data_as(C.POINTER(C.c_int)), sigma.data_ptr(),
                 int(n_2), self._s, C.byref(o), None, C.byref(ex), C.c_void_p(st.cuda_stream))
        if info < 0 and info != -24:
            raise JkError(info, "scored step loop: ")
        return info, ex.value

    def close(self):
        if self._s:
            lib().jk_scorer_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


PARAMS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "scorer_params.npy")


def training_set(count=64, nmin=64, nmax=512, seed=0):
    """`count` seeded training matrices with orders in [nmin, nmax]: half graded (column
    scales log-uniform down to 1e-2 .. 1e-8), half iid Gaussian, J of random signs."""
    from . import gen
    r = np.random.Generator(np.random.PCG64(seed))
    out = []
    for k in range(count):
        n = int(r.integers(nmin // 2, nmax // 2 + 1)) * 2
        if k % 2 == 0:
            Y, J = gen.graded(n, float(10.0 ** -r.integers(2, 9)), seed=int(r.integers(1 << 30)))
        else:
            Y, J = gen.gaussian(n, seed=int(r.integers(1 << 30)), n_plus=int(r.integers(n // 5, 4 * n // 5 + 1)))
        out.append((Y, J))
    return out


def load_params(path=PARAMS):
    """The committed trained parameters (see main())."""
    return np.load(path).astype(np.float32)


def main(argv=None):
    """Train the network on the exact method's trajectories of training_set() and save the
    FP32 master parameters:  python -m jkogb_b200.scorer [--solves C] [--iters I] [--out F]"""
    import argparse
    ap = argparse.ArgumentParser(prog="python -m jkogb_b200.scorer")
    ap.add_argument("--solves", type=int, default=64)
    ap.add_argument("--nmin", type=int, default=64)
    ap.add_argument("--nmax", type=int, default=512)
    ap.add_argument("--every", type=int, default=16)
    ap.add_argument("--pairs", type=int, default=512)
    ap.add_argument("--iters", type=int, default=3000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=PARAMS)
    a = ap.parse_args(argv)
    mats = training_set(a.solves, a.nmin, a.nmax, a.seed)
    X, T = training_data([m for m, _ in mats], [j for _, j in mats], every=a.every, max_pairs=a.pairs, seed=a.seed)
    P, hist = train(X, T, iters=a.iters, seed=a.seed, log=lambda it, l: print(f"iter {it} loss {l:.3e}", flush=True))
    np.save(a.out, P)
    print(f"{X.shape[0]} samples from {len(mats)} solves; loss {hist[0][1]:.3e} -> {hist[-1][1]:.3e}; saved {a.out}")


__all__ = ["NF", "nparams", "target_of", "init_params", "features", "forward", "grad", "training_data", "train",
           "Scorer", "Opts", "training_set", "load_params", "PARAMS", "main"]


if __name__ == "__main__":
    main()
