"""jk_dweights_noalloc (scratch in a static device array, no allocation) against
jk_handle_weights on the same inputs, through the C ABI.

Tolerance: none.  Both entry points run the same weight arithmetic, so the off-diagonal
weights must agree bit for bit (any two NaNs count as equal).  This file is collected last
so that it also runs after every other GPU test in the same process.
"""
import numpy as np
import pytest

from jkogb_b200 import gen

pytestmark = pytest.mark.gpu


def _jk():
    import jkogb_b200 as jk
    jk.lib()
    return jk


def _same(a, b):
    fa, fb = np.ascontiguousarray(a, np.float64), np.ascontiguousarray(b, np.float64)
    na, nb = np.isnan(fa), np.isnan(fb)
    if not np.array_equal(na, nb):
        return False
    return np.array_equal(np.where(na, 0.0, fa).view(np.uint64), np.where(nb, 0.0, fb).view(np.uint64))


def _dev(Y):
    import torch
    return torch.from_numpy(np.ascontiguousarray(Y.T)).cuda().t()  # column-major n x n


def _handle_weights(jk, Y, J):
    import torch
    n = Y.shape[0]
    A = _dev(Y)
    W = torch.zeros((n, n), dtype=torch.float64, device="cuda").t()
    h = jk.Handle(n, J)
    h.weights(A.data_ptr(), W.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    h.close()
    return W.cpu().numpy()


def _cases():
    # 8 x 8 tile kernel (n = 300); the handle's pipelined kernel vs the 16 x 16 one (n = 1000)
    Y1, J1 = gen.graded(300, 1e-8, seed=11)
    Y2, J2 = gen.gaussian(1000, seed=12, n_plus=500)
    return [(Y1, J1), (Y2, J2)]


def test_noalloc_matches_handle_two_calls():
    import torch
    jk = _jk()
    cases = _cases()
    stream = torch.cuda.current_stream().cuda_stream
    sentinel = 12345.0
    outs = []
    keep = []
    for Y, J in cases:  # two calls in a row on one stream, no synchronisation between them
        n = Y.shape[0]
        A = _dev(Y)
        W = torch.full((n, n), sentinel, dtype=torch.float64, device="cuda").t()
        jk.weights_noalloc(n, A.data_ptr(), J, W.data_ptr(), stream)
        keep.append(A)
        outs.append(W)
    torch.cuda.synchronize()
    for (Y, J), W in zip(cases, outs):
        n = Y.shape[0]
        got = W.cpu().numpy()
        ref = _handle_weights(jk, Y, J)
        off = ~np.eye(n, dtype=bool)
        assert _same(got[off], ref[off]), f"n={n}: weights differ from jk_handle_weights"
        assert np.all(np.diag(got) == sentinel), "the diagonal of W was written"


def test_noalloc_rejects_large_n_then_works():
    import torch
    jk = _jk()
    n = jk.NOALLOC_MAX_N + 1
    with pytest.raises(jk.JkError) as e:
        jk.weights_noalloc(n, 16, np.ones(n, np.int32), 16, 0)
    assert e.value.info == -34
    Y, J = gen.gaussian(64, seed=13, n_plus=20)
    A = _dev(Y)
    W = torch.zeros((64, 64), dtype=torch.float64, device="cuda").t()
    jk.weights_noalloc(64, A.data_ptr(), J, W.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    ref = _handle_weights(jk, Y, J)
    off = ~np.eye(64, dtype=bool)
    assert _same(W.cpu().numpy()[off], ref[off])
