"""The resumable step loop (jk_solver_*): a solve cut at any step boundaries, stopped at a
step limit, or continued from where a limited loop stopped, gives the results of one
uninterrupted DSTEP_LOOP, bit for bit; a step limit stops the loop exactly where the
oracle stops after the same number of steps."""
import numpy as np
import pytest

import oracle
from jkogb_b200 import gen

pytestmark = pytest.mark.gpu


def _jk():
    import jkogb_b200 as jk
    jk.lib()
    return jk


def _same(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    if a.shape != b.shape:
        return False
    fa, fb = a.view(np.float64), b.view(np.float64)
    na, nb = np.isnan(fa), np.isnan(fb)
    return np.array_equal(na, nb) and np.array_equal(np.where(na, 0.0, fa).view(np.uint64),
                                                      np.where(nb, 0.0, fb).view(np.uint64))


def _dev(Y):
    import torch
    n = Y.shape[0]
    dt = torch.complex128 if np.iscomplexobj(Y) else torch.float64
    A = torch.from_numpy(np.ascontiguousarray(Y.T)).cuda().t()
    U = torch.empty((n, n), dtype=dt, device="cuda").t()
    Z = torch.empty((n, n), dtype=dt, device="cuda").t()
    s = torch.empty(n, dtype=torch.float64, device="cuda")
    return A, U, Z, s


def _host(t):
    return np.asfortranarray(t.cpu().numpy())


@pytest.mark.parametrize("kind,n,slice_", [("d", 64, 7), ("d", 97, 1), ("z", 40, 5), ("d", 128, 33)])
def test_sliced_solve_equals_one_call(kind, n, slice_):
    import torch
    jk = _jk()
    Y, J = (gen.complex_gaussian if kind == "z" else gen.gaussian)(n, seed=50 + n)
    ref = jk.step_loop(Y, J)
    A, U, Z, s = _dev(Y)
    sv = jk.Solver(n, J, complex_=(kind == "z"))
    st = torch.cuda.current_stream().cuda_stream
    for rep in range(2):  # the same solver twice: the workspace is reused
        A.copy_(torch.from_numpy(np.ascontiguousarray(Y.T)).cuda().t())
        sv.begin(U.data_ptr(), A.data_ptr(), Z.data_ptr(), st)
        seen = []
        while not sv.advance(slice_):
            seen.append(sv.steps)
            assert seen[-1] == slice_ * len(seen)  # it waits exactly at the slice boundary
        info = sv.finish(s.data_ptr())
        assert info == ref["info"] > 0
        for k, t in (("A", A), ("U", U), ("Z", Z), ("sigma", s)):
            assert _same(_host(t), ref[k]), (rep, k)
    sv.close()


@pytest.mark.parametrize("kind,n,k", [("d", 64, 9), ("d", 256, 40), ("z", 48, 13)])
def test_step_limit_equals_oracle_prefix(kind, n, k):
    """max_steps = K stops after exactly K steps (INFO JK_ERR_MAX_STEPS) in the state the
    oracle reaches after K steps."""
    jk = _jk()
    Y, J = (gen.complex_gaussian if kind == "z" else gen.gaussian)(n, seed=60 + n)
    g = jk.step_loop(Y, J, max_steps=k, trace=True)
    o = oracle.step_loop(Y, J, nt=8, stop_after=k, trace=True)
    assert o["info"] == k and g["info"] == -24
    assert np.array_equal(g["trace"]["piv"], o["trace"]["piv"])
    for key in ("A", "U", "Z", "sigma"):
        assert _same(g[key], o[key]), key


def test_resume_after_limit_equals_full_solve():
    """A loop stopped at a step limit and continued by jk_solver_resume ends where the
    uninterrupted loop ends (the handover the batched solver uses for long tails)."""
    import torch
    jk = _jk()
    n = 80
    Y, J = gen.graded(n, 1e-6, seed=71)
    full = jk.step_loop(Y, J)
    k = full["info"] // 3
    part = jk.step_loop(Y, J, max_steps=k)
    assert part["info"] == -24
    A = torch.from_numpy(np.ascontiguousarray(part["A"].T)).cuda().t()
    U = torch.from_numpy(np.ascontiguousarray(part["U"].T)).cuda().t()
    Z = torch.from_numpy(np.ascontiguousarray(part["Z"].T)).cuda().t()
    s = torch.from_numpy(part["sigma"].copy()).cuda()
    sv = jk.Solver(n, J)
    sv.resume(U.data_ptr(), A.data_ptr(), Z.data_ptr(), s.data_ptr(), k, torch.cuda.current_stream().cuda_stream)
    assert sv.advance(0)
    info = sv.finish(s.data_ptr())
    assert info == full["info"]
    for key, t in (("A", A), ("U", U), ("Z", Z), ("sigma", s)):
        assert _same(_host(t), full[key]), key


def test_solver_call_order_and_complex_resume_rejected():
    import torch
    jk = _jk()
    n = 16
    Y, J = gen.complex_gaussian(n, seed=5)
    sv = jk.Solver(n, J, complex_=True)
    with pytest.raises(jk.JkError) as e:
        sv.advance(1)
    assert e.value.info == -27
    A, U, Z, s = _dev(Y)
    with pytest.raises(jk.JkError) as e:
        sv.resume(U.data_ptr(), A.data_ptr(), Z.data_ptr(), s.data_ptr(), 3, torch.cuda.current_stream().cuda_stream)
    assert e.value.info == -27
    sv.close()
