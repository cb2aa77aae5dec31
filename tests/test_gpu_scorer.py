"""The learned ranking (jk_mlp_*, jk_scorer_*): its kernels against the numpy oracle of
the network, and scored solves against the exact method.

Tolerances: features bit for bit; network outputs within 1e-5 of the output scale
(FP32 accumulation against float64); the gradient within 1e-4 in relative norm; one
Adam step within 1e-6 relative.  A scored solve ranks differently from the exact
method, so it is compared through its results, to the accuracy this ranking reaches:
every hyperbolic singular value within 1e-12 relative of the oracle's (per J class,
sorted) on iid Gaussian inputs (1e-10 for the untrained network, whose many more
hyperbolic steps add rounding), within 1e-8 on graded inputs with column scales down
to 1e-6 (the learned pivot order loses relative accuracy in the smallest values; the
exact method keeps bit parity with the oracle), and Y = U diag(SIGMA) Z to 1e-12
relative in the Frobenius norm (1e-10 untrained).
"""
import numpy as np
import pytest

import oracle
import oracle.mlp as om
from jkogb_b200 import gen

pytestmark = pytest.mark.gpu


def _env():
    import torch
    import jkogb_b200 as jk
    from jkogb_b200 import scorer
    jk.lib()
    return torch, jk, scorer, torch.device("cuda", 0)


def _dev(torch, dev, Y):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(Y).T)).to(dev).t()


def test_features_bitexact():
    torch, jk, scorer, dev = _env()
    Y, J = gen.graded(40, 1e-3, seed=5)
    Y[3, 7] = 0.0
    X, plus, minus = scorer.features(_dev(torch, dev, Y), J, 17)
    assert np.array_equal(X.cpu().numpy(), om.features(Y, J, 17))


def test_forward_grad_adam_match_oracle():
    torch, jk, scorer, dev = _env()
    r = np.random.default_rng(0)
    P = scorer.init_params(1)
    P[om.H * om.NF:om.H * om.NF + om.H] = r.standard_normal(om.H) * 0.1  # nonzero b1
    Pt = torch.from_numpy(P).to(dev)
    X = (r.standard_normal((3000, 7)) * 2).astype(np.float32)
    T = r.standard_normal(3000).astype(np.float32)
    Xt, Tt = torch.from_numpy(X).to(dev), torch.from_numpy(T).to(dev)
    y = scorer.forward(Xt, Pt).cpu().numpy()
    yn, _ = om.forward(X, P)
    assert np.max(np.abs(y - yn)) <= 1e-5 * np.max(np.abs(yn))
    loss, G = scorer.grad(Xt, Tt, Pt)
    ln, gn = om.loss_grad(X, T, P)
    g = G.cpu().numpy()
    assert abs(float(loss.item()) - ln) <= 1e-5 * ln
    assert np.linalg.norm(g - gn) <= 1e-4 * np.linalg.norm(gn)
    # one Adam step of the library against the oracle's
    M = torch.zeros_like(Pt)
    V = torch.zeros_like(Pt)
    P0 = Pt.clone()
    st = scorer._stream(torch, dev)
    assert jk.lib().jk_mlp_adam(P.size, scorer._vp(Pt), scorer._vp(G), scorer._vp(M), scorer._vp(V), 1, 1e-3, 0.9,
                                0.999, 1e-8, st) == 0
    Pn, _, _ = om.adam(P0.cpu().numpy(), g, np.zeros(P.size), np.zeros(P.size), 1, 1e-3)
    assert np.allclose(Pt.cpu().numpy(), Pn, rtol=1e-6, atol=1e-9)


def _train_small(scorer):
    mats = [gen.graded(n, lo, seed=200 + k) for k, (n, lo) in enumerate([(48, 1e-4), (64, 1e-6), (56, 1e-2)])]
    X, T = scorer.training_data([m for m, _ in mats], [j for _, j in mats], every=2, max_pairs=1024)
    P, hist = scorer.train(X, T, iters=600, batch=4096, lr=2e-3)
    assert hist[-1][1] < hist[0][1]
    return P


def _sigma_err(s, ref, J):
    e = 0.0
    for sgn in (1, -1):
        m = np.asarray(J) == sgn
        if m.any():
            a, b = np.sort(s[m]), np.sort(ref[m])
            e = max(e, float(np.max(np.abs(a - b) / np.abs(b))))
    return e


def _scored(torch, dev, sc, Y, J):
    n = Y.shape[0]
    A = _dev(torch, dev, Y).clone()
    U = torch.empty((n, n), dtype=torch.float64, device=dev).t()
    Z = torch.empty((n, n), dtype=torch.float64, device=dev).t()
    s = torch.empty(n, dtype=torch.float64, device=dev)
    info, ex = sc.step_loop_dev(A, U, Z, s, J)
    torch.cuda.synchronize(dev)
    return info, ex, U.cpu().numpy(), Z.cpu().numpy(), s.cpu().numpy()


def test_scored_solves_accurate_and_trained_beats_untrained():
    torch, jk, scorer, dev = _env()
    trained = scorer.Scorer(_train_small(scorer), stall_k=8)
    untrained = scorer.Scorer(scorer.init_params(7), stall_k=8)
    steps = {"trained": 0, "untrained": 0}
    cases = ((gen.gaussian(64, seed=301, n_plus=40), 1e-12), (gen.gaussian(96, seed=302, n_plus=48), 1e-12),
             (gen.graded(80, 1e-3, seed=303), 1e-8), (gen.graded(96, 1e-6, seed=304), 1e-8))
    for (Y, J), tol in cases:
        n = Y.shape[0]
        ref = oracle.step_loop(Y, J, nt=8)
        assert ref["info"] > 0
        for name, sc in (("trained", trained), ("untrained", untrained)):
            info, ex, U, Z, s = _scored(torch, dev, sc, Y, J)
            assert info > 0, f"{name} n={n}: INFO {info}"
            # the untrained network makes many more hyperbolic steps, each adding rounding
            bound = tol if name == "trained" else max(tol, 1e-10)
            assert _sigma_err(s, ref["sigma"], J) <= bound, f"{name} n={n}: sigma"
            R = U @ np.diag(s) @ Z - Y
            rbound = 1e-12 if name == "trained" else 1e-10
            assert np.linalg.norm(R) <= rbound * np.linalg.norm(Y), f"{name} n={n}: Y != U SIGMA Z"
            steps[name] += info
    trained.close()
    untrained.close()
    # what the training buys over the same network untrained (the exact method itself
    # needs fewer steps than either)
    assert steps["trained"] < steps["untrained"], steps
