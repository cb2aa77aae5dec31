"""Run one named workload through the library on the current GPU.

  python -m jkogb_b200.run WORKLOAD [--max-steps S] [--weights R] [--save-state F] [--load-state F]
                                    [--ranking exact|gram|learned] [--save-sigma F]
  python -m jkogb_b200.run batch4096 [--matrices M] [--min-n K] [--max-steps S]

Without --weights: one device-resident solve of the workload (jk_solver_*), stopped after S
steps when --max-steps is given, and prints the steps, INFO and the wall time.  --save-state
writes the loop's matrix (with its diagonal) where the run stopped to the .npy file F;
--load-state starts the run from such a matrix instead of the workload's input, so that a
profiler can look at a stretch deep inside the solve without replaying its start.  --save-sigma
writes the solve's SIGMA to the .npy file F.  --ranking
gram / learned: the scored solve (jk_dstep_loop_dev_scored) with the Gram form alone or with the
trained network's correction.  With --weights R: R launches of
one build's pair weights (jk_handle_weights) on the workload's input Y, the kernel-level
form of the weight phase.  For the batched workload: one launch of the batched solver
(jk_dstep_loop_batched) over its first M matrices of order >= K (all by default), each
stopped after S steps when given.  All are the small, bounded invocations a profiler is
pointed at.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import gen


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m jkogb_b200.run")
    ap.add_argument("workload", choices=sorted(gen.WORKLOADS) + ["batch4096"])
    ap.add_argument("--matrices", type=int, default=0)
    ap.add_argument("--min-n", type=int, default=0)
    ap.add_argument("--max-steps", type=int, default=0)
    ap.add_argument("--weights", type=int, default=0)
    ap.add_argument("--save-state", default="")
    ap.add_argument("--load-state", default="")
    ap.add_argument("--save-sigma", default="")
    ap.add_argument("--ranking", default="exact", choices=["exact", "gram", "learned"])
    a = ap.parse_args(argv)

    import torch

    import jkogb_b200 as jk

    if a.workload == "batch4096":
        b = [x for x in gen.batch(4096, 16, 128, seed=4) if x[0].shape[0] >= a.min_n]
        if a.matrices > 0:
            b = b[:a.matrices]
        t0 = time.perf_counter()
        res = jk.dstep_loop_batched([x[0] for x in b], [x[1] for x in b], max_steps=a.max_steps)
        info = np.array([r["info"] for r in res])
        print(f"batch4096: {len(b)} matrices in {time.perf_counter() - t0:.3f} s, INFO min {info.min()} max {info.max()}")
        return 0
    wl = gen.WORKLOADS[a.workload]
    Y, J = wl["make"]()
    n, n_2 = wl["n"], wl["n_2"]
    cplx = wl["kind"] == "complex"
    tdt = torch.complex128 if cplx else torch.float64
    dev = torch.device("cuda", 0)
    Y0 = torch.from_numpy(np.ascontiguousarray(Y.T)).to(dev).t()
    stream = torch.cuda.current_stream(dev)
    t0 = time.perf_counter()
    if a.weights > 0:
        h = jk.Handle(n, J, complex_=cplx)
        for _ in range(a.weights):
            h.weights(Y0.data_ptr(), None, stream.cuda_stream)
        torch.cuda.synchronize(dev)
        h.close()
        print(f"{a.workload}: {a.weights} weight launches in {time.perf_counter() - t0:.3f} s")
        return 0
    if a.load_state:
        A = torch.from_numpy(np.ascontiguousarray(np.load(a.load_state).T)).to(dev).t().contiguous().t()
    else:
        A = Y0.clone().t().contiguous().t()
    U = torch.empty((n, n), dtype=tdt, device=dev).t()
    Z = torch.empty((n, n), dtype=tdt, device=dev).t()
    s = torch.empty(n, dtype=torch.float64, device=dev)
    if a.ranking != "exact":
        from . import scorer
        sc = scorer.Scorer(None if a.ranking == "gram" else scorer.load_params(), stall_k=8)
        info, exact = sc.step_loop_dev(A, U, Z, s, J, n_2=n_2, stream=stream, max_steps=a.max_steps)
        sc.close()
        torch.cuda.synchronize(dev)
        if a.save_sigma:
            np.save(a.save_sigma, s.cpu().numpy())
        print(f"{a.workload} ({a.ranking}): INFO={info}, {exact} exact steps in {time.perf_counter() - t0:.3f} s")
        return 0
    sv = jk.Solver(n, J, n_2=n_2, complex_=cplx)
    sv.begin(U.data_ptr(), A.data_ptr(), Z.data_ptr(), stream.cuda_stream)
    sv.advance(a.max_steps)
    steps = sv.steps
    if a.save_state:
        torch.cuda.synchronize(dev)
        np.save(a.save_state, np.asfortranarray(A.cpu().numpy()))
    info = sv.finish(s.data_ptr())
    sv.close()
    torch.cuda.synchronize(dev)
    if a.save_sigma:
        np.save(a.save_sigma, s.cpu().numpy())
    print(f"{a.workload}: {steps} steps, INFO={info} in {time.perf_counter() - t0:.3f} s")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
