"""Benchmark of the J-Kogbetliantz HSVD step loop on B200 (time to converge, solves/s).

The workload is one full solve (DSTEP_LOOP from Y to U, Z, SIGMA) of the real
N = 2048 graded matrix Y = G D (G iid N(0,1), D log-uniform in [1e-6, 1], seeded),
J with 1024 entries of each sign in a seeded permutation, N_2 = 1024.  The timed
region is that one solve on device-resident inputs, cut at solver-step boundaries
into --steps slices (one benchmark step = one slice); `value` is solves/s.  `e2e`
times one solve through the host-pointer C ABI (the call a user makes), host
allocation and copies included.  Multi-GPU runs (torchrun, one process per GPU)
solve one replica per rank (weak scaling, no collective on the data path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from jkogb_b200 import gen  # noqa: E402

# workloads: name -> (kind, n, n_2, generator, steps to converge)
# The step count is a property of the (deterministic) algorithm on that input; the GPU
# arm measures it on every run, the CPU arms use the recorded value to turn their
# per-step time into a time to converge.
WORKLOADS = {
    "djk_n2048_graded": dict(kind="real", n=2048, n_2=1024, make=lambda: gen.graded(2048, 1e-6, seed=2),
                             desc="Y = G*D, G iid N(0,1), D log-uniform [1e-6,1], seed 2; J = 1024 x +1, 1024 x -1, "
                                  "seeded permutation; N_2 = 1024"),
    "djk_n256": dict(kind="real", n=256, n_2=128, make=lambda: gen.gaussian(256, seed=1, n_plus=192),
                     desc="Y iid N(0,1), seed 1; J = 192 x +1 then 64 x -1; N_2 = 128"),
    "zjk_n1024": dict(kind="complex", n=1024, n_2=512, make=lambda: gen.complex_gaussian(1024, seed=3),
                      desc="Y complex, Re/Im iid N(0,1/2), seed 3; J = 512 x +1 then 512 x -1; N_2 = 512"),
    "batch4096": dict(kind="batch", count=4096, make=lambda: gen.batch(4096, 16, 128, seed=4),
                      desc="4096 real matrices, even N uniform in [16,128], Y iid N(0,1), J iid +-1 with "
                           "P(+1) ~ U[0.2,0.8] per matrix, N_2 = N/2; seed 4; one persistent launch per rank "
                           "over the rank's share of the batch"),
}
STEPS_FILE = os.path.join(ROOT, "bench_steps.json")


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x, device=None):
    """The maximum of a per-rank number over all ranks: a multi-rank job takes as long as
    its slowest rank.  Without an initialised process group of more than one rank, x."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _clock_sampler(dev):
    """nvidia-smi sampling the GPU's clocks and throttle reasons every 200 ms into a
    temporary file, for the duration of the timed region."""
    import tempfile
    fd, name = tempfile.mkstemp(prefix="jk_clocks_", suffix=".csv")
    os.close(fd)
    f = open(name, "w")
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    try:
        p = subprocess.Popen(["nvidia-smi", "-i", str(dev), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                              "-lms", "200"], stdout=f, stderr=subprocess.DEVNULL)
    except OSError:
        p = None
    return p, f


def _clock_summary(p, f):
    if p is None:
        f.close()
        os.unlink(f.name)
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
    p.terminate()
    try:
        p.wait(5)
    except Exception:
        p.kill()
    f.close()
    sm, smax, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in open(f.name):
        c = [x.strip() for x in line.split(",")]
        if len(c) < 9:
            continue
        try:
            sm.append(float(c[1]))
            smax = float(c[2])
        except ValueError:
            continue
        for k, nm in enumerate(names):
            if c[5 + k].lower().startswith("active"):
                reasons.add(nm)
    os.unlink(f.name)
    return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons)}


def _steps_record():
    try:
        return json.load(open(STEPS_FILE))
    except Exception:
        return {}


def cpu_sample(Y, J, n_2, max_seconds=20.0):
    """The oracle port on all host cores: time whole solver steps on the workload for
    about max_seconds (at least 2 steps); returns (seconds per step, steps timed, threads)."""
    import oracle
    nt = os.cpu_count() or 1
    steps = 1
    t0 = time.perf_counter()
    oracle.step_loop(Y, J, n_2=n_2, nt=nt, stop_after=1)
    t1 = time.perf_counter() - t0
    steps = max(2, int(max_seconds / max(t1, 1e-3)))
    t0 = time.perf_counter()
    oracle.step_loop(Y, J, n_2=n_2, nt=nt, stop_after=steps)
    dt = time.perf_counter() - t0
    return dt / steps, steps, nt


def cpu_batch_estimate(mats, steps, max_seconds=20.0):
    """The oracle port on the host cores for a batch: per-step time measured at one thread
    for a few orders (whole solver steps from the start of a solve), interpolated as
    c N^3 + d, times each matrix's step count, divided by the cores (one matrix per core,
    perfect scaling assumed).  Returns (seconds for the batch, cores, sample description)."""
    import oracle
    cores = os.cpu_count() or 1
    ns = sorted({int(Y.shape[0]) for Y in mats})
    probe = [ns[0], ns[len(ns) // 2], ns[-1]]
    per = {}
    budget = max_seconds / len(probe)
    for n in probe:
        Y, J = next((Y, J) for Y, J in zip(mats, _batch_js) if Y.shape[0] == n)
        t0 = time.perf_counter()
        k = 4
        oracle.step_loop(Y, J, nt=1, stop_after=k)
        dt = time.perf_counter() - t0
        k = max(4, min(2000, int(budget / max(dt / 4, 1e-6))))
        t0 = time.perf_counter()
        oracle.step_loop(Y, J, nt=1, stop_after=k)
        per[n] = (time.perf_counter() - t0) / k
    x = np.array([float(n) ** 3 for n in probe])
    y = np.array([per[n] for n in probe])
    c, d = np.polyfit(x, y, 1)
    d = max(d, 0.0)
    cap = 4000 * max(int(Y.shape[0]) for Y in mats) + 100000  # the library's default step limit
    tot = sum((int(st) if st > 0 else (cap if st == -24 else 1)) * (c * float(Y.shape[0]) ** 3 + d)
              for Y, st in zip(mats, steps))
    desc = (f"oracle steps timed at 1 thread for N in {probe} ({', '.join(f'{per[n] * 1e3:.3f}' for n in probe)} "
            f"ms/step), fitted c N^3 + d, x each matrix's step count, / {cores} cores")
    return tot / cores, cores, desc


_batch_js = []


def run_reference(args, wl):
    """The oracle port (the reference's algorithm, restated in C with OpenMP) on all host
    cores: --warmup solver steps, then exactly --steps solver steps timed, both from the
    start of the solve; the time to converge is extrapolated with the recorded step count."""
    ws, rank, _ = _dist()
    if rank != 0:
        return
    if wl["kind"] == "batch":
        return run_reference_batch(args, wl)
    import oracle
    Y, J = wl["make"]()
    rec = _steps_record().get(args.workload)
    if not rec:
        print(json.dumps({"impl": "reference", "unavailable": "no recorded step count for this workload"}))
        return
    nt = os.cpu_count() or 1
    if args.warmup > 0:
        oracle.step_loop(Y, J, n_2=wl["n_2"], nt=nt, stop_after=args.warmup)
    t0 = time.perf_counter()
    oracle.step_loop(Y, J, n_2=wl["n_2"], nt=nt, stop_after=args.steps)
    dt = time.perf_counter() - t0
    sec = dt / args.steps
    solve_s = sec * rec
    out = {
        "impl": "reference", "metric": "HSVD time-to-converge & solves/s", "value": 1.0 / solve_s, "unit": "solves/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "desc": wl["desc"],
                   "step": "one benchmark step = one solver step (DSTEP_BUILD + DSTEP_TRANSF) from the start of the solve",
                   "solver_steps_to_converge": rec, "ms_per_solver_step": sec * 1e3,
                   "extrapolated_solve_s": solve_s},
        "cpu_baseline": {"value": 1.0 / solve_s, "unit": "solves/s", "cores": nt, "kind": "port",
                         "sample": f"{args.steps} solver steps from the start of the solve ({sec:.3f} s/step), "
                                   f"extrapolated to the {rec} steps the solve takes"},
        "e2e": {"value": 1.0 / solve_s, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def run_reference_batch(args, wl):
    rec = _steps_record().get(args.workload)
    if not rec:
        print(json.dumps({"impl": "reference", "unavailable": "no recorded step counts for this workload"}))
        return
    b = wl["make"]()
    mats = [Y for Y, _ in b]
    _batch_js[:] = [J for _, J in b]
    per = []
    for _ in range(args.warmup):
        cpu_batch_estimate(mats, rec, max_seconds=3.0)
    for _ in range(args.steps):
        sec, cores, desc = cpu_batch_estimate(mats, rec, max_seconds=20.0)
        per.append(sec)
    sec = float(np.mean(per))
    out = {
        "impl": "reference", "metric": "HSVD time-to-converge & solves/s", "value": len(mats) / sec, "unit": "solves/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": args.workload, "desc": wl["desc"]},
        "cpu_baseline": {"value": len(mats) / sec, "unit": "solves/s", "cores": cores, "kind": "port", "sample": desc},
        "e2e": {"value": len(mats) / sec, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def run_ours_batch(args, wl):
    """One 4096-matrix batch, partitioned over the ranks by estimated cost (N^4, the
    longest-processing-time rule); each rank solves its share in one persistent launch per
    benchmark step; rank 0 gathers every matrix's INFO.  `value` counts the matrices that
    converged (INFO >= 0) per second of the slowest rank."""
    import torch
    import torch.distributed as dist

    import jkogb_b200 as jk
    from jkogb_b200 import partition

    ws, rank, local = _dist()
    if ws > 1:
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=900), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    b = wl["make"]()
    total = len(b)
    share = partition.partition([Y.shape[0] for Y, _ in b], ws)[rank]
    mats = [b[i][0] for i in share]
    Js = [b[i][1] for i in share]
    A, J, n, off = jk.batch_pack(mats, Js)
    cnt = len(n)
    plan = jk.Batch(n, np.zeros(cnt, np.int32), J)
    A0 = torch.from_numpy(A).to(dev)
    dA = A0.clone()
    dU = torch.empty_like(dA)
    dZ = torch.empty_like(dA)
    ds = torch.empty(int(n.sum()), dtype=torch.float64, device=dev)
    di = torch.zeros(cnt, dtype=torch.int32, device=dev)
    side = torch.cuda.Stream(dev)
    st = side.cuda_stream
    ptrs = (dA.data_ptr(), dU.data_ptr(), dZ.data_ptr(), ds.data_ptr(), di.data_ptr())

    def barrier():
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    threads = plan.tune(*ptrs, st)
    for _ in range(args.warmup):
        with torch.cuda.stream(side):
            dA.copy_(A0)
        plan.run(*ptrs, st)
    barrier()
    smi, smf = _clock_sampler(local)
    ev = []
    launches = 0
    for k in range(args.steps):
        with torch.cuda.stream(side):
            dA.copy_(A0)  # restore the input, outside the timed launch
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(side)
        plan.run(*ptrs, st)
        e1.record(side)
        ev.append((e0, e1))
        launches += 1
    barrier()
    clocks = _clock_summary(smi, smf)
    dev_ms = sum(a.elapsed_time(b_) for a, b_ in ev)
    ms = max_over_ranks(dev_ms, dev) / args.steps
    info = di.cpu().numpy()

    # the learned form of the batch: the scanned weights ranked by their Gram form (the
    # batched kernel's scorer), one launch on the same share
    sc = scorer_mod().Scorer(None, stall_k=8)
    plan.set_scorer(sc)
    with torch.cuda.stream(side):
        dA.copy_(A0)
    barrier()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(side)
    plan.run(*ptrs, st)
    g1.record(side)
    barrier()
    g_ms = max_over_ranks(g0.elapsed_time(g1), dev)
    ginfo = di.cpu().numpy()
    plan.set_scorer(None)
    sc.close()
    plan.close()

    # end to end: the host-pointer entry (copies in and out inside the call)
    barrier()
    tt0 = time.perf_counter()
    res = jk.dstep_loop_batched(mats, Js)
    e2e_s = max_over_ranks(time.perf_counter() - tt0, dev)
    same = bool(np.array_equal(np.array([r["info"] for r in res]), info))

    # FP64 work of the weight scans of this rank's share: sum over matrices and steps of
    # NH (N - 2) 14 flop, with each matrix's NH and step count
    nplus = np.array([int(np.sum(j == 1)) for j in Js])
    steps_pos = np.where(info > 0, info, 0).astype(np.float64)
    flops = float(np.sum(steps_pos * nplus * (n - nplus) * (n - 2) * 14.0))
    achieved = flops / (ms * 1e-3) / 1e12
    peak = jk.lib().jk_fp64_peak()
    infos = partition.gather_results(share, [int(x) for x in info], total) if ws > 1 else [int(x) for x in info]
    ginfos = partition.gather_results(share, [int(x) for x in ginfo], total) if ws > 1 else [int(x) for x in ginfo]
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    infos = np.array(infos)
    ginfos = np.array(ginfos)
    conv = int(np.sum(infos >= 0))
    gconv = int(np.sum(ginfos >= 0))
    out = {
        "metric": "HSVD time-to-converge & solves/s", "value": conv * 1e3 / ms, "unit": "solves/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, the workload's distributions)",
        "config": {"workload": args.workload, "desc": wl["desc"], "matrices": total, "matrices_converged": conv,
                   "matrices_step_capped": int(np.sum(infos == -24)), "threads_per_block": threads,
                   "parallelism": f"partition{ws} (longest-processing-time on N^4)",
                   "steps_total_rank0": int(steps_pos.sum()),
                   "matrices_over_100N_steps_rank0": int(np.sum(info > 100 * n)),
                   "learned": {"ranking": "Gram form of the scanned hyperbolic weights (batched kernel)",
                               "solves_per_s": gconv * 1e3 / g_ms, "batch_ms": g_ms, "matrices_converged": gconv,
                               "matrices_step_capped": int(np.sum(ginfos == -24)),
                               "steps_total_rank0": int(np.where(ginfo > 0, ginfo, 0).sum()),
                               "speedup_vs_plain": ms / g_ms},
                   "l2": "each block's matrix lives in shared memory; U, Z (<= 0.5 GB) stream through L2"},
        "e2e": {"value": conv / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": int(A.nbytes + J.nbytes),
                "d2h_bytes_per_step": int(3 * A.nbytes + 8 * int(n.sum()) + 4 * cnt), "same_info": same},
        "gpu_launches": launches,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak > 0 else None, "traffic": None,
                     "kernel": "k_batch (the whole batched solve, one launch)",
                     "algorithmic_flop_per_launch": flops, "launch_ms": ms,
                     "peak_note": "counts only the weight scans (NH (N-2) 14 flop per step); FP64 FMA peak measured "
                                  "live by jk_fp64_peak"},
        "clocks": clocks,
    }
    if args.cpu_baseline:
        _batch_js[:] = Js
        sec, cores, desc = cpu_batch_estimate(mats, info, max_seconds=20.0)
        out["cpu_baseline"] = {"value": cnt / sec, "unit": "solves/s", "cores": cores, "kind": "port", "sample": desc}
    print(json.dumps(out))


def run_ours(args, wl):
    """One full device-resident solve, cut into --steps slices of solver steps (the
    recorded step count / K each, the last slice to the end), each slice timed with CUDA
    events on the solver's stream; --warmup bounded prefix solves (32 steps each) before
    it; then one end-to-end solve through the host-pointer C ABI."""
    import torch
    import torch.distributed as dist

    import jkogb_b200 as jk

    ws, rank, local = _dist()
    if ws > 1:
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    Y, J = wl["make"]()
    n, n_2 = wl["n"], wl["n_2"]
    cplx = wl["kind"] == "complex"
    tdt = torch.complex128 if cplx else torch.float64
    Y0 = torch.from_numpy(np.ascontiguousarray(Y.T)).to(dev).t()  # column-major resident copy of the input
    A = torch.empty((n, n), dtype=tdt, device=dev).t()
    U = torch.empty((n, n), dtype=tdt, device=dev).t()
    Z = torch.empty((n, n), dtype=tdt, device=dev).t()
    s = torch.empty(n, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    solver = jk.Solver(n, J, n_2=n_2, complex_=cplx)
    ptrs = (U.data_ptr(), A.data_ptr(), Z.data_ptr())

    def barrier():
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # warm-up: bounded prefixes of the same solve (graph capture, first launches)
    for _ in range(args.warmup):
        A.copy_(Y0)
        solver.begin(*ptrs, sp)
        solver.advance(32)
        solver.finish(s.data_ptr())
    rec = _steps_record().get(args.workload) or 32 * args.steps
    per_slice = -(-int(rec) // args.steps)
    A.copy_(Y0)  # the input, restored outside the timed region
    barrier()
    smi, smf = _clock_sampler(local)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    solver.begin(*ptrs, sp)
    for k in range(args.steps):
        solver.advance(per_slice if k < args.steps - 1 else 0)
        if k == args.steps - 1:
            info = solver.finish(s.data_ptr())
        ev[k + 1].record(stream)
    launches = int(jk.lib().jk_last_launch_count())  # the solve's launches, begin to finish
    barrier()
    clocks = _clock_summary(smi, smf)
    slice_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    dev_ms = sum(slice_ms)
    solve_ms = max_over_ranks(dev_ms, dev)
    sig_dev = s.cpu().numpy()
    solver.close()
    sig_ref = _sigma_reference(args.workload)
    sig_err = _sigma_err(sig_dev, sig_ref, J)

    # the learned form on the same input: the scored ranking (the trained network's
    # correction of the Gram form of the scanned weights), one device solve
    learned = None
    if os.path.exists(scorer_mod().PARAMS):
        sc = scorer_mod().Scorer(scorer_mod().load_params(), stall_k=8)
        A.copy_(Y0)
        barrier()
        l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0.record(stream)
        linfo, lexact = sc.step_loop_dev(A, U, Z, s, J, n_2=n_2, stream=stream)
        l1.record(stream)
        barrier()
        l_ms = max_over_ranks(l0.elapsed_time(l1), dev)
        sc.close()
        learned = {"ranking": "trained network correcting the Gram form of the scanned hyperbolic weights",
                   "solves_per_s": ws * 1e3 / l_ms, "solve_ms": l_ms, "solver_steps": linfo,
                   "exact_steps": lexact, "ms_per_solver_step": l_ms / max(linfo, 1),
                   "sigma_rel_err": _sigma_err(s.cpu().numpy(), sig_ref, J),
                   "speedup_vs_plain": solve_ms / l_ms}

    # end to end: one solve through the host-pointer C ABI (H2D of Y, D2H of A, U, Z, SIGMA inside)
    Yh = np.asfortranarray(Y)
    barrier()
    tt0 = time.perf_counter()
    r = jk.step_loop(Yh, J, n_2=n_2)
    e2e_s = max_over_ranks(time.perf_counter() - tt0, dev)
    same = bool(r["info"] == info and np.array_equal(r["sigma"].view(np.uint64), sig_dev.view(np.uint64)))

    # the dominant kernel (the pair weights) timed alone on the workload's input
    h = jk.Handle(n, J, complex_=cplx)
    for _ in range(3):
        h.weights(Y0.data_ptr(), None, sp)
    torch.cuda.synchronize(dev)
    w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 10
    w0.record(stream)
    for _ in range(reps):
        h.weights(Y0.data_ptr(), None, sp)
    w1.record(stream)
    torch.cuda.synchronize(dev)
    w_ms = w0.elapsed_time(w1) / reps
    h.close()
    nplus = int(np.sum(np.asarray(J) == 1))
    nh = nplus * (n - nplus)
    flops = nh * (n - 2) * (14 if not cplx else 36)  # NH (N - 2) rows x the per-row flops of the off-norm scan
    achieved = flops / (w_ms * 1e-3) / 1e12
    peak = jk.lib().jk_fp64_peak()
    traffic, traffic_warm = _recorded_traffic(args.workload)

    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    esize = 16 if cplx else 8
    h2d = n * n * esize + n * 4
    d2h = 3 * n * n * esize + n * 8
    out = {
        "metric": "HSVD time-to-converge & solves/s", "value": ws * 1e3 / solve_ms, "unit": "solves/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": solve_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128" if cplx else "f64",
        "data": "synthetic (seeded generator, the workload's distributions)",
        "config": {"workload": args.workload, "desc": wl["desc"], "n": n, "n_2": n_2,
                   "step": "one benchmark step = 1/K of one full solve (the solve cut at solver-step "
                           f"boundaries into K = {args.steps} slices of {per_slice} solver steps, the last to the end)",
                   "solver_steps_to_converge": info, "ms_per_solver_step": solve_ms / max(info, 1),
                   "sigma_rel_err": sig_err,
                   "sigma_reference": "extended-precision one-sided hyperbolic Jacobi of the same input "
                                      "(tests/golden/sigma_ref.npz), max relative error per J class",
                   "learned": learned,
                   "slice_ms": [round(x, 3) for x in slice_ms],
                   "warmup": f"{args.warmup} prefix solves of 32 solver steps",
                   "parallelism": f"replicas{ws}", "l2": "working set > L2 (A, U, Z, W: 4 x 32 MB + ranking lists)"},
        "e2e": {"value": ws / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "what": "one solve through jk_dstep_loop (host buffers, allocation and copies inside)",
                "same_result_as_device_solve": same},
        "gpu_launches": launches,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak > 0 else None, "traffic": traffic,
                     "traffic_warm_l2": traffic_warm,
                     "traffic_note": "traffic: ncu DRAM bytes of one k_hyp_pm launch with L2 flushed before it; "
                                     "traffic_warm_l2: the same launch after the trig-weight kernel, as in a build",
                     "kernel": "pair weights (k_weights_trig + k_hyp_pm), timed alone on the input Y",
                     "algorithmic_flop_per_launch": flops, "launch_ms": w_ms,
                     "peak_note": "FP64 FMA throughput measured live by jk_fp64_peak; the weight scan's op mix "
                                  "(4 fma, 2 mul, 4 add per 14 flop) bounds it at 0.70 of that peak"},
        "clocks": clocks,
    }
    if args.cpu_baseline and rank == 0:
        sec, nsteps, nt = cpu_sample(Y, J, n_2, max_seconds=20.0)
        steps_conv = info if info and info > 0 else _steps_record().get(args.workload)
        out["cpu_baseline"] = {"value": 1.0 / (sec * steps_conv), "unit": "solves/s", "cores": nt, "kind": "port",
                               "sample": f"{nsteps} solver steps of the same solve on all host cores "
                                         f"({sec:.3f} s/step) x {steps_conv} steps to converge (extrapolated)"}
    print(json.dumps(out))


def scorer_mod():
    from jkogb_b200 import scorer
    return scorer


def _sigma_reference(workload):
    """The workload's hyperbolic singular values from the accuracy oracle's fixture."""
    try:
        return np.load(os.path.join(ROOT, "tests", "golden", "sigma_ref.npz"))[workload]
    except Exception:
        return None


def _sigma_err(sig, ref, J):
    """Max relative error of sig against ref within each J sign class (both sorted)."""
    if ref is None:
        return None
    J = np.asarray(J)
    e = 0.0
    for c in (1, -1):
        m = J == c
        if m.any():
            a, b = np.sort(np.asarray(sig)[m]), np.sort(np.asarray(ref)[m])
            e = max(e, float(np.max(np.abs(a - b) / np.abs(b))))
    return e


def _recorded_traffic(workload):
    """DRAM bytes of one launch of the weight kernel from the committed ncu captures: (cold-cache
    capture, capture with the cache as a build leaves it), None where there is none."""
    try:
        rec = json.load(open(os.path.join(ROOT, "profiles", "traffic.json"))).get(workload)
    except Exception:
        return None, None
    if not rec:
        return None, None
    warm = rec.get("bytes_per_launch_warm_l2")
    return float(rec["bytes_per_launch"]), (float(warm) if warm is not None else None)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="djk_n2048_graded", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, wl)
    elif wl["kind"] == "batch":
        run_ours_batch(args, wl)
    else:
        run_ours(args, wl)


if __name__ == "__main__":
    main()
