"""Generate tests/golden/sigma_ref.npz: the hyperbolic singular values of the benchmark and
test inputs from the accuracy oracle (oracle/jk_accuracy.c, one-sided hyperbolic Jacobi in
__float128 or long double), rounded to float64.  The GPU tests and bench.py compare the
solver's SIGMA with these, per J sign class (sorted), as a relative error.

  python tests/golden/make_sigma.py [name ...]

Each entry is regenerated from the seeded generator in jkogb_b200/gen.py, so the inputs
need not be stored.  The long-double entries were checked against __float128 at N = 512.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from jkogb_b200 import gen  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "sigma_ref.npz")

# name -> (generator of (Y, J), precision)
CASES = {
    "djk_n256": (lambda: gen.gaussian(256, seed=1, n_plus=192), "q"),
    "graded512": (lambda: gen.graded(512, 1e-6, seed=3), "q"),
    "prescribed512": (lambda: gen.prescribed_graded(512, 1e-6, seed=8), "q"),
    "complex384": (lambda: gen.complex_gaussian(384, seed=3), "q"),
    "djk_n2048_graded": (lambda: gen.graded(2048, 1e-6, seed=2), "ld"),
    "zjk_n1024": (lambda: gen.complex_gaussian(1024, seed=3), "ld"),
    "djk_n4096_graded": (lambda: gen.WORKLOADS["djk_n4096_graded"]["make"](), "ld"),
}


def main(names):
    old = dict(np.load(OUT)) if os.path.exists(OUT) else {}
    for name in names or list(CASES):
        make, prec = CASES[name]
        Y, J = make()
        t0 = time.time()
        s, sweeps = oracle.accurate_sigma(Y, J, prec)
        print(f"{name}: n={Y.shape[0]} precision={prec} sweeps={sweeps} {time.time() - t0:.1f} s", flush=True)
        old[name] = s
        old[name + "__precision"] = np.array(prec)
        np.savez_compressed(OUT, **old)


if __name__ == "__main__":
    main(sys.argv[1:])
