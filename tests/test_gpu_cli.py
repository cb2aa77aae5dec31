"""The djk / zjk programs: the reference's command line and file contract over the C ABI.
Their FN.YU / FN.ZZ / FN.SY equal the library's own results bit for bit, the step log
is DSTEP_LOOP's CSV (one row per step and the closing row), and a prescribed spectrum
comes back to 1e-13 relative."""
import os
import subprocess

import numpy as np
import pytest

import jkogb_b200 as jk
from jkogb_b200 import gen

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "jkogb_b200", "_lib")


def _run(prog, fn, n, n_2=0):
    p = subprocess.run([os.path.join(BIN, prog), fn, str(n), str(n_2)], capture_output=True, text=True, timeout=300)
    return p.returncode, p.stdout, p.stderr


def _same(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


@pytest.mark.parametrize("cplx", [False, True])
def test_cli_matches_library(tmp_path, cplx):
    n = 24 if cplx else 40
    Y, J = gen.complex_gaussian(n, seed=11) if cplx else gen.gaussian(n, seed=11, n_plus=28)
    fn = str(tmp_path / "case")
    jk.write_yj(fn, Y, J)
    rc, out, err = _run("zjk" if cplx else "djk", fn, n)
    assert rc == 0, err
    ref = jk.step_loop(Y, J)
    assert f"Executed {ref['info']:11d} steps with transformations in" in out
    assert out.startswith("J has")
    dt = np.complex128 if cplx else np.float64
    U = np.fromfile(fn + ".YU", dt).reshape((n, n), order="F")
    Z = np.fromfile(fn + ".ZZ", dt).reshape((n, n), order="F")
    S = np.fromfile(fn + ".SY", np.float64)
    assert _same(U, ref["U"]) and _same(Z, ref["Z"]) and _same(S, ref["sigma"])
    lines = err.strip().splitlines()
    assert lines[0] == '"STEP","OLDLEN","BUILDs","TRANSFs","NEWLEN","NORMF2D","TRIG","HYP"'
    rows = [ln.split(",") for ln in lines[1:]]
    assert len(rows) == ref["info"] + 1
    assert [int(r[0]) for r in rows] == list(range(len(rows)))
    assert int(rows[-1][1]) == 0 and int(rows[-1][4]) == -1
    assert all(len(r) == 8 and len(r[5]) == 25 for r in rows)


def test_cli_prescribed_spectrum_and_errors(tmp_path):
    r = np.random.default_rng(2)
    n = 48
    J = np.array([1] * 30 + [-1] * 18)
    r.shuffle(J)
    sig = np.exp(r.uniform(-4, 4, n))
    fn = str(tmp_path / "pre")
    jk.write_yj(fn, gen.prescribed(sig, J, seed=9), J)
    rc, out, err = _run("djk", fn, n)
    assert rc == 0, err
    S = np.fromfile(fn + ".SY", np.float64)
    for g in (1, -1):
        m = J == g
        assert np.max(np.abs(np.sort(S[m]) - np.sort(sig[m])) / np.sort(sig[m])) < 1e-13
    rc, _, err = _run("djk", fn, 2)
    assert rc == 1 and "N should be at least 3" in err
    rc, _, err = _run("djk", str(tmp_path / "missing"), n)
    assert rc == 1 and "OPEN_YJ_RO" in err
