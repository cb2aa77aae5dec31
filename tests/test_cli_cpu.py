"""The djk / zjk programs' argument and file errors, which they report before any CUDA
call (no GPU needed): the reference drivers' STOP messages, exit status 1."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "jkogb_b200", "_lib")


@pytest.fixture(scope="module", autouse=True)
def _built():
    from jkogb_b200.build import build
    build()


def _run(*args):
    p = subprocess.run([os.path.join(BIN, args[0])] + [str(a) for a in args[1:]], capture_output=True, text=True,
                       timeout=60)
    return p.returncode, p.stdout, p.stderr


@pytest.mark.parametrize("prog", ["djk", "zjk"])
def test_usage_and_argument_errors(tmp_path, prog):
    rc, _, err = _run(prog)
    assert rc == 1 and f"{prog}.exe FN N N_2 [ID_NCP [ID_TRU]]" in err
    rc, _, err = _run(prog, tmp_path / "x", "abc", 0)
    assert rc == 1 and "FN N N_2" in err
    rc, _, err = _run(prog, tmp_path / "x", 2, 0)
    assert rc == 1 and "N should be at least 3" in err
    rc, _, err = _run(prog, tmp_path / "x", 8, -1)
    assert rc == 1 and "JSTEP_LEN" in err
    rc, _, err = _run(prog, tmp_path / "x", 8, 0, 4)
    assert rc == 1 and "DPROC_INIT" in err


def test_file_errors(tmp_path):
    fn = tmp_path / "case"
    rc, _, err = _run("djk", fn, 8, 0)
    assert rc == 1 and "OPEN_YJ_RO" in err and "INFO=          1" in err
    np.zeros(64).tofile(str(fn) + ".Y")
    rc, _, err = _run("djk", fn, 8, 0)
    assert rc == 1 and "OPEN_YJ_RO" in err and "INFO=          2" in err
    np.array([1, 1, -1, 2, 1, 1, -1, -1], np.int64).tofile(str(fn) + ".J")
    rc, _, err = _run("djk", fn, 8, 0)
    assert rc == 1 and "R%TRU" in err
