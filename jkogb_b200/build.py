"""Build libjkogb_b200.so in-tree (jkogb_b200/_lib/) for sm_100a with nvcc."""
from __future__ import annotations

import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))


def build(force: bool = False) -> str:
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    csrc = os.path.join(_HERE, "csrc")
    if force:
        subprocess.run(["make", "-s", "-C", csrc, "clean"], check=True, env=env)
    subprocess.run(["make", "-s", "-C", csrc], check=True, env=env)
    return os.path.join(_HERE, "_lib", "libjkogb_b200.so")


if __name__ == "__main__":
    print(build())
