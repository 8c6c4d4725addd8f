"""Builds the CUDA library in-tree: apirl_b200/_build/libapirl_b200.so (sm_100a)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(verbose=False):
    cmd = ["make", "-C", os.path.join(HERE, "csrc"), "-j4"]
    r = subprocess.run(cmd, capture_output=not verbose, text=True)
    if r.returncode != 0:
        sys.stderr.write((r.stdout or "") + (r.stderr or ""))
        raise RuntimeError("building libapirl_b200.so failed")
    return os.path.join(HERE, "_build", "libapirl_b200.so")


if __name__ == "__main__":
    print(build(verbose=True))
