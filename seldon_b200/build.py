"""Build libseldon_b200.so in-tree for sm_100a (nvcc via seldon_b200/csrc/Makefile)."""
import os
import subprocess

from . import PACKAGE_DIR, LIB_PATH


def build_library(jobs=8, verbose=False):
    csrc = os.path.join(PACKAGE_DIR, "csrc")
    cmd = ["make", "-C", csrc, f"-j{jobs}"]
    out = subprocess.run(cmd, capture_output=not verbose, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"building libseldon_b200.so failed:\n{out.stdout}\n{out.stderr}")
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} was not produced")
    return LIB_PATH
