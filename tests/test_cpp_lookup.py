"""The C++ drop-in's element access (operator(), Print of the device
matrix types) uses DeviceCsr::Lookup on downloaded arrays.  tests/cpp/
lookup_test.cpp checks it against Seldon's own operator() on random
RowSparse and RowSymSparse matrices; it makes no device call, so it runs on
the CPU where the reference's headers are present."""
import os
import subprocess

import pytest

from oracle.refpath import have_reference, reference_tree

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")
REF = reference_tree()


@pytest.mark.skipif(not have_reference(),
                    reason="the reference's headers are not present")
def test_lookup_matches_seldon():
    subprocess.run(["make", "-s", "_bin/lookup_test", f"REF={REF}"], cwd=CPP, check=True,
                   capture_output=True, timeout=600)
    out = subprocess.run([os.path.join(CPP, "_bin", "lookup_test")], capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "mismatches general 0 symmetric 0"
