"""seldon_b200: Seldon's sparse Krylov path on one B200 (sm_100a).

The engine is libseldon_b200.so (CUDA kernels behind the C ABI declared in
include/seldon_b200.h).  `seldon_b200.api` mirrors Seldon's free functions for
Python callers; include/SeldonB200.hxx plugs the same library into Seldon's
C++ templates.  Importing the package does not load the library; importing
`seldon_b200.api` does, and raises if it is missing (no CPU fallback).
"""
import os

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PACKAGE_DIR, "libseldon_b200.so")

__all__ = ["PACKAGE_DIR", "LIB_PATH"]
