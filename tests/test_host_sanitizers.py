"""The library's host code under AddressSanitizer and UBSan, on a machine
without a GPU.  Four drivers in tests/hostfuzz feed it random well-formed
and malformed inputs:

- sb2_csr_create's validator, symmetric expansion and layouts;
- the ILUT apply's planning (sb2_precond_create_ilut), with an independent
  check that every accepted factor's indices are in range;
- the host ILUT factorization (sb2_ilut_factor, sb2_ilut_factor_sym);
- sb2_batch_create's validation of the systems' CSR arrays.

Host memory operations stand in for the CUDA runtime calls of that code
(tests/hostfuzz/cuda_stubs.cpp), and no kernel runs."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.join(ROOT, "tests", "hostfuzz")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
CUDA_INC = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(NVCC))), "include")
SAN = ["-fsanitize=address", "-fsanitize=undefined", "-fno-omit-frame-pointer"]
ENV = dict(os.environ, UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1")

pytestmark = pytest.mark.skipif(not (os.path.exists(NVCC) and shutil.which("g++")),
                                reason="needs nvcc and g++")


def _run(cmd, cwd):
    out = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=600, env=ENV)
    assert out.returncode == 0, (cmd, out.stdout[-2000:], out.stderr[-4000:])
    return out.stdout


def _stubs(tmp):
    obj = os.path.join(tmp, "cuda_stubs.o")
    _run(["g++", "-std=c++17", "-g", *SAN, "-I" + CUDA_INC, "-c",
          os.path.join(HERE, "cuda_stubs.cpp"), "-o", obj], tmp)
    return obj


def _driver(tmp, name):
    obj = os.path.join(tmp, name + ".o")
    nv_san = [a for f in SAN for a in ("-Xcompiler", f)]
    _run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-g",
          "-I" + os.path.join(ROOT, "include"), *nv_san, "-c", os.path.join(HERE, name + ".cu"),
          "-o", obj], tmp)
    exe = os.path.join(tmp, name)
    _run(["g++", *SAN, obj, _stubs(tmp), "-o", exe, "-ldl", "-lpthread"], tmp)
    return exe


def _clean(out):
    assert "runtime error" not in out and "AddressSanitizer" not in out


def test_csr_create_host_code(tmp_path):
    out = _run([_driver(str(tmp_path), "fuzz_csr"), "1500"], str(tmp_path))
    _clean(out)
    created, refused = int(out.split()[1]), int(out.split()[3])
    assert created > 1000 and refused > 100


def test_ilut_plan_host_code(tmp_path):
    out = _run([_driver(str(tmp_path), "fuzz_ilut_plan"), "1500"], str(tmp_path))
    _clean(out)
    planned, refused = int(out.split()[1]), int(out.split()[3])
    assert planned > 500 and refused > 500


def test_batch_create_host_code(tmp_path):
    out = _run([_driver(str(tmp_path), "fuzz_batch"), "3000"], str(tmp_path))
    _clean(out)
    created, refused = int(out.split()[1]), int(out.split()[3])
    assert created > 500 and refused > 300


def test_ilut_factor_host_code(tmp_path):
    exe = os.path.join(str(tmp_path), "fuzz_ilut_factor")
    _run(["g++", "-std=c++17", "-O1", "-g", *SAN, "-x", "c++",
          os.path.join(ROOT, "seldon_b200", "csrc", "ilut.cu"), "-x", "none",
          os.path.join(HERE, "fuzz_ilut_factor.cpp"), "-I" + os.path.join(ROOT, "include"),
          "-I" + CUDA_INC, "-o", exe], str(tmp_path))
    out = _run([exe, "3000"], str(tmp_path))
    _clean(out)
    factored, refused = int(out.split()[1]), int(out.split()[3])
    assert factored > 1500 and refused > 100
