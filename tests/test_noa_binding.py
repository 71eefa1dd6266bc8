"""CPU test: the reference-side binding (include/noa_b200/noa_binding.hpp) compiles against noa's own
headers for every function and argument kind — with g++ for noa's CPU-only build, and with nvcc and
NOA_ENABLE_CUDA for the branch that stages texture inputs from their CUDA arrays. Needs the reference
sources; skipped where absent."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# The reference's src/ directory (environment variable NOA_REF_SRC; the default is where this build keeps it).
REF = os.environ.get("NOA_REF_SRC", "/root/reference/src")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "noa")), reason="reference sources not present")
def test_binding_compiles_against_noa_headers():
    import torch
    torch_inc = os.path.join(os.path.dirname(torch.__file__), "include")
    cmd = ["g++", "-std=c++20", "-fsyntax-only", "-DNOA_ERROR_POLICY=2", "-DNOA_ENABLE_CPU", "-DFMT_HEADER_ONLY",
           "-I", REF, "-I", os.path.join(ROOT, "include"), "-isystem", torch_inc,
           "-isystem", os.path.join(ROOT, "oracle", "ref_shim"),
           os.path.join(ROOT, "tests", "cpp", "noa_binding_compile.cpp")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "noa")), reason="reference sources not present")
def test_binding_compiles_with_noa_cuda_backend(tmp_path):
    import shutil
    import torch
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    torch_inc = os.path.join(os.path.dirname(torch.__file__), "include")
    cmd = [nvcc, "-std=c++20", "-x", "cu", "-gencode", "arch=compute_100a,code=sm_100a", "-w",
           "-DNOA_ERROR_POLICY=2", "-DNOA_ENABLE_CPU", "-DNOA_ENABLE_CUDA", "-DFMT_HEADER_ONLY",
           "-I", REF, "-I", os.path.join(ROOT, "include"), "-isystem", torch_inc,
           "-isystem", os.path.join(ROOT, "oracle", "ref_shim"),
           "-c", os.path.join(ROOT, "tests", "cpp", "noa_binding_compile.cpp"), "-o", str(tmp_path / "b.o")]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout + r.stderr)[-4000:]
