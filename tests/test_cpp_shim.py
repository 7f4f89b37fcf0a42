"""The header-only C++ drop-in (include/remifa_shim.hxx, with the
reference's header names in include/remifa/): compiled with g++ against
liblu_b200.so and run.

* CPU: argument errors surface as the reference's exception types
  (std::invalid_argument / std::runtime_error) before any device work, every
  lu_nopiv_ll_* wrapper has the reference's exact signature, and valid calls
  without a device fail instead of computing on the host.
* GPU: each shim call gives exactly what the C-ABI call it maps to gives."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = "/usr/local/cuda"
LIBDIR = os.path.join(ROOT, "remifa_b200")


def _compile(src: str, out: str) -> None:
    cxx = shutil.which("g++")
    if cxx is None or not os.path.isdir(os.path.join(CUDA, "include")):
        pytest.skip("g++ or the CUDA headers are not available")
    cmd = [cxx, "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include", "remifa"),
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "cpp", src), "-o", out, "-L", LIBDIR, "-llu_b200",
           "-L", os.path.join(CUDA, "lib64"), "-lcublas", "-lcudart",
           f"-Wl,-rpath,{LIBDIR}:{os.path.join(CUDA, 'lib64')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


def test_shim_argument_errors_and_signatures(built, tmp_path):
    exe = str(tmp_path / "shim_args")
    _compile("shim_args.cpp", exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "wrappers 35, failures 0" in r.stdout


@pytest.mark.gpu
def test_shim_calls_match_the_c_abi(built, tmp_path):
    exe = str(tmp_path / "shim_gpu")
    _compile("shim_gpu.cpp", exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "failures 0" in r.stdout
