"""The header-only C++ adapter (include/adamantine_b200.hpp) with the
reference's ThermalOperatorBase / ThermalPhysicsInterface method names: a
compiled C++ program (tests/cpp/adapter_test.cpp, g++) against
libadamantine_b200.so and the CPU oracle. Compiling and linking run on the
CPU; the program runs on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = "/usr/local/cuda"


def build(tmp_path):
    import oracle_py

    from adamantine_b200 import build as lib_build

    lib = lib_build.build()
    oracle_py.build()
    exe = os.path.join(str(tmp_path), "adapter_test")
    libdir, odir = os.path.dirname(lib), os.path.join(ROOT, "oracle", "_build")
    cmd = ["/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++", "-std=c++17", "-O2", "-Wall",
           os.path.join(ROOT, "tests", "cpp", "adapter_test.cpp"), "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "oracle"), "-I", os.path.join(CUDA, "include"),
           "-L", libdir, "-ladamantine_b200", "-L", odir, "-lthermal_oracle",
           "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{libdir}:{odir}:{os.path.join(CUDA, 'lib64')}", "-o", exe]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    return exe


def test_adapter_compiles_and_links(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_adapter_matches_oracle_on_the_gpu(tmp_path):
    exe = build(tmp_path)
    res = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(res.stdout)
    assert res.returncode == 0 and res.stdout.strip().endswith("OK"), res.stdout + res.stderr
