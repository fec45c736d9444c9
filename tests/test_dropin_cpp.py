"""The C++17 drop-in headers (include/limbforge/*.hpp): a program written against the reference's
class API compiles and links against liblimbforge_b200.so (CPU) and runs on the GPU (gpu)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_dropin(tmp_path):
    from limbforge_b200 import build
    build.build()
    exe = str(tmp_path / "dropin")
    libdir = os.path.join(ROOT, "limbforge_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{os.path.join(ROOT, 'include')}", os.path.join(ROOT, "tests", "cpp", "dropin.cpp"),
                    f"-L{libdir}", "-llimbforge_b200", f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    return exe


def test_dropin_compiles_and_links(tmp_path):
    assert os.path.exists(build_dropin(tmp_path))


@pytest.mark.gpu
def test_dropin_runs(tmp_path):
    exe = build_dropin(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all drop-in checks passed" in r.stdout
