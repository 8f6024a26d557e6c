"""The C sharded register with ranks split between two holders that talk
through the caller's transport (tests/c/sharded_threads.c): two host
threads stand for two processes on one GPU, their transport a barrier and
a device-to-device copy; both must report the overlaps of one holder of
every rank bit for bit (FP64 Trotter, second-order Trotter, qDRIFT; world
2 and 4, small exchange chunks).

CPU: the program compiles and links against include/ and the library.
GPU: it runs and reports ok.
"""

import shutil
import subprocess
from pathlib import Path

import pytest

from conftest import ROOT

SRC = ROOT / "tests" / "c" / "sharded_threads.c"
LIB = ROOT / "phase2_b200"
CUDA = Path("/usr/local/cuda")


def _build(out: Path) -> Path:
    if shutil.which("gcc") is None or not (CUDA / "include").is_dir():
        pytest.skip("gcc or the CUDA headers are not available")
    exe = out / "sharded_threads"
    cmd = ["gcc", "-std=gnu11", "-O2", "-Wall", "-Wextra", "-Werror",
           f"-I{ROOT / 'include'}", f"-I{CUDA / 'include'}", str(SRC),
           f"-L{LIB}", "-lphase2", f"-L{CUDA / 'lib64'}", "-lcudart",
           "-lpthread", f"-Wl,-rpath,{LIB}", f"-Wl,-rpath,{CUDA / 'lib64'}",
           "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    return exe


def test_builds(tmp_path):
    assert _build(tmp_path).is_file()


@pytest.mark.gpu
def test_runs(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), \
        r.stdout + r.stderr


NCCL_SRC = ROOT / "tests" / "c" / "sharded_nccl.c"


def test_nccl_program_builds(tmp_path):
    """The NCCL-transport program (tests/c/sharded_nccl.c) compiles and
    links against include/, the library and NCCL.  It runs one process per
    GPU and needs two or more GPUs (NCCL ranks must not share one), so
    only its build is checked here."""
    if not Path("/usr/include/nccl.h").is_file():
        pytest.skip("NCCL headers are not available")
    if shutil.which("gcc") is None or not (CUDA / "include").is_dir():
        pytest.skip("gcc or the CUDA headers are not available")
    exe = tmp_path / "sharded_nccl"
    cmd = ["gcc", "-std=gnu11", "-O2", "-Wall", "-Wextra", "-Werror",
           f"-I{ROOT / 'include'}", f"-I{CUDA / 'include'}", str(NCCL_SRC),
           f"-L{LIB}", "-lphase2", f"-L{CUDA / 'lib64'}", "-lcudart",
           "-lnccl", f"-Wl,-rpath,{LIB}", f"-Wl,-rpath,{CUDA / 'lib64'}",
           "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
