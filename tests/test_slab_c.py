"""The C host loop of a sharded register's qubit swap (tests/c/slab_exchange.c).

The program uses only the library's C-ABI (qreg_slab_get / qreg_slab_put
through caller-owned device buffers, qreg_slab_swap in place) the way a C
host that drives its own transport would: two ranks of one register on one
GPU, the partner's buffer delivered by a device-to-device copy where ranks
on different GPUs would use NCCL.  It checks the swapped and the restored
layouts against the host copy of the global state, bit for bit.

CPU: the program compiles and links against include/ and the library.
GPU: it runs and reports ok for several widths, positions and chunk sizes.
"""

import shutil
import subprocess
from pathlib import Path

import pytest

from conftest import ROOT

SRC = ROOT / "tests" / "c" / "slab_exchange.c"
LIB = ROOT / "phase2_b200"
CUDA = Path("/usr/local/cuda")


def _build(out: Path) -> Path:
    if shutil.which("gcc") is None or not (CUDA / "include").is_dir():
        pytest.skip("gcc or the CUDA headers are not available")
    exe = out / "slab_exchange"
    cmd = ["gcc", "-std=c11", "-O2", "-Wall", "-Wextra", "-Werror",
           f"-I{ROOT / 'include'}", f"-I{CUDA / 'include'}", str(SRC),
           f"-L{LIB}", "-lphase2", f"-L{CUDA / 'lib64'}", "-lcudart",
           f"-Wl,-rpath,{LIB}", f"-Wl,-rpath,{CUDA / 'lib64'}",
           "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    return exe


def test_builds(tmp_path):
    assert _build(tmp_path).is_file()


@pytest.mark.gpu
@pytest.mark.parametrize("nqb,pos,chunk", [(14, 3, 1000), (12, 0, 7),
                                           (16, 14, 1 << 20), (13, 5, 4096)])
def test_runs(tmp_path, nqb, pos, chunk):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe), str(nqb), str(pos), str(chunk)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), \
        r.stdout + r.stderr
