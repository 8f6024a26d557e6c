"""The reference's micro-benchmarks (bench/b-*.c) build against this
library: oracle/Makefile (target ``refbenches``) compiles them unchanged
against include/ and links them with phase2_b200/libphase2.so, so every
function of the C surface they call resolves in the product library.  The
check needs no GPU (the programs are not run here: they are timing loops
that write result files).  Skipped where the reference sources were not
available at build time."""

import subprocess
from pathlib import Path

import pytest

from conftest import ROOT

BIN = ROOT / "oracle" / "_ref" / "benches"
NAMES = ["b-paulis", "b-qreg", "b-log", "b-circ", "b-prob", "b-algos",
         "b-state-prep-coeff"]


@pytest.mark.parametrize("name", NAMES)
def test_reference_bench_links_product(name):
    exe = BIN / name
    if not exe.is_file():
        pytest.skip("reference benches not built (no reference sources at "
                    "build time)")
    out = subprocess.run(["ldd", str(exe)], capture_output=True, text=True,
                         timeout=60).stdout
    line = next((ln for ln in out.splitlines() if "libphase2.so" in ln), "")
    assert "=>" in line and "not found" not in out, out
    path = Path(line.split("=>")[1].split("(")[0].strip()).resolve()
    assert path == (ROOT / "phase2_b200" / "libphase2.so").resolve(), out
