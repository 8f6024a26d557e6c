"""The reference's own test suites, run against this library.

oracle/Makefile (target ``reftests``) compiles the reference test sources
test/t-{paulis,prob,circ_cache,qreg,circ_trott,circ_trott2,qdrift,cmpsit,
world,circ}.c unchanged against include/ and links them with
phase2_b200/libphase2.so.  Each program checks its own expectations
(dense mock-ups at 1e-14, analytic answers, bit-identical reproducibility,
exit status 0 on success).  They are built where the reference sources
are available and travel with the build; the test is skipped where they
were not built.

The reference's Python binding and its pytest suite
(python/phase2/__init__.py, python/tests/test_phase2.py; staged unchanged
by ``make -C oracle ref-python``) run the same way: the binding loads
this library through PHASE2_LIB, and every test of the suite must pass.
"""

import os
import subprocess

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

BIN = ROOT / "oracle" / "_ref" / "tests"
NAMES = ["t-paulis", "t-prob", "t-circ_cache", "t-world", "t-circ",
         "t-qreg", "t-circ_trott", "t-circ_trott2", "t-qdrift", "t-cmpsit"]


@pytest.mark.parametrize("name", NAMES)
def test_reference_program(name):
    exe = BIN / name
    if not exe.is_file():
        pytest.skip("reference test programs not built (no reference "
                    "sources at build time)")
    env = dict(os.environ, PHASE2_LOG="warn")
    r = subprocess.run([str(exe)], capture_output=True, text=True,
                       timeout=600, env=env, cwd=str(BIN))
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])


PYREF = ROOT / "oracle" / "_ref" / "python"


def test_reference_python_suite():
    suite = PYREF / "tests" / "test_phase2.py"
    if not suite.is_file():
        pytest.skip("reference Python suite not staged (no reference "
                    "sources at build time)")
    env = dict(os.environ, PHASE2_LIB=str(ROOT / "phase2_b200" /
                                          "libphase2.so"),
               PYTHONPATH=str(PYREF), PHASE2_LOG="warn")
    r = subprocess.run(["python", "-m", "pytest", "-q", "-p",
                        "no:cacheprovider", "--rootdir", str(PYREF),
                        "-c", os.devnull, str(suite)],
                       capture_output=True, text=True, timeout=900,
                       env=env, cwd=str(PYREF))
    assert r.returncode == 0, (r.stdout[-3000:], r.stderr[-2000:])
    assert " passed" in r.stdout and "failed" not in r.stdout, r.stdout[-500:]
