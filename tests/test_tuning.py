"""The launch table: the autotuner's files and their loading (CPU).

phase2_b200/autotune.py measures pass-kernel launch choices and writes
them as JSON (report) and as the flat table the library applies at
world_init (phase2_load_tuning, when the GPU name matches).  These tests
need no GPU: the table calls only touch the library's host-side launch
table (phase2_tune_set / phase2_tune_get).
"""

import ctypes as C
import json
from pathlib import Path

import pytest

from phase2_b200 import autotune
from phase2_b200._ffi import lib

PKG = Path(autotune.__file__).resolve().parent


def _table():
    L = lib()
    out = {}
    for prec in (0, 1):
        for m in range(6):
            v, s = C.c_int(), C.c_int()
            assert L.phase2_tune_get(prec, m, C.byref(v), C.byref(s)) == 0
            out[(prec, m)] = (v.value, s.value)
    return out


@pytest.fixture(autouse=True)
def _restore():
    saved = _table()
    runs = lib().phase2_get_batch_runs()
    yield
    L = lib()
    for (prec, m), (v, s) in saved.items():
        L.phase2_tune_set(prec, m, v, s)
    L.phase2_set_batch_runs(runs)


def test_load_matching_gpu(tmp_path):
    path = tmp_path / "t.tab"
    path.write_text("# test table\ngpu TEST GPU\nlaunch 0 3 1 8\n"
                    "  launch 1 5 2 3\n\nlaunch 1 4 0 16\n")
    assert lib().phase2_load_tuning(str(path).encode(), b"TEST GPU") == 3
    t = _table()
    assert t[(0, 3)] == (1, 8)
    assert t[(1, 5)] == (2, 3)
    assert t[(1, 4)] == (0, 16)


def test_batch_runs_line(tmp_path):
    """`batch_runs n` sets the persistent kernel's run length (1..64);
    a value out of range rejects the file."""
    path = tmp_path / "r.tab"
    path.write_text("gpu TEST GPU\nlaunch 0 3 1 8\nbatch_runs 4\n")
    assert lib().phase2_load_tuning(str(path).encode(), b"TEST GPU") == 2
    assert lib().phase2_get_batch_runs() == 4
    for body in ("gpu TEST GPU\nbatch_runs 0\n",
                 "gpu TEST GPU\nbatch_runs 65\n",
                 "gpu TEST GPU\nbatch_runs 2 3\n"):
        bad = tmp_path / "b.tab"
        bad.write_text(body)
        assert lib().phase2_load_tuning(str(bad).encode(), b"TEST GPU") \
            == -1, body
        assert lib().phase2_get_batch_runs() == 4, body


def test_other_gpu_and_bad_files_change_nothing(tmp_path):
    before = _table()
    other = tmp_path / "o.tab"
    other.write_text("gpu SOME OTHER GPU\nlaunch 0 3 1 8\n")
    assert lib().phase2_load_tuning(str(other).encode(), b"TEST GPU") == 0
    assert _table() == before
    for body in ("launch 0 3 1 8\n",                     # no gpu line
                 "gpu TEST GPU\nlaunch 0 9 0 8\n",        # span out of range
                 "gpu TEST GPU\nlaunch 0 3 1\n",          # short entry
                 "gpu TEST GPU\nlaunch 0 3 0 8\nfoo\n",   # unknown line
                 "gpu TEST GPU\nlaunch 1 5 7 8\n"):       # bad variant
        bad = tmp_path / "b.tab"
        bad.write_text(body)
        assert lib().phase2_load_tuning(str(bad).encode(), b"TEST GPU") \
            == -1, body
        assert _table() == before, body
    assert lib().phase2_load_tuning(str(tmp_path / "missing").encode(),
                                    b"TEST GPU") == -1


def test_shipped_table_matches_its_report():
    report = json.loads((PKG / "tuning_b200.json").read_text())
    tab = PKG / "tuning_b200.tab"
    n = lib().phase2_load_tuning(str(tab).encode(), report["gpu"].encode())
    entries = sum(len(v) for v in report["launch"].values())
    assert n == entries + ("batch_runs" in report)
    if "batch_runs" in report:
        assert lib().phase2_get_batch_runs() == report["batch_runs"]["best"]
    t = _table()
    for pname, per_m in report["launch"].items():
        prec = autotune.PRECS[pname]
        for m, e in per_m.items():
            assert t[(prec, int(m))] == (e["variant"], e["per_sm"])


def test_write_table_roundtrip(tmp_path):
    report = {"gpu": "TEST GPU", "nqb": 20, "launch": {
        "fp64": {"5": {"variant": 1, "per_sm": 0}},
        "fp32": {"3": {"variant": 2, "per_sm": 3},
                 "5": {"variant": 0, "per_sm": 32}}},
        "batch_runs": {"kernel_ms": {"1": 2.0, "8": 1.0}, "best": 8}}
    path = tmp_path / "w.tab"
    autotune.write_table(report, path)
    assert lib().phase2_load_tuning(str(path).encode(), b"TEST GPU") == 4
    assert lib().phase2_get_batch_runs() == 8
    t = _table()
    assert t[(0, 5)] == (1, 0)
    assert t[(1, 3)] == (2, 3)
    assert t[(1, 5)] == (0, 32)


def test_apply_sets_the_launch_table():
    report = {"launch": {"fp64": {"4": {"variant": 1, "per_sm": 4}},
                         "fp32": {"5": {"variant": 2, "per_sm": 3}}}}
    assert autotune.apply(report) is report
    t = _table()
    assert t[(0, 4)] == (1, 4)
    assert t[(1, 5)] == (2, 3)
    assert autotune.apply(Path("/nonexistent/table.json")) is None
