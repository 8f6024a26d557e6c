"""The persistent batch kernel: its bounded wait and its finish times.

* Bounded wait: phase2_batch_wait_check runs the kernel on a program that
  can never progress (its only tile taken, never completed).  Every warp
  must give up after the given number of idle rounds and report it; the
  call returns promptly and the device stays usable (a batch run right
  after it matches the oracle).  No GPU fault is involved: the wait simply
  runs out.
* Finish times: phase2_batch_finish_ms reports when each instance of the
  last persistent launch finished; every launched instance has one, and
  an instance with many times the work of the others finishes last.
"""

import time

import numpy as np
import pytest

import phase2_b200 as p2
from phase2_b200 import workloads
from phase2_b200._ffi import lib

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _world():
    p2.world_ensure()
    yield
    p2.set_precision(p2.PREC_FP64)


def test_wait_runs_out_and_is_reported(oracle_lib):
    t0 = time.perf_counter()
    assert lib().phase2_batch_wait_check(20000) == 1
    assert time.perf_counter() - t0 < 10.0
    # the device is usable afterwards
    t = workloads.jw_terms(10, 80, seed=0xB01)
    d = workloads.hamming_dets(10, 2, 5, seed=0xB02)
    zs = p2.batch("trott2", [dict(nqb=10, terms=t, dets=d, steps=2,
                                  delta=0.1)] * 2)
    want = oracle_lib.trott(10, t.flip, t.phase, t.cf, d.idx, d.cf, 2, 0.1,
                            order2=True)
    for z in zs:
        assert np.array_equal(z, want)


@pytest.mark.parametrize("prec", [p2.PREC_FP32, p2.PREC_FP64])
def test_finish_times(prec):
    p2.set_precision(prec)
    probs = []
    for k, steps in enumerate((2, 2, 24)):
        t = workloads.jw_terms(14, 400, seed=0xB10 + k)
        d = workloads.hamming_dets(14, 1, 7, seed=0xB20 + k)
        probs.append(dict(nqb=14, terms=t, dets=d, steps=steps,
                          delta=0.05))
    _, stats = p2.batch("trott", probs, with_stats=True)
    fin = [s["finish_ms"] for s in stats]
    assert all(f is not None and f > 0 for f in fin), fin
    assert fin[2] > max(fin[0], fin[1]), fin


@pytest.mark.parametrize("runs", [1, 64])
def test_run_lengths(runs, oracle_lib):
    """Every run length gives the oracle's bits (FP64): the tiles a warp
    claims at a time change only the schedule.  Out-of-range values are
    refused."""
    with pytest.raises(ValueError):
        p2.set_batch_runs(0)
    probs = []
    for k, n in enumerate((16, 9, 14)):
        t = workloads.jw_terms(n, 60 + 20 * k, seed=0xB30 + k)
        d = workloads.hamming_dets(n, 2, n // 2, seed=0xB40 + k)
        probs.append(dict(nqb=n, terms=t, dets=d, steps=3, delta=0.07))
    p2.set_batch_runs(runs)
    try:
        zs = p2.batch("trott", probs)
    finally:
        p2.set_batch_runs(2)
    for p, z in zip(probs, zs):
        t, d = p["terms"], p["dets"]
        want = oracle_lib.trott(p["nqb"], t.flip, t.phase, t.cf, d.idx, d.cf,
                                3, 0.07)
        assert np.array_equal(z, want)


def test_many_programs(oracle_lib):
    """More programs than a warp has lanes (the scan looks at 32 tickets
    at a time), of uneven sizes: every result is the oracle's (FP64)."""
    probs = []
    for k in range(45):
        n = 5 + k % 8
        t = workloads.jw_terms(n, 12 + k, seed=0xB50 + k)
        d = workloads.hamming_dets(n, 1, n // 2, seed=0xB90 + k)
        probs.append(dict(nqb=n, terms=t, dets=d, steps=1 + k % 4,
                          delta=0.11))
    zs, stats = p2.batch("trott2", probs, with_stats=True)
    assert sum(s["launches"] for s in stats) == 1
    for p, z in zip(probs, zs):
        t, d = p["terms"], p["dets"]
        want = oracle_lib.trott(p["nqb"], t.flip, t.phase, t.cf, d.idx, d.cf,
                                p["steps"], 0.11, order2=True)
        assert np.array_equal(z, want)


def test_hundreds_of_tiny_programs(oracle_lib):
    """Hundreds of programs of 4-9 qubits (registers smaller than one
    1024-amplitude tile; the look over tickets spans ten rounds of 32):
    every result is the oracle's (FP64), and every program has a finish
    time."""
    probs = []
    for k in range(300):
        n = 4 + k % 6
        t = workloads.jw_terms(n, 6 + k % 9, seed=0xC00 + k)
        d = workloads.hamming_dets(n, 1, max(1, n // 2), seed=0xE00 + k)
        probs.append(dict(nqb=n, terms=t, dets=d, steps=1 + k % 3,
                          delta=0.13))
    zs, stats = p2.batch("trott", probs, with_stats=True)
    assert sum(s["launches"] for s in stats) == 1
    assert all(s["finish_ms"] is not None and s["finish_ms"] >= 0
               for s in stats)
    for p, z in zip(probs, zs):
        t, d = p["terms"], p["dets"]
        want = oracle_lib.trott(p["nqb"], t.flip, t.phase, t.cf, d.idx, d.cf,
                                p["steps"], 0.13)
        assert np.array_equal(z, want)
