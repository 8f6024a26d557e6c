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
