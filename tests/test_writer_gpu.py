"""Per-step output (struct phase2_step_writer) on both sampling paths.

The reference's drivers call the step writer once per step or sample, in
order, as each completes (circ/qdrift.c:125, circ/cmpsit.c:231; ph2run's
writer flushes its file per call, ph2run/data.c:869-871).  Here qdrift and
cmpsit can also run every sample on the device.  These tests check that
a writer sees the same (index, overlap) sequence, in the same order, with
device sampling off, on and automatic; that the sequence equals the
driver's returned overlaps; and that under the automatic mode a run with a
writer keeps the host loop (its launches match the OFF run's), so the
writer is called as each sample completes.
"""

import numpy as np
import pytest

import phase2_b200 as p2
from phase2_b200 import workloads

pytestmark = pytest.mark.gpu

MODES = (p2.DEVICE_SAMPLING_OFF, p2.DEVICE_SAMPLING_AUTO,
         p2.DEVICE_SAMPLING_ON)


@pytest.fixture(autouse=True)
def _world():
    p2.world_ensure()
    yield
    p2.set_device_sampling(p2.DEVICE_SAMPLING_AUTO)
    p2.set_precision(p2.PREC_FP64)


def _run(kind, n, t, d, mode, writer):
    p2.set_device_sampling(mode)
    if kind == "qdrift":
        return p2.qdrift(n, t, d, 6, 40, 0.02, 0xD1, writer=writer,
                         with_stats=True)
    return p2.cmpsit(n, t, d, 4, 3, 20, 30, 0.05, 0.004, 0xD2,
                     writer=writer, with_stats=True)


@pytest.mark.parametrize("kind", ["qdrift", "cmpsit"])
@pytest.mark.parametrize("prec", [p2.PREC_FP64, p2.PREC_FP32])
def test_writer_sequence_on_every_path(kind, prec):
    n = 12
    t = workloads.jw_terms(n, 300, seed=0xA11)
    d = workloads.hamming_dets(n, 3, 6, seed=0xA12)
    p2.set_precision(prec)
    seen, stats = {}, {}
    for mode in MODES:
        calls = []
        z, st = _run(kind, n, t, d, mode,
                     lambda i, v, calls=calls: calls.append((i, v)))
        assert [i for i, _ in calls] == list(range(len(z)))
        assert np.array_equal(np.array([v for _, v in calls]), z)
        seen[mode], stats[mode] = calls, st
    # the same sequence on every path (device sampling reproduces the
    # host loop bit for bit)
    assert seen[p2.DEVICE_SAMPLING_OFF] == seen[p2.DEVICE_SAMPLING_ON]
    assert seen[p2.DEVICE_SAMPLING_OFF] == seen[p2.DEVICE_SAMPLING_AUTO]
    # automatic mode with a writer ran the host loop
    for key in ("launches", "passes", "rotations"):
        assert stats[p2.DEVICE_SAMPLING_AUTO][key] == \
            stats[p2.DEVICE_SAMPLING_OFF][key], key
    # without a writer, automatic mode samples on the device (this width
    # qualifies), and the overlaps are still the same
    z_auto, st_auto = _run(kind, n, t, d, p2.DEVICE_SAMPLING_AUTO, None)
    assert np.array_equal(z_auto, np.array(
        [v for _, v in seen[p2.DEVICE_SAMPLING_OFF]]))
    assert st_auto["launches"] != stats[p2.DEVICE_SAMPLING_OFF]["launches"]
