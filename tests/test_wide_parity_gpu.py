"""Parity at the benchmark widths against the reference's own CPU path.

The golden file tests/golden/wide.npz comes from the reference drivers
compiled from its sources (tests/golden/make_wide.py, oracle/_ref):

* 26 qubits: one second-order Trotter step of delta 0.05 over the first
  100 terms, in lexicographic order, of the 20,000-term JW Hamiltonian of
  the 26-qubit Strang configuration, 16 determinants (200 rotations).
* 30 qubits: one qDRIFT sample of depth 16 on the 100,000-term JW
  Hamiltonian of the 30-qubit configuration (its seed and step size).

The library runs the same inputs through its drivers (trott2_simul,
qdrift_simul).  FP64 must reproduce the reference bit for bit: the overlap
and every stored amplitude of the final state (a strided sample at 26
qubits; at 30 qubits every 16th non-zero amplitude, with the count and sum
of squares of the non-zero ones).  FP32 (both arithmetic forms) must stay
within 1e-5 of it, the tolerance of the other FP32 tests.
"""

from pathlib import Path

import numpy as np
import pytest

import phase2_b200 as p2
from phase2_b200 import Terms, workloads

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "wide.npz"
FP32_TOL = 1e-5


@pytest.fixture(scope="module")
def wide():
    if not GOLDEN.is_file():
        pytest.fail(f"{GOLDEN} missing: run tests/golden/make_wide.py")
    return dict(np.load(GOLDEN))


@pytest.fixture(autouse=True)
def _world():
    p2.world_ensure()
    yield
    p2.set_precision(p2.PREC_FP64)


def _run(prec, form, fn, *args, **kw):
    p2.set_precision(prec)
    saved = p2.get_fp32_form()
    p2.set_fp32_form(form)
    try:
        return fn(*args, with_stats=True, **kw)
    finally:
        p2.set_fp32_form(saved)
        p2.set_precision(p2.PREC_FP64)


CASES = [("fp64", p2.PREC_FP64, p2.FORM_LIFTED_F32),
         ("fp32_f32arith", p2.PREC_FP32, p2.FORM_LIFTED_F32),
         ("fp32_f64arith", p2.PREC_FP32, p2.FORM_LIFTED),
         ("fp32_mixed", p2.PREC_FP32, p2.FORM_LIFTED_MIXED)]


@pytest.mark.parametrize("name,prec,form", CASES, ids=[c[0] for c in CASES])
def test_trott2_26_first_lex_terms(wide, name, prec, form):
    cfg = workloads.strang26()
    sel = wide["trott2_26_terms"]
    t = cfg["terms"]
    sub = Terms(t.flip[sel], t.phase[sel], t.cf[sel])
    z, st = _run(prec, form, p2.trott2, 26, sub, cfg["dets"], 1,
                 cfg["delta"], state_idx=wide["trott2_26_idx"])
    want_z, want_a = wide["trott2_26_z"], wide["trott2_26_amp"]
    assert st["rotations"] == 2 * len(sel)
    if prec == p2.PREC_FP64:
        assert np.array_equal(z, want_z)
        assert np.array_equal(st["amps"], want_a)
    else:
        assert np.max(np.abs(z - want_z)) < FP32_TOL
        assert np.max(np.abs(st["amps"] - want_a)) < FP32_TOL


@pytest.mark.parametrize("name,prec,form", CASES, ids=[c[0] for c in CASES])
def test_qdrift_30_depth16(wide, name, prec, form):
    cfg = workloads.qdrift30()
    depth = int(wide["qdrift_30_depth"])
    z, st = _run(prec, form, p2.qdrift, 30, cfg["terms"], cfg["dets"], 1,
                 depth, cfg["step_size"], cfg["seed"],
                 state_idx=wide["qdrift_30_idx"])
    want_z, want_a = wide["qdrift_30_z"], wide["qdrift_30_amp"]
    assert st["rotations"] == depth
    if prec == p2.PREC_FP64:
        assert np.array_equal(z, want_z)
        assert np.array_equal(st["amps"], want_a)
    else:
        assert np.max(np.abs(z - want_z)) < FP32_TOL
        assert np.max(np.abs(st["amps"] - want_a)) < FP32_TOL
