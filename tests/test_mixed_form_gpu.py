"""The mixed FP32 form (PHASE2_FORM_LIFTED_MIXED).

On registers of 24 qubits or more its passes run k_pass_lift32h: a coset
whose amplitudes all stay below 2^-10 in magnitude (re and im) is rotated
with FP32 FMAs, as in the FP32-arithmetic form; a coset holding a larger
amplitude when the pass starts is rotated in FP64 by its warp and rounded
once per pass.  Smaller registers, the persistent batch kernel and device
sampling run mixed-form programs with FP64 arithmetic on every coset.

* A 24-qubit state of norm below 2^-10 has no heavy coset at any pass: the
  mixed form gives the FP32-arithmetic form's bits, at every span.
* A 24-qubit state held on 4096 basis states (heavy cosets), rotated by
  large angles: within the FP32 tolerance of FP64, and not the
  FP32-arithmetic form's bits.
* qDRIFT on a state concentrated on one determinant (24 qubits, 4096
  draws a sample at step size 1e-3, host loop): an FP32 shear absorbs the
  small increments of the dominant amplitude, so the FP32-arithmetic form
  drifts; the mixed form's overlaps stay within 1e-5 of FP64 and closer.
* A dense 12-qubit state (FP64 arithmetic on every coset): within the
  tolerance of the oracle and closer than the FP32-arithmetic form.
* The persistent batch kernel and device sampling: within 1e-5 of FP64.

The FP64 path these compare with is bit-identical to the oracle
(tests/test_parity_gpu.py, tests/test_wide_parity_gpu.py).
"""

import math

import numpy as np
import pytest

import phase2_b200 as p2
from phase2_b200 import Register, workloads

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-5


@pytest.fixture(autouse=True)
def _world():
    p2.world_ensure()
    old_form = p2.get_fp32_form()
    p2.set_precision(p2.PREC_FP64)
    p2.set_fusion(5, 0)
    yield
    p2.set_fp32_form(old_form)
    p2.set_precision(p2.PREC_FP64)
    p2.set_device_sampling(p2.DEVICE_SAMPLING_AUTO)


def _rots(n, k, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    t = workloads.random_terms(n, k, seed=int(rng.integers(1 << 30)))
    t.flip[rng.random(k) < 0.2] = 0
    return t.flip, t.phase, rng.uniform(-math.pi, math.pi, k)


def _state(n, seed, support=None):
    rng = np.random.Generator(np.random.PCG64(seed))
    m = (1 << n) if support is None else support
    a = np.zeros(1 << n, dtype=np.complex128)
    idx = (np.arange(m) if support is None else
           rng.choice(1 << n, size=m, replace=False))
    a[idx] = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    return a / np.linalg.norm(a)


def _run(n, prec, form, amp, flip, phase, phi, span=5):
    p2.set_fp32_form(form)
    with Register(n, prec) as r:
        r.set_fusion(span, 0)
        r.set_state(amp)
        r.paulirot(flip, phase, phi)
        return r.get_state()


@pytest.mark.parametrize("span", [1, 3, 5])
def test_light_state_is_the_fp32_form(span):
    n = 24
    # |a| <= ||psi|| = 2^-11 everywhere, at every pass
    amp = _state(n, 900 + span) * 2.0 ** -11
    flip, phase, phi = _rots(n, 120, 901 + span)
    f32 = _run(n, p2.PREC_FP32, p2.FORM_LIFTED_F32, amp, flip, phase, phi,
               span)
    mixed = _run(n, p2.PREC_FP32, p2.FORM_LIFTED_MIXED, amp, flip, phase,
                 phi, span)
    assert np.array_equal(mixed.view(np.float64), f32.view(np.float64))


def test_heavy_cosets_within_tolerance():
    n = 24
    amp = _state(n, 905, support=4096)
    flip, phase, phi = _rots(n, 150, 906)
    want = _run(n, p2.PREC_FP64, p2.FORM_LIFTED, amp, flip, phase, phi)
    f32 = _run(n, p2.PREC_FP32, p2.FORM_LIFTED_F32, amp, flip, phase, phi)
    mixed = _run(n, p2.PREC_FP32, p2.FORM_LIFTED_MIXED, amp, flip, phase,
                 phi)
    assert np.max(np.abs(mixed - want)) < FP32_TOL
    assert not np.array_equal(mixed.view(np.float64), f32.view(np.float64))


def _qdrift(form, prec, sampling, nqb):
    t = workloads.jw_terms(nqb, 2000, seed=0x3F0)
    d = workloads.hamming_dets(nqb, 1, nqb // 2, seed=0x3F1)
    p2.set_fp32_form(form)
    p2.set_precision(prec)
    p2.set_device_sampling(sampling)
    try:
        return p2.qdrift(nqb, t, d, 2, 4096, 1e-3, 0x5EED3)
    finally:
        p2.set_precision(p2.PREC_FP64)


def test_concentrated_qdrift_error():
    off = p2.DEVICE_SAMPLING_OFF
    z64 = _qdrift(p2.FORM_LIFTED, p2.PREC_FP64, off, 24)
    e32 = np.abs(_qdrift(p2.FORM_LIFTED_F32, p2.PREC_FP32, off, 24) - z64)
    emx = np.abs(_qdrift(p2.FORM_LIFTED_MIXED, p2.PREC_FP32, off, 24) - z64)
    assert emx.max() < FP32_TOL
    assert emx.max() < e32.max(), (emx, e32)


def test_small_register_is_fp64_arithmetic(oracle_lib):
    n = 12
    amp = _state(n, 910)
    flip, phase, phi = _rots(n, 300, 911)
    want = oracle_lib.rotate(amp, n, flip, phase, phi)
    err = {}
    for name, form in (("f32", p2.FORM_LIFTED_F32),
                       ("mixed", p2.FORM_LIFTED_MIXED)):
        got = _run(n, p2.PREC_FP32, form, amp, flip, phase, phi)
        err[name] = float(np.max(np.abs(got - want)))
    assert err["mixed"] < FP32_TOL
    assert err["mixed"] < err["f32"], err


def test_device_sampling_and_batch():
    z64 = _qdrift(p2.FORM_LIFTED, p2.PREC_FP64, p2.DEVICE_SAMPLING_OFF, 14)
    zmx = _qdrift(p2.FORM_LIFTED_MIXED, p2.PREC_FP32, p2.DEVICE_SAMPLING_ON,
                  14)
    assert np.max(np.abs(zmx - z64)) < FP32_TOL
    probs = []
    for k in range(6):
        n = 10 + k
        t = workloads.jw_terms(n, 200 + 40 * k, seed=0x3F8 + k)
        d = workloads.hamming_dets(n, 2, n // 2, seed=0x3FF + k)
        probs.append(dict(nqb=n, terms=t, dets=d, steps=3, delta=0.07))
    want = p2.batch("trott", probs)
    p2.set_fp32_form(p2.FORM_LIFTED_MIXED)
    p2.set_precision(p2.PREC_FP32)
    try:
        got, stats = p2.batch("trott", probs, with_stats=True)
    finally:
        p2.set_precision(p2.PREC_FP64)
    assert sum(s["launches"] for s in stats) == 1
    for g, w in zip(got, want):
        assert np.max(np.abs(np.asarray(g) - np.asarray(w))) < FP32_TOL
