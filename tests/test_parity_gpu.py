"""GPU parity of libphase2.so against the oracle (the parity tests proper).

Everything here runs the sm_100a kernels through the C-ABI and compares
with the CPU restatement (oracle/liboracle.so), the reference's golden
vectors (tests/golden/) or, for registers too wide for a dense CPU state,
an exact sparse restatement (tests/sparse.py).

Tolerances:
  FP64 state  -- bit-identical (np.array_equal) to the oracle; the bar the
                 path is held to is 1e-12 relative per overlap, which
                 bit-identity implies.
  FP32 state  -- 1e-5 absolute per amplitude / overlap for short runs, for
                 both FP32 forms (FP32 arithmetic: a few FP32 roundings per
                 rotation; FP64 arithmetic: one FP32 rounding per pass).
"""

import ctypes as C
import math

import numpy as np
import pytest

import phase2_b200 as p2
from phase2_b200 import Dets, Register, Terms, workloads

from conftest import GOLDEN
from sparse import rotate as sparse_rotate

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-5


def _cz(v):
    return complex(v[0], v[1])


def _rand_state(rng, n):
    a = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return a / np.linalg.norm(a)


def _rand_rots(rng, n, k, diag_frac=0.2):
    t = workloads.random_terms(n, k, seed=int(rng.integers(1 << 30)))
    t.flip[rng.random(k) < diag_frac] = 0
    return t.flip, t.phase, rng.uniform(-math.pi, math.pi, k)


@pytest.fixture(params=[p2.FORM_LIFTED_F32, p2.FORM_LIFTED,
                        p2.FORM_LIFTED_MIXED],
                ids=["f32arith", "f64arith", "mixed"])
def fp32_form(request):
    """Run an FP32 test under each FP32 arithmetic form."""
    old = p2.get_fp32_form()
    p2.set_fp32_form(request.param)
    yield request.param
    p2.set_fp32_form(old)


@pytest.fixture(scope="module", autouse=True)
def _world():
    p2.world_ensure()
    p2.set_precision(p2.PREC_FP64)
    p2.set_fusion(5, 0)
    yield


# ---- register level ----------------------------------------------------


def test_paulirot_golden_fixture(fp32_form):
    f = np.load(GOLDEN / "paulirot.npz")
    with Register(9, p2.PREC_FP64) as r:
        r.set_state(f["amp0"])
        r.paulirot(f["flip"], f["phase"], f["phi"])
        assert np.array_equal(r.get_state(), f["amp1"])
    with Register(9, p2.PREC_FP32) as r:
        r.set_state(f["amp0"])
        r.paulirot(f["flip"], f["phase"], f["phi"])
        assert np.max(np.abs(r.get_state() - f["amp1"])) < FP32_TOL


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7, 9, 12, 14])
@pytest.mark.parametrize("fusion", [(5, 0), (1, 1), (3, 0), (4, 2)])
def test_random_rotations_bit_exact(n, fusion, oracle_lib):
    rng = np.random.Generator(np.random.PCG64(7 * n + fusion[0]))
    amp = _rand_state(rng, n)
    flip, phase, phi = _rand_rots(rng, n, 120)
    want = oracle_lib.rotate(amp, n, flip, phase, phi)
    with Register(n, p2.PREC_FP64) as r:
        r.set_fusion(*fusion)
        r.set_state(amp)
        r.paulirot(flip, phase, phi, batch=37)
        got = r.get_state()
    assert np.array_equal(got, want)


@pytest.mark.parametrize("v64,v32,per_sm", [(0, 0, 0), (1, 1, 0), (0, 2, 0),
                                             (0, 0, 4), (1, 2, 2),
                                             (0, 3, 0)])
@pytest.mark.parametrize("n", [5, 11, 17])
def test_launch_variants(v64, v32, per_sm, n, fp32_form, oracle_lib):
    """The direct-load and shared-memory-prefetch FP64 kernels give the
    same bits for every span, at several grid densities; the FP32 lifted
    kernels (FP64-arithmetic form: direct, bulk-staged or cp.async-staged)
    stay within tolerance at the same densities."""
    from phase2_b200._ffi import lib
    L = lib()
    saved = []
    for prec, variant in ((0, v64), (1, v32)):
        for m in range(6):
            v, s = C.c_int(), C.c_int()
            L.phase2_tune_get(prec, m, C.byref(v), C.byref(s))
            saved.append((prec, m, v.value, s.value))
            assert L.phase2_tune_set(prec, m, variant, per_sm) == 0
    assert L.phase2_tune_set(0, 5, 2, 0) == -1
    assert L.phase2_tune_set(1, 5, 4, 0) == -1
    try:
        rng = np.random.Generator(np.random.PCG64(300 + n))
        amp = _rand_state(rng, n)
        flip, phase, phi = _rand_rots(rng, n, 150)
        want = oracle_lib.rotate(amp, n, flip, phase, phi)
        for span in (2, 3, 4, 5):
            with Register(n, p2.PREC_FP64) as r:
                r.set_fusion(span, 0)
                r.set_state(amp)
                r.paulirot(flip, phase, phi)
                assert np.array_equal(r.get_state(), want)
            with Register(n, p2.PREC_FP32) as r:
                r.set_fusion(span, 0)
                r.set_state(amp)
                r.paulirot(flip, phase, phi)
                assert np.max(np.abs(r.get_state() - want)) < FP32_TOL
    finally:
        for prec, m, v, s in saved:
            L.phase2_tune_set(prec, m, v, s)


@pytest.mark.parametrize("n", [3, 10, 15])
def test_fp32_state_close(n, fp32_form, oracle_lib):
    rng = np.random.Generator(np.random.PCG64(1000 + n))
    amp = _rand_state(rng, n)
    flip, phase, phi = _rand_rots(rng, n, 200)
    want = oracle_lib.rotate(amp, n, flip, phase, phi)
    with Register(n, p2.PREC_FP32) as r:
        assert r.precision == p2.PREC_FP32
        r.set_state(amp)
        r.paulirot(flip, phase, phi)
        got = r.get_state()
        nrm = r.norm2()
    err = np.max(np.abs(got - want))
    assert err < FP32_TOL * max(1.0, np.max(np.abs(want)) * 10), err
    assert abs(nrm - 1.0) < 1e-5


def test_identity_rotation_is_phase():
    """test/t-qreg.c:139-166: P = I multiplies every amplitude by e^{i phi}."""
    rng = np.random.Generator(np.random.PCG64(1))
    amp = rng.random(1 << 13) + 1j * rng.random(1 << 13)
    with Register(13) as r:
        r.set_state(amp)
        r.paulirot([0], [0], [0.711])
        got = r.get_state()
    assert np.max(np.abs(got - amp * np.exp(1j * 0.711))) < 1e-14


def test_y_and_yyy_explicit():
    """test/t-qreg.c:168-232: exp(i a Y)|0> and exp(i a YYY)|000>."""
    a = 0.11
    with Register(1) as r:
        r.zero()
        r.setamps([0], [2.0])
        r.paulirot([1], [1], [a])
        z = r.getamps([0, 1])
    assert abs(z[0] - 2 * math.cos(a)) < 1e-14
    assert abs(z[1] + 2 * math.sin(a)) < 1e-14
    with Register(3) as r:
        r.zero()
        r.setamps([0], [2.0])
        r.paulirot([7], [7], [a])
        z = r.getamps([0, 7])
    assert abs(z[0] - 2 * math.cos(a)) < 1e-14
    assert abs(z[1] - 2 * math.sin(a)) < 1e-14


def test_get_set_zero_roundtrip():
    rng = np.random.Generator(np.random.PCG64(2))
    n = 13
    amp = rng.random(1 << n) + 1j * rng.random(1 << n)
    with Register(n) as r:
        idx = np.arange(1 << n, dtype=np.uint64)
        r.setamps(idx, amp)
        assert np.array_equal(r.getamps(idx), amp)
        r.zero()
        assert not np.any(r.get_state())
        # later writes win on duplicate indices, as sequential setamp
        r.setamps([5, 5, 9], [1.0, 2.0, 3.0])
        assert np.array_equal(r.getamps([5, 9]), [2.0, 3.0])
        with pytest.raises(RuntimeError):
            r.getamps([1 << n])


def test_deterministic_across_runs():
    """test/t-qreg.c:456-503: identical inputs give identical bits."""
    rng = np.random.Generator(np.random.PCG64(3))
    amp = _rand_state(rng, 12)
    flip, phase, phi = _rand_rots(rng, 12, 300)
    outs = []
    for _ in range(2):
        with Register(12) as r:
            r.set_state(amp)
            r.paulirot(flip, phase, phi)
            outs.append(r.get_state())
    assert np.array_equal(outs[0], outs[1])


def test_stats_count_passes():
    t = workloads.jw_terms(16, 256, seed=5)
    with Register(16) as r:
        r.reset_stats()
        r.paulirot(t.flip, t.phase, np.full(len(t), 0.01))
        r.synchronize()
        st = r.stats()
    assert st["rotations"] == 256
    assert 0 < st["passes"] < 256
    assert st["bytes"] == st["passes"] * 2 * (1 << 16) * 16
    assert st["sweeps"] == st["passes"]


@pytest.fixture
def f32_arith():
    """The FP32-arithmetic form, the one sweeps run in."""
    old = p2.get_fp32_form()
    p2.set_fp32_form(p2.FORM_LIFTED_F32)
    yield
    p2.set_fp32_form(old)


def _fp32_run(n, amp, flip, phase, phi, shape, kernel=True):
    """FP32 register through the pass executor under a sweep shape, the
    planned sweeps run as one kernel each or one kernel per pass."""
    old = p2.get_sweep()
    p2.set_sweep(*shape)
    p2.set_sweep_kernel(kernel)
    try:
        with Register(n, p2.PREC_FP32) as r:
            r.set_state(amp)
            r.reset_stats()
            r.paulirot(flip, phase, phi)
            out = r.get_state()
            st = r.stats()
    finally:
        p2.set_sweep(*old)
        p2.set_sweep_kernel(True)
    return out, st


@pytest.mark.parametrize("tile,low", [(13, 5), (12, 4), (14, 6), (13, 4),
                                      (11, 3), (14, 5)])
@pytest.mark.parametrize("n", [17, 20])
def test_sweeps_bit_identical(tile, low, n, oracle_lib, f32_arith):
    """A plan's sweeps run as one kernel each (shared-memory tiles, one
    state round trip per sweep) give the same bits as one kernel per pass
    of the same plan, for every tile shape; and fewer round trips."""
    rng = np.random.Generator(np.random.PCG64(70 * n + tile))
    amp = _rand_state(rng, n)
    jw = workloads.jw_terms(n, 3000, seed=n * tile + low)
    pick = rng.integers(0, len(jw), 700)  # qDRIFT-like random draws
    flip, phase = jw.flip[pick], jw.phase[pick]
    phi = rng.uniform(-math.pi, math.pi, len(pick))
    want, st0 = _fp32_run(n, amp, flip, phase, phi, (tile, low), False)
    got, st1 = _fp32_run(n, amp, flip, phase, phi, (tile, low))
    assert np.array_equal(got, want)
    assert st0["sweeps"] == st0["passes"] == st1["passes"]
    assert st1["sweeps"] < st1["passes"]
    assert st1["bytes"] == st1["sweeps"] * 2 * (1 << n) * 8
    if n <= 17:
        ref = oracle_lib.rotate(amp, n, flip, phase, phi)
        assert np.max(np.abs(got - ref)) < FP32_TOL
    # the sweep-free plan of the same rotations agrees to FP32 rounding
    plain, _ = _fp32_run(n, amp, flip, phase, phi, (0, 5))
    assert np.max(np.abs(plain - got)) < FP32_TOL


@pytest.mark.parametrize("span,rots", [(5, 0), (3, 0), (2, 7), (1, 1)])
def test_sweeps_fusion_settings_and_random_strings(span, rots, f32_arith):
    """Sweep kernels under every fusion setting, with diagonal strings and
    random (wide) flip masks: bit-identical to one kernel per pass."""
    n = 18
    rng = np.random.Generator(np.random.PCG64(span * 10 + rots))
    amp = _rand_state(rng, n)
    jw = workloads.jw_terms(n, 300, seed=span)
    fl, ph, phi = _rand_rots(rng, n, 200, diag_frac=0.3)
    flip = np.concatenate([jw.flip, fl, jw.flip[:50]])
    phase = np.concatenate([jw.phase, ph, jw.phase[:50]])
    ang = np.concatenate([rng.uniform(-3, 3, len(jw)), phi,
                          rng.uniform(-3, 3, 50)])
    outs = []
    old = p2.get_sweep()
    p2.set_sweep(13, 5)
    try:
        for kernel in (False, True):
            p2.set_sweep_kernel(kernel)
            with Register(n, p2.PREC_FP32) as r:
                r.set_fusion(span, rots)
                r.set_state(amp)
                r.paulirot(flip, phase, ang)
                outs.append(r.get_state())
    finally:
        p2.set_sweep_kernel(True)
        p2.set_sweep(*old)
    assert np.array_equal(outs[0], outs[1])


def test_sweeps_drivers_and_graphs(oracle_lib, f32_arith):
    """Trotter steps replayed from CUDA graphs and qDRIFT samples (host and
    device sampling) with sweep kernels: the same overlaps as one kernel
    per pass of the same plans; within FP32 tolerance of the oracle."""
    t = workloads.jw_terms(18, 500, seed=44)
    d = workloads.hamming_dets(18, 3, 9, seed=45)
    res = {}
    old = p2.get_sweep()
    p2.set_precision(p2.PREC_FP32)
    p2.set_sweep(13, 5)
    try:
        for kernel in (False, True):
            p2.set_sweep_kernel(kernel)
            p2.set_device_sampling(False)
            z1, st = p2.trott2(18, t, d, 6, 0.1, with_stats=True)
            z2 = p2.qdrift(18, t, d, 3, 700, 0.02, 0x51)
            p2.set_device_sampling(True)
            z3 = p2.qdrift(18, t, d, 3, 700, 0.02, 0x51)
            res[kernel] = (z1, z2, st, z3)
    finally:
        p2.set_sweep_kernel(True)
        p2.set_sweep(*old)
        p2.set_device_sampling(p2.DEVICE_SAMPLING_AUTO)
        p2.set_precision(p2.PREC_FP64)
    assert np.array_equal(res[False][0], res[True][0])
    assert np.array_equal(res[False][1], res[True][1])
    # device sampling plans the same sweeps and runs them pass by pass
    assert np.array_equal(res[True][3], res[True][1])
    assert res[True][2]["graph_replays"] >= 3
    assert res[True][2]["sweeps"] < res[False][2]["sweeps"]
    want = oracle_lib.trott(18, t.flip, t.phase, t.cf, d.idx, d.cf, 6, 0.1,
                            order2=True)
    assert np.max(np.abs(res[True][0] - want)) < FP32_TOL
    want = oracle_lib.qdrift(18, t.flip, t.phase, t.cf, d.idx, d.cf, 3, 700,
                             0.02, 0x51)
    assert np.max(np.abs(res[True][1] - want)) < FP32_TOL


# ---- drivers -----------------------------------------------------------


def _driver_case(c):
    t = Terms(np.array(c["flip"], dtype=np.uint64),
              np.array(c["phase"], dtype=np.uint64), np.array(c["cf"]))
    d = Dets(np.array(c["det_idx"], dtype=np.uint64),
             np.array([_cz(v) for v in c["det_cf"]]))
    return t, d


def test_drivers_match_golden(golden):
    for c in golden["drivers"]:
        t, d = _driver_case(c)
        n = c["nqb"]
        if c["kind"] in ("trott", "trott2"):
            p2.set_term_order(0 if c["lex"] else 1)
            fn = p2.trott if c["kind"] == "trott" else p2.trott2
            z = fn(n, t, d, c["steps"], c["delta"])
        elif c["kind"] == "qdrift":
            p2.set_term_order(0)
            z = p2.qdrift(n, t, d, c["samples"], c["depth"], c["step_size"],
                          c["seed"])
        else:
            p2.set_term_order(0)
            z = p2.cmpsit(n, t, d, c["samples"], c["steps"], c["length"],
                          c["depth"], c["angle_det"], c["angle_rand"],
                          c["seed"])
        want = np.array([_cz(v) for v in c["z"]])
        assert np.all(np.abs(z - want) <= 1e-12 * np.maximum(1, abs(want)))
        assert np.array_equal(z, want), c["kind"]
    p2.set_term_order(0)


def test_trotter12_golden(golden):
    cfg = workloads.trotter12()
    z = p2.trott(12, cfg["terms"], cfg["dets"], cfg["steps"], cfg["delta"])
    want = np.array([_cz(v) for v in golden["trotter12"]["z"]])
    assert np.array_equal(z, want)


def test_trotter12_fp32(golden, fp32_form):
    cfg = workloads.trotter12()
    p2.set_precision(p2.PREC_FP32)
    try:
        z = p2.trott(12, cfg["terms"], cfg["dets"], cfg["steps"],
                     cfg["delta"])
    finally:
        p2.set_precision(p2.PREC_FP64)
    want = np.array([_cz(v) for v in golden["trotter12"]["z"]])
    assert np.max(np.abs(z - want)) < FP32_TOL


def _h2o(golden):
    h = golden["h2o"]
    return h, Terms(np.array(h["flip"], dtype=np.uint64),
                    np.array(h["phase"], dtype=np.uint64),
                    np.array(h["cf"])), \
        Dets(np.array(h["det_idx"], dtype=np.uint64),
             np.array([_cz(v) for v in h["det_cf"]]))


def _h2o_runs(t, d):
    return {
        "trott": lambda: p2.trott(10, t, d, 12, 0.5),
        "trott2": lambda: p2.trott2(10, t, d, 12, 0.5),
        "qdrift": lambda: p2.qdrift(10, t, d, 6, 300, 0.01, 0xC0FFEE),
        "cmpsit": lambda: p2.cmpsit(10, t, d, 3, 4, 60, 50, 0.1, 0.02,
                                    0xBEEF),
    }


@pytest.mark.parametrize("fusion", [(1, 1), (5, 0)])
def test_h2o_fixture_fp64(golden, fusion):
    """The reference's water CAS(5,6) Hamiltonian (251 terms, 10 qubits)
    through all four drivers: bit-identical to the reference's outputs."""
    h, t, d = _h2o(golden)
    p2.set_fusion(*fusion)
    try:
        for kind, run in _h2o_runs(t, d).items():
            want = np.array([_cz(v) for v in h[kind]])
            assert np.array_equal(run(), want), kind
    finally:
        p2.set_fusion(5, 0)


def test_h2o_fixture_fp32(golden, fp32_form):
    h, t, d = _h2o(golden)
    p2.set_precision(p2.PREC_FP32)
    try:
        for kind, run in _h2o_runs(t, d).items():
            want = np.array([_cz(v) for v in h[kind]])
            assert np.max(np.abs(run() - want)) < FP32_TOL, kind
    finally:
        p2.set_precision(p2.PREC_FP64)


@pytest.mark.parametrize("order2", [False, True])
def test_trott_jw_vs_oracle(order2, oracle_lib):
    t = workloads.jw_terms(12, 300, seed=11)
    d = workloads.hamming_dets(12, 6, 6, seed=12)
    fn = p2.trott2 if order2 else p2.trott
    z = fn(12, t, d, 5, 0.2)
    want = oracle_lib.trott(12, t.flip, t.phase, t.cf, d.idx, d.cf, 5, 0.2,
                            order2=order2)
    assert np.array_equal(z, want)


def test_qdrift_cmpsit_vs_oracle(oracle_lib):
    t = workloads.jw_terms(11, 500, seed=13)
    d = workloads.hamming_dets(11, 3, 5, seed=14)
    z = p2.qdrift(11, t, d, 5, 300, 0.01, 0xABC)
    want = oracle_lib.qdrift(11, t.flip, t.phase, t.cf, d.idx, d.cf, 5, 300,
                             0.01, 0xABC)
    assert np.array_equal(z, want)
    z = p2.cmpsit(11, t, d, 2, 3, 50, 100, 0.05, 0.002, 0xDEF)
    want = oracle_lib.cmpsit(11, t.flip, t.phase, t.cf, d.idx, d.cf, 2, 3,
                             50, 100, 0.05, 0.002, 0xDEF)
    assert np.array_equal(z, want)


def test_flip_order_vs_oracle_given_order(oracle_lib):
    t = workloads.jw_terms(13, 400, seed=15)
    d = workloads.hamming_dets(13, 4, 6, seed=16)
    p2.set_term_order(2)
    try:
        z = p2.trott2(13, t, d, 3, 0.1)
    finally:
        p2.set_term_order(0)
    s = workloads.sort_by_flip(t)
    want = oracle_lib.trott(13, s.flip, s.phase, s.cf, d.idx, d.cf, 3, 0.1,
                            order2=True, sort_lex=False)
    assert np.array_equal(z, want)


def test_graph_replay_is_exact(oracle_lib):
    """Repeated Trotter steps replay a captured CUDA graph; the result is
    unchanged (bit-identical to the oracle)."""
    t = workloads.jw_terms(14, 200, seed=41)
    d = workloads.hamming_dets(14, 3, 7, seed=42)
    z, st = p2.trott(14, t, d, 8, 0.1, with_stats=True)
    assert st["graph_replays"] >= 5
    want = oracle_lib.trott(14, t.flip, t.phase, t.cf, d.idx, d.cf, 8, 0.1)
    assert np.array_equal(z, want)


def test_batched_drivers_match_single(oracle_lib):
    """Independent problems of uneven size run together; every result is
    bit-identical to the oracle run of that problem alone."""
    probs = []
    for k, n in enumerate((8, 13, 10, 15, 9, 12)):
        t = workloads.jw_terms(n, 40 + 30 * k, seed=500 + k)
        d = workloads.hamming_dets(n, 1 + k % 3, n // 2, seed=600 + k)
        probs.append(dict(nqb=n, terms=t, dets=d, steps=3 + k, delta=0.1,
                          samples=2 + k % 2, depth=50 + 10 * k,
                          step_size=0.02, seed=700 + k))
    for kind in ("trott", "trott2"):
        got = p2.batch(kind, probs)
        for p, z in zip(probs, got):
            t, d = p["terms"], p["dets"]
            want = oracle_lib.trott(p["nqb"], t.flip, t.phase, t.cf, d.idx,
                                    d.cf, p["steps"], p["delta"],
                                    order2=kind == "trott2")
            assert np.array_equal(z, want), kind
    got = p2.batch("qdrift", probs)
    for p, z in zip(probs, got):
        t, d = p["terms"], p["dets"]
        want = oracle_lib.qdrift(p["nqb"], t.flip, t.phase, t.cf, d.idx,
                                 d.cf, p["samples"], p["depth"],
                                 p["step_size"], p["seed"])
        assert np.array_equal(z, want)
    cm = [dict(p, samples=2, steps=2, length=8, depth=20, angle_det=0.05,
               angle_rand=0.01) for p in probs]
    got = p2.batch("cmpsit", cm)
    for p, z in zip(cm, got):
        t, d = p["terms"], p["dets"]
        want = oracle_lib.cmpsit(p["nqb"], t.flip, t.phase, t.cf, d.idx,
                                 d.cf, 2, 2, 8, 20, 0.05, 0.01, p["seed"])
        assert np.array_equal(z, want)


def _uneven_problems():
    probs = []
    for k, n in enumerate((8, 13, 10, 15, 9, 12, 18, 11)):
        t = workloads.jw_terms(n, 40 + 30 * k, seed=900 + k)
        d = workloads.hamming_dets(n, 1 + k % 3, n // 2, seed=950 + k)
        probs.append(dict(nqb=n, terms=t, dets=d, steps=2 + k % 5,
                          delta=0.1, samples=1 + k % 3, depth=30 + 7 * k,
                          step_size=0.02, seed=990 + k, length=6,
                          angle_det=0.05, angle_rand=0.01))
    return probs


@pytest.mark.parametrize("kind", ["trott", "trott2", "qdrift", "cmpsit"])
def test_persistent_batch(kind, fp32_form, oracle_lib):
    """FP32 batches in one persistent launch (both FP32 forms): bit-identical
    to the same batch run on per-instance streams (same plans, same
    per-coset arithmetic), within the FP32 tolerance of the FP64 oracle,
    and one kernel launch for the whole batch."""
    probs = _uneven_problems()
    if kind == "cmpsit":
        probs = [dict(p, samples=2, steps=2, depth=12) for p in probs]
    p2.set_precision(p2.PREC_FP32)
    try:
        p2.set_batch_persistent(True)
        got, stats = p2.batch(kind, probs, with_stats=True)
        p2.set_batch_persistent(False)
        ref = p2.batch(kind, probs)
    finally:
        p2.set_batch_persistent(True)
        p2.set_precision(p2.PREC_FP64)
    assert sum(s["launches"] for s in stats) == 1
    assert all(s["passes"] > 0 for s in stats)
    for p, z, r in zip(probs, got, ref):
        assert np.array_equal(z, r), kind
        t, d = p["terms"], p["dets"]
        if kind in ("trott", "trott2"):
            want = oracle_lib.trott(p["nqb"], t.flip, t.phase, t.cf, d.idx,
                                    d.cf, p["steps"], p["delta"],
                                    order2=kind == "trott2")
        elif kind == "qdrift":
            want = oracle_lib.qdrift(p["nqb"], t.flip, t.phase, t.cf, d.idx,
                                     d.cf, p["samples"], p["depth"],
                                     p["step_size"], p["seed"])
        else:
            want = oracle_lib.cmpsit(p["nqb"], t.flip, t.phase, t.cf, d.idx,
                                     d.cf, 2, 2, p["length"], 12,
                                     p["angle_det"], p["angle_rand"],
                                     p["seed"])
        assert np.max(np.abs(z - want)) < FP32_TOL, kind


def _qdrift_both_ways(nqb, t, d, samples, depth, step, seed,
                      prec=p2.PREC_FP32):
    """qdrift with host sampling, then with device sampling."""
    p2.set_precision(prec)
    p2.set_device_sampling(False)
    try:
        host, hst = p2.qdrift(nqb, t, d, samples, depth, step, seed,
                              with_stats=True, with_state=True)
        p2.set_device_sampling(True)
        dev, st = p2.qdrift(nqb, t, d, samples, depth, step, seed,
                            with_stats=True, with_state=True)
    finally:
        p2.set_device_sampling(p2.DEVICE_SAMPLING_AUTO)
        p2.set_precision(p2.PREC_FP64)
    # the register ends holding the last sample's state either way
    assert np.array_equal(st["state"], hst["state"])
    return host, dev, st


@pytest.mark.parametrize("prec", [p2.PREC_FP32, p2.PREC_FP64],
                         ids=["fp32", "fp64"])
@pytest.mark.parametrize("nqb,nterms,ndet,samples,depth", [
    (9, 60, 1, 3, 40),        # one determinant, short circuits
    (11, 500, 5, 5, 300),
    (12, 200, 3, 2, 9000),    # planned in two chunks of the host queue
    (8, 30, 2, 4200, 3),      # two planning rounds, the last one short
    (16, 300, 4, 7, 700),
])
def test_qdrift_device_sampling(nqb, nterms, ndet, samples, depth, prec,
                                oracle_lib):
    """Device sampling (draws, plans and passes on the GPU; small registers
    run many samples at once on copies of the state) gives the host loop's
    overlaps and final register bit for bit; FP64 registers also match the
    oracle bit for bit, FP32 ones within the FP32 tolerance."""
    t = workloads.jw_terms(nqb, nterms, seed=nqb * 7 + depth)
    # a term below DBL_EPSILON draws the zero angle
    t.cf[3] = 1e-17
    d = workloads.hamming_dets(nqb, ndet, nqb // 2, seed=nqb + ndet)
    host, dev, st = _qdrift_both_ways(nqb, t, d, samples, depth, 0.02,
                                      0x5EED + nqb, prec)
    assert np.array_equal(dev, host)
    assert st["passes"] > 0 and st["launches"] >= 3
    if samples * depth <= 20000 or prec == p2.PREC_FP64 and nqb <= 12:
        want = oracle_lib.qdrift(nqb, t.flip, t.phase, t.cf, d.idx, d.cf,
                                 samples, depth, 0.02, 0x5EED + nqb)
        if prec == p2.PREC_FP64:
            assert np.array_equal(dev, want)
        else:
            assert np.max(np.abs(dev - want)) < FP32_TOL


@pytest.mark.parametrize("prec", [p2.PREC_FP32, p2.PREC_FP64],
                         ids=["fp32", "fp64"])
def test_device_sampling_edges(prec, oracle_lib):
    """Edges under forced device sampling, as the host loop has them: a
    determinant outside the register is refused; zero samples give no
    output; cmpsit with zero steps (prepst and measure only) and qdrift
    with depth 1 match the oracle."""
    n = 10
    t = workloads.jw_terms(n, 80, seed=3)
    d = workloads.hamming_dets(n, 2, 5, seed=4)
    bad = Dets(np.array([3, 1 << n], dtype=np.uint64),
               np.array([0.6 + 0j, 0.8 + 0j]))
    p2.set_precision(prec)
    tol = 0.0 if prec == p2.PREC_FP64 else FP32_TOL
    try:
        for mode in (False, True):
            p2.set_device_sampling(mode)
            with pytest.raises(RuntimeError):
                p2.qdrift(n, t, bad, 2, 10, 0.01, 5)
            assert len(p2.qdrift(n, t, d, 0, 10, 0.01, 5)) == 0
            z = p2.cmpsit(n, t, d, 2, 0, 5, 8, 0.05, 0.01, 7)
            want = oracle_lib.cmpsit(n, t.flip, t.phase, t.cf, d.idx, d.cf,
                                     2, 0, 5, 8, 0.05, 0.01, 7)
            assert np.max(np.abs(z - want)) <= tol
            z = p2.qdrift(n, t, d, 3, 1, 0.01, 6)
            want = oracle_lib.qdrift(n, t.flip, t.phase, t.cf, d.idx, d.cf,
                                     3, 1, 0.01, 6)
            assert np.max(np.abs(z - want)) <= tol
    finally:
        p2.set_device_sampling(p2.DEVICE_SAMPLING_AUTO)
        p2.set_precision(p2.PREC_FP64)


def test_device_sampling_on_a_nearly_full_device():
    """With too little free memory for state copies, device sampling runs
    its samples on the register alone (smaller rounds if need be) and
    still gives the host loop's overlaps bit for bit."""
    torch = pytest.importorskip("torch")
    n = 24
    t = workloads.jw_terms(n, 600, seed=24)
    d = workloads.hamming_dets(n, 2, 12, seed=25)
    p2.set_precision(p2.PREC_FP32)
    try:
        p2.set_device_sampling(False)
        host = p2.qdrift(n, t, d, 6, 500, 0.01, 0xF011)
        free, _ = torch.cuda.mem_get_info()
        # room for the 128 MiB register and a little scratch, not for
        # the three 128 MiB copies four concurrent samples would need
        hold = torch.empty(free - (400 << 20), dtype=torch.uint8,
                           device="cuda")
        try:
            p2.set_device_sampling(True)
            dev = p2.qdrift(n, t, d, 6, 500, 0.01, 0xF011)
        finally:
            del hold
            torch.cuda.empty_cache()
    finally:
        p2.set_device_sampling(p2.DEVICE_SAMPLING_AUTO)
        p2.set_precision(p2.PREC_FP64)
    assert np.array_equal(dev, host)


def _cmpsit_both_ways(nqb, t, d, samples, steps, length, depth, adet,
                      arand, seed, prec=p2.PREC_FP32):
    """cmpsit with host sampling, then with device sampling."""
    args = (nqb, t, d, samples, steps, length, depth, adet, arand, seed)
    p2.set_precision(prec)
    p2.set_device_sampling(False)
    try:
        host, hst = p2.cmpsit(*args, with_stats=True, with_state=True)
        p2.set_device_sampling(True)
        dev, st = p2.cmpsit(*args, with_stats=True, with_state=True)
    finally:
        p2.set_device_sampling(p2.DEVICE_SAMPLING_AUTO)
        p2.set_precision(p2.PREC_FP64)
    assert np.array_equal(st["state"], hst["state"])
    return host, dev, st


@pytest.mark.parametrize("nqb,nterms,ndet,samples,steps,length,depth", [
    (9, 60, 1, 3, 2, 8, 12),
    (11, 400, 3, 2, 3, 50, 100),
    (12, 1500, 2, 2, 2, 1000, 3000),  # halves straddle queue chunks
    (8, 40, 2, 300, 1, 5, 3),        # many samples on register copies
    (10, 50, 2, 3, 2, 10, 0),        # head terms only
    (10, 50, 2, 3, 2, 0, 20),        # draws only
])
@pytest.mark.parametrize("prec", [p2.PREC_FP32, p2.PREC_FP64],
                         ids=["fp32", "fp64"])
def test_cmpsit_device_sampling(nqb, nterms, ndet, samples, steps, length,
                                depth, prec, oracle_lib):
    """cmpsit with device sampling (forward and reversed halves of head
    terms and fresh draws on the GPU) gives the host loop's overlaps and
    final register bit for bit; FP64 also the oracle's bits, FP32 within
    the FP32 tolerance."""
    t = workloads.jw_terms(nqb, nterms, seed=nqb * 11 + depth)
    t.cf[5] = -1e-17  # a drawn term in the sign dead zone
    d = workloads.hamming_dets(nqb, ndet, nqb // 2, seed=nqb + 2 * ndet)
    args = (samples, steps, length, depth, 0.05, 0.004, 0xC0DE + nqb)
    host, dev, st = _cmpsit_both_ways(nqb, t, d, *args, prec=prec)
    assert np.array_equal(dev, host)
    assert st["passes"] > 0
    if samples * steps * (length + depth) <= 20000:
        want = oracle_lib.cmpsit(nqb, t.flip, t.phase, t.cf, d.idx, d.cf,
                                 *args)
        if prec == p2.PREC_FP64:
            assert np.array_equal(dev, want)
        else:
            assert np.max(np.abs(dev - want)) < FP32_TOL


@pytest.mark.parametrize("kind", ["qdrift", "cmpsit"])
def test_device_sampling_fp64_arith(kind, oracle_lib):
    """Device sampling of an FP32 register in the FP64-arithmetic form
    (the persistent kernel's FP64-arithmetic instance): the host loop's
    overlaps and final register bit for bit, within the FP32 tolerance of
    the oracle."""
    old = p2.get_fp32_form()
    p2.set_fp32_form(p2.FORM_LIFTED)
    try:
        t = workloads.jw_terms(11, 400, seed=0xF64A)
        d = workloads.hamming_dets(11, 3, 5, seed=0xF64B)
        if kind == "qdrift":
            args = (5, 300, 0.02, 0x5EE1)
            host, dev, _ = _qdrift_both_ways(11, t, d, *args)
            want = oracle_lib.qdrift(11, t.flip, t.phase, t.cf, d.idx,
                                     d.cf, *args)
        else:
            args = (3, 2, 40, 120, 0.05, 0.004, 0xC0DF)
            host, dev, _ = _cmpsit_both_ways(11, t, d, *args,
                                             prec=p2.PREC_FP32)
            want = oracle_lib.cmpsit(11, t.flip, t.phase, t.cf, d.idx,
                                     d.cf, *args)
    finally:
        p2.set_fp32_form(old)
    assert np.array_equal(dev, host)
    assert np.max(np.abs(dev - want)) < FP32_TOL


def test_device_sampling_h2o(golden):
    """The water fixture (real molecular terms) under device sampling."""
    _, t, d = _h2o(golden)
    host, dev, _ = _qdrift_both_ways(10, t, d, 6, 300, 0.01, 0xC0FFEE)
    assert np.array_equal(dev, host)
    want = np.array([_cz(v) for v in golden["h2o"]["qdrift"]])
    assert np.max(np.abs(dev - want)) < FP32_TOL
    host, dev, _ = _cmpsit_both_ways(10, t, d, 3, 4, 60, 50, 0.1, 0.02,
                                     0xBEEF)
    assert np.array_equal(dev, host)
    want = np.array([_cz(v) for v in golden["h2o"]["cmpsit"]])
    assert np.max(np.abs(dev - want)) < FP32_TOL


@pytest.mark.parametrize("kind", ["trott", "trott2", "qdrift", "cmpsit"])
def test_persistent_batch_fp64(kind, oracle_lib):
    """FP64 batches in one persistent launch (the exact per-coset
    arithmetic of the pass kernel): every result bit-identical to the
    oracle and to the per-instance stream mode, one kernel launch."""
    probs = _uneven_problems()[:5]
    if kind == "cmpsit":
        probs = [dict(p, samples=2, steps=2, depth=12) for p in probs]
    try:
        p2.set_batch_persistent(True)
        got, stats = p2.batch(kind, probs, with_stats=True)
        p2.set_batch_persistent(False)
        ref = p2.batch(kind, probs)
    finally:
        p2.set_batch_persistent(True)
    assert sum(s["launches"] for s in stats) == 1
    for p, z, r in zip(probs, got, ref):
        assert np.array_equal(z, r), kind
        t, d = p["terms"], p["dets"]
        if kind in ("trott", "trott2"):
            want = oracle_lib.trott(p["nqb"], t.flip, t.phase, t.cf, d.idx,
                                    d.cf, p["steps"], p["delta"],
                                    order2=kind == "trott2")
        elif kind == "qdrift":
            want = oracle_lib.qdrift(p["nqb"], t.flip, t.phase, t.cf, d.idx,
                                     d.cf, p["samples"], p["depth"],
                                     p["step_size"], p["seed"])
        else:
            want = oracle_lib.cmpsit(p["nqb"], t.flip, t.phase, t.cf, d.idx,
                                     d.cf, 2, 2, p["length"], 12,
                                     p["angle_det"], p["angle_rand"],
                                     p["seed"])
        assert np.array_equal(z, want), kind


def test_persistent_batch_empty_and_single():
    """Edge cases: an empty batch, one instance, an instance with no
    outputs (zero steps) beside others."""
    assert p2.batch("trott", []) == []
    probs = _uneven_problems()[:3]
    probs[1] = dict(probs[1], steps=0)
    p2.set_precision(p2.PREC_FP32)
    try:
        one = p2.batch("trott", probs[:1])
        got = p2.batch("trott", probs)
    finally:
        p2.set_precision(p2.PREC_FP64)
    assert np.array_equal(one[0], got[0])
    assert len(got[1]) == 0


# ---- coefficient-matrix trial states ----------------------------------


def _coeff_state(c):
    cm = p2.CoeffMatrix(
        n_sites=c["n_sites"], n_alpha=c["n_alpha"], n_beta=c["n_beta"],
        C_alpha=[np.array(a) for a in c["C_alpha"]],
        C_beta=(None if c["C_beta"] is None
                else [np.array(b) for b in c["C_beta"]]),
        weights=c["weights"], tapered=c["tapered"])
    g = np.random.Generator(np.random.PCG64(c["psi_seed"]))
    n = c["nqb"]
    return n, cm, g.standard_normal(1 << n) + 1j * g.standard_normal(1 << n)


def test_coeff_matrix_golden(golden, fp32_form):
    """Device expansion bit-identical to the reference's (FP64) and its
    device overlap within 1e-12 relative of the reference's sequential sum;
    FP32 registers within the FP32 tolerance."""
    for c in golden["coeff_matrix"]:
        n, cm, psi = _coeff_state(c)
        want = np.zeros(1 << n, dtype=np.complex128)
        want[c["expand_idx"]] = c["expand_val"]
        z_ref = _cz(c["inner"])
        with Register(n, p2.PREC_FP64) as r:
            r.coeff_expand(cm)
            assert np.array_equal(r.get_state(), want)
            r.set_state(psi)
            z = r.coeff_inner(cm)
        assert abs(z - z_ref) <= 1e-12 * max(1.0, abs(z_ref))
        with Register(n, p2.PREC_FP32) as r:
            r.coeff_expand(cm)
            got = r.get_state()
            assert np.max(np.abs(got - want)) <= 1e-6 * max(
                1.0, np.max(np.abs(want)))


@pytest.mark.parametrize("kind", ["trott", "trott2"])
def test_coeff_matrix_drivers(kind, oracle_lib):
    """Drivers with a coefficient-matrix initial state and overlap (the
    coeff_matrix branch of circ_prepst / circ_measure): equal to the
    oracle's expand -> sorted rotations -> sequential overlap, to 1e-12."""
    rng = np.random.Generator(np.random.PCG64(77))
    ns, na, nb = 5, 2, 2
    blocks = 2
    cm = p2.CoeffMatrix(ns, na, nb,
                        [rng.standard_normal((ns, na)) for _ in range(blocks)],
                        [rng.standard_normal((ns, nb)) for _ in range(blocks)],
                        [0.8, -0.6])
    n = 2 * ns
    t = workloads.jw_terms(n, 60, seed=78)
    steps, delta = 3, 0.2
    z = (p2.trott if kind == "trott" else p2.trott2)(n, t, cm, steps, delta)
    rec = oracle_lib.sort_lex(t.flip, t.phase, t.cf)
    amp = oracle_lib.coeff_expand(n, cm)
    want = []
    for _ in range(steps):
        if kind == "trott":
            amp = oracle_lib.rotate(amp, n, rec["flip"], rec["phase"],
                                    delta * rec["cf"])
        else:
            amp = oracle_lib.rotate(amp, n, rec["flip"], rec["phase"],
                                    0.5 * delta * rec["cf"])
            amp = oracle_lib.rotate(amp, n, rec["flip"][::-1],
                                    rec["phase"][::-1],
                                    0.5 * delta * rec["cf"][::-1])
        want.append(oracle_lib.coeff_inner(n, cm, amp))
    want = np.array(want)
    assert np.all(np.abs(z - want) <= 1e-12 * np.maximum(1.0, np.abs(want)))


def test_coeff_matrix_rejects_small_register():
    """An expansion needing more qubits than the register is refused."""
    cm = p2.CoeffMatrix(5, 2, 2, [np.eye(5, 2)], None, None)
    with Register(8, p2.PREC_FP64) as r:
        with pytest.raises(RuntimeError):
            r.coeff_expand(cm)


def test_sharded_qdrift_equals_single_run():
    """Replica sharding (phase2_b200.replicas): the blocks of 3 ranks,
    each with its generator advanced to its first sample, concatenate to
    the single-process run bit for bit."""
    from phase2_b200 import replicas
    t = workloads.jw_terms(12, 150, seed=61)
    d = workloads.hamming_dets(12, 2, 6, seed=62)
    full = p2.qdrift(12, t, d, 8, 40, 0.03, 0x600D)
    parts = []
    for rank in range(3):
        start, z = replicas.qdrift_local(12, t, d, 8, 40, 0.03, 0x600D,
                                         rank, 3)
        parts.append((start, z))
    got = np.concatenate([z for _, z in sorted(parts, key=lambda b: b[0])])
    assert np.array_equal(got, full)


def test_empty_hamiltonian_and_edges():
    t = Terms(np.zeros(0, np.uint64), np.zeros(0, np.uint64), np.zeros(0))
    d = Dets(np.array([3], np.uint64), np.array([1.0 + 0j]))
    z = p2.trott(4, t, d, 3, 0.1)
    assert np.array_equal(z, np.ones(3, dtype=complex))
    with pytest.raises(RuntimeError):  # qdrift needs a non-empty CDF
        p2.qdrift(4, t, d, 1, 4, 0.1, 1)


# ---- one-shot entry (python/tests/test_phase2.py of the reference) -----


def test_phase2_run_golden(golden):
    for c in golden["phase2_run"]:
        if c["rc"] != 0:
            with pytest.raises(ValueError):
                p2.run(c["paulis"], c["coeffs"], c["delta"], c["psi"])
            continue
        z = p2.run(c["paulis"], c["coeffs"], c["delta"], c["psi"])
        assert z == _cz(c["z"]), c


def test_phase2_run_analytic():
    TOL = 1e-12
    assert isinstance(p2.run(["Z0"], [1.0], 0.1, "0"), complex)
    a = 0.3
    z = p2.run(["Z0"], [1.0], a, "0")
    assert abs(z - complex(math.cos(a), math.sin(a))) < TOL
    z = p2.run(["Z0"], [1.0], 0.7, "1")
    assert abs(z - complex(math.cos(0.7), -math.sin(0.7))) < TOL
    z = p2.run(["X0", "X0"], [1.0, 1.0], 0.4, "0")
    assert abs(z.real - math.cos(0.8)) < TOL
    h = [0.1 * (k + 1) for k in range(10)]
    z = p2.run([f"X{k}" for k in range(10)], h, 0.05, "0" * 10)
    assert abs(z.real - math.prod(math.cos(0.05 * x) for x in h)) < TOL
    assert abs(p2.run([], [], 1.0, "00") - 1.0) < TOL
    assert abs(p2.run(["Z0"], [1.0], math.pi / 2, "0") - 1j) < TOL
    for bad in ((["Z0"], [1.0, 2.0], 0.1, "0"), (["W0"], [1.0], 0.1, "0"),
                (["X5"], [1.0], 0.1, "0"), (["Z0"], [1.0], 0.1, "2")):
        with pytest.raises(ValueError):
            p2.run(*bad)
    args = (["X0", "Z1"], [0.3, -0.7], 0.25, "01")
    assert p2.run(*args) == p2.run(*args)


# ---- wide registers: exact sparse checks, size-independent properties --


@pytest.mark.parametrize("n,prec", [(26, 0), (30, 0), (30, 1), (32, 1),
                                    (33, 0)])
def test_wide_register_sparse_exact(n, prec):
    t = workloads.jw_terms(n, 400, seed=20 + n)
    rng = np.random.Generator(np.random.PCG64(n))
    pick = rng.choice(len(t), 10, replace=False)
    flip, phase = t.flip[pick], t.phase[pick]
    flip[3] = 1 << (n - 1) | 1   # top and bottom qubit
    phase[3] = 1 << (n - 2)
    flip[6] = 0                  # one diagonal term
    phi = rng.uniform(-1, 1, 10)
    start = {int(1 << (n - 1)) | 5: 0.6 + 0.0j, 3: 0.0 + 0.8j}
    want = dict(start)
    for k in range(10):
        want = sparse_rotate(want, int(flip[k]), int(phase[k]), float(phi[k]))
    idx = np.array(sorted(want), dtype=np.uint64)
    with Register(n, prec) as r:
        r.zero()
        r.setamps(list(start), list(start.values()))
        r.paulirot(flip, phase, phi)
        got = r.getamps(idx)
        nrm = r.norm2()
    exp = np.array([want[int(i)] for i in idx])
    if prec == 0:
        assert np.array_equal(got, exp)
        assert abs(nrm - 1.0) < 1e-12
    else:
        assert np.max(np.abs(got - exp)) < FP32_TOL


def test_fused_equals_plain_and_inverse_at_scale():
    """24 qubits, dense state: fused FP64 == one-rotation-per-pass FP64 bit
    for bit; applying the reversed sequence at -phi restores the state."""
    n = 24
    rng = np.random.Generator(np.random.PCG64(24))
    amp = _rand_state(rng, n)
    t = workloads.jw_terms(n, 600, seed=24)
    phi = rng.uniform(-0.5, 0.5, len(t))
    outs = []
    for fusion in ((5, 0), (1, 1)):
        with Register(n) as r:
            r.set_fusion(*fusion)
            r.set_state(amp)
            r.paulirot(t.flip, t.phase, phi)
            outs.append(r.get_state())
            if fusion == (5, 0):
                r.paulirot(t.flip[::-1], t.phase[::-1], -phi[::-1])
                back = r.get_state()
                nrm = r.norm2()
    assert np.array_equal(outs[0], outs[1])
    assert np.max(np.abs(back - amp)) < 1e-12
    assert abs(nrm - 1.0) < 1e-12


def test_inner_dense_matches_numpy():
    rng = np.random.Generator(np.random.PCG64(31))
    n = 16
    a, b = _rand_state(rng, n), _rand_state(rng, n)
    with Register(n) as r:
        r.set_state(a)
        z = r.inner_dense(b)
    assert abs(z - np.vdot(b, a)) < 1e-13
