"""Host-side checks of libphase2.so that need no GPU.

* the library loads and exports every function declared in include/;
* ctypes struct layouts equal the C ones;
* Pauli algebra, xoshiro256**, CDF sampling and the batch cache reproduce
  the reference's golden vectors exactly;
* the pass planner: its descriptors, executed by a numpy emulation of the
  device kernel (tests/emulate.py), reproduce the oracle bit for bit.
"""

import ctypes as C
import re
import subprocess

import numpy as np
import pytest

import phase2_b200 as p2
from phase2_b200 import _ffi, plan, workloads
from phase2_b200._ffi import lib

from conftest import ROOT
from emulate import emulate


def _declared_functions() -> set[str]:
    names = set()
    for h in sorted((ROOT / "include").rglob("*.h")):
        src = h.read_text()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"^\s*#.*?(?<!\\)$", "", src, flags=re.M)
        # drop static inline definitions (header-only helpers)
        src = re.sub(r"static\s+inline[^{;]*\{.*?\n\}", "", src, flags=re.S)
        for m in re.finditer(
                r"([A-Za-z_][A-Za-z0-9_]*)\s*\(([^;{}()]|\([^;{}()]*\))*\)"
                r"\s*(__attribute__\s*\(\(.*?\)\))?\s*;", src, flags=re.S):
            name = m.group(1)
            if name not in ("__attribute__", "format", "sizeof"):
                names.add(name)
    return names


def test_library_loads():
    L = lib()
    assert b"sm_100a" in L.phase2_version()


def test_exports_every_declared_function():
    declared = _declared_functions()
    assert "qreg_paulirot" in declared and "phase2_run" in declared
    assert len(declared) > 80
    out = subprocess.run(["nm", "-D", "--defined-only", str(_ffi.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = sorted(declared - exported)
    assert not missing, missing
    # internals stay hidden
    assert not any(s.startswith(("p2d_", "p2_")) for s in exported)


def test_struct_layouts():
    for k, (py, c) in _ffi.check_layout().items():
        assert py == c, (k, py, c)


def _paulis(f, p):
    return _ffi.Paulis((C.c_uint64 * 2)(f, p))


def test_paulis_effect_and_cmp(golden):
    L = lib()
    for e in golden["paulis_effect"]:
        z = (C.c_double * 2)(1.0, 0.0)
        j = L.paulis_effect(_paulis(e["flip"], e["phase"]), e["i"], z)
        assert j == e["j"]
        assert (z[0] + 0.0, z[1] + 0.0) == (e["z"][0] + 0.0,
                                            e["z"][1] + 0.0)
    for c in golden["paulis_cmp"]:
        a, b = c["a"], c["b"]
        assert L.paulis_cmp(_paulis(*a), _paulis(*b)) == c["cmp"]


def test_paulis_get_set_split():
    L = lib()
    p = L.paulis_new()
    for q, op in ((0, 1), (1, 2), (2, 3), (63, 2), (40, 1)):
        L.paulis_set(C.byref(p), op, q)
        assert L.paulis_get(p, q) == op
    L.paulis_set(C.byref(p), 0, 1)
    assert L.paulis_get(p, 1) == 0
    L.paulis_set(C.byref(p), 7, 2)  # unknown op: unchanged
    assert L.paulis_get(p, 2) == 3
    lo, hi = _ffi.Paulis(), _ffi.Paulis()
    L.paulis_split(p, 3, 38, C.byref(lo), C.byref(hi))
    assert lo.pak[0] == p.pak[0] & 7 and lo.pak[1] == p.pak[1] & 7
    assert hi.pak[0] == p.pak[0] & ((1 << 41) - 8)
    q = _ffi.Paulis((C.c_uint64 * 2)(p.pak[0], p.pak[1]))
    L.paulis_shr(C.byref(q), 5)
    L.paulis_shl(C.byref(q), 5)
    assert q.pak[0] == p.pak[0] & ~31 & (2**64 - 1)


def test_xoshiro(golden):
    L = lib()
    for case in golden["xoshiro"]:
        st = _ffi.Xoshiro()
        L.xoshiro256ss_init(C.byref(st), case["seed"])
        got = [L.xoshiro256ss_next(C.byref(st)) for _ in range(32)]
        assert got == case["next"]


def test_prob(golden):
    L = lib()
    assert L.prob_cdf_init(C.byref(_ffi.ProbCdf()), 0) == -1
    for c in golden["prob"]:
        w = (C.c_double * len(c["w"]))(*c["w"])
        cdf = _ffi.ProbCdf()
        assert L.prob_cdf_init(C.byref(cdf), len(c["w"])) == 0
        lam = C.c_double(-1)
        rc = L.prob_cdf_from_array_strided(C.byref(cdf), w, 8, C.byref(lam))
        assert rc == c["rc"]
        if rc == 0:
            assert lam.value == c["lambda"]
            assert [cdf.y[k] for k in range(cdf.len)] == c["y"]
            for q, want in zip(c["q"], c["inv"]):
                assert L.prob_cdf_inverse(C.byref(cdf), q) == want
        L.prob_cdf_free(C.byref(cdf))
        assert cdf.len == 0 and not cdf.y
        L.prob_cdf_free(C.byref(cdf))  # idempotent


def test_cache_capacity_and_flush():
    """Batch semantics of test/t-circ_cache.c: 1024 terms, hi-code split."""
    L = lib()
    c = L.circ_cache_init(0, 20)
    for k in range(1024):
        assert L.circ_cache_insert(c, _paulis(k & 0xFFFFF, 0), 0.1) == 0
    assert L.circ_cache_len(c) == 1024
    assert L.circ_cache_insert(c, _paulis(1, 0), 0.1) == -1
    L.circ_cache_free(c)
    c = L.circ_cache_init(2, 4)
    assert L.circ_cache_insert(c, _paulis(0b010000, 0), 0.1) == 0
    assert L.circ_cache_insert(c, _paulis(0b010001, 0), 0.1) == 0
    assert L.circ_cache_insert(c, _paulis(0b100001, 0), 0.1) == -1
    L.circ_cache_free(c)


def _hamil(nqb, t):
    L = lib()
    hm = _ffi.CircHamil()
    assert L.circ_hamil_init(C.byref(hm), nqb, len(t)) == 0
    rec = t.records()
    C.memmove(hm.terms, rec.ctypes.data, rec.nbytes)
    return hm


def _terms_of(hm):
    n = hm.len
    buf = np.ctypeslib.as_array(C.cast(hm.terms, C.POINTER(C.c_uint8)),
                                shape=(24 * n,))
    return np.frombuffer(buf.tobytes(), dtype=[("cf", "<f8"),
                                               ("flip", "<u8"),
                                               ("phase", "<u8")])


def test_sort_lex_matches_oracle(oracle_lib):
    L = lib()
    t = workloads.random_terms(20, 500, seed=3)
    # duplicate operators with different coefficients exercise ties
    t.flip[::7], t.phase[::7] = t.flip[0], t.phase[0]
    hm = _hamil(20, t)
    L.circ_hamil_sort_lex(C.byref(hm))
    got = _terms_of(hm)
    want = oracle_lib.sort_lex(t.flip, t.phase, t.cf)
    assert got.tobytes() == want.tobytes()
    L.circ_hamil_free(C.byref(hm))


def test_sort_flip_is_stable():
    L = lib()
    t = workloads.jw_terms(12, 400, seed=9)
    hm = _hamil(12, t)
    L.circ_hamil_sort_flip(C.byref(hm))
    got = _terms_of(hm)
    want = workloads.sort_by_flip(t)
    assert np.array_equal(got["flip"], want.flip)
    assert np.array_equal(got["phase"], want.phase)
    assert np.array_equal(got["cf"], want.cf)
    L.circ_hamil_free(C.byref(hm))


def test_cmpsit_split_matches_oracle(oracle_lib):
    """cmpsit_ranct_init: the `length` largest |c| lexicographically
    sorted, the rest in |c|-descending order with their CDF and lambda
    (circ/cmpsit.c:65-111), the split cmpsit_init makes."""
    L = lib()
    t = workloads.jw_terms(12, 300, seed=17)
    order0 = L.phase2_get_term_order()
    L.phase2_set_term_order(0)
    hm = _hamil(12, t)
    rc = _ffi.CmpsitRanct()
    dt = _ffi.CmpsitData(1, 1, 40, 8, 0.05, 0.01, 5)
    try:
        assert L.cmpsit_ranct_init(C.byref(rc), C.byref(hm),
                                   C.byref(dt)) == 0
        idx = np.argsort(-np.abs(t.cf), kind="stable")
        assert len(np.unique(np.abs(t.cf))) == len(t)  # no ties here
        head = oracle_lib.sort_lex(t.flip[idx[:40]], t.phase[idx[:40]],
                                   t.cf[idx[:40]])
        assert _terms_of(rc.hm_det).tobytes() == head.tobytes()
        tail = _terms_of(rc.hm_ran)
        assert np.array_equal(tail["cf"], t.cf[idx[40:]])
        assert np.array_equal(tail["flip"], t.flip[idx[40:]])
        _, y, lam = oracle_lib.cdf(t.cf[idx[40:]])
        got = np.ctypeslib.as_array(rc.cdf.y, shape=(int(rc.cdf.len),))
        assert np.array_equal(got, y) and rc.lambda_r == lam
    finally:
        L.cmpsit_ranct_free(C.byref(rc))
        L.cmpsit_ranct_free(C.byref(rc))  # idempotent
        L.phase2_set_term_order(order0)
    bad = _ffi.CmpsitData(1, 1, 300, 8, 0.05, 0.01, 5)
    assert L.cmpsit_ranct_init(C.byref(rc), C.byref(hm), C.byref(bad)) == -1
    L.cmpsit_ranct_free(C.byref(rc))
    L.circ_hamil_free(C.byref(hm))


def _rand_rotations(rng, n, k, diag_frac=0.2):
    t = workloads.random_terms(n, k, seed=int(rng.integers(1 << 30)))
    mask = rng.random(k) < diag_frac
    t.flip[mask] = 0
    phi = rng.uniform(-np.pi, np.pi, k)
    return t.flip, t.phase, phi


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 11])
@pytest.mark.parametrize("span,max_rots", [(1, 1), (2, 0), (3, 0), (5, 0),
                                           (5, 1), (4, 3)])
def test_planner_emulation_bit_exact(n, span, max_rots, oracle_lib):
    rng = np.random.Generator(np.random.PCG64(n * 100 + span * 10 + max_rots))
    flip, phase, phi = _rand_rotations(rng, n, 60)
    amp = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    passes, recs = plan(n, flip, phase, phi, span, max_rots)
    assert sum(p["nrot"] for p in passes) == 60
    for p in passes:
        assert p["span"] <= max(span, min(3, n))
        if max_rots:
            assert p["nrot"] <= max_rots
    got = emulate(amp, n, passes, recs)
    want = oracle_lib.rotate(amp, n, flip, phase, phi)
    assert np.array_equal(got, want)


def test_fp32_form_setting():
    """The three FP32 forms are accepted, anything else refused."""
    old = p2.get_fp32_form()
    try:
        for form in (p2.FORM_LIFTED, p2.FORM_LIFTED_F32,
                     p2.FORM_LIFTED_MIXED):
            p2.set_fp32_form(form)
            assert p2.get_fp32_form() == form
        for bad in (p2.FORM_EXACT, 4, -1):
            with pytest.raises(ValueError):
                p2.set_fp32_form(bad)
        assert p2.get_fp32_form() == p2.FORM_LIFTED_MIXED
    finally:
        p2.set_fp32_form(old)


@pytest.mark.parametrize("n", [2, 6, 11])
@pytest.mark.parametrize("form", [p2.FORM_LIFTED, p2.FORM_LIFTED_F32,
                                  p2.FORM_LIFTED_MIXED])
def test_planner_fp32_forms(n, form, oracle_lib):
    """FP32 plans (lifted shears with a pass-wide sign) reproduce the
    oracle when executed in FP64: to FP64 rounding with FP64 coefficients,
    and to the rounding of s to FP32 (relative angle error <= 2^-24 per
    rotation) with the FP32-arithmetic coefficients; angles in [-pi, pi]
    cover both signs of cos."""
    rng = np.random.Generator(np.random.PCG64(500 + n))
    flip, phase, phi = _rand_rotations(rng, n, 80)
    amp = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    old = p2.get_fp32_form()
    p2.set_fp32_form(form)
    try:
        passes, recs = plan(n, flip, phase, phi, 5, 0, prec=1)
    finally:
        p2.set_fp32_form(old)
    assert {r["form"] for r in recs} == {1}
    assert {p["form"] for p in passes} == {form}
    assert {p["scale"] for p in passes} <= {1.0, -1.0}
    assert all(abs(r["c"]) <= 1.0 + 1e-7 for r in recs)
    got = emulate(amp, n, passes, recs)
    want = oracle_lib.rotate(amp, n, flip, phase, phi)
    if form == p2.FORM_LIFTED:
        tol = 1e-12
    else:
        assert all(np.float32(r["s"]) == r["s"] for r in recs)
        # t * s = 1 - cos(phi) exactly: s rounding only tilts the shears
        tol = 80 * 2.0 ** -24
    assert np.max(np.abs(got - want)) < tol * np.max(np.abs(want))


@pytest.mark.parametrize("n", [6, 24])
def test_mixed_plan_is_the_f32_plan(n):
    """The mixed form's kernel rotates light cosets from the FP32 form's
    records and heavy ones from the same records in FP64: its plan must be
    the FP32-arithmetic form's, record for record, with only each pass's
    form changed."""
    rng = np.random.Generator(np.random.PCG64(700 + n))
    flip, phase, phi = _rand_rotations(rng, n, 120)
    old = p2.get_fp32_form()
    try:
        p2.set_fp32_form(p2.FORM_LIFTED_F32)
        pf, rf = plan(n, flip, phase, phi, 5, 0, prec=1)
        p2.set_fp32_form(p2.FORM_LIFTED_MIXED)
        pm, rm = plan(n, flip, phase, phi, 5, 0, prec=1)
    finally:
        p2.set_fp32_form(old)
    assert rm == rf
    assert {p["form"] for p in pm} == {p2.FORM_LIFTED_MIXED}
    for a, b in zip(pm, pf):
        assert dict(a, form=0) == dict(b, form=0)
    assert len(pm) == len(pf)


def test_planner_fuses_jw_runs():
    t = workloads.jw_terms(20, 2000, seed=4)
    phi = np.full(len(t), 0.01)
    passes, _ = plan(20, t.flip, t.phase, phi, 5, 0)
    # 8 strings share each excitation's flip mask: runs fuse
    assert len(passes) < len(t) / 8
    one, _ = plan(20, t.flip, t.phase, phi, 5, 1)
    assert len(one) == len(t)


def _rank(vectors):
    rows = []
    for v in vectors:
        v = int(v)
        for r in rows:
            v = min(v, v ^ r)
        if v:
            rows.append(v)
    return len(rows)


@pytest.mark.parametrize("tile,low", [(13, 5), (12, 4), (11, 3)])
def test_planner_sweep_grouping(tile, low, oracle_lib):
    """FP32 plans (FP32-arithmetic form, the one sweeps run in) of
    registers of tile + 3 qubits or more group passes into sweeps: every
    sweep's bases, modulo the low qubits, span at most tile - low
    dimensions; the plan still applies every rotation in order (emulated
    execution matches the oracle)."""
    n = 17
    rng = np.random.Generator(np.random.PCG64(tile * 7 + low))
    jw = workloads.jw_terms(n, 3000, seed=tile)
    pick = rng.integers(0, len(jw), 400)  # qDRIFT-like random draws
    flip, phase = jw.flip[pick], jw.phase[pick]
    phi = rng.uniform(-np.pi, np.pi, len(pick))
    old = p2.get_sweep()
    form = p2.get_fp32_form()
    p2.set_fp32_form(p2.FORM_LIFTED_F32)
    p2.set_sweep(tile, low)
    try:
        passes, recs = plan(n, flip, phase, phi, 5, 0, prec=1)
        p2.set_sweep(0, 5)
        plain, _ = plan(n, flip, phase, phi, 5, 0, prec=1)
    finally:
        p2.set_sweep(*old)
        p2.set_fp32_form(form)
    assert passes[0]["sweep"] == 1
    assert sum(p["sweep"] for p in plain) == 1
    heads = [i for i, p in enumerate(passes) if p["sweep"]] + [len(passes)]
    assert len(heads) - 1 < len(plain)  # fewer round trips than passes
    lowm = (1 << low) - 1
    for a, b in zip(heads[:-1], heads[1:]):
        vecs = [int(v) & ~lowm for p in passes[a:b]
                for v in p["basis"][:p["span"]]]
        assert _rank(vecs) <= tile - low
    assert sum(p["nrot"] for p in passes) == len(pick)
    amp = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    got = emulate(amp, n, passes, recs)
    want = oracle_lib.rotate(amp, n, flip, phase, phi)
    assert np.max(np.abs(got - want)) < 100 * 2.0 ** -24 * np.max(np.abs(want))


def test_sweep_setting_validates():
    old = p2.get_sweep()
    for bad in ((15, 5), (13, 3), (10, 2), (7, 3)):
        with pytest.raises(ValueError):
            p2.set_sweep(*bad)
    p2.set_sweep(13, 5)
    assert p2.get_sweep() == (13, 5)
    p2.set_sweep(0, 5)
    assert p2.get_sweep()[0] == 0
    p2.set_sweep(*old)
    assert p2.get_sweep() == old


def test_planner_rejects_bad_width():
    L = lib()
    rin = (_ffi.RotIn * 1)()
    assert L.phase2_plan(0, rin, 1, 5, 0, 0, (_ffi.Pass * 1)(),
                         (_ffi.RotRec * 1)()) == -1


def test_settings_validate():
    L = lib()
    assert L.phase2_set_precision(7) == -1
    assert L.phase2_set_fusion(0, 0) == -1
    assert L.phase2_set_fusion(6, 0) == -1
    assert L.phase2_set_term_order(9) == -1
    assert L.phase2_set_term_order(2) == 0
    assert L.phase2_get_term_order() == 2
    assert L.phase2_set_term_order(0) == 0
    assert L.phase2_set_device_sampling(3) == -1
    for mode in (0, 1, 2):
        assert L.phase2_set_device_sampling(mode) == 0


def test_phase2_run_rejects_without_touching_device():
    """Inputs rejected before the world starts (psi NULL or bad length)."""
    L = lib()
    re_, im_ = C.c_double(), C.c_double()
    arr = (C.c_char_p * 1)(b"Z0")
    cf = (C.c_double * 1)(1.0)
    assert L.phase2_run(arr, cf, 1, 0.1, None, C.byref(re_),
                        C.byref(im_)) == -1
    assert L.phase2_run(arr, cf, 1, 0.1, b"", C.byref(re_),
                        C.byref(im_)) == -1
    assert L.phase2_run(arr, cf, 1, 0.1, b"0" * 31, C.byref(re_),
                        C.byref(im_)) == -1


def test_slab_calls_reject_uninitialised_registers():
    """qreg_slab_get/put/swap on a register that was never initialised
    return -1 before touching any device (no GPU needed)."""
    L = lib()
    a, b = _ffi.Qreg(), _ffi.Qreg()
    buf = C.c_void_p(0)
    assert L.qreg_slab_get(C.byref(a), 0, 0, 0, 1, buf) == -1
    assert L.qreg_slab_put(C.byref(a), 0, 0, 0, 1, buf) == -1
    assert L.qreg_slab_swap(C.byref(a), C.byref(b), 0, 0, 1) == -1
    rc = _ffi.CmpsitRanct()
    empty = _ffi.CircHamil()
    dt = _ffi.CmpsitData(1, 1, 0, 4, 0.05, 0.01, 5)
    assert L.cmpsit_ranct_init(C.byref(rc), C.byref(empty), C.byref(dt)) == -1
    L.cmpsit_ranct_free(C.byref(rc))
