"""Pin the CPU restatement (oracle/oracle.c) against the reference.

Every golden vector in tests/golden/ was produced by the reference's own
CPU path (tests/golden/make_golden.py).  The restatement must reproduce
each of them exactly: integers and indices equal, doubles bit-identical.
Where oracle/_ref is built (reference sources available) the same checks
also run live on fresh random inputs.
"""

import numpy as np
import pytest

from oracle import REF_SO, Oracle, Reference
from phase2_b200 import workloads

from conftest import GOLDEN


def _cz(pair):
    return complex(pair[0], pair[1])


def test_xoshiro_sequences(golden, oracle_lib):
    for case in golden["xoshiro"]:
        assert oracle_lib.rng_sequence(case["seed"], 32) == case["next"]


def test_paulis_effect_table(golden, oracle_lib):
    for e in golden["paulis_effect"]:
        j, r = oracle_lib.effect(e["flip"], e["phase"], e["i"])
        assert j == e["j"]
        z = [(1, 0), (0, 1), (-1, 0), (0, -1)][r]
        assert (float(z[0]), float(z[1])) == (e["z"][0] + 0.0,
                                              e["z"][1] + 0.0)


def test_paulis_cmp_table(golden, oracle_lib):
    for c in golden["paulis_cmp"]:
        a, b = c["a"], c["b"]
        assert oracle_lib.L.orc_pauli_cmp(a[0], a[1], b[0], b[1]) == c["cmp"]


def test_prob_cdf(golden, oracle_lib):
    for c in golden["prob"]:
        rc, y, lam = oracle_lib.cdf(c["w"])
        assert rc == c["rc"]
        if rc:
            continue
        assert lam == c["lambda"]
        assert y.tolist() == c["y"]
        for q, want in zip(c["q"], c["inv"]):
            assert oracle_lib.cdf_inverse(y, q) == want


def test_phase2_run_cases(golden, oracle_lib):
    for c in golden["phase2_run"]:
        rc, z = oracle_lib.phase2_run(c["paulis"], c["coeffs"], c["delta"],
                                      c["psi"])
        assert rc == c["rc"], c
        if rc == 0:
            assert z == _cz(c["z"]), c


def test_paulirot_fixture(oracle_lib):
    f = np.load(GOLDEN / "paulirot.npz")
    out = oracle_lib.rotate(f["amp0"], 9, f["flip"], f["phase"], f["phi"])
    assert np.array_equal(out, f["amp1"])


def test_drivers(golden, oracle_lib):
    for c in golden["drivers"]:
        di = np.array(c["det_idx"], dtype=np.uint64)
        dc = np.array([_cz(v) for v in c["det_cf"]])
        fl = np.array(c["flip"], dtype=np.uint64)
        ph = np.array(c["phase"], dtype=np.uint64)
        cf = np.array(c["cf"])
        if c["kind"] in ("trott", "trott2"):
            z = oracle_lib.trott(c["nqb"], fl, ph, cf, di, dc, c["steps"],
                                 c["delta"], order2=c["kind"] == "trott2",
                                 sort_lex=c["lex"])
        elif c["kind"] == "qdrift":
            z = oracle_lib.qdrift(c["nqb"], fl, ph, cf, di, dc, c["samples"],
                                  c["depth"], c["step_size"], c["seed"])
        else:
            z = oracle_lib.cmpsit(c["nqb"], fl, ph, cf, di, dc, c["samples"],
                                  c["steps"], c["length"], c["depth"],
                                  c["angle_det"], c["angle_rand"], c["seed"])
        want = np.array([_cz(v) for v in c["z"]])
        assert np.array_equal(z, want), c["kind"]


def test_trotter12(golden, oracle_lib):
    cfg = workloads.trotter12()
    t, d = cfg["terms"], cfg["dets"]
    z = oracle_lib.trott(12, t.flip, t.phase, t.cf, d.idx, d.cf,
                         cfg["steps"], cfg["delta"])
    want = np.array([_cz(v) for v in golden["trotter12"]["z"]])
    assert np.array_equal(z, want)


def h2o_case(golden):
    """The reference's water CAS(5,6) fixture as numpy arrays."""
    h = golden["h2o"]
    return (h["nqb"], np.array(h["flip"], dtype=np.uint64),
            np.array(h["phase"], dtype=np.uint64), np.array(h["cf"]),
            np.array(h["det_idx"], dtype=np.uint64),
            np.array([_cz(v) for v in h["det_cf"]]))


def test_h2o_fixture(golden, oracle_lib):
    h = golden["h2o"]
    n, fl, ph, cf, di, dc = h2o_case(golden)
    assert n == 10 and len(cf) == 251 and int(di[0]) == 0b0011100111
    # Pauli strings are distinct; the identity is not among them (its
    # coefficient is the file's separate `offset` attribute).
    assert len(set(zip(fl.tolist(), ph.tolist()))) == 251
    assert not np.any((fl == 0) & (ph == 0))
    runs = {
        "trott": oracle_lib.trott(n, fl, ph, cf, di, dc, 12, 0.5),
        "trott2": oracle_lib.trott(n, fl, ph, cf, di, dc, 12, 0.5,
                                   order2=True),
        "qdrift": oracle_lib.qdrift(n, fl, ph, cf, di, dc, 6, 300, 0.01,
                                    0xC0FFEE),
        "cmpsit": oracle_lib.cmpsit(n, fl, ph, cf, di, dc, 3, 4, 60, 50, 0.1,
                                    0.02, 0xBEEF),
    }
    for kind, z in runs.items():
        want = np.array([_cz(v) for v in h[kind]])
        assert np.array_equal(z, want), kind
        assert np.all(np.abs(z) <= 1 + 1e-12), kind


def coeff_case(c):
    """A golden coefficient-matrix case as (nqb, state object, psi)."""
    from types import SimpleNamespace
    cm = SimpleNamespace(
        n_sites=c["n_sites"], n_alpha=c["n_alpha"], n_beta=c["n_beta"],
        C_alpha=[np.array(a) for a in c["C_alpha"]],
        C_beta=(None if c["C_beta"] is None
                else [np.array(b) for b in c["C_beta"]]),
        weights=c["weights"], tapered=c["tapered"])
    g = np.random.Generator(np.random.PCG64(c["psi_seed"]))
    n = c["nqb"]
    psi = g.standard_normal(1 << n) + 1j * g.standard_normal(1 << n)
    return n, cm, psi


def test_coeff_matrix_fixtures(golden, oracle_lib):
    """The restated Slater-Condon expansion and overlap reproduce the
    reference's (state_prep_coeff.c) bit for bit."""
    for c in golden["coeff_matrix"]:
        n, cm, psi = coeff_case(c)
        amp = oracle_lib.coeff_expand(n, cm)
        nz = np.nonzero(amp)[0]
        assert nz.tolist() == c["expand_idx"]
        assert np.array_equal(amp[nz].real, np.array(c["expand_val"]))
        assert not np.any(amp.imag)
        assert oracle_lib.coeff_inner(n, cm, psi) == _cz(c["inner"])


needs_ref = pytest.mark.skipif(not REF_SO.is_file(),
                               reason="oracle/_ref not built here")


@needs_ref
@pytest.mark.parametrize("seed", range(4))
def test_live_paulirot_vs_reference(seed, oracle_lib):
    ref = Reference()
    rng = np.random.Generator(np.random.PCG64(seed))
    n = int(rng.integers(1, 11))
    amp = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    t = workloads.random_terms(n, 150, seed=100 + seed)
    phi = rng.uniform(-2, 2, len(t))
    assert np.array_equal(oracle_lib.rotate(amp, n, t.flip, t.phase, phi),
                          ref.paulirot(amp, n, t.flip, t.phase, phi))


@needs_ref
def test_live_drivers_vs_reference(oracle_lib):
    ref = Reference()
    t = workloads.jw_terms(9, 80, seed=77)
    d = workloads.hamming_dets(9, 4, 4, seed=78)
    for order2 in (False, True):
        a = oracle_lib.trott(9, t.flip, t.phase, t.cf, d.idx, d.cf, 3, 0.3,
                             order2=order2)
        b = ref.trott(9, t.flip, t.phase, t.cf, d.idx, d.cf, 3, 0.3,
                      order2=order2)
        assert np.array_equal(a, b)
    a = oracle_lib.qdrift(9, t.flip, t.phase, t.cf, d.idx, d.cf, 3, 40, 0.1,
                          99)
    b = ref.qdrift(9, t.flip, t.phase, t.cf, d.idx, d.cf, 3, 40, 0.1, 99)
    assert np.array_equal(a, b)
    a = oracle_lib.cmpsit(9, t.flip, t.phase, t.cf, d.idx, d.cf, 2, 2, 8, 12,
                          0.1, 0.01, 5)
    b = ref.cmpsit(9, t.flip, t.phase, t.cf, d.idx, d.cf, 2, 2, 8, 12, 0.1,
                   0.01, 5)
    assert np.array_equal(a, b)


def test_oracle_is_not_the_product():
    """The product library must not link the oracle."""
    from phase2_b200._ffi import LIB_PATH
    data = LIB_PATH.read_bytes()
    assert b"orc_rotate" not in data and b"refh_" not in data
