"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference's own CPU path (oracle/_ref/libphase2_ref.so, built from
the reference sources by ``make -C oracle ref``) on small seeded inputs and
records inputs and outputs:

  golden.json     phase2_run cases (the reference Python test suite's
                  analytic cases plus random multi-qubit ones), paulis_effect
                  and paulis_cmp tables, xoshiro256** sequences, CDF builds
                  and inverse queries, driver overlaps (trott in lex and
                  given order, trott2, qdrift, cmpsit) and the full 12-qubit
                  200-term Trotter case.
  paulirot.npz    a 9-qubit random state before and after 300 random
                  rotations through qreg_paulirot.

Usage:  python tests/golden/make_golden.py   (needs oracle/_ref built)
"""

from __future__ import annotations

import ctypes as C
import json
import math
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import Reference  # noqa: E402
from phase2_b200 import workloads  # noqa: E402

OUT = Path(__file__).resolve().parent


class RPaulis(C.Structure):
    _fields_ = [("pak", C.c_uint64 * 2)]


class RXo(C.Structure):
    _fields_ = [("s", C.c_uint64 * 4)]


class RCdf(C.Structure):
    _fields_ = [("y", C.POINTER(C.c_double)), ("len", C.c_size_t)]


def cplx(z) -> list:
    return [float(np.real(z)), float(np.imag(z))]


def _reference_tree() -> Path:
    """$PHASE2_REF, else the oracle recipes' default (oracle/Makefile REF)."""
    env = os.environ.get("PHASE2_REF")
    if env:
        return Path(env)
    root = Path(__file__).resolve().parents[2]
    return Path(subprocess.run(["make", "-s", "-C", "oracle", "print-ref"],
                               cwd=root, check=True, capture_output=True,
                               text=True).stdout.strip())


H2O_DUMP = _reference_tree() / "test" / "data" / "H2O_CAS56.h5dump"


def _dataset_values(text: str, name: str) -> list[float]:
    """Numbers of DATASET `name` in an h5dump text (index prefixes
    like "(12):" or "(3,0):" removed)."""
    import re
    start = text.index(f'DATASET "{name}"')
    body = text[text.index("DATA {", start) + 6:]
    body = body[:body.index("}")]
    body = re.sub(r"\(\s*\d+(\s*,\s*\d+)*\s*\):", " ", body)
    return [float(v) for v in body.replace(",", " ").split()]


def h2o_fixture() -> dict:
    """The reference's 10-qubit water CAS(5,6) Hamiltonian (251 terms) and
    determinant from test/data/H2O_CAS56.h5dump, loaded as the reference's
    data_hamil_load / data_muldet_load do (ph2run/data.c:515-540, 625-660):
    coefficient times the `normalization` attribute, byte j of a row is the
    operator on qubit j (I=0, X=1, Y=2, Z=3), determinant bit j = byte j."""
    import re
    text = H2O_DUMP.read_text()
    i = text.index('ATTRIBUTE "normalization"')
    norm = float(re.search(r"\(0\):\s*([-0-9.eE+]+)", text[i:]).group(1))
    coeffs = _dataset_values(text, "coeffs")[:251]
    paulis = [int(v) for v in _dataset_values(text, "paulis")]
    sp = text.index('GROUP "state_prep"')
    det_cf = _dataset_values(text[sp:], "coeffs")
    det_bits = [int(v) for v in _dataset_values(text[sp:], "dets")]
    nqb = 10
    flip, phase = [], []
    for t in range(len(coeffs)):
        f = p = 0
        for j in range(nqb):
            b = paulis[t * nqb + j]
            if b in (1, 2):
                f |= 1 << j
            if b in (2, 3):
                p |= 1 << j
        flip.append(f)
        phase.append(p)
    idx = sum(b << j for j, b in enumerate(det_bits))
    return {"nqb": nqb, "flip": flip, "phase": phase,
            "cf": [c * norm for c in coeffs], "det_idx": [idx],
            "det_cf": [[det_cf[0], det_cf[1]]], "normalization": norm}


def _psi_from_seed(nqb: int, seed: int) -> np.ndarray:
    """The complex test state of a coefficient-matrix golden case."""
    g = np.random.Generator(np.random.PCG64(seed))
    return g.standard_normal(1 << nqb) + 1j * g.standard_normal(1 << nqb)


def main() -> None:
    ref = Reference()
    L = ref.L
    L.paulis_effect.argtypes = [RPaulis, C.c_uint64,
                                C.POINTER(C.c_double)]
    L.paulis_effect.restype = C.c_uint64
    L.paulis_cmp.argtypes = [RPaulis, RPaulis]
    L.paulis_cmp.restype = C.c_int
    L.xoshiro256ss_init.argtypes = [C.POINTER(RXo), C.c_uint64]
    L.xoshiro256ss_next.argtypes = [C.POINTER(RXo)]
    L.xoshiro256ss_next.restype = C.c_uint64
    L.prob_cdf_init.argtypes = [C.POINTER(RCdf), C.c_size_t]
    L.prob_cdf_from_array_strided.argtypes = [
        C.POINTER(RCdf), C.POINTER(C.c_double), C.c_size_t,
        C.POINTER(C.c_double)]
    L.prob_cdf_inverse.argtypes = [C.POINTER(RCdf), C.c_double]
    L.prob_cdf_inverse.restype = C.c_size_t

    rng = np.random.Generator(np.random.PCG64(0x601DE))
    gold: dict = {}

    # -- phase2_run: analytic suite of python/tests/test_phase2.py + random
    cases = [
        (["Z0"], [1.0], 0.1, "0"), (["X0", "Z1"], [0.3, -0.7], 0.25, "01"),
        ([], [], 1.0, "00"), ([], [], 1.0, "0"), (["Z0"], [1.0], 0.3, "0"),
        (["Z0"], [1.0], 0.7, "1"), (["X0"], [1.0], 0.5, "0"),
        (["Z0"], [1.0], -0.6, "0"), (["Z0"], [0.5], 2.0, "0"),
        (["X0", "X0"], [1.0, 1.0], 0.4, "0"),
        (["Z0", "Z0"], [1.0, 1.0], 0.35, "0"),
        (["Z0 Z1"], [1.0], 0.8, "00"),
        (["X0 Y1", "Z1 Z2"], [0.3, -0.5], 0.2, "010"),
        ([f"X{k}" for k in range(10)], [0.1 * (k + 1) for k in range(10)],
         0.05, "0" * 10),
        ([f"Z{k}" for k in range(10)], [0.1 * (k + 1) for k in range(10)],
         0.1, "0101010101"),
        (["X0"], [1.0], 0.0, "0"), (["Z0"], [1.0], math.pi, "0"),
        (["Z0"], [1.0], math.pi / 2, "0"),
        (["W0"], [1.0], 0.1, "0"), (["X5"], [1.0], 0.1, "0"),
        (["Z0"], [1.0], 0.1, "2"), (["Z0"], [1.0], 0.1, ""),
        (["X"], [1.0], 0.1, "0"), (["X0x"], [1.0], 0.1, "0"),
        # token edges of the index grammar (strtoul inside a token)
        (["X+1"], [1.0], 0.3, "01"), (["X-0"], [1.0], 0.3, "0"),
        (["X-1"], [1.0], 0.3, "01"), (["X\r1"], [1.0], 0.3, "01"),
        (["X00 Z01"], [1.0], 0.3, "01"), (["X0 I0"], [1.0], 0.3, "0"),
        (["Y1 X1 Z0"], [0.7], 0.3, "01"), (["\tZ0\n Y1 "], [1.0], 0.3, "01"),
        (["X 0"], [1.0], 0.1, "0"), (["x0"], [1.0], 0.1, "0"),
        (["X+"], [1.0], 0.1, "0"), (["X1"], [1.0], 0.1, "0"),
        (["Z0", "W1"], [1.0, 1.0], 0.1, "00"),
        ([" ", ""], [1.0, 2.0], 0.1, "1"),
    ]
    xz = []
    for k in range(10):
        xz += [(f"X{k}", 0.01 * (k + 1)), (f"Z{k}", 0.02 * (k + 1))]
    cases.append(([p for p, _ in xz], [c for _, c in xz], 1.0, "0" * 10))
    ops = "IXYZ"
    for n in (3, 5, 8, 11):
        nt = int(rng.integers(5, 40))
        ps, cs = [], []
        for _ in range(nt):
            toks = [f"{ops[int(rng.integers(4))]}{q}" for q in range(n)]
            ps.append(" ".join(toks))
            cs.append(float(rng.standard_normal()))
        psi = "".join(str(int(b)) for b in rng.integers(0, 2, n))
        cases.append((ps, cs, float(rng.uniform(0.05, 0.5)), psi))
    runs = []
    for ps, cs, d, psi in cases:
        rc, z = ref.phase2_run(ps, cs, d, psi)
        runs.append({"paulis": ps, "coeffs": cs, "delta": d, "psi": psi,
                     "rc": rc, "z": cplx(z)})
    gold["phase2_run"] = runs

    # -- paulis_effect / cmp tables (test/t-paulis.c kinds of cases)
    eff = []
    for _ in range(200):
        f = int(rng.integers(0, 2**63)) | (int(rng.integers(0, 2)) << 63)
        p = int(rng.integers(0, 2**63)) | (int(rng.integers(0, 2)) << 63)
        i = int(rng.integers(0, 2**63)) | (int(rng.integers(0, 2)) << 63)
        code = RPaulis((C.c_uint64 * 2)(f, p))
        z = (C.c_double * 2)(1.0, 0.0)
        j = L.paulis_effect(code, i, z)
        eff.append({"flip": f, "phase": p, "i": i, "j": j,
                    "z": [z[0], z[1]]})
    for f, p in ((1, 1), (3, 3), (0b1011, 0), (0b1011, 0b10), (0b1011, 0b1011)):
        for i in range(4):
            code = RPaulis((C.c_uint64 * 2)(f, p))
            z = (C.c_double * 2)(1.0, 0.0)
            j = L.paulis_effect(code, i, z)
            eff.append({"flip": f, "phase": p, "i": i, "j": j,
                        "z": [z[0], z[1]]})
    gold["paulis_effect"] = eff
    cmps = []
    for _ in range(300):
        a = [int(x) for x in rng.integers(0, 2**16, 2)]
        b = list(a) if rng.random() < 0.1 else \
            [int(x) for x in rng.integers(0, 2**16, 2)]
        hi = int(rng.integers(0, 48))
        a = [v << hi for v in a]
        b = [v << hi for v in b]
        r = L.paulis_cmp(RPaulis((C.c_uint64 * 2)(*a)),
                         RPaulis((C.c_uint64 * 2)(*b)))
        cmps.append({"a": a, "b": b, "cmp": r})
    gold["paulis_cmp"] = cmps

    # -- xoshiro256**
    seqs = []
    for seed in (1, 0x34EAAA33, 0xD3B9268B8737DDC0, 0xFFFFFFFFFFFFFFFF):
        st = RXo()
        L.xoshiro256ss_init(C.byref(st), seed)
        seqs.append({"seed": seed,
                     "next": [L.xoshiro256ss_next(C.byref(st))
                              for _ in range(32)]})
    gold["xoshiro"] = seqs

    # -- prob CDF
    cdfs = []
    for w in ([1.0, 1.0, 1.0, 1.0], [5.0], [1.0, 2.0, 1.0],
              [-1.0, 2.0, -1.0], [0.0, 0.0, 0.0], [1.0, 3.0, 1.0],
              [0.0, 1.0, 0.0, 2.0, 0.0],
              rng.standard_normal(37).tolist()):
        arr = (C.c_double * len(w))(*w)
        cdf = RCdf()
        L.prob_cdf_init(C.byref(cdf), len(w))
        lam = C.c_double(-1.0)
        rc = L.prob_cdf_from_array_strided(C.byref(cdf), arr, 8,
                                           C.byref(lam))
        ys = [cdf.y[k] for k in range(len(w))]
        qs = [0.0, 1.0, 0.25, 0.26, 0.5, 0.51, 0.75, 1e-15, 0.999] + \
            rng.random(20).tolist()
        inv = [int(L.prob_cdf_inverse(C.byref(cdf), q)) for q in qs] \
            if rc == 0 else []
        cdfs.append({"w": list(w), "rc": rc, "lambda": lam.value,
                     "y": ys if rc == 0 else [], "q": qs, "inv": inv})
    gold["prob"] = cdfs

    # -- drivers on small random inputs
    drv = []
    for case in range(6):
        n = 8
        t = workloads.random_terms(n, 12 + case, seed=1000 + case)
        d = workloads.hamming_dets(n, 5, 4, seed=2000 + case)
        steps = 6
        delta = float(0.5 + 0.1 * case)
        for order2 in (False, True):
            for lex in (True, False):
                z = ref.trott(n, t.flip, t.phase, t.cf, d.idx, d.cf, steps,
                              delta, order2=order2, sort_lex=lex)
                drv.append({"kind": "trott2" if order2 else "trott",
                            "lex": lex, "nqb": n,
                            "flip": t.flip.tolist(),
                            "phase": t.phase.tolist(), "cf": t.cf.tolist(),
                            "det_idx": d.idx.tolist(),
                            "det_cf": [cplx(c) for c in d.cf],
                            "steps": steps, "delta": delta,
                            "z": [cplx(v) for v in z]})
    for case in range(3):
        n = 10
        t = workloads.jw_terms(n, 60, seed=3000 + case)
        d = workloads.hamming_dets(n, 3, 5, seed=4000 + case)
        z = ref.qdrift(n, t.flip, t.phase, t.cf, d.idx, d.cf, 4, 64, 0.05,
                       0x1234 + case)
        drv.append({"kind": "qdrift", "nqb": n, "flip": t.flip.tolist(),
                    "phase": t.phase.tolist(), "cf": t.cf.tolist(),
                    "det_idx": d.idx.tolist(),
                    "det_cf": [cplx(c) for c in d.cf], "samples": 4,
                    "depth": 64, "step_size": 0.05, "seed": 0x1234 + case,
                    "z": [cplx(v) for v in z]})
        z = ref.cmpsit(n, t.flip, t.phase, t.cf, d.idx, d.cf, 3, 2, 10, 16,
                       0.1, 0.02, 0x5678 + case)
        drv.append({"kind": "cmpsit", "nqb": n, "flip": t.flip.tolist(),
                    "phase": t.phase.tolist(), "cf": t.cf.tolist(),
                    "det_idx": d.idx.tolist(),
                    "det_cf": [cplx(c) for c in d.cf], "samples": 3,
                    "steps": 2, "length": 10, "depth": 16,
                    "angle_det": 0.1, "angle_rand": 0.02,
                    "seed": 0x5678 + case, "z": [cplx(v) for v in z]})
    gold["drivers"] = drv

    # -- the full 12-qubit Trotter workload
    cfg = workloads.trotter12()
    t, d = cfg["terms"], cfg["dets"]
    z = ref.trott(12, t.flip, t.phase, t.cf, d.idx, d.cf, cfg["steps"],
                  cfg["delta"], order2=False, sort_lex=True)
    gold["trotter12"] = {"z": [cplx(v) for v in z]}

    # -- the reference's water fixture through all four drivers
    h = h2o_fixture()
    fl = np.array(h["flip"], dtype=np.uint64)
    ph = np.array(h["phase"], dtype=np.uint64)
    cf = np.array(h["cf"])
    di = np.array(h["det_idx"], dtype=np.uint64)
    dc = np.array([complex(*c) for c in h["det_cf"]])
    h["trott"] = [cplx(v) for v in ref.trott(10, fl, ph, cf, di, dc, 12,
                                            0.5)]
    h["trott2"] = [cplx(v) for v in ref.trott(10, fl, ph, cf, di, dc, 12,
                                             0.5, order2=True)]
    h["qdrift"] = [cplx(v) for v in ref.qdrift(10, fl, ph, cf, di, dc, 6,
                                              300, 0.01, 0xC0FFEE)]
    h["cmpsit"] = [cplx(v) for v in ref.cmpsit(10, fl, ph, cf, di, dc, 3,
                                              4, 60, 50, 0.1, 0.02,
                                              0xBEEF)]
    gold["h2o"] = h

    # -- coefficient-matrix trial states: the reference's expansion
    # (state_prep_coeff_expand_all) and overlap (circ.c measure_coeff)
    from types import SimpleNamespace
    crng = np.random.Generator(np.random.PCG64(0xC0EFF))
    cms = []
    for ns, na, nb, closed, tap, nc in ((4, 2, 2, True, False, 0),
                                        (5, 2, 3, False, False, 0),
                                        (5, 2, 2, True, True, 0),
                                        (4, 2, 1, False, False, 3),
                                        (6, 3, 3, False, True, 2),
                                        (3, 0, 1, False, False, 0)):
        nblk = max(nc, 1)
        cm = SimpleNamespace(
            n_sites=ns, n_alpha=na, n_beta=nb,
            C_alpha=[crng.standard_normal((ns, na)) for _ in range(nblk)],
            C_beta=(None if closed else
                    [crng.standard_normal((ns, nb)) for _ in range(nblk)]),
            weights=None if nc == 0 else list(crng.standard_normal(nc)),
            tapered=tap)
        nqb = 2 * ns - (2 if tap else 0)
        amp = ref.coeff_expand(nqb, cm)
        nz = np.nonzero(amp)[0]
        seed = int(crng.integers(1 << 30))
        cms.append({
            "nqb": nqb, "n_sites": ns, "n_alpha": na, "n_beta": nb,
            "tapered": tap,
            "C_alpha": [c.tolist() for c in cm.C_alpha],
            "C_beta": (None if cm.C_beta is None
                       else [c.tolist() for c in cm.C_beta]),
            "weights": cm.weights,
            "expand_idx": nz.tolist(),
            "expand_val": [float(v.real) for v in amp[nz]],
            "psi_seed": seed,
            "inner": cplx(ref.coeff_inner(nqb, cm,
                                          _psi_from_seed(nqb, seed)))})
    gold["coeff_matrix"] = cms

    (OUT / "golden.json").write_text(json.dumps(gold, indent=0))

    # -- qreg_paulirot on a random 9-qubit state
    n = 9
    amp0 = rng.random(1 << n) + 1j * rng.random(1 << n)
    t = workloads.random_terms(n, 300, seed=5000)
    phi = rng.uniform(-1.0, 1.0, 300)
    amp1 = ref.paulirot(amp0, n, t.flip, t.phase, phi)
    np.savez_compressed(OUT / "paulirot.npz", amp0=amp0, flip=t.flip,
                        phase=t.phase, phi=phi, amp1=amp1)
    print("wrote", OUT / "golden.json", OUT / "paulirot.npz")


if __name__ == "__main__":
    main()
