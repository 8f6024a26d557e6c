"""The seeded synthetic inputs that stand in for the reference's
Hamiltonians (phase2_b200.workloads): Jordan-Wigner-like excitation
strings with the structure the benchmark configurations specify, and
determinants of a given Hamming weight.  CPU only."""

import numpy as np

from phase2_b200 import workloads


def _bits(v):
    return [k for k in range(64) if v >> k & 1]


def _inside(p, q):
    return sum(1 << k for k in range(p + 1, q))


def test_jw_terms_structure():
    nqb, n = 16, 3000
    t = workloads.jw_terms(nqb, n, seed=77)
    assert len(t) == n
    flips = [int(f) for f in t.flip]
    phases = [int(p) for p in t.phase]
    nz = sum(1 for f in flips if f == 0)
    assert nz == round(0.1 * n)
    for f, ph in zip(flips, phases):
        assert (f | ph) >> nqb == 0
        if f == 0:  # Z_p or Z_p Z_q
            assert len(_bits(ph)) in (1, 2)
            continue
        pos = _bits(f)
        assert len(pos) in (2, 4)
        assert len(_bits(f & ph)) % 2 == 0  # even number of Y
        z = ph & ~f
        if len(pos) == 2:
            assert z == _inside(pos[0], pos[1])
        else:
            assert z == _inside(pos[0], pos[1]) | _inside(pos[2], pos[3])
    a = np.abs(t.cf)
    assert a.min() >= 1e-6 and a.max() <= 1.0
    assert (t.cf < 0).any() and (t.cf > 0).any()


def test_jw_terms_excitations_come_in_full_sets():
    """A one-body excitation gives XX and YY, a two-body one all eight X/Y
    assignments with an even Y count (the last set may be cut at the
    requested length)."""
    t = workloads.jw_terms(12, 800, seed=5)
    seen = {}
    for f, ph in zip(t.flip.tolist(), t.phase.tolist()):
        if f:
            seen.setdefault(f, set()).add(ph & f)
    full = [ys for f, ys in seen.items()
            if len(ys) == (2 if len(_bits(f)) == 2 else 8)]
    assert len(full) >= len(seen) - 1


def test_workloads_are_seeded():
    a = workloads.jw_terms(10, 500, seed=3)
    b = workloads.jw_terms(10, 500, seed=3)
    c = workloads.jw_terms(10, 500, seed=4)
    assert np.array_equal(a.flip, b.flip) and np.array_equal(a.cf, b.cf)
    assert not np.array_equal(a.cf, c.cf)


def test_hamming_dets():
    d = workloads.hamming_dets(20, 32, 10, seed=9)
    idx = [int(i) for i in d.idx]
    assert len(set(idx)) == 32
    assert all(len(_bits(i)) == 10 and i >> 20 == 0 for i in idx)
    assert abs(np.sum(np.abs(d.cf) ** 2) - 1.0) < 1e-12
