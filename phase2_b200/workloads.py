"""Seeded synthetic inputs with the shapes of the benchmark workloads.

There is no dataset for this path: the workloads are generated.  All
generators use numpy's PCG64 with explicit seeds, so every run (tests,
bench, oracle) sees identical inputs.

* ``random_terms``   each qubit's operator uniform over {I, X, Y, Z};
                     coefficients N(0,1)/sqrt(nterms) (the 12-qubit Trotter
                     case: 200 terms, one determinant with 6 ones).
* ``jw_terms``       Jordan-Wigner-like excitation strings: one-body
                     (2 strings per pair: XX, YY on p<q) and two-body
                     (8 strings per quadruple: every X/Y assignment with an
                     even number of Y on p<q<r<s), Z on every qubit strictly
                     inside each paired interval, plus pure-Z terms (Z_p,
                     Z_p Z_q) for the last 10 %.  Coefficients +-10^U(-6,0).
                     Position sets are drawn with replacement.
* ``hamming_dets``   determinants of a given Hamming weight with
                     complex-normal amplitudes, normalised.
"""

from __future__ import annotations

import numpy as np

from . import Dets, Terms

_XY8 = [(a, b, c, d) for a in (0, 1) for b in (0, 1) for c in (0, 1)
        for d in (0, 1) if (a + b + c + d) % 2 == 0]  # 1 = Y


def random_terms(nqb: int, nterms: int, seed: int) -> Terms:
    rng = np.random.Generator(np.random.PCG64(seed))
    ops = rng.integers(0, 4, size=(nterms, nqb))  # 0 I, 1 X, 2 Y, 3 Z
    bit = (np.uint64(1) << np.arange(nqb, dtype=np.uint64))
    flip = ((ops == 1) | (ops == 2)).astype(np.uint64) @ bit
    phase = ((ops == 2) | (ops == 3)).astype(np.uint64) @ bit
    cf = rng.standard_normal(nterms) / np.sqrt(nterms)
    return Terms(flip.astype(np.uint64), phase.astype(np.uint64), cf)


def _chain(lo: int, hi: int) -> int:
    """Z mask strictly between qubits lo < hi."""
    if hi - lo < 2:
        return 0
    return ((1 << hi) - 1) & ~((1 << (lo + 1)) - 1)


def jw_terms(nqb: int, nterms: int, seed: int,
             one_body_frac: float = 0.1, z_frac: float = 0.1) -> Terms:
    if nqb < 4:
        raise ValueError("jw_terms needs at least 4 qubits")
    rng = np.random.Generator(np.random.PCG64(seed))
    n_z = int(round(nterms * z_frac))
    flips, phases = [], []
    while len(flips) < nterms - n_z:
        if rng.random() < one_body_frac:
            p, q = sorted(rng.choice(nqb, size=2, replace=False).tolist())
            z = _chain(p, q)
            for y in (0, 1):
                f = (1 << p) | (1 << q)
                ph = z | (((1 << p) | (1 << q)) if y else 0)
                flips.append(f)
                phases.append(ph)
        else:
            pos = sorted(rng.choice(nqb, size=4, replace=False).tolist())
            z = _chain(pos[0], pos[1]) | _chain(pos[2], pos[3])
            f = sum(1 << k for k in pos)
            for ys in _XY8:
                ph = z
                for k, y in zip(pos, ys):
                    if y:
                        ph |= 1 << k
                flips.append(f)
                phases.append(ph)
    flips = flips[:nterms - n_z]
    phases = phases[:nterms - n_z]
    for _ in range(n_z):
        if rng.random() < 0.5:
            p = int(rng.integers(nqb))
            flips.append(0)
            phases.append(1 << p)
        else:
            p, q = rng.choice(nqb, size=2, replace=False).tolist()
            flips.append(0)
            phases.append((1 << p) | (1 << q))
    mag = 10.0 ** rng.uniform(-6.0, 0.0, size=nterms)
    sign = np.where(rng.random(nterms) < 0.5, -1.0, 1.0)
    return Terms(np.array(flips, dtype=np.uint64),
                 np.array(phases, dtype=np.uint64), mag * sign)


def hamming_dets(nqb: int, ndets: int, weight: int, seed: int) -> Dets:
    rng = np.random.Generator(np.random.PCG64(seed))
    seen: set[int] = set()
    idx = []
    while len(idx) < ndets:
        pos = rng.choice(nqb, size=weight, replace=False)
        v = int(sum(1 << int(k) for k in pos))
        if v not in seen:
            seen.add(v)
            idx.append(v)
    cf = rng.standard_normal(ndets) + 1j * rng.standard_normal(ndets)
    cf /= np.linalg.norm(cf)
    return Dets(np.array(idx, dtype=np.uint64), cf.astype(np.complex128))


def sort_by_flip(t: Terms) -> Terms:
    """Stable order by (flip, phase), as circ_hamil_sort_flip."""
    order = np.lexsort((t.phase, t.flip))
    return Terms(t.flip[order], t.phase[order], t.cf[order])


# ---- the benchmark configurations --------------------------------------

def trotter12():
    """12 qubits, 200 random terms, 1 determinant with 6 ones, delta 0.1,
    4 first-order steps (lexicographic order, as trott_init sorts)."""
    t = random_terms(12, 200, seed=0x12C0FFEE)
    d = hamming_dets(12, 1, 6, seed=0x12DE7)
    d = Dets(d.idx, np.ones(1, dtype=np.complex128))
    return dict(nqb=12, terms=t, dets=d, steps=4, delta=0.1)


def strang26(nterms: int = 20000, steps: int = 256):
    """26 qubits, 20,000 JW terms sorted by flip mask, 16 determinants of
    weight 13, delta 0.05, second-order steps."""
    t = sort_by_flip(jw_terms(26, nterms, seed=0x26A11CE))
    d = hamming_dets(26, 16, 13, seed=0x26DE75)
    return dict(nqb=26, terms=t, dets=d, steps=steps, delta=0.05)


def qdrift30(nqb: int = 30, nterms: int = 100000, depth: int = 4096,
             samples: int = 64):
    """30 qubits, 100,000 JW terms, 4096 draws per sample, 64 samples,
    step_size 1e-3, one determinant of weight nqb/2."""
    t = jw_terms(nqb, nterms, seed=0x30D41F7)
    d = hamming_dets(nqb, 1, nqb // 2, seed=0x30DE7)
    d = Dets(d.idx, np.ones(1, dtype=np.complex128))
    return dict(nqb=nqb, terms=t, dets=d, samples=samples, depth=depth,
                step_size=1e-3, seed=0x5EEDD41F7)


def cmpsit33(nqb: int = 33, nterms: int = 200000, steps: int = 64):
    """33 qubits, 200,000 JW terms, top 2,000 deterministic, 8,192 draws
    per half step, 32 determinants, angle_det 0.05,
    angle_rand 0.05 * lambda_rand / 8192."""
    t = jw_terms(nqb, nterms, seed=0x33C0317)
    d = hamming_dets(nqb, 32, nqb // 2, seed=0x33DE7)
    length, depth = 2000, 8192
    lam = float(np.sort(np.abs(t.cf))[::-1][length:].sum())
    return dict(nqb=nqb, terms=t, dets=d, samples=1, steps=steps,
                length=length, depth=depth, angle_det=0.05,
                angle_rand=0.05 * lam / depth, seed=0x5EEDC317)
