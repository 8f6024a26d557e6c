"""Full-width golden vectors from the reference's own CPU path
(TEST INFRASTRUCTURE; runs where oracle/_ref/libphase2_ref.so is built).

Two runs of the reference drivers at the benchmark widths, on the seeded
benchmark Hamiltonians (phase2_b200.workloads):

* trott2_26   26 qubits: the first 100 terms, in the reference's
              lexicographic order, of the 20,000-term JW Hamiltonian of the
              26-qubit Strang configuration, with its 16 determinants; one
              second-order step of delta 0.05 (200 rotations,
              circ/trott2.c:44-74).  Stored: the overlap and every 2^14-th
              amplitude of the final state (4096 values).
* qdrift_30   30 qubits: one qDRIFT sample of depth 16 on the
              100,000-term JW Hamiltonian of the 30-qubit configuration
              (its determinant, step_size and seed; circ/qdrift.c:95-134).
              Stored: the overlap, the number and the sum of squares of the
              non-zero amplitudes of the final state, and every 16th of
              them in index order.

Writes tests/golden/wide.npz.  The reference needs 2 GiB (26 qubits) and
32 GiB (30 qubits: amplitudes and exchange buffer) of host memory and a
few minutes per run on one core.
"""

from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import Reference  # noqa: E402
from phase2_b200 import Terms, workloads  # noqa: E402

TROTT_TERMS = 100
QDRIFT_DEPTH = 16


def lex_key(t: Terms, nqb: int) -> np.ndarray:
    """Sort key of the reference's lexicographic order: per-qubit operator
    codes I<X<Y<Z compared from the highest qubit down
    (phase2/paulis.c:190-205)."""
    key = np.zeros(len(t.cf), dtype=np.uint64)
    for q in range(nqb):
        f = (t.flip >> np.uint64(q)) & np.uint64(1)
        p = (t.phase >> np.uint64(q)) & np.uint64(1)
        code = np.where(f == 1, 1 + p, 3 * p).astype(np.uint64)
        key |= code << np.uint64(2 * q)
    return key


def trott_subset() -> tuple[dict, np.ndarray]:
    """The 26-qubit configuration and the indices of its first TROTT_TERMS
    terms in lexicographic order."""
    cfg = workloads.strang26()
    order = np.argsort(lex_key(cfg["terms"], 26), kind="stable")
    return cfg, np.sort(order[:TROTT_TERMS])


def main() -> None:
    ref = Reference()
    out = {}

    cfg, sel = trott_subset()
    t, d = cfg["terms"], cfg["dets"]
    sub = Terms(t.flip[sel], t.phase[sel], t.cf[sel])
    taken = ref.capture(1 << 14, 4096)
    t0 = time.perf_counter()
    z = ref.trott(26, sub.flip, sub.phase, sub.cf, d.idx, d.cf, 1,
                  cfg["delta"], order2=True)
    idx, amp = taken()
    print(f"trott2_26: {time.perf_counter() - t0:.0f} s, z = {z[0]}",
          flush=True)
    out.update(trott2_26_terms=sel, trott2_26_z=z, trott2_26_idx=idx,
               trott2_26_amp=amp)

    cfg = workloads.qdrift30()
    t, d = cfg["terms"], cfg["dets"]
    cap = 1 << QDRIFT_DEPTH
    taken = ref.capture(0, cap)
    t0 = time.perf_counter()
    z = ref.qdrift(30, t.flip, t.phase, t.cf, d.idx, d.cf, 1, QDRIFT_DEPTH,
                   cfg["step_size"], cfg["seed"])
    idx, amp = taken()
    print(f"qdrift_30: {time.perf_counter() - t0:.0f} s, z = {z[0]}, "
          f"{len(idx)} non-zero amplitudes", flush=True)
    out.update(qdrift_30_depth=np.int64(QDRIFT_DEPTH), qdrift_30_z=z,
               qdrift_30_nnz=np.int64(len(idx)),
               qdrift_30_norm2=np.float64(np.sum(np.abs(amp) ** 2)),
               qdrift_30_idx=idx[::16], qdrift_30_amp=amp[::16])

    np.savez_compressed(HERE / "wide.npz", **out)
    print("wrote", HERE / "wide.npz")


if __name__ == "__main__":
    main()
