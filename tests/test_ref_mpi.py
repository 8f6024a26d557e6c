"""The reference's CPU drivers as R ranks of one job (oracle/_ref/ref_mpi).

The CPU baseline runs the reference's own qdrift and trott2 drivers as R
MPI ranks on the host's cores through the shared-memory stand-in
(oracle/mpi_shm).  These tests check, on CPU, that the stand-in carries
the reference's exchanges correctly: at 1, 2, 4 and 8 ranks (the state
split by its high qubits, every flush exchanging slabs between partner
ranks) and on both transports (single-copy cross-process reads and the
shared mailboxes), the drivers' overlaps agree with the oracle to 1e-12
(multi-rank runs round differently: the reference's projector mix and
add).  Skipped where the reference was not built.
"""

import numpy as np
import pytest

from oracle import REF_MPI, Oracle, run_ref_mpi, write_ref_input
from phase2_b200 import workloads

pytestmark = pytest.mark.skipif(not REF_MPI.is_file(),
                                reason="oracle/_ref/ref_mpi not built")

TOL = 1e-12


@pytest.fixture(scope="module")
def case():
    t = workloads.jw_terms(14, 800, seed=0x3E1)
    d = workloads.hamming_dets(14, 3, 7, seed=0x3E2)
    return t, d


@pytest.mark.parametrize("ranks", [1, 2, 4, 8])
def test_qdrift_ranks(tmp_path, case, ranks):
    t, d = case
    want = Oracle().qdrift(14, t.flip, t.phase, t.cf, d.idx, d.cf, 1, 48,
                           0.02, 0x77)
    path = tmp_path / "q.in"
    write_ref_input(path, "qdrift", 14, t.flip, t.phase, t.cf, d.idx, d.cf,
                    48, 0.02, 0x77)
    r = run_ref_mpi(ranks, path, 1, timeout=120)
    assert r["ranks"] == ranks and r["rotations"] == 48
    assert abs(r["z"] - want[0]) <= TOL
    assert r["rot_amp_s"] > 0


@pytest.mark.parametrize("mailbox", [False, True])
def test_trott2_ranks(tmp_path, case, mailbox):
    t, d = case
    n = 40
    want = Oracle().trott(14, t.flip[:n], t.phase[:n], t.cf[:n], d.idx,
                          d.cf, 2, 0.05, order2=True)
    path = tmp_path / "t.in"
    write_ref_input(path, "trott2", 14, t.flip[:n], t.phase[:n], t.cf[:n],
                    d.idx, d.cf, 2, 0.05)
    env = {"MPI_SHM_MAILBOX": "1"} if mailbox else None
    r = run_ref_mpi(4, path, 2, timeout=120, env=env)
    if mailbox:
        assert r["mailbox"]
    assert r["rotations"] == 2 * n * 2
    assert abs(r["z"] - want[-1]) <= TOL


def test_bad_input_is_refused(tmp_path):
    path = tmp_path / "bad.in"
    path.write_bytes(b"not an input file")
    with pytest.raises(RuntimeError):
        run_ref_mpi(2, path, 1, timeout=60)
