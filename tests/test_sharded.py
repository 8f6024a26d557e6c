"""Sharded registers (phase2_b200/sharded.py) on CPU.

Each rank's slab here is a numpy array rotated by the oracle (test
infrastructure), so these tests check the host logic of the sharding: the
qubit layout, the choice and execution of qubit swaps, the per-rank sign
of Z on high qubits, chunked half-slab exchange, state preparation and
overlaps.  Virtual ranks in one process (in-place pair swaps and chunked
buffers) and two or four gloo ranks must reproduce the oracle's
full-register results bit for bit.  The CUDA slabs are checked in
test_sharded_gpu.py.
"""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from phase2_b200 import Dets, Terms, sharded, workloads


class OracleSlab:
    """One rank's 2^L amplitudes on the CPU, rotated by the oracle."""

    def __init__(self, nlocal, oracle):
        self.nqb, self.o = nlocal, oracle
        self.a = np.zeros(1 << nlocal, dtype=np.complex128)
        self.dtype, self.device = torch.float64, torch.device("cpu")

    def buffer(self, count):
        return torch.empty(2 * count, dtype=torch.float64)

    def paulirot(self, flip, phase, phi):
        self.a = self.o.rotate(self.a, self.nqb, flip, phase, phi)

    def zero(self):
        self.a[:] = 0

    def setamps(self, idx, z):
        self.a[np.asarray(idx, dtype=np.int64)] = z

    def getamps(self, idx):
        return self.a[np.asarray(idx, dtype=np.int64)].copy()

    def get_state(self):
        return self.a.copy()

    def norm2(self):
        return float(np.sum(np.abs(self.a) ** 2))

    def synchronize(self):
        pass

    def _half(self, bit, val):
        return self.a.reshape(-1, 2, 1 << bit)[:, val, :].reshape(-1)

    def slab_get(self, bit, val, first, count, buf):
        buf.numpy().view(np.complex128)[:] = \
            self._half(bit, val)[first:first + count]

    def slab_put(self, bit, val, first, count, buf):
        v = self.a.reshape(-1, 2, 1 << bit)[:, val, :]
        flat = v.reshape(-1).copy()
        flat[first:first + count] = buf.numpy().view(np.complex128)
        v[...] = flat.reshape(v.shape)

    def swap_halves(self, other, bit, val, other_val):
        x = self.a.reshape(-1, 2, 1 << bit)[:, val, :]
        y = other.a.reshape(-1, 2, 1 << bit)[:, other_val, :]
        t = x.copy()
        x[...] = y
        y[...] = t


def _local_reg(nqb, world, oracle, chunk=sharded.CHUNK, in_place=True):
    g = world.bit_length() - 1
    slabs = {r: OracleSlab(nqb - g, oracle) for r in range(world)}
    return sharded.ShardedRegister(nqb, world, slabs,
                                   sharded.LocalTransport(), chunk,
                                   in_place)


def _narrow_terms(nqb, n, max_flip, seed):
    """Random Pauli strings with at most max_flip X/Y (any Z elsewhere)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    flip = np.zeros(n, dtype=np.uint64)
    phase = np.zeros(n, dtype=np.uint64)
    for k in range(n):
        w = int(rng.integers(0, max_flip + 1))
        qs = rng.choice(nqb, size=w, replace=False)
        f = 0
        for q in qs:
            f |= 1 << int(q)
        z = int(rng.integers(0, 1 << nqb))
        flip[k], phase[k] = f, z
    return flip, phase, rng.standard_normal(n)


def _start_state(nqb, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    a = rng.standard_normal(1 << nqb) + 1j * rng.standard_normal(1 << nqb)
    return a / np.linalg.norm(a)


def _load(reg, amp):
    nz = np.arange(len(amp), dtype=np.uint64)
    reg.prepst(Dets(nz, amp))


def test_layout_maps_are_inverse():
    lay = sharded.Layout(9, 6)
    rng = np.random.Generator(np.random.PCG64(4))
    for _ in range(20):
        lay.swap(int(rng.integers(0, 9)), int(rng.integers(0, 9)))
    m = rng.integers(0, 1 << 9, size=200).astype(np.uint64)
    assert np.array_equal(lay.glob(lay.phys(m)), m)
    assert sorted(lay.pos) == list(range(9))
    assert all(lay.at[lay.pos[q]] == q for q in range(9))


@pytest.mark.parametrize("in_place", [True, False])
@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_rotations_bitwise_equal_full_register(oracle_lib, world, in_place):
    nqb = 9
    flip, phase, phi = _narrow_terms(nqb, 120, 3, seed=11)
    amp = _start_state(nqb, 5)
    want = oracle_lib.rotate(amp, nqb, flip, phase, phi)
    reg = _local_reg(nqb, world, oracle_lib, in_place=in_place)
    assert reg.in_place == in_place
    _load(reg, amp)
    reg.paulirot(flip, phase, phi)
    got = reg.get_state()
    assert np.array_equal(got.view(np.float64), want.view(np.float64))
    if world > 1:
        assert reg.swaps > 0
        assert not reg.layout.identity()


@pytest.mark.parametrize("chunk", [1, 3, 64])
def test_chunked_exchange_same_bits(oracle_lib, chunk):
    nqb, world = 8, 4
    flip, phase, phi = _narrow_terms(nqb, 60, 4, seed=12)
    amp = _start_state(nqb, 6)
    want = oracle_lib.rotate(amp, nqb, flip, phase, phi)
    reg = _local_reg(nqb, world, oracle_lib, chunk=chunk, in_place=False)
    _load(reg, amp)
    reg.paulirot(flip, phase, phi)
    assert np.array_equal(reg.get_state(), want)


def test_high_z_and_y_only_signs(oracle_lib):
    """Strings with Z/Y on the high qubits: Y needs a swap, Z only a
    per-rank sign."""
    nqb, world = 6, 4
    hi = 1 << 5 | 1 << 4
    flip = np.array([0, 1 << 5, 1 | 1 << 4, 0], dtype=np.uint64)
    phase = np.array([hi, 1 << 5, hi | 2, 1 << 4 | 1], dtype=np.uint64)
    phi = np.array([0.3, -0.7, 1.1, 0.25])
    amp = _start_state(nqb, 8)
    want = oracle_lib.rotate(amp, nqb, flip, phase, phi)
    reg = _local_reg(nqb, world, oracle_lib)
    _load(reg, amp)
    reg.paulirot(flip[:1], phase[:1], phi[:1])
    assert reg.swaps == 0  # Z only: no exchange
    reg.paulirot(flip[1:], phase[1:], phi[1:])
    assert reg.swaps == 2
    assert np.array_equal(reg.get_state(), want)


def test_norm2_over_ranks(oracle_lib):
    nqb = 9
    flip, phase, phi = _narrow_terms(nqb, 50, 3, seed=13)
    amp = 0.7 * _start_state(nqb, 14)
    reg = _local_reg(nqb, 4, oracle_lib)
    _load(reg, amp)
    reg.paulirot(flip, phase, phi)
    assert abs(reg.norm2() - 0.49) < 1e-13


def test_swapped_qubit_stays_local(oracle_lib):
    nqb, world = 7, 2
    reg = _local_reg(nqb, world, oracle_lib)
    _load(reg, _start_state(nqb, 9))
    f = np.array([1 << 6 | 1] * 5, dtype=np.uint64)
    reg.paulirot(f, np.zeros(5, dtype=np.uint64), np.full(5, 0.1))
    assert reg.swaps == 1
    assert reg.layout.pos[6] < reg.nlocal


@pytest.mark.parametrize("order2", [False, True])
def test_trott_overlaps_bitwise(oracle_lib, order2):
    nqb = 10
    terms = workloads.jw_terms(nqb, 60, seed=21)
    dets = workloads.hamming_dets(nqb, 5, 3, seed=22)
    want = oracle_lib.trott(nqb, terms.flip, terms.phase, terms.cf,
                            dets.idx, dets.cf, 3, 0.05, order2=order2)
    reg = _local_reg(nqb, 4, oracle_lib)
    got = sharded.trott(reg, terms, dets, 3, 0.05, order2=order2)
    assert np.array_equal(got.view(np.float64), want.view(np.float64))


@pytest.mark.parametrize("world", [2, 4])
def test_qdrift_overlaps_bitwise(oracle_lib, world):
    nqb = 10
    terms = workloads.jw_terms(nqb, 80, seed=23)
    dets = workloads.hamming_dets(nqb, 2, 5, seed=24)
    want = oracle_lib.qdrift(nqb, terms.flip, terms.phase, terms.cf,
                             dets.idx, dets.cf, 3, 40, 0.01, 0xD41F7)
    reg = _local_reg(nqb, world, oracle_lib)
    got = sharded.qdrift(reg, terms, dets, 3, 40, 0.01, 0xD41F7)
    assert np.array_equal(got.view(np.float64), want.view(np.float64))
    assert reg.swaps > 0
    with pytest.raises(ValueError):
        sharded.qdrift(reg, terms, dets, 1, 4, 0.01, 0)
    eps = np.finfo(np.float64).eps
    assert list(sharded._sign_dz(np.array(
        [eps, eps / 2, -eps / 2, -eps, 0.0, -0.0, 3.0, -2.0]))) == \
        [1.0, 0.0, 0.0, -1.0, 0.0, 0.0, 1.0, -1.0]


@pytest.mark.parametrize("world", [2, 4])
def test_cmpsit_overlaps_bitwise(oracle_lib, world):
    nqb = 10
    terms = workloads.jw_terms(nqb, 90, seed=25)
    dets = workloads.hamming_dets(nqb, 3, 5, seed=26)
    args = (2, 2, 12, 20, 0.05, 0.003, 0xC0317)
    want = oracle_lib.cmpsit(nqb, terms.flip, terms.phase, terms.cf,
                             dets.idx, dets.cf, *args)
    reg = _local_reg(nqb, world, oracle_lib)
    got = sharded.cmpsit(reg, terms, dets, *args)
    assert np.array_equal(got.view(np.float64), want.view(np.float64))
    with pytest.raises(ValueError):
        sharded.cmpsit(reg, terms, dets, 1, 1, 90, 4, 0.05, 0.003, 7)


def test_errors(oracle_lib):
    with pytest.raises(ValueError):
        _local_reg(4, 3, oracle_lib)  # not a power of two
    with pytest.raises(ValueError):
        sharded.ShardedRegister(3, 8, {}, sharded.LocalTransport())
    reg = _local_reg(5, 8, oracle_lib)  # two local qubits
    _load(reg, _start_state(5, 1))
    with pytest.raises(ValueError, match="local qubits"):
        reg.paulirot(np.array([0b10111], dtype=np.uint64),
                     np.zeros(1, dtype=np.uint64), np.array([0.1]))
    with pytest.raises(ValueError, match="beyond"):
        reg.paulirot(np.array([1 << 5], dtype=np.uint64),
                     np.zeros(1, dtype=np.uint64), np.array([0.1]))


# ---- two gloo ranks ---------------------------------------------------


def _gloo_main(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import Oracle
        o = Oracle()
        nqb = 8
        g = world.bit_length() - 1
        reg = sharded.ShardedRegister(
            nqb, world, {rank: OracleSlab(nqb - g, o)},
            sharded.DistTransport(), chunk=5)
        terms = workloads.jw_terms(nqb, 40, seed=31)
        dets = workloads.hamming_dets(nqb, 4, 2, seed=32)
        vals = sharded.trott(reg, terms, dets, 2, 0.07, order2=True)
        state = reg.get_state()
        q.put((rank, vals, state, reg.swaps))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_gloo_ranks_match_oracle(oracle_lib, world):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_main, args=(r, world, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    nqb = 8
    terms = workloads.jw_terms(nqb, 40, seed=31)
    dets = workloads.hamming_dets(nqb, 4, 2, seed=32)
    want = oracle_lib.trott(nqb, terms.flip, terms.phase, terms.cf,
                            dets.idx, dets.cf, 2, 0.07, order2=True)
    sorted_t = sharded.sort_lex(nqb, terms)
    amp = np.zeros(1 << nqb, dtype=np.complex128)
    amp[dets.idx.astype(np.int64)] = dets.cf
    for _ in range(2):
        amp = oracle_lib.rotate(amp, nqb, sorted_t.flip, sorted_t.phase,
                                sorted_t.cf * 0.035)
        amp = oracle_lib.rotate(amp, nqb, sorted_t.flip[::-1],
                                sorted_t.phase[::-1],
                                sorted_t.cf[::-1] * 0.035)
    for rank, vals, state, swaps in res:
        assert np.array_equal(vals, want)
        assert np.array_equal(state, amp)
        assert swaps == res[0][3] and swaps > 0


def _subgroup_main(rank, world, port, q):
    """Four gloo ranks as two sharded registers of two ranks each: ranks
    {0, 2} and {1, 3}, so a group rank differs from the global one."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import Oracle
        o = Oracle()
        groups = [dist.new_group([0, 2]), dist.new_group([1, 3])]
        grp = groups[rank % 2]
        grank = dist.get_rank(grp)
        nqb = 8
        reg = sharded.ShardedRegister(
            nqb, 2, {grank: OracleSlab(nqb - 1, o)},
            sharded.DistTransport(group=grp), chunk=7)
        terms = workloads.jw_terms(nqb, 30, seed=33 + rank % 2)
        dets = workloads.hamming_dets(nqb, 2, 3, seed=34)
        vals = sharded.trott(reg, terms, dets, 2, 0.06)
        q.put((rank, vals, reg.swaps))
    finally:
        dist.destroy_process_group()


def test_gloo_subgroups_match_oracle(oracle_lib):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_subgroup_main, args=(r, 4, port, q))
             for r in range(4)]
    for p in procs:
        p.start()
    res = {r: (v, sw) for r, v, sw in (q.get(timeout=240) for _ in range(4))}
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    nqb = 8
    dets = workloads.hamming_dets(nqb, 2, 3, seed=34)
    for parity in (0, 1):
        terms = workloads.jw_terms(nqb, 30, seed=33 + parity)
        want = oracle_lib.trott(nqb, terms.flip, terms.phase, terms.cf,
                                dets.idx, dets.cf, 2, 0.06)
        for r in (parity, parity + 2):
            assert np.array_equal(res[r][0], want)
            assert res[r][1] > 0
