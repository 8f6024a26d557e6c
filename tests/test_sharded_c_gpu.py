"""The C sharded register (include/phase2_sharded.h) on one GPU.

Every rank held by one object (pairs trade halves in place): FP64
rotations and the four drivers equal the oracle's full-register results
bit for bit for 1 to 8 ranks, the swap decisions match the Python layer
(phase2_b200/sharded.py: same layout, same swap count), FP32 within 1e-5,
and bad shapes are refused.  The transport path between processes is
exercised by tests/c/sharded_threads.c (test_sharded_c.py).
"""

import ctypes as C

import numpy as np
import pytest

import phase2_b200 as p2
from phase2_b200 import Dets, _hamil, _muldet, sharded, workloads
from phase2_b200._ffi import CmpsitData, lib

pytestmark = pytest.mark.gpu

U64 = C.POINTER(C.c_uint64)
F64 = C.POINTER(C.c_double)


class CSharded:
    def __init__(self, nqb, world, prec, ranks=None, chunk=0):
        p2.world_ensure()
        ranks = list(range(world)) if ranks is None else ranks
        arr = (C.c_uint32 * len(ranks))(*ranks)
        self.L = lib()
        self.h = self.L.phase2_sharded_new(nqb, world, arr, len(ranks), prec,
                                           None, chunk)
        if not self.h:
            raise ValueError("phase2_sharded_new refused")
        self.nqb = nqb

    def close(self):
        if self.h:
            self.L.phase2_sharded_free(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def prepst(self, idx, cf):
        idx = np.ascontiguousarray(idx, dtype=np.uint64)
        cf = np.ascontiguousarray(cf, dtype=np.complex128)
        assert self.L.phase2_sharded_prepst(
            self.h, idx.ctypes.data_as(U64), cf.ctypes.data_as(F64),
            len(idx)) == 0

    def paulirot(self, flip, phase, phi):
        flip = np.ascontiguousarray(flip, dtype=np.uint64)
        phase = np.ascontiguousarray(phase, dtype=np.uint64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        return self.L.phase2_sharded_paulirot(
            self.h, flip.ctypes.data_as(U64), phase.ctypes.data_as(U64),
            phi.ctypes.data_as(F64), len(phi))

    def state(self):
        idx = np.arange(1 << self.nqb, dtype=np.uint64)
        out = np.zeros(len(idx), dtype=np.complex128)
        assert self.L.phase2_sharded_getamps(
            self.h, idx.ctypes.data_as(U64), out.ctypes.data_as(F64),
            len(idx)) == 0
        return out

    def counters(self):
        sw, ex = C.c_uint64(), C.c_uint64()
        self.L.phase2_sharded_counters(self.h, C.byref(sw), C.byref(ex))
        return sw.value, ex.value

    def layout(self):
        pos = (C.c_uint32 * self.nqb)()
        assert self.L.phase2_sharded_layout(self.h, pos) == 0
        return list(pos)


def _narrow_terms(nqb, n, max_flip, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    flip = np.zeros(n, dtype=np.uint64)
    phase = rng.integers(0, 1 << nqb, size=n).astype(np.uint64)
    for k in range(n):
        w = int(rng.integers(0, max_flip + 1))
        for q in rng.choice(nqb, size=w, replace=False):
            flip[k] |= np.uint64(1 << int(q))
    return flip, phase, rng.standard_normal(n)


def _start_state(nqb, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    a = rng.standard_normal(1 << nqb) + 1j * rng.standard_normal(1 << nqb)
    return a / np.linalg.norm(a)


@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_fp64_rotations_bitwise_and_same_swaps(oracle_lib, world):
    nqb = 13
    flip, phase, phi = _narrow_terms(nqb, 300, 4, seed=41)
    amp = _start_state(nqb, 42)
    want = oracle_lib.rotate(amp, nqb, flip, phase, phi)
    with CSharded(nqb, world, p2.PREC_FP64) as reg:
        reg.prepst(np.arange(1 << nqb), amp)
        assert reg.paulirot(flip, phase, phi) == 0
        got = reg.state()
        swaps, _ = reg.counters()
        layout = reg.layout()
    assert np.array_equal(got.view(np.float64), want.view(np.float64))
    if world > 1:
        with sharded.ShardedRegister.on_one_gpu(nqb, world,
                                                p2.PREC_FP64) as py:
            py.prepst(Dets(np.arange(1 << nqb, dtype=np.uint64), amp))
            py.paulirot(flip, phase, phi)
            assert py.swaps == swaps > 0
            assert py.layout.pos == layout


def _drivers(nqb, world, kind, oracle_lib):
    terms = workloads.jw_terms(nqb, 400, seed=43)
    dets = workloads.hamming_dets(nqb, 4, nqb // 2, seed=44)
    hm, md = _hamil(nqb, terms), _muldet(dets)
    L = lib()
    try:
        with CSharded(nqb, world, p2.PREC_FP64) as reg:
            if kind in ("trott", "trott2"):
                out = np.zeros(3, dtype=np.complex128)
                assert L.phase2_sharded_trott(
                    reg.h, C.byref(hm), C.byref(md), 3, 0.05,
                    int(kind == "trott2"), out.ctypes.data_as(F64)) == 0
                ref = oracle_lib.trott(nqb, terms.flip, terms.phase, terms.cf,
                                       dets.idx, dets.cf, 3, 0.05,
                                       order2=kind == "trott2")
            elif kind == "qdrift":
                out = np.zeros(2, dtype=np.complex128)
                assert L.phase2_sharded_qdrift(
                    reg.h, C.byref(hm), C.byref(md), 2, 300, 1e-2,
                    0x5EED51, out.ctypes.data_as(F64)) == 0
                ref = oracle_lib.qdrift(nqb, terms.flip, terms.phase, terms.cf,
                                        dets.idx, dets.cf, 2, 300, 1e-2,
                                        0x5EED51)
            else:
                args = (2, 2, 40, 60, 0.05, 0.002, 0xC3317)
                dt = CmpsitData(*args)
                out = np.zeros(2, dtype=np.complex128)
                assert L.phase2_sharded_cmpsit(
                    reg.h, C.byref(hm), C.byref(md), C.byref(dt),
                    out.ctypes.data_as(F64)) == 0
                ref = oracle_lib.cmpsit(nqb, terms.flip, terms.phase,
                                        terms.cf, dets.idx, dets.cf, *args)
            swaps, _ = reg.counters()
    finally:
        L.circ_hamil_free(C.byref(hm))
        L.circ_muldet_free(C.byref(md))
    return out, ref, swaps


@pytest.mark.parametrize("kind", ["trott", "trott2", "qdrift", "cmpsit"])
@pytest.mark.parametrize("world", [2, 4])
def test_fp64_drivers_bitwise(oracle_lib, kind, world):
    out, ref, swaps = _drivers(13, world, kind, oracle_lib)
    assert swaps > 0
    assert np.array_equal(out.view(np.float64), ref.view(np.float64))


def test_fp32_within_tolerance(oracle_lib):
    nqb = 16
    flip, phase, phi = _narrow_terms(nqb, 200, 4, seed=45)
    amp = _start_state(nqb, 46)
    want = oracle_lib.rotate(amp, nqb, flip, phase, phi)
    with CSharded(nqb, 4, p2.PREC_FP32) as reg:
        reg.prepst(np.arange(1 << nqb), amp)
        assert reg.paulirot(flip, phase, phi) == 0
        got = reg.state()
        n2 = C.c_double()
        assert lib().phase2_sharded_norm2(reg.h, C.byref(n2)) == 0
    assert np.max(np.abs(got - want)) < 1e-5
    assert abs(n2.value - 1.0) < 1e-5


def test_refusals():
    p2.world_ensure()
    L = lib()
    one = (C.c_uint32 * 1)(0)
    two = (C.c_uint32 * 2)(0, 0)
    assert not L.phase2_sharded_new(10, 3, one, 1, p2.PREC_FP64, None, 0)
    assert not L.phase2_sharded_new(2, 4, one, 1, p2.PREC_FP64, None, 0)
    assert not L.phase2_sharded_new(10, 2, two, 2, p2.PREC_FP64, None, 0)
    # one of two ranks held and no transport
    assert not L.phase2_sharded_new(10, 2, one, 1, p2.PREC_FP64, None, 0)
    with CSharded(8, 4, p2.PREC_FP64) as reg:
        # a flip over 7 qubits does not fit 6 local qubits
        assert reg.paulirot([0x7F], [0], [0.1]) == -1
        # a string beyond the register
        assert reg.paulirot([1 << 9], [0], [0.1]) == -1
