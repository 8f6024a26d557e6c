"""Sharded registers on the GPU: virtual ranks in one process, each a
device register of this library, exchanging half slabs through
qreg_slab_get / qreg_slab_put.

FP64 results must equal the oracle's full-register results (and the
unsharded engine's) bit for bit; FP32 within 1e-5 of them.  The
half-slab calls are checked against numpy and for the host-side errors
(host pointer, misaligned buffer, range past the buffer's allocation)
that they turn into -1 before any copy runs.
"""

import ctypes as C

import numpy as np
import pytest
import torch

import phase2_b200 as p2
from phase2_b200 import Dets, Register, sharded, workloads
from phase2_b200._ffi import lib

pytestmark = pytest.mark.gpu


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


def _load(reg, amp):
    reg.prepst(Dets(np.arange(len(amp), dtype=np.uint64), amp))


@pytest.mark.parametrize("in_place", [True, False])
@pytest.mark.parametrize("world", [2, 4, 8])
def test_fp64_rotations_bitwise(oracle_lib, world, in_place):
    nqb = 13
    flip, phase, phi = _narrow_terms(nqb, 300, 4, seed=41)
    amp = _start_state(nqb, 42)
    want = oracle_lib.rotate(amp, nqb, flip, phase, phi)
    with sharded.ShardedRegister.on_one_gpu(nqb, world, p2.PREC_FP64,
                                            chunk=1000,
                                            in_place=in_place) as reg:
        assert reg.in_place == in_place
        _load(reg, amp)
        reg.paulirot(flip, phase, phi)
        got = reg.get_state()
        assert reg.swaps > 0
    assert np.array_equal(got.view(np.float64), want.view(np.float64))


@pytest.mark.parametrize("order2", [False, True])
def test_fp64_trott_equals_unsharded_engine(oracle_lib, order2):
    nqb = 14
    terms = workloads.jw_terms(nqb, 400, seed=43)
    dets = workloads.hamming_dets(nqb, 4, 7, seed=44)
    fn = p2.trott2 if order2 else p2.trott
    p2.set_precision(p2.PREC_FP64)
    want = fn(nqb, terms, dets, 3, 0.05)
    ref = oracle_lib.trott(nqb, terms.flip, terms.phase, terms.cf,
                           dets.idx, dets.cf, 3, 0.05, order2=order2)
    with sharded.ShardedRegister.on_one_gpu(nqb, 4, p2.PREC_FP64) as reg:
        got = sharded.trott(reg, terms, dets, 3, 0.05, order2=order2)
    assert np.array_equal(np.asarray(want).view(np.float64),
                          ref.view(np.float64))
    assert np.array_equal(got.view(np.float64), ref.view(np.float64))


def test_fp64_qdrift_equals_unsharded_engine(oracle_lib):
    nqb = 14
    terms = workloads.jw_terms(nqb, 500, seed=51)
    dets = workloads.hamming_dets(nqb, 1, 7, seed=52)
    p2.set_precision(p2.PREC_FP64)
    want = p2.qdrift(nqb, terms, dets, 2, 300, 1e-2, 0x5EED51)
    ref = oracle_lib.qdrift(nqb, terms.flip, terms.phase, terms.cf,
                            dets.idx, dets.cf, 2, 300, 1e-2, 0x5EED51)
    with sharded.ShardedRegister.on_one_gpu(nqb, 4, p2.PREC_FP64) as reg:
        got = sharded.qdrift(reg, terms, dets, 2, 300, 1e-2, 0x5EED51)
        assert reg.swaps > 0
    assert np.array_equal(np.asarray(want).view(np.float64),
                          ref.view(np.float64))
    assert np.array_equal(got.view(np.float64), ref.view(np.float64))


def test_fp64_cmpsit_equals_unsharded_engine(oracle_lib):
    nqb = 13
    terms = workloads.jw_terms(nqb, 400, seed=53)
    dets = workloads.hamming_dets(nqb, 4, 6, seed=54)
    args = (2, 2, 40, 60, 0.05, 0.002, 0xC3317)
    p2.set_precision(p2.PREC_FP64)
    want = p2.cmpsit(nqb, terms, dets, *args)
    ref = oracle_lib.cmpsit(nqb, terms.flip, terms.phase, terms.cf,
                            dets.idx, dets.cf, *args)
    with sharded.ShardedRegister.on_one_gpu(nqb, 2, p2.PREC_FP64) as reg:
        got = sharded.cmpsit(reg, terms, dets, *args)
    assert np.array_equal(np.asarray(want).view(np.float64),
                          ref.view(np.float64))
    assert np.array_equal(got.view(np.float64), ref.view(np.float64))


@pytest.mark.parametrize("in_place", [True, False])
def test_fp32_within_tolerance(oracle_lib, in_place):
    nqb = 16
    flip, phase, phi = _narrow_terms(nqb, 200, 4, seed=45)
    amp = _start_state(nqb, 46)
    want = oracle_lib.rotate(amp, nqb, flip, phase, phi)
    with sharded.ShardedRegister.on_one_gpu(nqb, 4, p2.PREC_FP32,
                                            chunk=777,
                                            in_place=in_place) as reg:
        _load(reg, amp)
        reg.paulirot(flip, phase, phi)
        got = reg.get_state()
        assert abs(reg.norm2() - 1.0) < 1e-5
    assert np.max(np.abs(got - want)) < 1e-5


@pytest.mark.parametrize("prec", [p2.PREC_FP64, p2.PREC_FP32])
def test_slab_get_put_roundtrip(prec):
    nqb = 11
    amp = _start_state(nqb, 47)
    L = lib()
    with Register(nqb, prec) as r:
        r.set_state(amp)
        fp64 = r.precision == p2.PREC_FP64
        dt = torch.float64 if fp64 else torch.float32
        cdt = np.complex128 if fp64 else np.complex64
        cur = amp.astype(cdt)
        # even offsets and counts take the 16-byte path of FP32 halves
        # with bit >= 1; odd ones and bit 0 the per-amplitude path
        for bit in (0, 1, 3, nqb - 1):
            for val in (0, 1):
                for a, n in ((100, 300), (101, 299)):
                    half = cur.reshape(-1, 2, 1 << bit)[:, val, :]
                    half = half.reshape(-1)
                    buf = torch.empty(2 * n, dtype=dt, device="cuda")
                    assert L.qreg_slab_get(C.byref(r.reg), bit, val, a, n,
                                           C.c_void_p(buf.data_ptr())) == 0
                    got = buf.cpu().numpy().view(cdt)
                    assert np.array_equal(got, half[a:a + n])
                    new = (got * 1j).astype(cdt)
                    buf.copy_(torch.from_numpy(new.view(
                        np.float64 if fp64 else np.float32)).cuda())
                    assert L.qreg_slab_put(C.byref(r.reg), bit, val, a, n,
                                           C.c_void_p(buf.data_ptr())) == 0
                    v = cur.reshape(-1, 2, 1 << bit)[:, val, :]
                    flat = v.reshape(-1).copy()
                    flat[a:a + n] = new
                    v[...] = flat.reshape(v.shape)
                st = r.get_state()
                assert np.array_equal(st.astype(cdt), cur)


def test_slab_errors_copy_nothing():
    nqb = 22
    L = lib()
    with Register(nqb, p2.PREC_FP64) as r:
        r.set_state(np.zeros(1 << nqb, dtype=np.complex128))
        reg = C.byref(r.reg)
        small = torch.zeros(32, dtype=torch.float64, device="cuda")
        host = np.zeros(32, dtype=np.float64)
        p = C.c_void_p(small.data_ptr())
        # host pointer, misaligned pointer, bad bit / value / range
        assert L.qreg_slab_get(reg, 0, 0, 0, 16,
                               C.c_void_p(host.ctypes.data)) == -1
        assert L.qreg_slab_get(reg, 0, 0, 0, 8,
                               C.c_void_p(small.data_ptr() + 8)) == -1
        assert L.qreg_slab_get(reg, nqb, 0, 0, 16, p) == -1
        assert L.qreg_slab_get(reg, 0, 2, 0, 16, p) == -1
        assert L.qreg_slab_get(reg, 0, 0, 1 << (nqb - 1), 1, p) == -1
        # 2^21 complex128 = 32 MiB against a buffer in a 2 MiB segment
        assert L.qreg_slab_put(reg, 0, 0, 0, 1 << (nqb - 1), p) == -1
        assert L.qreg_slab_get(reg, 0, 0, 0, 0, None) == 0
        assert r.norm2() == 0.0
        torch.cuda.synchronize()
        assert torch.count_nonzero(small).item() == 0


@pytest.mark.parametrize("prec", [p2.PREC_FP64, p2.PREC_FP32])
def test_slab_swap_in_place(prec):
    nqb = 10
    x, y = _start_state(nqb, 48), _start_state(nqb, 49)
    L = lib()
    with Register(nqb, prec) as a, Register(nqb, prec) as b:
        cdt = np.complex128 if a.precision == p2.PREC_FP64 else np.complex64
        xa, yb = x.astype(cdt), y.astype(cdt)
        a.set_state(x)
        b.set_state(y)
        for bit, va, vb in ((0, 1, 0), (1, 0, 1), (4, 1, 1), (nqb - 1, 0, 0)):
            assert L.qreg_slab_swap(C.byref(a.reg), C.byref(b.reg), bit,
                                    va, vb) == 0
            hx = xa.reshape(-1, 2, 1 << bit)[:, va, :]
            hy = yb.reshape(-1, 2, 1 << bit)[:, vb, :]
            t = hx.copy()
            hx[...] = hy
            hy[...] = t
            assert np.array_equal(a.get_state().astype(cdt), xa)
            assert np.array_equal(b.get_state().astype(cdt), yb)


def test_slab_swap_errors():
    L = lib()
    with Register(8, p2.PREC_FP64) as a, Register(9, p2.PREC_FP64) as b, \
            Register(8, p2.PREC_FP32) as c:
        a.set_state(_start_state(8, 50))
        before = a.get_state()
        assert L.qreg_slab_swap(C.byref(a.reg), C.byref(a.reg), 0, 0, 1) == -1
        assert L.qreg_slab_swap(C.byref(a.reg), C.byref(b.reg), 0, 0, 1) == -1
        assert L.qreg_slab_swap(C.byref(a.reg), C.byref(c.reg), 0, 0, 1) == -1
        assert L.qreg_slab_swap(C.byref(a.reg), C.byref(a.reg), 8, 0, 1) == -1
        assert np.array_equal(a.get_state(), before)
