"""phase2_norm2_noalloc: the reduction for callers that cannot allocate.

Some callers cannot call cudaMalloc (their device memory belongs to their
own pool, or they cannot take the synchronisation an allocation implies),
so the library offers one entry point that keeps its scratch in a fixed
static device array.  This test calls it through the C-ABI on device
states held by the test, several times in a row on different sizes, and
checks every sum against an independent FP64 sum of the host array
(math.fsum of |z|^2, correctly rounded) and, for register-sized states,
against the allocating entry point qreg_norm2 on the same state
(tolerance 1e-12 relative, the FP64 tolerance of the other GPU tests).
It sorts last so that a run stopping at the first failure has already
run every other test; it also passes alone in a fresh process.
"""

import ctypes as C
import math

import numpy as np
import pytest

import phase2_b200 as p2
from phase2_b200._ffi import lib

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _fn():
    fn = lib().phase2_norm2_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_void_p, C.c_void_p]
    return fn


def _noalloc(fn, d_state, prec, namp, d_out, stream) -> int:
    return fn(C.c_void_p(d_state), prec, C.c_uint64(namp), C.c_void_p(d_out),
              C.c_void_p(stream))


def _fsum_norm(host: np.ndarray) -> float:
    return math.fsum((host.real * host.real + host.imag * host.imag).tolist())


def _register_norm(host: np.ndarray, prec: int) -> float:
    nqb = int(np.log2(len(host)))
    with p2.Register(nqb, prec) as r:
        r.set_state(host)
        return r.norm2()


def test_norm2_noalloc_matches_independent_sums():
    import torch

    p2.world_ensure()
    fn = _fn()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.Generator(np.random.PCG64(0x5C7A))
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    # calls in a row on the same static array: a large FP64 state, a small
    # FP32 one that uses fewer slots, and an FP32 state of a size that is
    # not a power of two, spread over many blocks
    for namp, prec in ((1 << 23, p2.PREC_FP64), (1 << 11, p2.PREC_FP32),
                       (3 * (1 << 21) + 12345, p2.PREC_FP32)):
        host = rng.standard_normal(namp) + 1j * rng.standard_normal(namp)
        if prec == p2.PREC_FP32:
            host = host.astype(np.complex64).astype(np.complex128)
            dev = torch.from_numpy(host.astype(np.complex64)).cuda()
        else:
            dev = torch.from_numpy(host).cuda()
        torch.cuda.synchronize()
        rc = _noalloc(fn, dev.data_ptr(), prec, namp, out.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        want = _fsum_norm(host)
        assert abs(got[0] - want) <= TOL * want, (namp, got[0], want)
        assert got[1] == 0.0
        if namp & (namp - 1) == 0:
            reg = _register_norm(host, prec)
            assert abs(got[0] - reg) <= TOL * reg, (namp, got[0], reg)


def test_norm2_noalloc_rejects_bad_inputs():
    import torch

    p2.world_ensure()
    fn = _fn()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    dev = torch.zeros(4, dtype=torch.complex128, device="cuda")
    # sizes and pointers are checked before anything is launched
    assert _noalloc(fn, dev.data_ptr(), 0, (1 << 34) + 1, out.data_ptr(),
                    0) == -1
    assert _noalloc(fn, dev.data_ptr(), 0, 0, out.data_ptr(), 0) == -1
    assert _noalloc(fn, dev.data_ptr(), 9, 4, out.data_ptr(), 0) == -1
    # a host pointer, and a buffer far shorter than namp amplitudes
    host = np.zeros(8, dtype=np.complex128)
    assert _noalloc(fn, host.ctypes.data, 0, 4, out.data_ptr(), 0) == -1
    assert _noalloc(fn, dev.data_ptr(), 0, 1 << 22, out.data_ptr(), 0) == -1
    assert _noalloc(fn, dev.data_ptr(), 0, 4, host.ctypes.data, 0) == -1
    # the entry point still works after the refusals
    assert _noalloc(fn, dev.data_ptr(), 0, 4, out.data_ptr(), 0) == 0
    torch.cuda.synchronize()
    assert out.cpu().numpy()[0] == 0.0
