"""phase2_norm2_noalloc: the reduction for callers that cannot allocate.

Some callers cannot call cudaMalloc (their device memory belongs to their
own pool, or they cannot take the synchronisation an allocation implies),
so the library offers one entry point that keeps its scratch in a fixed
static device array.  This test calls it through the C-ABI on device
states held by the test, twice in a row on different sizes, and checks
both sums against the allocating entry point qreg_norm2 on the same state
(tolerance 1e-12 relative, the FP64 tolerance of the other GPU tests).
It sorts last so that a run stopping at the first failure has already
run every other test; it also passes alone in a fresh process.
"""

import ctypes as C

import numpy as np
import pytest

import phase2_b200 as p2
from phase2_b200._ffi import lib

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _noalloc(fn, d_state, prec, namp, d_out, stream) -> int:
    return fn(C.c_void_p(d_state), prec, C.c_uint64(namp), C.c_void_p(d_out),
              C.c_void_p(stream))


def _reference_norm(host: np.ndarray, prec: int) -> float:
    nqb = int(np.log2(len(host)))
    with p2.Register(nqb, prec) as r:
        r.set_state(host)
        return r.norm2()


def test_norm2_noalloc_matches_qreg_norm2():
    import torch

    p2.world_ensure()
    fn = lib().phase2_norm2_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_void_p, C.c_void_p]
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.Generator(np.random.PCG64(0x5C7A))
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    # two calls in a row: a large state (many partial sums), then a small
    # one that reuses fewer slots of the same static array
    for nqb, prec in ((23, p2.PREC_FP64), (11, p2.PREC_FP32)):
        host = (rng.standard_normal(1 << nqb) +
                1j * rng.standard_normal(1 << nqb))
        if prec == p2.PREC_FP32:
            host = host.astype(np.complex64).astype(np.complex128)
            dev = torch.from_numpy(host.astype(np.complex64)).cuda()
        else:
            dev = torch.from_numpy(host).cuda()
        torch.cuda.synchronize()
        rc = _noalloc(fn, dev.data_ptr(), prec, 1 << nqb, out.data_ptr(),
                      stream)
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        want = _reference_norm(host, prec)
        assert abs(got[0] - want) <= TOL * want, (nqb, got[0], want)
        assert got[1] == 0.0


def test_norm2_noalloc_rejects_oversize():
    import torch

    p2.world_ensure()
    fn = lib().phase2_norm2_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_void_p, C.c_void_p]
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    dev = torch.zeros(4, dtype=torch.complex128, device="cuda")
    # sizes are checked before anything is launched
    assert _noalloc(fn, dev.data_ptr(), 0, (1 << 34) + 1, out.data_ptr(),
                    0) == -1
    assert _noalloc(fn, dev.data_ptr(), 0, 0, out.data_ptr(), 0) == -1
    assert _noalloc(fn, dev.data_ptr(), 9, 4, out.data_ptr(), 0) == -1
