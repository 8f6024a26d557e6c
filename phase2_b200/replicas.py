"""Multi-GPU execution by replicas: one process per GPU, no data-path
collective.

qDRIFT (and composite) samples are independent, so a run of S samples is
split into contiguous blocks, one per rank.  Rank r draws from the same
xoshiro256** stream as a single-process run would, advanced past the draws
of the samples before its block, so the union of all ranks' samples is
exactly the single-process run's sample sequence.  Results are gathered
with torch.distributed (gloo or nccl) only at the end.
"""

from __future__ import annotations

import ctypes as C

from . import _ffi
from ._ffi import lib


def shard(total: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous block of `total` items for `rank`: (start, count)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def skip_draws(rng: _ffi.Xoshiro, n: int) -> None:
    """Advance an xoshiro256** state by n draws (the stream position a
    single-process run reaches after n draws)."""
    L = lib()
    for _ in range(n):
        L.xoshiro256ss_next(C.byref(rng))


def qdrift_stream_state(seed: int, depth: int, start: int) -> _ffi.Xoshiro:
    """Generator state at the first draw of sample `start` (each qDRIFT
    sample consumes `depth` draws, circ/qdrift.c:95-103)."""
    st = _ffi.Xoshiro()
    lib().xoshiro256ss_init(C.byref(st), seed)
    skip_draws(st, start * depth)
    return st


def qdrift_local(nqb, terms, dets, samples, depth, step_size, seed, rank,
                 world):
    """This rank's block of a sharded qDRIFT run, as overlaps (complex)."""
    import numpy as np

    from . import _hamil, _muldet, _values, world_ensure
    start, count = shard(samples, rank, world)
    if count == 0:
        return start, np.zeros(0, dtype=np.complex128)
    world_ensure()
    L = lib()
    obj = _ffi.Qdrift()
    dt = _ffi.QdriftData(count, depth, step_size, seed)
    if L.qdrift_init(C.byref(obj), C.byref(dt), _hamil(nqb, terms),
                     _ffi.STPREP_MULTIDET,
                     C.cast(C.pointer(_muldet(dets)), C.c_void_p),
                     None) != 0:
        raise RuntimeError("qdrift_init failed")
    try:
        obj.rng = qdrift_stream_state(seed, depth, start)
        if L.qdrift_simul(C.byref(obj)) != 0:
            raise RuntimeError("qdrift_simul failed")
        return start, _values(obj.ct.vals)
    finally:
        L.qdrift_free(C.byref(obj))


def gather_blocks(start: int, values, world: int):
    """All ranks' (start, values) blocks concatenated in sample order."""
    import numpy as np
    import torch.distributed as dist
    blocks = [None] * world
    dist.all_gather_object(blocks, (start, list(values)))
    out = []
    for _, vals in sorted(blocks, key=lambda b: b[0]):
        out.extend(vals)
    return np.array(out, dtype=np.complex128)
