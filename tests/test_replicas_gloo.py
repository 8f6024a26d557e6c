"""Multi-rank host logic on CPU: two gloo ranks shard a qDRIFT run.

Each rank takes a contiguous block of samples and advances the library's
xoshiro256** stream past the draws of the samples before its block; the
sampled term sequences of both ranks, gathered with torch.distributed,
must equal the single-process run's sequence (oracle) exactly.  Only the
host-side generator and CDF are exercised, so no GPU is needed.
"""

import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from phase2_b200 import _ffi, replicas, workloads
from phase2_b200._ffi import lib

SAMPLES, DEPTH, SEED = 7, 33, 0x5EED7


def _draw_block(terms, start, count):
    """Draw `count` samples from the stream positioned at sample `start`,
    using the library's CDF and generator as qdrift_simul does."""
    L = lib()
    cf = np.ascontiguousarray(terms.cf)
    cdf = _ffi.ProbCdf()
    assert L.prob_cdf_init(C.byref(cdf), len(cf)) == 0
    L.prob_cdf_from_array_strided(
        C.byref(cdf), cf.ctypes.data_as(C.POINTER(C.c_double)), 8, None)
    st = replicas.qdrift_stream_state(SEED, DEPTH, start)
    out = []
    for _ in range(count * DEPTH):
        x = (L.xoshiro256ss_next(C.byref(st)) >> 11) * 2.0 ** -53
        k = L.prob_cdf_inverse(C.byref(cdf), x)
        out.append((int(terms.flip[k]), int(terms.phase[k]),
                    float(np.sign(terms.cf[k]))))
    L.prob_cdf_free(C.byref(cdf))
    return out


def _rank_main(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        terms = workloads.jw_terms(12, 90, seed=3)
        start, count = replicas.shard(SAMPLES, rank, world)
        mine = _draw_block(terms, start, count)
        blocks = [None] * world
        dist.all_gather_object(blocks, (start, mine))
        if rank == 0:
            seq = []
            for _, b in sorted(blocks, key=lambda b: b[0]):
                seq.extend(b)
            q.put(seq)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_covers_all():
    for total in (0, 1, 7, 64):
        for world in (1, 2, 3, 8):
            blocks = [replicas.shard(total, r, world) for r in range(world)]
            assert sum(c for _, c in blocks) == total
            pos = 0
            for s, c in blocks:
                assert s == pos
                pos += c
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def test_two_gloo_ranks_reproduce_single_stream(oracle_lib):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q))
             for r in range(2)]
    for p in procs:
        p.start()
    seq = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    terms = workloads.jw_terms(12, 90, seed=3)
    want = oracle_lib.qdrift_draws(terms.flip, terms.phase, terms.cf,
                                   SAMPLES, DEPTH, SEED)
    assert len(seq) == len(want)
    for (f, p, s), w in zip(seq, want):
        assert (f, p, s) == (int(w["flip"]), int(w["phase"]), float(w["cf"]))
