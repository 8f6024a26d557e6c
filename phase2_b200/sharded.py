"""Registers sharded by high qubits, with qubit-swap exchange.

A register of nqb qubits over W = 2^g ranks keeps L = nqb - g qubits on
each rank: rank r holds the 2^L amplitudes whose physical index has r in
its g high bits (the reference's layout, phase2/qreg.c:46-66: qb_lo local
qubits, qb_hi = log2(ranks)).

The reference applies a rotation whose flip touches a high qubit by
exchanging the whole slab with the partner rank (rank ^ flip_hi), mixing,
rotating both copies and adding (phase2/qreg.c:124-142,
phase2/qreg_qreg.c:123-166): two slabs of traffic per flush that touches a
high qubit, every time.  Here a high qubit is made local instead: a
physical high position h (rank bit b = h - L) trades places with a local
position l, which moves half of every slab across the pair (rank,
rank ^ 2^b) once; the qubit then stays local for every later rotation
until it is swapped out again.  Global qubit q sits at physical position
pos[q]; the layout is the same on every rank, since every rank takes the
same swap decisions from the same rotation sequence.

After the swaps a rotation's flip lies in the local positions.  A Z on a
high position then contributes the fixed sign (-1)^popc(rank & z_hi) to
P on this rank's slab (r4 = popc(flip & ph) + 2 popc(i & ph) mod 4,
include/phase2/paulis.h:137-144), so the rank applies exp(i sigma phi
P_lo) to its slab with the ordinary engine.  cos(-phi) = cos(phi) and
sin(-phi) = -sin(phi) exactly, and every amplitude's update reads the same
pair with the same phases, so an FP64 sharded register gives the same bits
as one register of nqb qubits.

Which local position trades places: among those outside the rotation's
flip, the one whose qubit the rotation sequence flips again farthest ahead
(or never, within the look-ahead window): Belady's choice, since the
register sees the whole sequence it is given.  On random qDRIFT draws
every qubit is flipped by about one draw in eight, so a
least-recently-used choice swaps at nearly every draw that reaches the
high qubit, while the farthest next use is some tens of draws away.

Each rank moves its outgoing half in chunks: qreg_slab_get gathers a chunk
into a device buffer, the transport exchanges it with the partner (NCCL
send/recv through torch.distributed between GPUs; gloo on CPU), and
qreg_slab_put scatters the received chunk into the same places.  Two send
buffers alternate: chunk k+1 is gathered while chunk k is in flight, and
chunk k is scattered after that, so between GPUs the HBM gather and
scatter hide behind the NVLink transfer.  When both ranks of a pair live
in this process on one GPU, qreg_slab_swap trades the two halves in place
instead (one read and one write of each, no buffers).  One
process may also hold several ranks (LocalTransport): their exchange is a
hand-over of buffers, which runs a sharded register on one GPU.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import PREC_FP64, Dets, Register, Terms, _ffi, _hamil, world_ensure
from ._ffi import lib

#: default exchange chunk, in amplitudes (1 GiB of FP64 per buffer)
CHUNK = 1 << 26

_WINDOW = 4096     # rotations mapped to physical positions at a time
_LOOKAHEAD = 4096  # rotations searched for the next use of a local qubit


def _log2_exact(w: int) -> int:
    g = w.bit_length() - 1
    if w <= 0 or (1 << g) != w:
        raise ValueError(f"world size {w} is not a power of two")
    return g


def _popcount(a: np.ndarray) -> np.ndarray:
    return np.bitwise_count(a)


def _swap_bits(m: np.ndarray, a: int, b: int) -> None:
    """Exchange bit positions a and b of every mask in m, in place."""
    one = np.uint64(1)
    x = ((m >> np.uint64(a)) ^ (m >> np.uint64(b))) & one
    m ^= (x << np.uint64(a)) | (x << np.uint64(b))


class Layout:
    """Global qubit <-> physical position map of a sharded register."""

    def __init__(self, nqb: int, nlocal: int):
        self.nqb, self.nlocal = nqb, nlocal
        self.pos = list(range(nqb))  # global qubit -> physical position
        self.at = list(range(nqb))   # physical position -> global qubit

    def identity(self) -> bool:
        return all(p == q for q, p in enumerate(self.pos))

    def swap(self, a: int, b: int) -> None:
        """Exchange the qubits at physical positions a and b."""
        qa, qb = self.at[a], self.at[b]
        self.at[a], self.at[b] = qb, qa
        self.pos[qa], self.pos[qb] = b, a

    def phys(self, masks) -> np.ndarray:
        """Bit masks over global qubits -> masks over physical positions."""
        m = np.ascontiguousarray(masks, dtype=np.uint64)
        if self.identity():
            return m.copy()
        out = np.zeros_like(m)
        one = np.uint64(1)
        for q, p in enumerate(self.pos):
            out |= ((m >> np.uint64(q)) & one) << np.uint64(p)
        return out

    def glob(self, masks) -> np.ndarray:
        """Physical masks (indices) -> global masks (indices)."""
        m = np.ascontiguousarray(masks, dtype=np.uint64)
        if self.identity():
            return m.copy()
        out = np.zeros_like(m)
        one = np.uint64(1)
        for q, p in enumerate(self.pos):
            out |= ((m >> np.uint64(p)) & one) << np.uint64(q)
        return out


# ---- slabs: one rank's local register ---------------------------------


class CudaSlab:
    """One rank's 2^L amplitudes in a device register of this library."""

    def __init__(self, nlocal: int, prec: int | None = None):
        import torch
        self.reg = Register(nlocal, prec)
        self.nqb = nlocal
        self._L = lib()
        fp64 = self.reg.precision == PREC_FP64
        self.dtype = torch.float64 if fp64 else torch.float32
        self.device = torch.device("cuda", torch.cuda.current_device())

    def close(self) -> None:
        self.reg.close()

    def buffer(self, count: int):
        import torch
        return torch.empty(2 * count, dtype=self.dtype, device=self.device)

    def paulirot(self, flip, phase, phi) -> None:
        self.reg.paulirot(flip, phase, phi)

    def zero(self) -> None:
        self.reg.zero()

    def setamps(self, idx, z) -> None:
        self.reg.setamps(idx, z)

    def getamps(self, idx) -> np.ndarray:
        return self.reg.getamps(idx)

    def get_state(self) -> np.ndarray:
        return self.reg.get_state()

    def norm2(self) -> float:
        return self.reg.norm2()

    def synchronize(self) -> None:
        self.reg.synchronize()

    def slab_get(self, bit, val, first, count, buf) -> None:
        if self._L.qreg_slab_get(C.byref(self.reg.reg), bit, val, first,
                                 count, C.c_void_p(buf.data_ptr())):
            raise RuntimeError("qreg_slab_get failed")

    def slab_put(self, bit, val, first, count, buf) -> None:
        if self._L.qreg_slab_put(C.byref(self.reg.reg), bit, val, first,
                                 count, C.c_void_p(buf.data_ptr())):
            raise RuntimeError("qreg_slab_put failed")

    def swap_halves(self, other: "CudaSlab", bit, val, other_val) -> None:
        if self._L.qreg_slab_swap(C.byref(self.reg.reg),
                                  C.byref(other.reg.reg), bit, val,
                                  other_val):
            raise RuntimeError("qreg_slab_swap failed")


# ---- transports: how paired ranks trade their halves ------------------


class LocalTransport:
    """All ranks in this process: a half moves by handing over its buffer."""

    def post(self, sends: dict, mask: int):
        return {r: sends[r ^ mask] for r in sends}

    def wait(self, handle) -> dict:
        return handle

    def sum_over_ranks(self, v: np.ndarray, device=None) -> np.ndarray:
        return v


class DistTransport:
    """One rank per process over torch.distributed (NCCL between GPUs, gloo
    on CPU).  Every rank makes the same calls in the same order."""

    def __init__(self, group=None, device=None):
        import torch
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.device = torch.device("cpu") if device is None else device

    def _sync(self) -> None:
        if self.device.type == "cuda":
            import torch
            torch.cuda.synchronize(self.device)

    def post(self, sends: dict, mask: int):
        """Start the pair exchange of this rank's chunk."""
        import torch
        dist = self.dist
        (r, buf), = sends.items()
        partner = r ^ mask
        if self.group is not None:
            partner = dist.get_global_rank(self.group, partner)
        recv = torch.empty_like(buf)
        ops = [dist.P2POp(dist.isend, buf, partner, self.group),
               dist.P2POp(dist.irecv, recv, partner, self.group)]
        return r, recv, dist.batch_isend_irecv(ops)

    def wait(self, handle) -> dict:
        r, recv, reqs = handle
        for req in reqs:
            req.wait()
        self._sync()
        return {r: recv}

    def sum_over_ranks(self, v: np.ndarray, device=None) -> np.ndarray:
        import torch
        t = torch.from_numpy(np.ascontiguousarray(v).view(np.float64).copy())
        t = t.to(self.device)
        self.dist.all_reduce(t, group=self.group)
        self._sync()
        return t.cpu().numpy().view(np.complex128)


# ---- the sharded register ---------------------------------------------


class ShardedRegister:
    """nqb qubits over `world` ranks; this process holds the ranks in
    `slabs` (rank -> slab).  Rotations, state preparation and overlaps
    take global qubit indices."""

    def __init__(self, nqb: int, world: int, slabs: dict, transport,
                 chunk: int = CHUNK, in_place: bool = True):
        g = _log2_exact(world)
        if not slabs or any(not 0 <= r < world for r in slabs):
            raise ValueError("slab ranks outside the world")
        if nqb - g < 1:
            raise ValueError(f"{nqb} qubits over {world} ranks leaves no"
                             " local qubit")
        for s in slabs.values():
            if s.nqb != nqb - g:
                raise ValueError("slab size does not match the layout")
        if chunk < 1:
            raise ValueError("chunk must be positive")
        self.nqb, self.world, self.nlocal = nqb, world, nqb - g
        self.slabs, self.transport, self.chunk = dict(slabs), transport, chunk
        # pairs held by this process trade halves in place
        self.in_place = (in_place and isinstance(transport, LocalTransport)
                         and all(hasattr(s, "swap_halves")
                                 for s in self.slabs.values()))
        self.layout = Layout(nqb, self.nlocal)
        self.swaps = 0           # qubit swaps performed
        self.exchanged = 0       # amplitudes this process sent

    # -- construction
    @classmethod
    def on_one_gpu(cls, nqb: int, world: int, prec: int | None = None,
                   chunk: int = CHUNK,
                   in_place: bool = True) -> "ShardedRegister":
        """All `world` ranks in this process, on the current GPU."""
        world_ensure()
        g = _log2_exact(world)
        slabs = {r: CudaSlab(nqb - g, prec) for r in range(world)}
        return cls(nqb, world, slabs, LocalTransport(), chunk, in_place)

    @classmethod
    def distributed(cls, nqb: int, prec: int | None = None, group=None,
                    chunk: int = CHUNK) -> "ShardedRegister":
        """One rank per process (torch.distributed initialised, NCCL, with
        this process's GPU current)."""
        import torch
        import torch.distributed as dist
        world_ensure()
        world = dist.get_world_size(group)
        rank = dist.get_rank(group)
        g = _log2_exact(world)
        slab = CudaSlab(nqb - g, prec)
        dev = torch.device("cuda", torch.cuda.current_device())
        return cls(nqb, world, {rank: slab}, DistTransport(group, dev),
                   chunk)

    def close(self) -> None:
        for s in self.slabs.values():
            if hasattr(s, "close"):
                s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- rotations
    def paulirot(self, flip, phase, phi) -> None:
        """exp(+i phi_k P_k) for k in order; flip/phase over global
        qubits (struct paulis pak[0] / pak[1])."""
        flip = np.ascontiguousarray(flip, dtype=np.uint64)
        phase = np.ascontiguousarray(phase, dtype=np.uint64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        if not len(flip) == len(phase) == len(phi):
            raise ValueError("flip, phase and phi differ in length")
        if self.nqb < 64 and len(flip):
            top = np.uint64(self.nqb)
            if (flip >> top).any() or (phase >> top).any():
                raise ValueError("Pauli string acts beyond the register")
        L = np.uint64(self.nlocal)
        n, k = len(phi), 0
        while k < n:
            # map a window plus its look-ahead once; a swap then only
            # exchanges two bit positions of the mapped masks
            limit = min(n, k + _WINDOW) - k
            span = min(n, k + _WINDOW + _LOOKAHEAD)
            pf = self.layout.phys(flip[k:span])
            pp = self.layout.phys(phase[k:span])
            off = 0
            while off < limit:
                far = np.flatnonzero(pf[off:limit] >> L)
                stop = limit if len(far) == 0 else off + int(far[0])
                if stop > off:
                    self._apply_local(pf[off:stop], pp[off:stop],
                                      phi[k + off:k + stop])
                if stop < limit:
                    ahead = pf[stop + 1:stop + 1 + _LOOKAHEAD]
                    for h, l in self._make_local(int(pf[stop]), ahead):
                        _swap_bits(pf[stop:], h, l)
                        _swap_bits(pp[stop:], h, l)
                off = stop
            k += limit

    def _apply_local(self, pf, pp, phi) -> None:
        L = np.uint64(self.nlocal)
        lo = np.uint64((1 << self.nlocal) - 1)
        z_hi = pp >> L
        for r, slab in self.slabs.items():
            odd = _popcount(z_hi & np.uint64(r)) & 1
            slab.paulirot(pf, pp & lo, np.where(odd == 1, -phi, phi))

    def _make_local(self, pflip: int, ahead: np.ndarray) -> list:
        """Swap every high position of pflip with a local one outside it;
        `ahead` holds the physical flips of the rotations that follow.
        Returns the (high, local) position pairs swapped, in order."""
        L = self.nlocal
        need = [h for h in range(L, self.nqb) if pflip >> h & 1]
        taken = {p for p in range(L) if pflip >> p & 1}
        # first use of each position ahead: where the running OR of the
        # flips gains that bit
        first = {}
        if len(ahead):
            cum = np.bitwise_or.accumulate(ahead)
            gain = cum.copy()
            gain[1:] ^= cum[:-1]
            for i in np.flatnonzero(gain):
                g = int(gain[i])
                while g:
                    p = (g & -g).bit_length() - 1
                    first[p] = int(i)
                    g &= g - 1
        nxt = {p: first.get(p, len(ahead)) for p in range(L)
               if p not in taken}
        done = []
        for h in need:
            free = [p for p in nxt if p not in taken]
            if not free:
                raise ValueError(
                    f"a flip over {bin(pflip).count('1')} qubits does not"
                    f" fit the {L} local qubits of each rank")
            l = max(free, key=lambda p: (nxt[p], p))
            self._swap(h, l)
            taken.add(l)
            done.append((h, l))
        return done

    def _swap(self, h: int, l: int) -> None:
        """Trade the qubits at high position h and local position l: every
        rank swaps the half of its slab with bit l != its rank bit b with
        the partner rank ^ 2^b (double-buffered chunks)."""
        b = h - self.nlocal
        mask = 1 << b
        nhalf = 1 << (self.nlocal - 1)
        val = {r: 1 - (r >> b & 1) for r in self.slabs}
        if self.in_place:
            for r, slab in self.slabs.items():
                if r < r ^ mask:
                    slab.swap_halves(self.slabs[r ^ mask], l, val[r],
                                     val[r ^ mask])
            self.exchanged += nhalf * len(self.slabs)
            self.layout.swap(h, l)
            self.swaps += 1
            return
        count0 = min(self.chunk, nhalf)
        bufs = [{r: s.buffer(count0) for r, s in self.slabs.items()}, None]
        pending = None
        for k, first in enumerate(range(0, nhalf, self.chunk)):
            count = min(self.chunk, nhalf - first)
            if bufs[k & 1] is None:
                bufs[k & 1] = {r: s.buffer(count0)
                               for r, s in self.slabs.items()}
            sends = {}
            for r, slab in self.slabs.items():
                buf = bufs[k & 1][r][:2 * count]
                slab.slab_get(l, val[r], first, count, buf)
                sends[r] = buf
            posted = (first, count, self.transport.post(sends, mask))
            if pending is not None:
                self._land(l, val, *pending)
            pending = posted
        self._land(l, val, *pending)
        self.layout.swap(h, l)
        self.swaps += 1

    def _land(self, l, val, first, count, handle) -> None:
        recvs = self.transport.wait(handle)
        for r, slab in self.slabs.items():
            slab.slab_put(l, val[r], first, count, recvs[r])
        self.exchanged += count * len(self.slabs)

    # -- state preparation and overlaps (multidet, phase2/circ.c:215-224,
    #    338-350)
    def _owners(self, idx):
        p = self.layout.phys(idx)
        L = np.uint64(self.nlocal)
        return p >> L, p & np.uint64((1 << self.nlocal) - 1)

    def prepst(self, dets: Dets) -> None:
        owner, local = self._owners(dets.idx)
        cf = np.ascontiguousarray(dets.cf, dtype=np.complex128)
        for r, slab in self.slabs.items():
            slab.zero()
            sel = owner == np.uint64(r)
            if sel.any():
                slab.setamps(local[sel], cf[sel])

    def getamps(self, idx) -> np.ndarray:
        """Amplitudes at global indices, on every rank."""
        owner, local = self._owners(idx)
        out = np.zeros(len(owner), dtype=np.complex128)
        for r, slab in self.slabs.items():
            sel = owner == np.uint64(r)
            if sel.any():
                out[sel] = slab.getamps(local[sel])
        return self.transport.sum_over_ranks(out)

    def measure(self, dets: Dets) -> complex:
        """sum_d conj(cf_d) a[idx_d], summed in det order."""
        a = self.getamps(dets.idx)
        pr = pi = 0.0
        for ad, cd in zip(a, np.asarray(dets.cf, dtype=np.complex128)):
            ar, ai = float(ad.real), float(ad.imag)
            cr, ci = float(cd.real), -float(cd.imag)
            pr += ar * cr - ai * ci
            pi += ar * ci + ai * cr
        return complex(pr, pi)

    def get_state(self) -> np.ndarray:
        """The whole state in global index order, on every rank (small
        registers: every rank receives 2^nqb amplitudes)."""
        full = np.zeros(1 << self.nqb, dtype=np.complex128)
        k = np.arange(1 << self.nlocal, dtype=np.uint64)
        for r, slab in self.slabs.items():
            phys = (np.uint64(r) << np.uint64(self.nlocal)) | k
            full[self.layout.glob(phys)] = slab.get_state()
        return self.transport.sum_over_ranks(full)

    def norm2(self) -> float:
        """sum |a_i|^2 over all ranks: each rank's device reduction
        (qreg_norm2), then the ranks' sums added in rank order."""
        part = np.zeros(self.world, dtype=np.complex128)
        for r, slab in self.slabs.items():
            part[r] = slab.norm2()
        part = self.transport.sum_over_ranks(part)
        tot = 0.0
        for v in part.real:
            tot += float(v)
        return tot

    def synchronize(self) -> None:
        for s in self.slabs.values():
            s.synchronize()


# ---- drivers ----------------------------------------------------------


def sort_lex(nqb: int, terms: Terms) -> Terms:
    """terms in the order circ_hamil_sort_lex gives them (the library's
    sort, phase2/circ.c:60-81)."""
    L = lib()
    hm = _hamil(nqb, terms)
    try:
        L.circ_hamil_sort_lex(C.byref(hm))
        n = int(hm.len)
        rec = np.zeros(n, dtype=[("cf", "<f8"), ("flip", "<u8"),
                                 ("phase", "<u8")])
        if n:
            C.memmove(rec.ctypes.data, hm.terms, rec.nbytes)
    finally:
        L.circ_hamil_free(C.byref(hm))
    return Terms(rec["flip"].copy(), rec["phase"].copy(), rec["cf"].copy())


def trott(reg: ShardedRegister, terms: Terms, dets: Dets, steps: int,
          delta: float, order2: bool = False,
          sort: bool = True) -> np.ndarray:
    """trott_simul / trott2_simul on a sharded register (circ/trott.c:44-65,
    circ/trott2.c:44-74): one overlap per step."""
    t = sort_lex(reg.nqb, terms) if sort else terms
    reg.prepst(dets)
    out = np.zeros(steps, dtype=np.complex128)
    if order2:
        half = delta / 2.0
        fwd = t.cf * half
        rev = (t.flip[::-1], t.phase[::-1], t.cf[::-1] * half)
    else:
        fwd = t.cf * delta
    for s in range(steps):
        reg.paulirot(t.flip, t.phase, fwd)
        if order2:
            reg.paulirot(*rev)
        out[s] = reg.measure(dets)
    return out


def _sign_dz(a: np.ndarray) -> np.ndarray:
    """|a| < DBL_EPSILON -> 0, else -1 or +1 (circ/internal.h:26-32)."""
    f = np.abs(a)
    return np.where(f < np.finfo(np.float64).eps, 0.0,
                    np.where(a < f, -1.0, 1.0))


def qdrift(reg: ShardedRegister, terms: Terms, dets: Dets, samples: int,
           depth: int, step_size: float, seed: int) -> np.ndarray:
    """qdrift_simul on a sharded register (circ/qdrift.c:95-134): per
    sample, state preparation, `depth` draws from the |c| CDF with the
    library's prob_cdf and xoshiro256** (the draws of qdrift_simul for the
    same seed), rotations at asin(step_size) sign_dz(c), one overlap.
    Every rank draws the same sequence.  seed must be non-zero: the
    library's qdrift replaces 0 by the last non-zero seed it was given,
    which is process state."""
    if seed == 0:
        raise ValueError("seed must be non-zero")
    if len(terms) == 0 or depth < 0 or samples < 0:
        raise ValueError("no terms, or a negative depth or sample count")
    L = lib()
    cf = np.ascontiguousarray(terms.cf, dtype=np.float64)
    cdf = _ffi.ProbCdf()
    if L.prob_cdf_init(C.byref(cdf), len(cf)) != 0:
        raise MemoryError("prob_cdf_init")
    out = np.zeros(samples, dtype=np.complex128)
    try:
        L.prob_cdf_from_array_strided(
            C.byref(cdf), cf.ctypes.data_as(C.POINTER(C.c_double)), 8,
            None)
        rng = _ffi.Xoshiro()
        L.xoshiro256ss_init(C.byref(rng), seed)
        omega = math.asin(step_size)
        k = np.empty(depth, dtype=np.int64)
        for s in range(samples):
            reg.prepst(dets)
            for i in range(depth):
                x = (L.xoshiro256ss_next(C.byref(rng)) >> 11) * 2.0 ** -53
                k[i] = L.prob_cdf_inverse(C.byref(cdf), x)
            reg.paulirot(terms.flip[k], terms.phase[k],
                         omega * _sign_dz(cf[k]))
            out[s] = reg.measure(dets)
    finally:
        L.prob_cdf_free(C.byref(cdf))
    return out


def _hamil_terms(hm) -> Terms:
    n = int(hm.len)
    rec = np.zeros(n, dtype=[("cf", "<f8"), ("flip", "<u8"),
                             ("phase", "<u8")])
    if n:
        C.memmove(rec.ctypes.data, hm.terms, rec.nbytes)
    return Terms(rec["flip"].copy(), rec["phase"].copy(), rec["cf"].copy())


def cmpsit(reg: ShardedRegister, terms: Terms, dets: Dets, samples: int,
           steps: int, length: int, depth: int, angle_det: float,
           angle_rand: float, seed: int) -> np.ndarray:
    """cmpsit_simul on a sharded register (circ/cmpsit.c:151-235): the
    library's own split (cmpsit_ranct_init: the `length` largest |c| as
    the deterministic head at c angle_det, the rest sampled through its
    |c| CDF at sign_dz(c) angle_rand); per sample, state preparation, then
    per step a fresh sample applied forward at 0.5 and another applied in
    reverse at 0.5; one overlap per sample.  seed must be non-zero (see
    qdrift)."""
    if seed == 0:
        raise ValueError("seed must be non-zero")
    L = lib()
    hm = _hamil(reg.nqb, terms)
    rc = _ffi.CmpsitRanct()
    dt = _ffi.CmpsitData(samples, steps, length, depth, angle_det,
                         angle_rand, seed)
    out = np.zeros(samples, dtype=np.complex128)
    try:
        if L.cmpsit_ranct_init(C.byref(rc), C.byref(hm), C.byref(dt)):
            raise ValueError("cmpsit split failed (length >= terms?)")
        det = _hamil_terms(rc.hm_det)
        ran = _hamil_terms(rc.hm_ran)
        det_phi = det.cf * angle_det
        rng = _ffi.Xoshiro()
        L.xoshiro256ss_init(C.byref(rng), seed)
        k = np.empty(depth, dtype=np.int64)

        def sample():
            for i in range(depth):
                x = (L.xoshiro256ss_next(C.byref(rng)) >> 11) * 2.0 ** -53
                k[i] = L.prob_cdf_inverse(C.byref(rc.cdf), x)
            return (np.concatenate([det.flip, ran.flip[k]]),
                    np.concatenate([det.phase, ran.phase[k]]),
                    np.concatenate([det_phi,
                                    _sign_dz(ran.cf[k]) * angle_rand]))

        for s in range(samples):
            reg.prepst(dets)
            for _ in range(steps):
                f, p, c = sample()
                reg.paulirot(f, p, 0.5 * c)
                f, p, c = sample()
                reg.paulirot(f[::-1], p[::-1], 0.5 * c[::-1])
            out[s] = reg.measure(dets)
    finally:
        L.cmpsit_ranct_free(C.byref(rc))
        L.circ_hamil_free(C.byref(hm))
    return out
