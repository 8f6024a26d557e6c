"""B200-native phase2 state-vector hot path (Python side).

``run`` is the drop-in for the phase2 Python entry point
(python/phase2/__init__.py:71-124 of Quantum-for-Life/phase2): same
arguments, same return type, same ``ValueError`` on bad input.  It calls
``phase2_run`` in this package's ``libphase2.so`` (sm_100a kernels).

The other helpers drive the library's C surface (register, circuit
drivers, planner) for tests and benchmarks.  All computation happens in
libphase2.so on the GPU; nothing here computes amplitudes.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _ffi
from ._ffi import lib

__all__ = ["run", "world_ensure", "Register", "Terms", "Dets", "trott",
           "trott2", "qdrift", "cmpsit", "plan", "set_precision",
           "set_fusion", "set_term_order", "PREC_FP64", "PREC_FP32"]

PREC_FP64 = _ffi.PREC_FP64
PREC_FP32 = _ffi.PREC_FP32
FORM_EXACT, FORM_LIFTED, FORM_LIFTED_F32, FORM_LIFTED_MIXED = 0, 1, 2, 3
_WORLD_SEED = 0x2B200C0DE5EED001


def world_ensure() -> None:
    """Initialise the library world (CUDA device) once; raise if no GPU."""
    L = lib()
    if L.world_info(None) == _ffi.WORLD_READY:
        return
    if L.world_init(None, None, _WORLD_SEED) != _ffi.WORLD_READY:
        raise RuntimeError("phase2 world_init failed (no usable CUDA "
                           "device?)")


def run(paulis: list[str], coeffs: list[float], delta: float,
        psi: str) -> complex:
    """<psi| prod_k exp(i*delta*coeffs[k]*P_k) |psi>, as phase2.run."""
    nterms = len(paulis)
    if nterms != len(coeffs):
        raise ValueError(f"len(paulis)={nterms} != len(coeffs)="
                         f"{len(coeffs)}")
    L = lib()
    c_paulis = (C.c_char_p * max(nterms, 1))(
        *(s.encode("ascii") for s in paulis))
    c_coeffs = (C.c_double * max(nterms, 1))(*coeffs)
    out_re, out_im = C.c_double(0.0), C.c_double(0.0)
    rc = L.phase2_run(c_paulis, c_coeffs, C.c_size_t(nterms),
                      C.c_double(delta), psi.encode("ascii"),
                      C.byref(out_re), C.byref(out_im))
    if rc == -1:
        raise ValueError("phase2_run returned -1: invalid input")
    return complex(out_re.value, out_im.value)


def set_precision(prec: int) -> None:
    if lib().phase2_set_precision(prec) != 0:
        raise ValueError(f"bad precision {prec}")


def set_fp32_form(form: int) -> None:
    """Arithmetic of FP32 passes: FORM_LIFTED_MIXED (default: FP32 FMAs,
    except cosets holding an amplitude >= 2^-10, which take FP64
    arithmetic and one rounding per pass; registers below 24 qubits FP64
    arithmetic throughout), FORM_LIFTED (coefficients from FP64 cos/sin,
    FP64 arithmetic, one rounding to FP32 per pass) or FORM_LIFTED_F32
    (FP32 FMAs on FP32 coefficients)."""
    if lib().phase2_set_fp32_form(form) != 0:
        raise ValueError(f"bad FP32 form {form}")


def get_fp32_form() -> int:
    return lib().phase2_get_fp32_form()


def set_batch_persistent(on: bool) -> None:
    """Batched drivers: one persistent launch for all instances (default)
    or per-instance streams."""
    lib().phase2_set_batch_persistent(1 if on else 0)


def set_batch_runs(per_warp: int) -> None:
    """Persistent launch run length: a warp claims what is left of an op
    times the programs running, over (resident warps x per_warp), tiles of
    1024 amplitudes, 1 to 16 (default 2; 1..64)."""
    if lib().phase2_set_batch_runs(per_warp) != 0:
        raise ValueError(f"batch runs per warp {per_warp} not in 1..64")


def set_sweep(tile_qubits: int, low_qubits: int = 5) -> None:
    """FP32 sweeps: plans group passes that fit a tile of 2^tile_qubits
    amplitudes (low_qubits of them the lowest qubits), and each group runs
    as one kernel, one read and one write of the state.  tile_qubits 0
    turns them off."""
    if lib().phase2_set_sweep(int(tile_qubits), int(low_qubits)) != 0:
        raise ValueError(f"bad sweep shape {tile_qubits}, {low_qubits}")


def get_sweep() -> tuple:
    a, b = C.c_int(), C.c_int()
    lib().phase2_get_sweep(C.byref(a), C.byref(b))
    return a.value, b.value


def set_sweep_kernel(on: bool) -> None:
    """False: keep the plans' sweep grouping but run one kernel per pass
    (same bits; for comparisons)."""
    lib().phase2_set_sweep_kernel(1 if on else 0)


DEVICE_SAMPLING_OFF, DEVICE_SAMPLING_ON, DEVICE_SAMPLING_AUTO = 0, 1, 2


def set_device_sampling(mode) -> None:
    """qdrift and cmpsit: draw, plan and run the samples on the GPU (same
    results as the host loop, bit for bit).  True/False force it on or
    off; DEVICE_SAMPLING_AUTO (default) uses it for registers of at most
    21 qubits."""
    mode = {True: 1, False: 0}.get(mode, mode)
    if lib().phase2_set_device_sampling(int(mode)) != 0:
        raise ValueError(f"bad device sampling mode {mode}")


def set_fusion(max_span: int, max_rots: int = 0) -> None:
    if lib().phase2_set_fusion(max_span, max_rots) != 0:
        raise ValueError("bad fusion setting")


def set_term_order(order: int) -> None:
    if lib().phase2_set_term_order(order) != 0:
        raise ValueError("bad term order")


# ---- inputs ------------------------------------------------------------


@dataclass
class Terms:
    """Hamiltonian terms: flip/phase masks (uint64) and real coefficients."""
    flip: np.ndarray
    phase: np.ndarray
    cf: np.ndarray

    def __len__(self) -> int:
        return len(self.cf)

    def records(self) -> np.ndarray:
        """24-byte records laid out as struct circ_hamil_term."""
        rec = np.zeros(len(self), dtype=[("cf", "<f8"), ("flip", "<u8"),
                                         ("phase", "<u8")])
        rec["cf"], rec["flip"], rec["phase"] = self.cf, self.flip, self.phase
        return rec


@dataclass
class Dets:
    """Initial state sum_d cf_d |idx_d>."""
    idx: np.ndarray
    cf: np.ndarray  # complex128

    def __len__(self) -> int:
        return len(self.idx)


@dataclass
class CoeffMatrix:
    """Coefficient-matrix trial state (Slater-Condon expansion): blocks of
    real orbital coefficients C_alpha[k] (n_sites x n_alpha) and C_beta[k]
    (n_sites x n_beta; None = closed shell, C_beta = C_alpha) with weights
    (None = the single block of weight 1).  tapered drops qubits 0 and
    n_sites.  Used as the initial state / overlap trial of the drivers in
    place of Dets."""
    n_sites: int
    n_alpha: int
    n_beta: int
    C_alpha: list
    C_beta: list | None = None
    weights: list | None = None
    tapered: bool = False

    def blocks(self):
        nb = len(self.C_alpha)
        w = self.weights if self.weights is not None else [1.0]
        cb = self.C_beta if self.C_beta is not None else [None] * nb
        return list(zip(w, self.C_alpha, cb))


_libc = None


def _malloc_copy(arr) -> int:
    """A malloc'ed copy of a float64 array (the library frees it)."""
    global _libc
    if _libc is None:
        _libc = C.CDLL(None)
        _libc.malloc.restype = C.c_void_p
        _libc.malloc.argtypes = [C.c_size_t]
    a = np.ascontiguousarray(arr, dtype=np.float64)
    p = _libc.malloc(max(1, a.nbytes))
    if not p:
        raise MemoryError("malloc")
    C.memmove(p, a.ctypes.data, a.nbytes)
    return p


def _coeff_matrix(nqb: int, cm: CoeffMatrix) -> _ffi.CoeffMatrix:
    """struct data_coeff_matrix with malloc'ed arrays, adopted by circ_init
    (freed by data_coeff_matrix_free)."""
    out = _ffi.CoeffMatrix()
    out.nqb, out.n_sites = nqb, cm.n_sites
    out.n_alpha, out.n_beta = cm.n_alpha, cm.n_beta
    out.closed_shell = 1 if cm.C_beta is None else 0
    out.tapered = 1 if cm.tapered else 0
    if cm.weights is None:
        out.n_components = 0
        out.C_alpha = _malloc_copy(cm.C_alpha[0])
        out.C_beta = (None if cm.C_beta is None
                      else _malloc_copy(cm.C_beta[0]))
        out.blocks = None
        return out
    n = len(cm.weights)
    out.n_components = n
    out.C_alpha = out.C_beta = None
    bl = _libc.malloc(C.sizeof(_ffi.CoeffBlock) * n)
    arr = (_ffi.CoeffBlock * n).from_address(bl)
    for k, (w, ca, cb) in enumerate(cm.blocks()):
        arr[k].cf = float(w)
        arr[k].C_alpha = _malloc_copy(ca)
        arr[k].C_beta = None if cb is None else _malloc_copy(cb)
    out.blocks = bl
    return out


def _initial_state(nqb: int, dets):
    """(stprep kind, pointer, keep-alive) for Dets or CoeffMatrix."""
    if isinstance(dets, CoeffMatrix):
        cm = _coeff_matrix(nqb, dets)
        return _ffi.STPREP_COEFF_MATRIX, C.cast(C.pointer(cm), C.c_void_p), cm
    md = _muldet(dets)
    return _ffi.STPREP_MULTIDET, C.cast(C.pointer(md), C.c_void_p), md


def _hamil(nqb: int, terms: Terms) -> _ffi.CircHamil:
    L = lib()
    hm = _ffi.CircHamil()
    if L.circ_hamil_init(C.byref(hm), nqb, len(terms)) != 0:
        raise MemoryError("circ_hamil_init")
    rec = terms.records()
    if len(terms):
        C.memmove(hm.terms, rec.ctypes.data, rec.nbytes)
    return hm


def _muldet(dets: Dets) -> _ffi.CircMuldet:
    L = lib()
    md = _ffi.CircMuldet()
    if L.circ_muldet_init(C.byref(md), len(dets)) != 0:
        raise MemoryError("circ_muldet_init")
    rec = np.zeros(len(dets), dtype=[("idx", "<u8"), ("cf", "<c16")])
    rec["idx"], rec["cf"] = dets.idx, dets.cf
    if len(dets):
        C.memmove(md.dets, rec.ctypes.data, rec.nbytes)
    return md


def _values(v: _ffi.CircValues) -> np.ndarray:
    n = int(v.len)
    arr = np.ctypeslib.as_array(v.z, shape=(2 * n,)) if n else np.zeros(0)
    return arr.view(np.complex128).copy()


# ---- register ----------------------------------------------------------


class Register:
    """A device-resident register (struct qreg) of nqb qubits."""

    def __init__(self, nqb: int, prec: int | None = None):
        world_ensure()
        self._L = lib()
        self.reg = _ffi.Qreg()
        if prec is None:
            rc = self._L.qreg_init(C.byref(self.reg), nqb)
        else:
            rc = self._L.qreg_init_prec(C.byref(self.reg), nqb, prec)
        if rc != 0:
            raise RuntimeError(f"qreg_init({nqb}) failed")
        self.nqb = nqb

    def close(self) -> None:
        if self.reg.backend:
            self._L.qreg_free(C.byref(self.reg))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def precision(self) -> int:
        return self._L.qreg_precision(C.byref(self.reg))

    def set_state(self, amp: np.ndarray) -> None:
        a = np.ascontiguousarray(amp, dtype=np.complex128)
        if self._L.qreg_set_state(C.byref(self.reg),
                                  a.ctypes.data_as(C.POINTER(C.c_double))):
            raise RuntimeError("qreg_set_state failed")

    def get_state(self) -> np.ndarray:
        out = np.empty(1 << self.nqb, dtype=np.complex128)
        if self._L.qreg_get_state(C.byref(self.reg),
                                  out.ctypes.data_as(C.POINTER(C.c_double))):
            raise RuntimeError("qreg_get_state failed")
        return out

    def zero(self) -> None:
        self._L.qreg_zero(C.byref(self.reg))

    def paulirot(self, flip, phase, phi, batch: int = 1024) -> None:
        """qreg_paulirot with code_hi = identity, `batch` terms per call."""
        flip = np.ascontiguousarray(flip, dtype=np.uint64)
        phase = np.ascontiguousarray(phase, dtype=np.uint64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        codes = np.empty((len(phi), 2), dtype=np.uint64)
        codes[:, 0], codes[:, 1] = flip, phase
        hi = _ffi.Paulis()
        for k in range(0, len(phi), batch):
            m = min(batch, len(phi) - k)
            self._L.qreg_paulirot(
                C.byref(self.reg), hi,
                codes[k:].ctypes.data_as(C.POINTER(_ffi.Paulis)),
                phi[k:].ctypes.data_as(C.POINTER(C.c_double)), m)

    def getamps(self, idx) -> np.ndarray:
        idx = np.ascontiguousarray(idx, dtype=np.uint64)
        out = np.empty(len(idx), dtype=np.complex128)
        if self._L.qreg_getamps(C.byref(self.reg),
                                idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                out.ctypes.data_as(C.POINTER(C.c_double)),
                                len(idx)):
            raise RuntimeError("qreg_getamps failed")
        return out

    def setamps(self, idx, z) -> None:
        idx = np.ascontiguousarray(idx, dtype=np.uint64)
        z = np.ascontiguousarray(z, dtype=np.complex128)
        if self._L.qreg_setamps(C.byref(self.reg),
                                idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                z.ctypes.data_as(C.POINTER(C.c_double)),
                                len(idx)):
            raise RuntimeError("qreg_setamps failed")

    def set_fusion(self, max_span: int, max_rots: int = 0) -> None:
        if self._L.qreg_set_fusion(C.byref(self.reg), max_span, max_rots):
            raise ValueError("qreg_set_fusion failed")

    def synchronize(self) -> None:
        if self._L.qreg_synchronize(C.byref(self.reg)):
            raise RuntimeError("qreg_synchronize reported a CUDA error")

    def norm2(self) -> float:
        v = C.c_double()
        if self._L.qreg_norm2(C.byref(self.reg), C.byref(v)):
            raise RuntimeError("qreg_norm2 failed")
        return v.value

    def inner_dense(self, trial: np.ndarray) -> complex:
        t = np.ascontiguousarray(trial, dtype=np.complex128)
        out = (C.c_double * 2)()
        if self._L.qreg_inner_dense(C.byref(self.reg),
                                    t.ctypes.data_as(C.POINTER(C.c_double)),
                                    out):
            raise RuntimeError("qreg_inner_dense failed")
        return complex(out[0], out[1])

    def _coeff_call(self, fn, cm: CoeffMatrix, *tail):
        sc = _ffi.CoeffScratch()
        if self._L.state_prep_coeff_scratch_init(
                C.byref(sc), cm.n_sites, cm.n_alpha, cm.n_beta) != 0:
            raise ValueError("coefficient matrix sizes out of range")
        try:
            return fn(sc, *tail)
        finally:
            self._L.state_prep_coeff_scratch_free(C.byref(sc))

    def coeff_expand(self, cm: CoeffMatrix) -> None:
        """Zero the register and expand the trial state on the device
        (state_prep_coeff_expand_all)."""
        m = _coeff_matrix(self.nqb, cm)
        try:
            def run(sc):
                if self._L.state_prep_coeff_expand_all(
                        C.byref(self.reg), C.byref(sc), C.byref(m)) != 0:
                    raise RuntimeError("state_prep_coeff_expand_all failed")
            self._coeff_call(run, cm)
        finally:
            self._L.data_coeff_matrix_free(C.byref(m))

    def coeff_inner(self, cm: CoeffMatrix) -> complex:
        """<trial|psi> summed over the blocks in order (device reduction;
        the measure of the coefficient-matrix drivers)."""
        def run(sc):
            tot = 0j
            for w, ca, cb in cm.blocks():
                a = np.ascontiguousarray(ca, dtype=np.float64)
                b = (None if cb is None
                     else np.ascontiguousarray(cb, dtype=np.float64))
                z = (C.c_double * 2)()
                if self._L.state_prep_coeff_inner(
                        C.byref(self.reg), C.byref(sc),
                        a.ctypes.data_as(C.POINTER(C.c_double)),
                        None if b is None else
                        b.ctypes.data_as(C.POINTER(C.c_double)),
                        float(w), int(cm.tapered), z) != 0:
                    raise RuntimeError("state_prep_coeff_inner failed")
                tot += complex(z[0], z[1])
            return tot
        return self._coeff_call(run, cm)

    def set_timing(self, on: bool) -> None:
        self._L.qreg_set_timing(C.byref(self.reg), int(on))

    def stats(self) -> dict:
        st = _ffi.Stats()
        self._L.qreg_get_stats(C.byref(self.reg), C.byref(st))
        return {k: getattr(st, k) for k, _ in _ffi.Stats._fields_}

    def reset_stats(self) -> None:
        self._L.qreg_reset_stats(C.byref(self.reg))


# ---- drivers -----------------------------------------------------------


def _run_driver(kind: str, nqb: int, terms: Terms, dets, **kw):
    world_ensure()
    L = lib()
    hm = _hamil(nqb, terms)
    sp_kind, sp_ptr, _keep = _initial_state(nqb, dets)
    if kind in ("trott", "trott2"):
        obj = (_ffi.Trott if kind == "trott" else _ffi.Trott2)()
        dt = _ffi.TrottData(kw["steps"], kw["delta"])
    elif kind == "qdrift":
        obj = _ffi.Qdrift()
        dt = _ffi.QdriftData(kw["samples"], kw["depth"], kw["step_size"],
                             kw["seed"])
    else:
        obj = _ffi.Cmpsit()
        dt = _ffi.CmpsitData(kw["samples"], kw["steps"], kw["length"],
                             kw["depth"], kw["angle_det"], kw["angle_rand"],
                             kw["seed"])
    init = getattr(L, f"{kind}_init")
    sw = None
    if kw.get("writer") is not None:
        # per-step output: writer(step_index, overlap) for every step or
        # sample, as the driver produces it (the callback must outlive the
        # run, hence kept here)
        py_writer = kw["writer"]

        def _write(_ctx, i, z):
            py_writer(int(i), complex(z.re, z.im))
            return 0
        sw = _ffi.StepWriter(None, _ffi.STEP_WRITE_FN(_write))
    if init(C.byref(obj), C.byref(dt), hm, sp_kind, sp_ptr,
            C.cast(C.pointer(sw), C.c_void_p) if sw else None) != 0:
        raise RuntimeError(f"{kind}_init failed")
    try:
        if kw.get("fusion") is not None:
            span, rots = kw["fusion"]
            L.qreg_set_fusion(C.byref(obj.ct.reg), span, rots)
        if kw.get("timing"):
            L.qreg_set_timing(C.byref(obj.ct.reg), 1)
        if getattr(L, f"{kind}_simul")(C.byref(obj)) != 0:
            raise RuntimeError(f"{kind}_simul failed")
        vals = _values(obj.ct.vals)
        st = _ffi.Stats()
        L.qreg_get_stats(C.byref(obj.ct.reg), C.byref(st))
        stats = {k: getattr(st, k) for k, _ in _ffi.Stats._fields_}
        if kw.get("state_idx") is not None:
            # selected amplitudes of the register after the run
            idx = np.ascontiguousarray(kw["state_idx"], dtype=np.uint64)
            amps = np.zeros(len(idx), dtype=np.complex128)
            if len(idx) and L.qreg_getamps(
                    C.byref(obj.ct.reg),
                    idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                    amps.ctypes.data_as(C.POINTER(C.c_double)), len(idx)):
                raise RuntimeError("qreg_getamps failed")
            stats["amps"] = amps
        if kw.get("with_state"):
            # the register after the run (small registers)
            stats["state"] = np.empty(1 << nqb, dtype=np.complex128)
            if L.qreg_get_state(C.byref(obj.ct.reg),
                                stats["state"].ctypes.data_as(
                                    C.POINTER(C.c_double))):
                raise RuntimeError("qreg_get_state failed")
    finally:
        getattr(L, f"{kind}_free")(C.byref(obj))
    return (vals, stats) if kw.get("with_stats") else vals


_KIND = {"trott": (_ffi.Trott, "steps"), "trott2": (_ffi.Trott2, "steps"),
         "qdrift": (_ffi.Qdrift, None), "cmpsit": (_ffi.Cmpsit, None)}


def _driver_data(kind: str, p: dict):
    if kind in ("trott", "trott2"):
        return _ffi.TrottData(p["steps"], p["delta"])
    if kind == "qdrift":
        return _ffi.QdriftData(p["samples"], p["depth"], p["step_size"],
                               p["seed"])
    return _ffi.CmpsitData(p["samples"], p["steps"], p["length"], p["depth"],
                           p["angle_det"], p["angle_rand"], p["seed"])


def batch(kind: str, problems: list[dict], with_stats: bool = False):
    """Run independent problems of one driver kind together through
    <kind>_simul_batch.  Each problem dict holds nqb, terms, dets and the
    driver's parameters (as the single-problem helpers take them)."""
    world_ensure()
    L = lib()
    cls = _KIND[kind][0]
    objs = []
    try:
        for p in problems:
            obj = cls()
            hm = _hamil(p["nqb"], p["terms"])
            sp_kind, sp_ptr, _keep = _initial_state(p["nqb"], p["dets"])
            dt = _driver_data(kind, p)
            if getattr(L, f"{kind}_init")(
                    C.byref(obj), C.byref(dt), hm, sp_kind, sp_ptr,
                    None) != 0:
                raise RuntimeError(f"{kind}_init failed")
            objs.append(obj)
        arr = (C.c_void_p * max(1, len(objs)))(
            *[C.cast(C.pointer(o), C.c_void_p) for o in objs])
        if getattr(L, f"{kind}_simul_batch")(arr, len(objs)) != 0:
            raise RuntimeError(f"{kind}_simul_batch failed")
        # per-instance finish times of the persistent launch (if it ran)
        fin = (C.c_double * max(1, len(objs)))()
        nfin = L.phase2_batch_finish_ms(fin, len(objs))
        vals = [_values(o.ct.vals) for o in objs]
        stats = []
        for k, o in enumerate(objs):
            st = _ffi.Stats()
            L.qreg_get_stats(C.byref(o.ct.reg), C.byref(st))
            stats.append({k: getattr(st, k) for k, _ in _ffi.Stats._fields_})
            stats[-1]["finish_ms"] = fin[k] if nfin == len(objs) else None
    finally:
        for o in objs:
            getattr(L, f"{kind}_free")(C.byref(o))
    return (vals, stats) if with_stats else vals


def trott(nqb, terms, dets, steps, delta, **kw):
    return _run_driver("trott", nqb, terms, dets, steps=steps, delta=delta,
                       **kw)


def trott2(nqb, terms, dets, steps, delta, **kw):
    return _run_driver("trott2", nqb, terms, dets, steps=steps, delta=delta,
                       **kw)


def qdrift(nqb, terms, dets, samples, depth, step_size, seed, **kw):
    return _run_driver("qdrift", nqb, terms, dets, samples=samples,
                       depth=depth, step_size=step_size, seed=seed, **kw)


def cmpsit(nqb, terms, dets, samples, steps, length, depth, angle_det,
           angle_rand, seed, **kw):
    return _run_driver("cmpsit", nqb, terms, dets, samples=samples,
                       steps=steps, length=length, depth=depth,
                       angle_det=angle_det, angle_rand=angle_rand, seed=seed,
                       **kw)


# ---- planner (host only) -----------------------------------------------


def plan(nqb: int, flip, phase, phi, max_span: int = 5, max_rots: int = 0,
         prec: int = PREC_FP64):
    """Run the host planner; returns (passes, records) as lists of dicts."""
    L = lib()
    n = len(phi)
    rin = (_ffi.RotIn * max(n, 1))()
    for k in range(n):
        rin[k].flip, rin[k].phase, rin[k].phi = int(flip[k]), int(phase[k]), \
            float(phi[k])
    passes = (_ffi.Pass * max(n, 1))()
    recs = (_ffi.RotRec * max(n, 1))()
    np_ = L.phase2_plan(nqb, rin, n, max_span, max_rots, prec, passes, recs)
    if np_ < 0:
        raise ValueError("phase2_plan failed")
    out_p = [{"span": p.span, "nrot": p.nrot, "rot_off": p.rot_off,
              "piv": list(p.piv)[:p.span], "basis": list(p.basis)[:p.span],
              "scale": p.scale, "form": p.form, "sweep": p.sweep}
             for p in passes[:np_]]
    out_r = [{"z": r.z, "c": r.c, "s": r.s, "smask": r.smask, "U": r.U,
              "odd": r.odd, "form": r.form} for r in recs[:n]]
    return out_p, out_r
