"""Python access to the oracle libraries.  TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
bench.py use this module, and only as the checker.  The product library
(phase2_b200/libphase2.so) never calls into it.

* ``Oracle`` wraps oracle/liboracle.so, the CPU restatement in oracle.c.
* ``Reference`` wraps oracle/_ref/libphase2_ref.so, the reference's own
  CPU path compiled from its sources by ``make -C oracle ref`` (present
  only where the reference sources were available at build time).
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libphase2_ref.so"

_P = C.POINTER
_D = _P(C.c_double)
_U = _P(C.c_uint64)

TERM_DTYPE = np.dtype([("cf", "<f8"), ("flip", "<u8"), ("phase", "<u8")])


def _dptr(a):
    return a.ctypes.data_as(_D)


def _uptr(a):
    return a.ctypes.data_as(_U)


def term_records(flip, phase, cf) -> np.ndarray:
    rec = np.zeros(len(cf), dtype=TERM_DTYPE)
    rec["flip"], rec["phase"], rec["cf"] = flip, phase, cf
    return rec


def coeff_arrays(cm):
    """(ncomp, weights, Ca, Cb) flat float64 arrays of a coefficient-matrix
    state given as an object with n_sites, n_alpha, n_beta, C_alpha (list),
    C_beta (list or None), weights (list or None)."""
    ncomp = 0 if cm.weights is None else len(cm.weights)
    w = np.asarray(cm.weights if ncomp else [1.0], dtype=np.float64)
    ca = np.concatenate([np.ascontiguousarray(a, dtype=np.float64).ravel()
                         for a in cm.C_alpha])
    cb = None
    if cm.C_beta is not None:
        cb = np.concatenate([np.ascontiguousarray(b, dtype=np.float64).ravel()
                             for b in cm.C_beta])
    return ncomp, w, ca, cb


def _dets(idx, cf):
    idx = np.ascontiguousarray(idx, dtype=np.uint64)
    cf = np.ascontiguousarray(cf, dtype=np.complex128).view(np.float64)
    return idx, cf


class Oracle:
    """ctypes wrapper of the CPU restatement (oracle.c)."""

    def __init__(self, path: Path = ORACLE_SO):
        if not Path(path).is_file():
            raise RuntimeError(f"{path} missing: run `make -C oracle`")
        L = C.CDLL(str(path))
        L.orc_rng_init.argtypes = [_U, C.c_uint64]
        L.orc_rng_next.argtypes = [_U]
        L.orc_rng_next.restype = C.c_uint64
        L.orc_rng_dbl01.argtypes = [_U]
        L.orc_rng_dbl01.restype = C.c_double
        L.orc_effect.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64,
                                 _P(C.c_int)]
        L.orc_effect.restype = C.c_uint64
        L.orc_pauli_cmp.argtypes = [C.c_uint64] * 4
        L.orc_pauli_cmp.restype = C.c_int
        L.orc_cdf_build.argtypes = [_D, C.c_size_t, C.c_size_t, _D, _D]
        L.orc_cdf_build.restype = C.c_int
        L.orc_cdf_inverse.argtypes = [_D, C.c_size_t, C.c_double]
        L.orc_cdf_inverse.restype = C.c_size_t
        L.orc_signof.argtypes = [C.c_double]
        L.orc_signof.restype = C.c_double
        L.orc_rotate_many.argtypes = [_D, C.c_uint32, _U, _U, _D, C.c_size_t]
        L.orc_sort_lex.argtypes = [C.c_void_p, C.c_size_t]
        for name in ("orc_trott", "orc_trott2"):
            fn = getattr(L, name)
            fn.argtypes = [C.c_uint32, C.c_void_p, C.c_size_t, C.c_size_t,
                           _U, _D, C.c_size_t, C.c_double, C.c_int, _D]
            fn.restype = C.c_int
        L.orc_qdrift.argtypes = [C.c_uint32, C.c_void_p, C.c_size_t,
                                 C.c_size_t, _U, _D, C.c_size_t, C.c_size_t,
                                 C.c_double, C.c_uint64, _D]
        L.orc_qdrift.restype = C.c_int
        L.orc_qdrift_draws.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t,
                                       C.c_size_t, C.c_uint64, C.c_void_p]
        L.orc_qdrift_draws.restype = C.c_int
        L.orc_cmpsit.argtypes = [C.c_uint32, C.c_void_p, C.c_size_t,
                                 C.c_size_t, _U, _D, C.c_size_t, C.c_size_t,
                                 C.c_size_t, C.c_size_t, C.c_double,
                                 C.c_double, C.c_uint64, _D]
        L.orc_cmpsit.restype = C.c_int
        L.orc_phase2_run.argtypes = [_P(C.c_char_p), _D, C.c_size_t,
                                     C.c_double, C.c_char_p, _D, _D]
        L.orc_phase2_run.restype = C.c_int
        cm_args = [C.c_uint32] * 4 + [C.c_int, C.c_size_t, _D, _D, _D]
        L.orc_coeff_expand_all.argtypes = cm_args + [_D]
        L.orc_coeff_expand_all.restype = C.c_int
        L.orc_coeff_inner.argtypes = cm_args + [_D, _D]
        L.orc_coeff_inner.restype = C.c_int
        self.L = L

    # -- coefficient-matrix trial state
    def coeff_expand(self, nqb, cm) -> np.ndarray:
        ncomp, w, ca, cb = coeff_arrays(cm)
        amp = np.zeros(1 << nqb, dtype=np.complex128)
        if self.L.orc_coeff_expand_all(
                nqb, cm.n_sites, cm.n_alpha, cm.n_beta, int(cm.tapered),
                ncomp, _dptr(w), _dptr(ca),
                None if cb is None else _dptr(cb),
                _dptr(amp.view(np.float64))):
            raise RuntimeError("oracle coeff_expand failed")
        return amp

    def coeff_inner(self, nqb, cm, amp) -> complex:
        ncomp, w, ca, cb = coeff_arrays(cm)
        a = np.ascontiguousarray(amp, dtype=np.complex128)
        out = np.zeros(2)
        if self.L.orc_coeff_inner(
                nqb, cm.n_sites, cm.n_alpha, cm.n_beta, int(cm.tapered),
                ncomp, _dptr(w), _dptr(ca),
                None if cb is None else _dptr(cb),
                _dptr(a.view(np.float64)), _dptr(out)):
            raise RuntimeError("oracle coeff_inner failed")
        return complex(out[0], out[1])

    # -- primitives
    def rng_sequence(self, seed: int, n: int) -> list[int]:
        s = (C.c_uint64 * 4)()
        self.L.orc_rng_init(s, seed)
        return [self.L.orc_rng_next(s) for _ in range(n)]

    def effect(self, flip: int, phase: int, i: int) -> tuple[int, int]:
        r = C.c_int()
        j = self.L.orc_effect(flip, phase, i, C.byref(r))
        return j, r.value

    def cdf(self, w) -> tuple[int, np.ndarray, float]:
        w = np.ascontiguousarray(w, dtype=np.float64)
        y = np.zeros(len(w))
        lam = C.c_double(-1.0)
        rc = self.L.orc_cdf_build(_dptr(w), 8, len(w), _dptr(y),
                                  C.byref(lam))
        return rc, y, lam.value

    def cdf_inverse(self, y: np.ndarray, x: float) -> int:
        y = np.ascontiguousarray(y, dtype=np.float64)
        return int(self.L.orc_cdf_inverse(_dptr(y), len(y), x))

    def rotate(self, amp: np.ndarray, nqb: int, flip, phase, phi):
        a = np.ascontiguousarray(amp, dtype=np.complex128).copy()
        flip = np.ascontiguousarray(flip, dtype=np.uint64)
        phase = np.ascontiguousarray(phase, dtype=np.uint64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        self.L.orc_rotate_many(_dptr(a.view(np.float64)), nqb, _uptr(flip),
                               _uptr(phase), _dptr(phi), len(phi))
        return a

    def sort_lex(self, flip, phase, cf):
        rec = term_records(flip, phase, cf)
        self.L.orc_sort_lex(rec.ctypes.data, len(rec))
        return rec

    # -- drivers
    def trott(self, nqb, flip, phase, cf, det_idx, det_cf, steps, delta,
              order2=False, sort_lex=True) -> np.ndarray:
        rec = term_records(flip, phase, cf)
        di, dc = _dets(det_idx, det_cf)
        out = np.zeros(2 * steps)
        fn = self.L.orc_trott2 if order2 else self.L.orc_trott
        rc = fn(nqb, rec.ctypes.data, len(rec), len(di), _uptr(di),
                _dptr(dc), steps, delta, int(sort_lex), _dptr(out))
        if rc:
            raise RuntimeError("oracle trott failed")
        return out.view(np.complex128)

    def qdrift(self, nqb, flip, phase, cf, det_idx, det_cf, samples, depth,
               step_size, seed) -> np.ndarray:
        rec = term_records(flip, phase, cf)
        di, dc = _dets(det_idx, det_cf)
        out = np.zeros(2 * samples)
        rc = self.L.orc_qdrift(nqb, rec.ctypes.data, len(rec), len(di),
                               _uptr(di), _dptr(dc), samples, depth,
                               step_size, seed, _dptr(out))
        if rc:
            raise RuntimeError("oracle qdrift failed")
        return out.view(np.complex128)

    def qdrift_draws(self, flip, phase, cf, samples, depth, seed):
        rec = term_records(flip, phase, cf)
        out = np.zeros(samples * depth, dtype=TERM_DTYPE)
        if self.L.orc_qdrift_draws(rec.ctypes.data, len(rec), samples, depth,
                                   seed, out.ctypes.data):
            raise RuntimeError("oracle qdrift_draws failed")
        return out

    def cmpsit(self, nqb, flip, phase, cf, det_idx, det_cf, samples, steps,
               length, depth, angle_det, angle_rand, seed) -> np.ndarray:
        rec = term_records(flip, phase, cf)
        di, dc = _dets(det_idx, det_cf)
        out = np.zeros(2 * samples)
        rc = self.L.orc_cmpsit(nqb, rec.ctypes.data, len(rec), len(di),
                               _uptr(di), _dptr(dc), samples, steps, length,
                               depth, angle_det, angle_rand, seed,
                               _dptr(out))
        if rc:
            raise RuntimeError("oracle cmpsit failed")
        return out.view(np.complex128)

    def phase2_run(self, paulis, coeffs, delta, psi):
        n = len(paulis)
        arr = (C.c_char_p * max(n, 1))(*(p.encode() for p in paulis))
        cf = (C.c_double * max(n, 1))(*coeffs)
        re, im = C.c_double(), C.c_double()
        rc = self.L.orc_phase2_run(arr, cf, n, delta, psi.encode(),
                                   C.byref(re), C.byref(im))
        return rc, complex(re.value, im.value)


class Reference:
    """ctypes wrapper of the reference CPU path (oracle/_ref)."""

    def __init__(self, path: Path = REF_SO):
        if not Path(path).is_file():
            raise RuntimeError(f"{path} missing: run `make -C oracle ref`")
        L = C.CDLL(str(path))
        L.refh_paulirot.argtypes = [C.c_uint32, _D, _U, _U, _D, C.c_size_t]
        L.refh_paulirot.restype = C.c_int
        L.refh_trott.argtypes = [C.c_int, C.c_uint32, C.c_void_p, C.c_size_t,
                                 C.c_size_t, _U, _D, C.c_size_t, C.c_double,
                                 C.c_int, _D]
        L.refh_trott.restype = C.c_int
        L.refh_qdrift.argtypes = [C.c_uint32, C.c_void_p, C.c_size_t,
                                  C.c_size_t, _U, _D, C.c_size_t, C.c_size_t,
                                  C.c_double, C.c_uint64, _D]
        L.refh_qdrift.restype = C.c_int
        L.refh_cmpsit.argtypes = [C.c_uint32, C.c_void_p, C.c_size_t,
                                  C.c_size_t, _U, _D, C.c_size_t, C.c_size_t,
                                  C.c_size_t, C.c_size_t, C.c_double,
                                  C.c_double, C.c_uint64, _D]
        L.refh_cmpsit.restype = C.c_int
        L.phase2_run.argtypes = [_P(C.c_char_p), _D, C.c_size_t, C.c_double,
                                 C.c_char_p, _D, _D]
        L.phase2_run.restype = C.c_int
        L.refh_capture.argtypes = [C.c_uint64, C.c_size_t, _U, _D]
        L.refh_capture.restype = C.c_int
        L.refh_captured.argtypes = []
        L.refh_captured.restype = C.c_size_t
        cm_args = [C.c_uint32] * 4 + [C.c_int, C.c_size_t, _D, _D, _D]
        L.refh_coeff_expand_all.argtypes = cm_args + [_D]
        L.refh_coeff_expand_all.restype = C.c_int
        L.refh_coeff_inner.argtypes = cm_args + [_D, _D]
        L.refh_coeff_inner.restype = C.c_int
        self.L = L

    def coeff_expand(self, nqb, cm) -> np.ndarray:
        ncomp, w, ca, cb = coeff_arrays(cm)
        amp = np.zeros(1 << nqb, dtype=np.complex128)
        if self.L.refh_coeff_expand_all(
                nqb, cm.n_sites, cm.n_alpha, cm.n_beta, int(cm.tapered),
                ncomp, _dptr(w), _dptr(ca),
                None if cb is None else _dptr(cb),
                _dptr(amp.view(np.float64))):
            raise RuntimeError("reference coeff_expand failed")
        return amp

    def coeff_inner(self, nqb, cm, amp) -> complex:
        ncomp, w, ca, cb = coeff_arrays(cm)
        a = np.ascontiguousarray(amp, dtype=np.complex128)
        out = np.zeros(2)
        if self.L.refh_coeff_inner(
                nqb, cm.n_sites, cm.n_alpha, cm.n_beta, int(cm.tapered),
                ncomp, _dptr(w), _dptr(ca),
                None if cb is None else _dptr(cb),
                _dptr(a.view(np.float64)), _dptr(out)):
            raise RuntimeError("reference coeff_inner failed")
        return complex(out[0], out[1])

    def capture(self, stride: int, cap: int):
        """Arm the amplitude capture of the next driver run; returns a
        function giving (indices, amplitudes) after the run (stride 0:
        the non-zero amplitudes in index order)."""
        idx = np.zeros(cap, dtype=np.uint64)
        amp = np.zeros(cap, dtype=np.complex128)
        self.L.refh_capture(stride, cap, _uptr(idx),
                            _dptr(amp.view(np.float64)))

        def taken():
            n = self.L.refh_captured()
            return idx[:n].copy(), amp[:n].copy()
        return taken

    def paulirot(self, amp, nqb, flip, phase, phi):
        a = np.ascontiguousarray(amp, dtype=np.complex128).copy()
        flip = np.ascontiguousarray(flip, dtype=np.uint64)
        phase = np.ascontiguousarray(phase, dtype=np.uint64)
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        if self.L.refh_paulirot(nqb, _dptr(a.view(np.float64)), _uptr(flip),
                                _uptr(phase), _dptr(phi), len(phi)):
            raise RuntimeError("reference paulirot failed")
        return a

    def trott(self, nqb, flip, phase, cf, det_idx, det_cf, steps, delta,
              order2=False, sort_lex=True):
        rec = term_records(flip, phase, cf)
        di, dc = _dets(det_idx, det_cf)
        out = np.zeros(2 * steps)
        rc = self.L.refh_trott(int(order2), nqb, rec.ctypes.data, len(rec),
                               len(di), _uptr(di), _dptr(dc), steps, delta,
                               int(sort_lex), _dptr(out))
        if rc:
            raise RuntimeError("reference trott failed")
        return out.view(np.complex128)

    def qdrift(self, nqb, flip, phase, cf, det_idx, det_cf, samples, depth,
               step_size, seed):
        rec = term_records(flip, phase, cf)
        di, dc = _dets(det_idx, det_cf)
        out = np.zeros(2 * samples)
        if self.L.refh_qdrift(nqb, rec.ctypes.data, len(rec), len(di),
                              _uptr(di), _dptr(dc), samples, depth,
                              step_size, seed, _dptr(out)):
            raise RuntimeError("reference qdrift failed")
        return out.view(np.complex128)

    def cmpsit(self, nqb, flip, phase, cf, det_idx, det_cf, samples, steps,
               length, depth, angle_det, angle_rand, seed):
        rec = term_records(flip, phase, cf)
        di, dc = _dets(det_idx, det_cf)
        out = np.zeros(2 * samples)
        if self.L.refh_cmpsit(nqb, rec.ctypes.data, len(rec), len(di),
                              _uptr(di), _dptr(dc), samples, steps, length,
                              depth, angle_det, angle_rand, seed,
                              _dptr(out)):
            raise RuntimeError("reference cmpsit failed")
        return out.view(np.complex128)

    def phase2_run(self, paulis, coeffs, delta, psi):
        n = len(paulis)
        arr = (C.c_char_p * max(n, 1))(*(p.encode() for p in paulis))
        cf = (C.c_double * max(n, 1))(*coeffs)
        re, im = C.c_double(), C.c_double()
        rc = self.L.phase2_run(arr, cf, n, delta, psi.encode(), C.byref(re),
                               C.byref(im))
        return rc, complex(re.value, im.value)


# ---- the reference as R ranks on the host cores (oracle/_ref/ref_mpi) ----

REF_MPI = HERE / "_ref" / "ref_mpi"
_REF_IN_HDR = np.dtype([("magic", "S8"), ("mode", "<u4"), ("nqb", "<u4"),
                        ("nterms", "<u8"), ("ndets", "<u8"),
                        ("count", "<u8"), ("angle", "<f8"), ("seed", "<u8")])
_REF_IN_DET = np.dtype([("idx", "<u8"), ("re", "<f8"), ("im", "<f8")])


def write_ref_input(path, mode: str, nqb: int, flip, phase, cf, det_idx,
                    det_cf, count: int, angle: float, seed: int = 0) -> None:
    """Input file of ref_mpi: mode "qdrift" (count = depth, angle =
    step_size, one sample per run) or "trott2" (count = steps, angle =
    delta)."""
    h = np.zeros(1, dtype=_REF_IN_HDR)
    h["magic"], h["mode"], h["nqb"] = b"P2REFIN1", \
        {"qdrift": 0, "trott2": 1}[mode], nqb
    h["nterms"], h["ndets"], h["count"] = len(cf), len(det_idx), count
    h["angle"], h["seed"] = angle, seed
    d = np.zeros(len(det_idx), dtype=_REF_IN_DET)
    dc = np.asarray(det_cf, dtype=np.complex128)
    d["idx"], d["re"], d["im"] = det_idx, dc.real, dc.imag
    with open(path, "wb") as f:
        f.write(h.tobytes())
        f.write(term_records(flip, phase, cf).tobytes())
        f.write(d.tobytes())


def run_ref_mpi(ranks: int, path, reps: int, timeout: float = 1800,
                env: dict | None = None, warmup: int = 0) -> dict:
    """Run ref_mpi: the reference's driver as `ranks` ranks of one job,
    `warmup` untimed runs then the minimum over `reps` timed ones; returns
    its timing line as a dict."""
    import os
    import subprocess
    if not REF_MPI.is_file():
        raise RuntimeError(f"{REF_MPI} missing: run `make -C oracle ref-mpi`")
    e = dict(os.environ)
    e.update(env or {})
    out = subprocess.run([str(REF_MPI), str(ranks), str(path), str(reps),
                          str(warmup)],
                         capture_output=True, text=True, timeout=timeout,
                         env=e)
    if out.returncode != 0:
        raise RuntimeError(f"ref_mpi failed ({out.returncode}): "
                           f"{out.stderr.strip()[-400:]}")
    # the reference logs to stdout too: the timing line is the last one
    f = out.stdout.strip().splitlines()[-1].split()
    return {"ranks": int(f[0]), "rotations": int(f[1]),
            "seconds": float(f[2]), "rot_amp_s": float(f[3]),
            "mailbox": bool(int(f[4])), "z": complex(float(f[5]),
                                                    float(f[6]))}
