"""ctypes mirror of the C surface of libphase2.so.

Struct layouts follow include/phase2/*.h, include/circ/*.h and
include/phase2_b200.h of this repository (which in turn mirror the phase2
reference headers); ``check_layout`` compares every size against
``phase2_sizeof`` from the library itself.

The library is loaded from this package directory (``libphase2.so`` built
in-tree by ``make -C phase2_b200/csrc``).  Loading fails loudly when it is
missing: there is no Python or CPU fallback for any operation.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libphase2.so"

# ---- structs -----------------------------------------------------------


class Paulis(C.Structure):
    _fields_ = [("pak", C.c_uint64 * 2)]


class WorldInfo(C.Structure):
    _fields_ = [("stat", C.c_int), ("size", C.c_int), ("rank", C.c_int),
                ("seed", C.c_uint64)]


class Qreg(C.Structure):
    _fields_ = [("wd", WorldInfo), ("qb_lo", C.c_uint32),
                ("qb_hi", C.c_uint32), ("amp", C.c_void_p),
                ("buf", C.c_void_p), ("namp", C.c_uint64),
                ("msg_count", C.c_int), ("reqs_snd", C.c_void_p),
                ("reqs_rcv", C.c_void_p), ("nreqs", C.c_size_t),
                ("backend", C.c_void_p)]


class HamilTerm(C.Structure):
    _fields_ = [("cf", C.c_double), ("op", Paulis)]


class CircHamil(C.Structure):
    _fields_ = [("qb", C.c_uint32), ("terms", C.POINTER(HamilTerm)),
                ("len", C.c_size_t)]


class Det(C.Structure):
    _fields_ = [("idx", C.c_uint64), ("cf", C.c_double * 2)]


class CircMuldet(C.Structure):
    _fields_ = [("dets", C.POINTER(Det)), ("len", C.c_size_t)]


class CircValues(C.Structure):
    _fields_ = [("z", C.POINTER(C.c_double)), ("len", C.c_size_t)]


class CoeffMatrix(C.Structure):
    _fields_ = [("nqb", C.c_uint32), ("n_sites", C.c_uint32),
                ("n_alpha", C.c_uint32), ("n_beta", C.c_uint32),
                ("closed_shell", C.c_int), ("tapered", C.c_int),
                ("n_components", C.c_size_t), ("C_alpha", C.c_void_p),
                ("C_beta", C.c_void_p), ("blocks", C.c_void_p)]


class CoeffBlock(C.Structure):
    _fields_ = [("cf", C.c_double), ("C_alpha", C.c_void_p),
                ("C_beta", C.c_void_p)]


class CoeffScratch(C.Structure):
    _fields_ = [("n_sites", C.c_uint32), ("n_alpha", C.c_uint32),
                ("n_beta", C.c_uint32), ("tup_a", C.c_void_p),
                ("tup_b", C.c_void_p), ("det_a", C.c_void_p),
                ("det_b", C.c_void_p), ("Ma", C.c_size_t),
                ("Mb", C.c_size_t)]


class Circ(C.Structure):
    _fields_ = [("hm", CircHamil), ("md", CircMuldet),
                ("cache", C.c_void_p), ("vals", CircValues),
                ("reg", Qreg), ("stprep_kind", C.c_int),
                ("cm", CoeffMatrix), ("sp_scratch", CoeffScratch)]


class TrottData(C.Structure):
    _fields_ = [("steps", C.c_size_t), ("delta", C.c_double)]


class Trott(C.Structure):
    _fields_ = [("ct", Circ), ("dt", TrottData), ("sw", C.c_void_p)]


class Trott2(C.Structure):
    _fields_ = [("ct", Circ), ("dt", TrottData), ("sw", C.c_void_p)]


class ProbCdf(C.Structure):
    _fields_ = [("y", C.POINTER(C.c_double)), ("len", C.c_size_t)]


class Xoshiro(C.Structure):
    _fields_ = [("s", C.c_uint64 * 4)]


class QdriftData(C.Structure):
    _fields_ = [("samples", C.c_size_t), ("depth", C.c_size_t),
                ("step_size", C.c_double), ("seed", C.c_uint64)]


class QdriftRanct(C.Structure):
    _fields_ = [("hm_ran", CircHamil), ("cdf", ProbCdf)]


class Qdrift(C.Structure):
    _fields_ = [("ct", Circ), ("dt", QdriftData), ("ranct", QdriftRanct),
                ("rng", Xoshiro), ("sw", C.c_void_p)]


class CmpsitData(C.Structure):
    _fields_ = [("samples", C.c_size_t), ("steps", C.c_size_t),
                ("length", C.c_size_t), ("depth", C.c_size_t),
                ("angle_det", C.c_double), ("angle_rand", C.c_double),
                ("seed", C.c_uint64)]


class CmpsitRanct(C.Structure):
    _fields_ = [("hm_det", CircHamil), ("hm_ran", CircHamil),
                ("hm_smpl", CircHamil), ("cdf", ProbCdf),
                ("lambda_r", C.c_double), ("depth", C.c_size_t),
                ("angle_rand", C.c_double)]


class Cmpsit(C.Structure):
    _fields_ = [("ct", Circ), ("dt", CmpsitData), ("ranct", CmpsitRanct),
                ("rng", Xoshiro), ("sw", C.c_void_p)]


class Complex(C.Structure):
    """_Complex double as returned in registers (two doubles)."""
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


# struct phase2_step_writer (include/phase2/step_writer.h): the callback
# receives the step's overlap as a _Complex double, passed as two doubles
STEP_WRITE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_size_t, Complex)


class StepWriter(C.Structure):
    _fields_ = [("ctx", C.c_void_p), ("write", STEP_WRITE_FN)]


class RotIn(C.Structure):
    _fields_ = [("flip", C.c_uint64), ("phase", C.c_uint64),
                ("phi", C.c_double)]


MAX_SPAN = 5


class Pass(C.Structure):
    _fields_ = [("span", C.c_uint32), ("nrot", C.c_uint32),
                ("rot_off", C.c_uint32), ("piv", C.c_uint8 * MAX_SPAN),
                ("form", C.c_uint8), ("sweep", C.c_uint8),
                ("pad", C.c_uint8),
                ("basis", C.c_uint64 * MAX_SPAN),
                ("scale", C.c_double)]


class RotRec(C.Structure):
    _fields_ = [("z", C.c_uint64), ("c", C.c_double), ("s", C.c_double),
                ("smask", C.c_uint32), ("U", C.c_uint8), ("W", C.c_uint8),
                ("odd", C.c_uint8), ("form", C.c_uint8)]


class Stats(C.Structure):
    _fields_ = [("rotations", C.c_uint64), ("passes", C.c_uint64),
                ("launches", C.c_uint64), ("bytes", C.c_uint64),
                ("timed_passes", C.c_uint64), ("pass_ms", C.c_double),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64),
                ("graph_replays", C.c_uint64), ("sweeps", C.c_uint64),
                ("timed_sweeps", C.c_uint64)]


LAYOUT = {0: Qreg, 1: Circ, 2: Trott, 3: Trott2, 4: Qdrift, 5: Cmpsit,
          6: HamilTerm, 7: Pass, 8: RotRec, 9: Stats}

PREC_FP64 = 0
PREC_FP32 = 1
ORDER_LEX, ORDER_GIVEN, ORDER_FLIP = 0, 1, 2
STPREP_MULTIDET = 1
STPREP_COEFF_MATRIX = 2
WORLD_READY = 0

# ---- loading -----------------------------------------------------------

_P = C.POINTER
_SIGS = {
    "paulis_new": (Paulis, []),
    "paulis_get": (C.c_int, [Paulis, C.c_uint32]),
    "paulis_set": (None, [_P(Paulis), C.c_int, C.c_uint32]),
    "paulis_eq": (C.c_int, [Paulis, Paulis]),
    "paulis_shl": (None, [_P(Paulis), C.c_uint32]),
    "paulis_shr": (None, [_P(Paulis), C.c_uint32]),
    "paulis_effect": (C.c_uint64, [Paulis, C.c_uint64, _P(C.c_double)]),
    "paulis_split": (None, [Paulis, C.c_uint32, C.c_uint32, _P(Paulis),
                            _P(Paulis)]),
    "paulis_cmp": (C.c_int, [Paulis, Paulis]),
    "world_init": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "world_free": (C.c_int, []),
    "world_info": (C.c_int, [_P(WorldInfo)]),
    "qreg_init": (C.c_int, [_P(Qreg), C.c_uint32]),
    "qreg_init_prec": (C.c_int, [_P(Qreg), C.c_uint32, C.c_int]),
    "qreg_free": (None, [_P(Qreg)]),
    "qreg_getamp": (None, [_P(Qreg), C.c_uint64, _P(C.c_double)]),
    "qreg_setamp": (None, [_P(Qreg), C.c_uint64, C.c_double, C.c_double]),
    "qreg_zero": (None, [_P(Qreg)]),
    "qreg_sync_host_to_device": (None, [_P(Qreg)]),
    "qreg_sync_device_to_host": (None, [_P(Qreg)]),
    "qreg_paulirot": (None, [_P(Qreg), Paulis, _P(Paulis), _P(C.c_double),
                             C.c_size_t]),
    "qreg_precision": (C.c_int, [_P(Qreg)]),
    "qreg_set_fusion": (C.c_int, [_P(Qreg), C.c_int, C.c_int]),
    "qreg_flush": (C.c_int, [_P(Qreg)]),
    "qreg_synchronize": (C.c_int, [_P(Qreg)]),
    "qreg_getamps": (C.c_int, [_P(Qreg), _P(C.c_uint64), _P(C.c_double),
                               C.c_size_t]),
    "qreg_setamps": (C.c_int, [_P(Qreg), _P(C.c_uint64), _P(C.c_double),
                               C.c_size_t]),
    "qreg_get_state": (C.c_int, [_P(Qreg), _P(C.c_double)]),
    "qreg_set_state": (C.c_int, [_P(Qreg), _P(C.c_double)]),
    "qreg_norm2": (C.c_int, [_P(Qreg), _P(C.c_double)]),
    "qreg_slab_get": (C.c_int, [_P(Qreg), C.c_uint32, C.c_uint32,
                                C.c_uint64, C.c_uint64, C.c_void_p]),
    "qreg_slab_put": (C.c_int, [_P(Qreg), C.c_uint32, C.c_uint32,
                                C.c_uint64, C.c_uint64, C.c_void_p]),
    "qreg_slab_swap": (C.c_int, [_P(Qreg), _P(Qreg), C.c_uint32,
                                 C.c_uint32, C.c_uint32]),
    "phase2_sharded_new": (C.c_void_p, [C.c_uint32, C.c_uint32,
                                        _P(C.c_uint32), C.c_uint32, C.c_int,
                                        C.c_void_p, C.c_uint64]),
    "phase2_sharded_free": (None, [C.c_void_p]),
    "phase2_sharded_paulirot": (C.c_int, [C.c_void_p, _P(C.c_uint64),
                                          _P(C.c_uint64), _P(C.c_double),
                                          C.c_size_t]),
    "phase2_sharded_prepst": (C.c_int, [C.c_void_p, _P(C.c_uint64),
                                        _P(C.c_double), C.c_size_t]),
    "phase2_sharded_getamps": (C.c_int, [C.c_void_p, _P(C.c_uint64),
                                         _P(C.c_double), C.c_size_t]),
    "phase2_sharded_measure": (C.c_int, [C.c_void_p, _P(C.c_uint64),
                                         _P(C.c_double), C.c_size_t,
                                         _P(C.c_double)]),
    "phase2_sharded_norm2": (C.c_int, [C.c_void_p, _P(C.c_double)]),
    "phase2_sharded_synchronize": (C.c_int, [C.c_void_p]),
    "phase2_sharded_layout": (C.c_int, [C.c_void_p, _P(C.c_uint32)]),
    "phase2_sharded_counters": (None, [C.c_void_p, _P(C.c_uint64),
                                       _P(C.c_uint64)]),
    "qreg_inner_dense": (C.c_int, [_P(Qreg), _P(C.c_double),
                                   _P(C.c_double)]),
    "qreg_get_stats": (C.c_int, [_P(Qreg), _P(Stats)]),
    "qreg_reset_stats": (None, [_P(Qreg)]),
    "qreg_set_timing": (C.c_int, [_P(Qreg), C.c_int]),
    "qreg_stream": (C.c_void_p, [_P(Qreg)]),
    "circ_hamil_init": (C.c_int, [_P(CircHamil), C.c_uint32, C.c_size_t]),
    "circ_hamil_free": (None, [_P(CircHamil)]),
    "circ_hamil_sort_lex": (None, [_P(CircHamil)]),
    "circ_hamil_sort_flip": (None, [_P(CircHamil)]),
    "circ_muldet_init": (C.c_int, [_P(CircMuldet), C.c_size_t]),
    "circ_muldet_free": (None, [_P(CircMuldet)]),
    "circ_values_init": (C.c_int, [_P(CircValues), C.c_size_t]),
    "circ_values_free": (None, [_P(CircValues)]),
    "circ_init": (C.c_int, [_P(Circ), CircHamil, C.c_int, C.c_void_p,
                            C.c_size_t]),
    "circ_free": (None, [_P(Circ)]),
    "circ_prepst": (C.c_int, [_P(Circ)]),
    "circ_step": (C.c_int, [_P(Circ), _P(CircHamil), C.c_double]),
    "circ_step_reverse": (C.c_int, [_P(Circ), _P(CircHamil), C.c_double]),
    "circ_measure": (Complex, [_P(Circ)]),
    "trott_init": (C.c_int, [_P(Trott), _P(TrottData), CircHamil, C.c_int,
                             C.c_void_p, C.c_void_p]),
    "trott_free": (None, [_P(Trott)]),
    "trott_simul": (C.c_int, [_P(Trott)]),
    "trott2_init": (C.c_int, [_P(Trott2), _P(TrottData), CircHamil,
                              C.c_int, C.c_void_p, C.c_void_p]),
    "trott2_free": (None, [_P(Trott2)]),
    "trott2_simul": (C.c_int, [_P(Trott2)]),
    "qdrift_init": (C.c_int, [_P(Qdrift), _P(QdriftData), CircHamil,
                              C.c_int, C.c_void_p, C.c_void_p]),
    "qdrift_free": (None, [_P(Qdrift)]),
    "qdrift_simul": (C.c_int, [_P(Qdrift)]),
    "cmpsit_init": (C.c_int, [_P(Cmpsit), _P(CmpsitData), CircHamil,
                              C.c_int, C.c_void_p, C.c_void_p]),
    "cmpsit_free": (None, [_P(Cmpsit)]),
    "cmpsit_simul": (C.c_int, [_P(Cmpsit)]),
    "cmpsit_ranct_init": (C.c_int, [_P(CmpsitRanct), _P(CircHamil),
                                    _P(CmpsitData)]),
    "cmpsit_ranct_free": (None, [_P(CmpsitRanct)]),
    "phase2_sharded_trott": (C.c_int, [C.c_void_p, _P(CircHamil),
                                       _P(CircMuldet), C.c_size_t,
                                       C.c_double, C.c_int, _P(C.c_double)]),
    "phase2_sharded_qdrift": (C.c_int, [C.c_void_p, _P(CircHamil),
                                        _P(CircMuldet), C.c_size_t,
                                        C.c_size_t, C.c_double, C.c_uint64,
                                        _P(C.c_double)]),
    "phase2_sharded_cmpsit": (C.c_int, [C.c_void_p, _P(CircHamil),
                                        _P(CircMuldet), _P(CmpsitData),
                                        _P(C.c_double)]),
    "prob_cdf_init": (C.c_int, [_P(ProbCdf), C.c_size_t]),
    "prob_cdf_free": (None, [_P(ProbCdf)]),
    "prob_cdf_from_array_strided": (C.c_int, [_P(ProbCdf), _P(C.c_double),
                                              C.c_size_t, _P(C.c_double)]),
    "prob_cdf_inverse": (C.c_size_t, [_P(ProbCdf), C.c_double]),
    "xoshiro256ss_init": (None, [_P(Xoshiro), C.c_uint64]),
    "xoshiro256ss_next": (C.c_uint64, [_P(Xoshiro)]),
    "xoshiro256ss_jump": (None, [_P(Xoshiro)]),
    "xoshiro256ss_longjump": (None, [_P(Xoshiro)]),
    "circ_cache_init": (C.c_void_p, [C.c_int, C.c_int]),
    "circ_cache_free": (None, [C.c_void_p]),
    "circ_cache_insert": (C.c_int, [C.c_void_p, Paulis, C.c_double]),
    "circ_cache_len": (C.c_size_t, [C.c_void_p]),
    "phase2_run": (C.c_int, [_P(C.c_char_p), _P(C.c_double), C.c_size_t,
                             C.c_double, C.c_char_p, _P(C.c_double),
                             _P(C.c_double)]),
    "phase2_set_precision": (C.c_int, [C.c_int]),
    "phase2_get_precision": (C.c_int, []),
    "phase2_set_fp32_form": (C.c_int, [C.c_int]),
    "phase2_set_batch_persistent": (C.c_int, [C.c_int]),
    "phase2_set_batch_runs": (C.c_int, [C.c_uint]),
    "phase2_get_batch_runs": (C.c_uint, []),
    "phase2_set_device_sampling": (C.c_int, [C.c_int]),
    "phase2_set_sweep": (C.c_int, [C.c_int, C.c_int]),
    "phase2_get_sweep": (None, [C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "phase2_set_sweep_kernel": (C.c_int, [C.c_int]),
    "state_prep_coeff_scratch_init": (C.c_int, [C.c_void_p, C.c_uint32,
                                                C.c_uint32, C.c_uint32]),
    "state_prep_coeff_scratch_free": (None, [C.c_void_p]),
    "state_prep_coeff_expand_all": (C.c_int, [C.c_void_p, C.c_void_p,
                                              C.c_void_p]),
    "state_prep_coeff_expand": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_double, C.c_int,
                                          C.c_int]),
    "state_prep_coeff_inner": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_double, C.c_int,
                                         C.c_void_p]),
    "data_coeff_matrix_free": (None, [C.c_void_p]),
    "phase2_get_fp32_form": (C.c_int, []),
    "phase2_set_fusion": (C.c_int, [C.c_int, C.c_int]),
    "phase2_set_term_order": (C.c_int, [C.c_int]),
    "phase2_get_term_order": (C.c_int, []),
    "phase2_plan": (C.c_long, [C.c_uint32, _P(RotIn), C.c_size_t, C.c_int,
                               C.c_int, C.c_int, _P(Pass), _P(RotRec)]),
    "phase2_norm2_noalloc": (C.c_int, [C.c_void_p, C.c_int, C.c_uint64,
                                       C.c_void_p, C.c_void_p]),
    "trott_simul_batch": (C.c_int, [_P(C.c_void_p), C.c_size_t]),
    "trott2_simul_batch": (C.c_int, [_P(C.c_void_p), C.c_size_t]),
    "qdrift_simul_batch": (C.c_int, [_P(C.c_void_p), C.c_size_t]),
    "cmpsit_simul_batch": (C.c_int, [_P(C.c_void_p), C.c_size_t]),
    "phase2_tune_set": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int]),
    "phase2_load_tuning": (C.c_int, [C.c_char_p, C.c_char_p]),
    "phase2_batch_finish_ms": (C.c_size_t, [_P(C.c_double), C.c_size_t]),
    "phase2_batch_wait_check": (C.c_int, [C.c_uint]),
    "phase2_tune_get": (C.c_int, [C.c_int, C.c_int, _P(C.c_int),
                                  _P(C.c_int)]),
    "phase2_version": (C.c_char_p, []),
    "phase2_sizeof": (C.c_size_t, [C.c_int]),
}

_LIB = None


def lib() -> C.CDLL:
    """Load the in-tree libphase2.so (once) and declare its signatures."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.environ.get("PHASE2_B200_LIB") or str(LIB_PATH)
    if not Path(path).is_file():
        raise RuntimeError(
            f"libphase2.so not found at {path}; build it with "
            "`make -C phase2_b200/csrc` (there is no fallback)")
    L = C.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def check_layout() -> dict:
    """Return {id: (python size, C size)} for every mirrored struct."""
    L = lib()
    return {k: (C.sizeof(v), int(L.phase2_sizeof(k)))
            for k, v in LAYOUT.items()}
