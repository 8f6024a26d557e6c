"""Exact rotation on a sparse state (TEST INFRASTRUCTURE).

For registers too large for the dense oracle, a state that starts on a few
basis vectors stays sparse under a few rotations.  This applies
exp(+i phi P) to a dict {index: complex} with the reference's rounding
(products and sums rounded separately, phase2/qreg_qreg.c:149-160), so
the device's FP64 amplitudes must match it bit for bit at any width.
"""

import math


def _popc(v: int) -> int:
    return bin(v).count("1")


def _mul_ipow(s: float, k: int, re: float, im: float):
    k &= 3
    if k == 0:
        return s * re, s * im
    if k == 1:
        return -(s * im), s * re
    if k == 2:
        return -(s * re), -(s * im)
    return s * im, -(s * re)


def rotate(state: dict, flip: int, phase: int, phi: float) -> dict:
    c, s = math.cos(phi), math.sin(phi)
    ny = _popc(flip & phase)
    out = dict(state)
    done = set()
    for g in list(state.keys()):
        lo = min(g, g ^ flip)
        if lo in done:
            continue
        done.add(lo)
        hi = lo ^ flip
        a = state.get(lo, 0j)
        b = state.get(hi, 0j)
        r4 = (ny + 2 * _popc(lo & phase)) & 3
        tr, ti = _mul_ipow(s, 1 - r4, b.real, b.imag)
        out[lo] = complex(c * a.real + tr, c * a.imag + ti)
        if hi != lo:
            ur, ui = _mul_ipow(s, 1 + r4, a.real, a.imag)
            out[hi] = complex(c * b.real + ur, c * b.imag + ui)
    return out
