"""numpy execution of planned passes (TEST INFRASTRUCTURE).

Applies the pass descriptors and rotation records produced by
phase2_plan exactly as the device kernel interprets them: each
representative x (zeros at the pivots) owns the slots x ^ off(u), and
rotation r updates slot u as
    a_u <- c a_u + (-1)^sigma_u s (odd ? i : 1) a_{u ^ U},
    sigma_u = bit u of (smask ^ -parity(x & z)).
Products and sums are rounded separately (numpy never fuses), as the
FP64 kernel does with __dmul_rn/__dadd_rn, so results must match the
oracle bit for bit.  Lifted records (FP32 state) are executed in FP64 here
and agree with the oracle to FP64 rounding.
"""

import numpy as np


def _parity(v: np.ndarray) -> np.ndarray:
    v = v.copy()
    for sh in (32, 16, 8, 4, 2, 1):
        v ^= v >> np.uint64(sh)
    return (v & np.uint64(1)).astype(np.int64)


def _lifted(R, I, M, U, odd, t, s, sm):
    """Form 1 in place: per pair (u, w = u ^ U) with q_u = sigma_u (i if
    odd), q_w = -conj(q_u): y_u += t q_u y_w; y_w += s q_w y_u;
    y_u += t q_u y_w.  U = 0 multiplies by c + s q_u, c = 1 - t s."""
    H = U.bit_length() - 1
    for u in range(1 << M):
        if U and (u >> H) & 1:
            continue
        sig = np.where((sm >> u) & 1, -1.0, 1.0)
        qu = sig * (1j if odd else 1.0)
        yu = R[:, u] + 1j * I[:, u]
        if U == 0:
            yu = yu * ((1.0 - t * s) + s * qu)
            R[:, u], I[:, u] = yu.real, yu.imag
            continue
        w = u ^ U
        qw = -np.conj(qu)
        yw = R[:, w] + 1j * I[:, w]
        yu = yu + t * qu * yw
        yw = yw + s * qw * yu
        yu = yu + t * qu * yw
        R[:, u], I[:, u] = yu.real, yu.imag
        R[:, w], I[:, w] = yw.real, yw.imag


def emulate(amp: np.ndarray, nqb: int, passes, recs) -> np.ndarray:
    a = np.array(amp, dtype=np.complex128)
    re, im = a.real.copy(), a.imag.copy()
    for p in passes:
        M = p["span"]
        x = np.arange(1 << (nqb - M), dtype=np.uint64)
        for q in p["piv"]:
            q = np.uint64(q)
            low = x & ((np.uint64(1) << q) - np.uint64(1))
            x = ((x >> q) << (q + np.uint64(1))) | low
        offs = []
        for u in range(1 << M):
            o = 0
            for k in range(M):
                if u >> k & 1:
                    o ^= int(p["basis"][k])
            offs.append(o)
        idx = x[:, None] ^ np.array(offs, dtype=np.uint64)[None, :]
        R, I = re[idx], im[idx]
        for r in recs[p["rot_off"]:p["rot_off"] + p["nrot"]]:
            px = _parity(x & np.uint64(r["z"]))
            sm = (np.int64(r["smask"]) ^ (-px)) & 0xFFFFFFFF
            c, s, U, odd = r["c"], r["s"], r["U"], r["odd"]
            form = r.get("form", 0)
            nR, nI = R.copy(), I.copy()
            if form == 1:
                _lifted(nR, nI, M, U, odd, c, s, sm)
            else:
                for u in range(1 << M):
                    w = u ^ U
                    sig = np.where((sm >> u) & 1, -1.0, 1.0)
                    pr, pi = (-I[:, w], R[:, w]) if odd else (R[:, w], I[:, w])
                    su = sig * s
                    nR[:, u] = c * R[:, u] + su * pr
                    nI[:, u] = c * I[:, u] + su * pi
            R, I = nR, nI
        if p.get("form", 0) != 0:
            R, I = R * p["scale"], I * p["scale"]
        re[idx], im[idx] = R, I
    return re + 1j * im
