"""Autotuner for the pass kernel launch table, the fusion cap and the
persistent batch kernel's run length.

For each state precision and span M (amplitudes per thread = 2^M) it times
passes of the kernel variants (FP64: direct loads / shared-memory prefetch;
FP32: the lifted kernel of the current FP32 form) at several grid densities
on probe rotations whose flip masks span exactly M dimensions, then keeps
the fastest.  It then compares fusion caps
(max_span 4 vs 5) on a stream of qDRIFT-like draws, by rotations per second.

FP32 passes: the grid density is tuned on the FP32-arithmetic kernel
(one variant), then, at that density, the FP64-arithmetic form's variants
(0 direct loads, 1 bulk-copy staging, 2 cp.async staging, 3 the same in
a build for two blocks per SM) are compared;
the entry keeps both choices (the variant only steers the FP64-arithmetic
form).

Last, the persistent batch kernel's run length (phase2_set_batch_runs:
runs per warp's share of an op, 1, 2, 4 or 8) is timed on a batch of 16
small trott instances (18-21 qubits, FP32 in the current form) and the
fastest kept.

Results are written as JSON (the full report) and as the flat launch table
the library applies at world_init when the GPU name matches
(``tuning_b200.tab`` beside libphase2.so, ``write_table``; C loader
phase2_load_tuning).  ``apply`` loads a table into the running library
(phase2_tune_set / phase2_set_fusion).  ``python -m phase2_b200.autotune
--nqb 28 --out phase2_b200/tuning_b200.json`` runs a sweep on the current
GPU and writes both files.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import time
from pathlib import Path

import numpy as np

from . import PREC_FP32, PREC_FP64, Register, lib, world_ensure

DEFAULT_FILE = Path(__file__).resolve().parent / "tuning_b200.json"
TABLE_FILE = Path(__file__).resolve().parent / "tuning_b200.tab"
PRECS = {"fp64": PREC_FP64, "fp32": PREC_FP32}
# per precision: variant -> per_sm candidates
GRIDS = {"fp64": {0: [0, 4, 8, 32], 1: [0, 1]},
         "fp32": {0: [0, 8, 16, 32]}}
# FP32 variants of the FP64-arithmetic form, compared at the tuned density
FP32_F64_VARIANTS = (0, 1, 2, 3)
FORM_LIFTED, FORM_LIFTED_F32 = 1, 2


def _probe_rotations(nqb: int, M: int, groups: int, seed: int):
    """`groups` runs of M rotations with independent random flips (2-4
    qubits each) plus one diagonal term: each run plans to one pass of
    span M."""
    rng = np.random.Generator(np.random.PCG64(seed))
    flip, phase = [], []
    for _ in range(groups):
        for _ in range(M):
            k = int(rng.choice([2, 4]))
            q = rng.choice(nqb, size=k, replace=False)
            f = int(sum(1 << int(x) for x in q))
            flip.append(f)
            phase.append(f & int(rng.integers(0, 1 << nqb)))
        flip.append(0)
        phase.append(int(rng.integers(0, 1 << nqb)))
    n = len(flip)
    return (np.array(flip, dtype=np.uint64), np.array(phase, dtype=np.uint64),
            rng.uniform(-0.3, 0.3, n))


def _time_passes(reg: Register, flip, phase, phi) -> tuple[float, int]:
    reg.reset_stats()
    reg.set_timing(True)
    reg.paulirot(flip, phase, phi)
    reg.synchronize()
    st = reg.stats()
    reg.set_timing(False)
    return st["pass_ms"] / max(1, st["timed_passes"]), st["passes"]


def sweep_launch(nqb: int, groups: int = 12, reps: int = 2) -> dict:
    L = lib()
    out: dict = {}
    for pname, prec in PRECS.items():
        out[pname] = {}
        elem = 16 if prec == PREC_FP64 else 8
        with Register(nqb, prec) as reg:
            for M in range(1, 6):
                reg.set_fusion(M, 0)
                flip, phase, phi = _probe_rotations(nqb, M, groups, 7 + M)
                best = None
                trials = []
                for variant, grids in GRIDS[pname].items():
                    for per_sm in grids:
                        L.phase2_tune_set(prec, M, variant, per_sm)
                        _time_passes(reg, flip[:M + 1], phase[:M + 1],
                                     phi[:M + 1])  # warm
                        ms = min(_time_passes(reg, flip, phase, phi)[0]
                                 for _ in range(reps))
                        gbs = 2 * (1 << nqb) * elem / (ms * 1e-3) / 1e9
                        trials.append([variant, per_sm, ms * 1e3, gbs])
                        if best is None or ms < best[2] / 1e3:
                            best = [variant, per_sm, ms * 1e3, gbs]
                L.phase2_tune_set(prec, M, best[0], best[1])
                out[pname][str(M)] = {"variant": best[0],
                                      "per_sm": best[1],
                                      "us_per_pass": best[2],
                                      "gbs": best[3], "trials": trials}
                if prec == PREC_FP32 and M >= 3:
                    out[pname][str(M)].update(_fp64_arith_variant(
                        reg, M, best[1], flip, phase, phi, nqb, reps))
    return out


def _fp64_arith_variant(reg, M, per_sm, flip, phase, phi, nqb, reps):
    """The FP64-arithmetic form's kernel variant at the tuned density."""
    L = lib()
    form = L.phase2_get_fp32_form()
    L.phase2_set_fp32_form(FORM_LIFTED)
    trials, best = [], None
    try:
        for variant in FP32_F64_VARIANTS:
            L.phase2_tune_set(PREC_FP32, M, variant, per_sm)
            _time_passes(reg, flip[:M + 1], phase[:M + 1], phi[:M + 1])
            ms = min(_time_passes(reg, flip, phase, phi)[0]
                     for _ in range(reps))
            gbs = 2 * (1 << nqb) * 8 / (ms * 1e-3) / 1e9
            trials.append([variant, per_sm, ms * 1e3, gbs])
            if best is None or ms * 1e3 < best[2]:
                best = trials[-1]
    finally:
        L.phase2_set_fp32_form(form)
    L.phase2_tune_set(PREC_FP32, M, best[0], per_sm)
    return {"variant": best[0], "f64arith_us_per_pass": best[2],
            "f64arith_gbs": best[3], "f64arith_trials": trials}


def sweep_fusion(nqb: int, depth: int = 1024) -> dict:
    """Rotations per second for fusion caps 3..5 on qDRIFT-like draws."""
    from . import workloads
    t = workloads.jw_terms(nqb, 20000, seed=11)
    rng = np.random.Generator(np.random.PCG64(12))
    p = np.abs(t.cf) / np.abs(t.cf).sum()
    pick = rng.choice(len(t), size=depth, p=p)
    flip, phase = t.flip[pick], t.phase[pick]
    phi = np.full(depth, 1e-3)
    out: dict = {}
    for pname, prec in PRECS.items():
        out[pname] = {}
        with Register(nqb, prec) as reg:
            for span in (3, 4, 5):
                reg.set_fusion(span, 0)
                _time_passes(reg, flip[:64], phase[:64], phi[:64])
                ms, passes = _time_passes(reg, flip, phase, phi)
                total_ms = ms * passes
                out[pname][str(span)] = {
                    "passes": passes, "rot_per_pass": depth / passes,
                    "rot_amp_per_s": depth * (1 << nqb) / (total_ms * 1e-3)}
    return out


BATCH_RUNS = (1, 2, 4, 8)


def sweep_batch_runs(ninst: int = 16, reps: int = 2) -> dict:
    """Kernel milliseconds of one persistent launch per run length, on
    `ninst` trott instances of 18-21 qubits (2,000 JW terms, 2 steps,
    FP32 state in the current form); the best of `reps` launches each."""
    from . import batch, set_batch_runs, set_precision, workloads
    g = np.random.Generator(np.random.PCG64(21))
    probs = []
    for k in range(ninst):
        n = int(g.integers(18, 22))
        probs.append(dict(nqb=n, terms=workloads.jw_terms(n, 2000,
                                                          seed=300 + k),
                          dets=workloads.hamming_dets(n, 1, n // 2,
                                                      seed=400 + k),
                          steps=2, delta=0.05))
    before = lib().phase2_get_batch_runs()
    out: dict = {"workload": f"{ninst} trott instances, 18-21 qubits, "
                 "2000 JW terms, 2 steps, FP32", "kernel_ms": {}}
    set_precision(PREC_FP32)
    try:
        for runs in BATCH_RUNS:
            set_batch_runs(runs)
            best = None
            for _ in range(reps + 1):  # the first launch warms up
                _, st = batch("trott", probs, with_stats=True)
                ms = float(sum(s["pass_ms"] for s in st))
                best = ms if best is None or ms < best else best
            out["kernel_ms"][str(runs)] = best
    finally:
        set_batch_runs(before)
        set_precision(PREC_FP64)
    out["best"] = int(min(out["kernel_ms"], key=lambda r:
                          out["kernel_ms"][r]))
    return out


def run(nqb: int) -> dict:
    world_ensure()
    t0 = time.time()
    launch = sweep_launch(nqb)
    fusion = sweep_fusion(nqb)
    runs = sweep_batch_runs()
    best_span = {p: int(max(v, key=lambda s: v[s]["rot_amp_per_s"]))
                 for p, v in fusion.items()}
    import subprocess
    try:
        gpu = subprocess.run(["nvidia-smi", "--query-gpu=name",
                              "--format=csv,noheader"], capture_output=True,
                             text=True).stdout.strip().splitlines()[0]
    except (OSError, IndexError):
        gpu = "unknown"
    return {"gpu": gpu, "nqb": nqb, "seconds": time.time() - t0,
            "launch": launch, "fusion": fusion, "max_span": best_span,
            "batch_runs": runs}


def apply(table: dict | str | Path | None = None, prec: int | None = None):
    """Load a tuning table (dict or JSON path; default the shipped B200
    table) into the library; sets the fusion cap for `prec` (or the FP32
    cap when prec is None and only the launch table otherwise)."""
    if table is None:
        table = DEFAULT_FILE
    if not isinstance(table, dict):
        p = Path(table)
        if not p.is_file():
            return None
        table = json.loads(p.read_text())
    L = lib()
    for pname, per_m in table.get("launch", {}).items():
        pr = PRECS[pname]
        for M, e in per_m.items():
            L.phase2_tune_set(pr, int(M), int(e["variant"]),
                              int(e["per_sm"]))
    if "batch_runs" in table:
        L.phase2_set_batch_runs(int(table["batch_runs"]["best"]))
    if prec is not None:
        pname = "fp32" if prec == PREC_FP32 else "fp64"
        span = table.get("max_span", {}).get(pname)
        if span:
            L.phase2_set_fusion(int(span), 0)
    return table


def write_table(table: dict, path: str | Path = TABLE_FILE) -> None:
    """The flat launch table the library loads at world_init (C loader
    phase2_load_tuning): the GPU name and one line per precision and
    span."""
    lines = ["# phase2 launch table, written by phase2_b200.autotune "
             f"({table.get('nqb', '?')} qubits)",
             f"gpu {table['gpu']}"]
    for pname, per_m in table.get("launch", {}).items():
        for M, e in sorted(per_m.items(), key=lambda kv: int(kv[0])):
            lines.append(f"launch {PRECS[pname]} {int(M)} "
                         f"{int(e['variant'])} {int(e['per_sm'])}")
    if "batch_runs" in table:
        lines.append(f"batch_runs {int(table['batch_runs']['best'])}")
    Path(path).write_text("\n".join(lines) + "\n")


def probe(nqb: int, pname: str, M: int, variant: int, per_sm: int,
          groups: int) -> dict:
    """Time `groups` passes of span M with a fixed launch choice (for
    targeted profiler captures)."""
    world_ensure()
    prec = PRECS[pname]
    lib().phase2_tune_set(prec, M, variant, per_sm)
    flip, phase, phi = _probe_rotations(nqb, M, groups, 7 + M)
    elem = 16 if prec == PREC_FP64 else 8
    with Register(nqb, prec) as reg:
        reg.set_fusion(M, 0)
        _time_passes(reg, flip[:M + 1], phase[:M + 1], phi[:M + 1])
        ms, passes = _time_passes(reg, flip, phase, phi)
    return {"prec": pname, "M": M, "variant": variant, "per_sm": per_sm,
            "passes": passes, "us_per_pass": ms * 1e3,
            "gbs": 2 * (1 << nqb) * elem / (ms * 1e-3) / 1e9}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--nqb", type=int, default=28)
    ap.add_argument("--out", default=str(DEFAULT_FILE))
    ap.add_argument("--probe", nargs=4, metavar=("PREC", "M", "VARIANT",
                                                 "PER_SM"))
    ap.add_argument("--groups", type=int, default=8)
    args = ap.parse_args()
    if args.probe:
        p = args.probe
        print(json.dumps(probe(args.nqb, p[0], int(p[1]), int(p[2]),
                               int(p[3]), args.groups)))
        return
    res = run(args.nqb)
    Path(args.out).write_text(json.dumps(res, indent=1))
    write_table(res, Path(args.out).with_suffix(".tab"))
    for pname in PRECS:
        for M, e in res["launch"][pname].items():
            print(f"{pname} M={M}: variant={e['variant']} "
                  f"per_sm={e['per_sm']} {e['us_per_pass']:.1f} us/pass "
                  f"{e['gbs']:.0f} GB/s")
        print(pname, "fusion", json.dumps(res["fusion"][pname]))
    print("batch_runs", json.dumps(res["batch_runs"]))
    print("max_span", res["max_span"], f"({res['seconds']:.0f} s)")


if __name__ == "__main__":
    main()
