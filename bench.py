"""Benchmark of the phase2 state-vector hot path on B200.

Metric: Pauli-rotation x amplitudes per second (and HBM GB/s) at 30 qubits,
FP32 state ("FP32-batched": fused passes) against the FP64 path, on the
qDRIFT workload: 30 qubits, 100,000 Jordan-Wigner-like terms (seeded
synthetic, phase2_b200.workloads), 4096 draws per sample, step_size 1e-3.
The headline runs the library's FP32 form (--fp32-form; the line's
``fp32_form`` and ``storage`` say what it computes).  The line also
carries comparison arms on the same draws -- FP64 one rotation per pass
("plain"), FP64 fused, FP32 one rotation per pass, and the three FP32
forms fused (FP32 arithmetic with FP32 coefficients; FP64 arithmetic with
FP64 coefficients and one rounding per pass; FP32 arithmetic with FP64 on
the cosets that hold an amplitude >= 2^-10) -- with each FP32 form's
ratio to the fused FP64 path (like for like) and the headline's ratio to
the plain FP64 path, the reference's own CUDA kernel built from its
sources, the FP32 error of every form on the headline samples and on a
1000-step Trotter run, and, at N=1, studies within a time budget (--studies,
--study-budget): the 26-qubit second-order Trotter configuration over
all 256 steps with the FP32 error after every step, the batched
configuration (64 uneven instances in one persistent launch, with finish
times), the 33-qubit composite configuration and sharded registers.

A step is one qDRIFT sample through the library's C-ABI driver
(qdrift_simul): state prep, 4096 rotations, overlap.  ``value`` is timed
with CUDA events recorded on the register's own stream; ``e2e`` is the same
steps timed around the host call (host-side sampling and planning, record
upload, overlap download included).  The 8 GiB state is larger than L2, so
no L2 flush is needed between steps.

Multi-GPU (torchrun): each rank runs independent qDRIFT samples of its own
seed on its own GPU (replicas, weak scaling); no data-path collective.
Timing is the max over ranks.

``cpu_baseline`` and ``--impl reference`` time the reference's own CPU
path: its qdrift driver (oracle/_ref/ref_mpi, built from the reference
sources) on the same workload as R MPI ranks of one job on the host cores,
each step a sample truncated to a few draws (the metric is a rate).
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = ("Pauli-rot·amplitudes/s and HBM GB/s at 30 qb: FP32-batched "
          "vs FP64 plain")
UNIT = "rot·amp/s"


def _peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.is_file():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class Clocks:
    """Samples nvidia-smi every 200 ms while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,"
         "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev: int):
        self.dev = dev
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _max_over_ranks(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(ws: int) -> None:
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ---- the GPU arm -------------------------------------------------------


def _qdrift_obj(p2, cfg, prec, fusion, seed):
    """Build a one-sample qDRIFT driver through the C-ABI."""
    from phase2_b200 import _ffi
    L = p2.lib()
    p2.set_precision(prec)
    hm, md = p2._hamil(cfg["nqb"], cfg["terms"]), p2._muldet(cfg["dets"])
    obj = _ffi.Qdrift()
    dt = _ffi.QdriftData(1, cfg["depth"], cfg["step_size"], seed)
    if L.qdrift_init(C.byref(obj), C.byref(dt), hm, _ffi.STPREP_MULTIDET,
                     C.cast(C.pointer(md), C.c_void_p), None) != 0:
        raise RuntimeError("qdrift_init failed")
    L.qreg_set_fusion(C.byref(obj.ct.reg), *fusion)
    return obj


def _run_steps(p2, obj, steps: int, timing: bool):
    """Run `steps` samples; return (device_ms, wall_s, stats delta, z)."""
    import torch
    L = p2.lib()
    reg = C.byref(obj.ct.reg)
    L.qreg_set_timing(reg, int(timing))
    stream = torch.cuda.ExternalStream(L.qreg_stream(reg))
    L.qreg_reset_stats(reg)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    ev0.record(stream)
    zs = []
    for _ in range(steps):
        if L.qdrift_simul(C.byref(obj)) != 0:
            raise RuntimeError("qdrift_simul failed")
        zs.append(complex(obj.ct.vals.z[0], obj.ct.vals.z[1]))
    ev1.record(stream)
    ev1.synchronize()
    wall = time.perf_counter() - w0
    st = _ffi_stats(p2, obj)
    return ev0.elapsed_time(ev1), wall, st, zs


def _ffi_stats(p2, obj):
    from phase2_b200 import _ffi
    st = _ffi.Stats()
    p2.lib().qreg_get_stats(C.byref(obj.ct.reg), C.byref(st))
    return {k: getattr(st, k) for k, _ in _ffi.Stats._fields_}


# what the headline FP32 form computes, for the line's "storage" key
STORAGE = {
    2: ("complex64 state; each pair rotated by three shears in FP32 FMAs "
        "whose coefficients s and t = tan(phi/2) are computed in FP64 and "
        "rounded to FP32 (planner); norms and overlaps in FP64"),
    1: ("complex64 state; each pass widens its amplitudes to FP64, applies "
        "all its rotations in FP64 arithmetic with the FP64 coefficients "
        "(s and t = tan(phi/2) from FP64 cos/sin), and rounds to FP32 once "
        "at the store; norms and overlaps in FP64"),
    3: ("complex64 state; cosets whose amplitudes are all below 2^-10 in "
        "magnitude rotated as form 2 (FP32 FMAs, coefficients rounded to "
        "FP32), cosets holding a larger amplitude rotated in FP64 "
        "arithmetic by their warp and rounded to FP32 once per pass; norms "
        "and overlaps in FP64"),
}
FORM_NAME = {1: "f64 arithmetic (PHASE2_FORM_LIFTED)",
             2: "f32 arithmetic (PHASE2_FORM_LIFTED_F32)",
             3: "f32 arithmetic, f64 on heavy cosets (PHASE2_FORM_LIFTED_MIXED)"}


def _headline_kernel(p2, form: int) -> str:
    """The pass kernel that carries the headline's span-5 passes."""
    if form == p2.FORM_LIFTED_F32:
        return "k_pass_lift32<M,uint32_t>"
    if form == p2.FORM_LIFTED_MIXED:
        return "k_pass_lift32h<M,uint32_t>"
    v, per = C.c_int(), C.c_int()
    p2.lib().phase2_tune_get(p2.PREC_FP32, 5, C.byref(v), C.byref(per))
    return {0: "k_pass_lift<M,uint32_t>", 1: "k_pass_lift_bulk<M>",
            2: "k_pass_lift_pf<M,3>", 3: "k_pass_lift_pf<M,2>"}[v.value]


def _traffic_per_launch(kernel: str):
    """ncu DRAM bytes of one 30-qubit launch of the kernel (profiles/,
    scaled from a 26-qubit capture), or None without a capture."""
    name = kernel.split("<")[0]
    p = ROOT / "profiles" / f"{name}_traffic.json"
    if p.is_file():
        try:
            return json.loads(p.read_text()).get("bytes_per_launch_30q_fp32")
        except (ValueError, KeyError):
            return None
    return None


def _reference_gpu(nqb: int, nrot: int = 16, reps: int = 3):
    """The reference's own CUDA backend (phase2/qreg_cuda_lo.cu: one thread
    per amplitude, two kernelPauliRot launches per rotation for its amp and
    buf slabs, plus the mix/add/exchange of a flush), compiled from its
    sources for sm_100a (oracle/Makefile ref-cuda) and timed with the same
    driver as the CPU baseline: one flush of nrot JW-like rotations on an
    nqb-qubit FP64 register, min of reps, device-synchronised."""
    exe = ROOT / "oracle" / "_ref" / "ref_bench_cuda"
    if not exe.is_file():
        return None
    try:
        out = subprocess.run([str(exe), str(nqb), str(nrot), str(reps)],
                             capture_output=True, text=True, timeout=600)
        best, rate = out.stdout.split()[-2:]
    except (subprocess.SubprocessError, ValueError, OSError):
        return None
    namp = 1 << nqb
    return {"value": float(rate), "unit": UNIT, "rotations": nrot,
            "seconds_per_flush": float(best),
            "kernel_gbs_effective": nrot * 2 * namp * 16 / float(best) / 1e9,
            "what": ("reference CUDA backend, FP64, one flush of "
                     f"{nrot} rotations at {nqb} qubits")}


def _config(cfg: dict) -> dict:
    """The workload both arms report (the same dict in each line)."""
    return {"workload": (f"qdrift {cfg['nqb']} qubits, {len(cfg['terms'])} "
                         f"JW terms, {cfg['depth']} draws per sample"),
            "nqb": cfg["nqb"], "terms": len(cfg["terms"]),
            "depth": cfg["depth"],
            "step": "one qDRIFT sample: prepst + rotations + overlap"}


# CPU baseline: the reference's own qdrift driver on the headline
# workload, as R ranks of one job on the host cores
CPU_DEPTH = 4    # draws per timed sample (of the workload's 4096)
CPU_REPS = 3     # min of K, the reference's convention (bench/bench.h)


def _cpu_ranks() -> int:
    cores = os.cpu_count() or 1
    return 1 << int(math.log2(max(1, min(cores, 256))))


def _cpu_reference(cfg: dict, depth: int, reps: int, warmup: int,
                   ranks: int | None = None) -> dict:
    """The reference's qdrift_simul (phase2/circ/qdrift.c, CPU backend,
    built from its sources with its release optimisation) on the
    headline's Hamiltonian, determinant, step size and seed, as R MPI ranks
    of one job on this host's cores (oracle/_ref/ref_mpi over the
    shared-memory MPI stand-in), each holding its 2^(n - log2 R)
    amplitudes as the reference distributes them; one sample per run,
    truncated to `depth` of its draws (prepst, draws, rotations with their
    slab exchanges, overlap), min over `reps` runs after `warmup`."""
    import tempfile

    from oracle import REF_MPI, run_ref_mpi, write_ref_input
    nqb = cfg["nqb"]
    R = ranks or _cpu_ranks()
    base = {"unit": UNIT, "cores": R, "kind": "reference"}
    if not REF_MPI.is_file():
        return dict(base, value=None, sample=(
            "oracle/_ref/ref_mpi not built (reference sources absent at "
            "build time)"))
    t, d = cfg["terms"], cfg["dets"]
    with tempfile.TemporaryDirectory() as tmp:
        path = Path(tmp) / "qdrift.in"
        write_ref_input(path, "qdrift", nqb, t.flip, t.phase, t.cf, d.idx,
                        d.cf, depth, cfg["step_size"], cfg["seed"])
        r = run_ref_mpi(R, path, reps, warmup=warmup, timeout=3600)
    return dict(base, value=r["rot_amp_s"], seconds_per_sample=r["seconds"],
                rotations_per_sample=r["rotations"], sample=(
                    f"reference qdrift_simul, CPU backend (-O3, AVX2/FMA), "
                    f"as {R} MPI ranks of one job on {R} host cores "
                    f"(shared-memory MPI stand-in, "
                    f"{'mailbox' if r['mailbox'] else 'single-copy'} slab "
                    f"exchange), on the {nqb}-qubit headline workload "
                    f"({len(t.cf)} JW terms, same determinant, step size "
                    f"and seed): one sample truncated to {depth} of its "
                    f"{cfg['depth']} draws (prepst, draws, rotations, "
                    f"overlap), min of {reps} runs after {warmup} warm-up"))


def gpu_arm(args) -> None:
    ws, rank, local = _dist()
    import torch
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(
            seconds=300))
    import phase2_b200 as p2
    from phase2_b200 import workloads
    p2.world_ensure()
    if args.fp32_form:
        p2.set_fp32_form({"f32": p2.FORM_LIFTED_F32,
                          "f64": p2.FORM_LIFTED,
                          "mixed": p2.FORM_LIFTED_MIXED}[args.fp32_form])
    if args.lift_kernel:
        # FP64-arithmetic passes of span 3-5: direct loads, or the next
        # cosets staged by bulk copies or by cp.async
        v = {"direct": 0, "bulk": 1, "staged": 2,
             "staged2": 3}[args.lift_kernel]
        for span in (3, 4, 5):
            p2.lib().phase2_tune_set(p2.PREC_FP32, span, v, 32)
    head_form = p2.get_fp32_form()
    cfg = workloads.qdrift30(nqb=args.nqb, depth=args.depth)
    nqb, depth = cfg["nqb"], cfg["depth"]
    namp = 1 << nqb
    seed = cfg["seed"] + 1000003 * rank

    # headline: FP32 state, fused passes
    obj = _qdrift_obj(p2, cfg, p2.PREC_FP32, (5, 0), seed)
    try:
        _run_steps(p2, obj, args.warmup, timing=False)
        _barrier(ws)
        torch.cuda.synchronize()
        with Clocks(local) as clk:
            dev_ms, wall, st, zs = _run_steps(p2, obj, args.steps,
                                              timing=False)
        _barrier(ws)
        # per-launch kernel timing in a separate, untimed step
        _, _, st_t, _ = _run_steps(p2, obj, 1, timing=True)
    finally:
        p2.lib().qdrift_free(C.byref(obj))
    dev_ms = _max_over_ranks(dev_ms, ws)
    wall = _max_over_ranks(wall, ws)
    rot_amp = args.steps * depth * namp
    value = ws * rot_amp / (dev_ms / 1e3)
    e2e_value = ws * rot_amp / wall

    # comparison arms on a bounded number of rotations (same sample shape)
    cmp_depth = max(64, min(depth, args.cmp_depth))
    cmp_cfg = dict(cfg, depth=cmp_depth)
    arms = {}
    form0 = p2.get_fp32_form()
    for name, prec, fusion, form in (
            ("fp64_plain", p2.PREC_FP64, (1, 1), form0),
            ("fp64_fused", p2.PREC_FP64, (5, 0), form0),
            ("fp32_plain", p2.PREC_FP32, (1, 1), form0),
            ("fp32_fused_f32arith", p2.PREC_FP32, (5, 0),
             p2.FORM_LIFTED_F32),
            ("fp32_fused_f64arith", p2.PREC_FP32, (5, 0), p2.FORM_LIFTED),
            ("fp32_fused_mixed", p2.PREC_FP32, (5, 0),
             p2.FORM_LIFTED_MIXED)):
        if args.quick and name != "fp64_plain":
            continue
        p2.set_fp32_form(form)
        o = _qdrift_obj(p2, cmp_cfg, prec, fusion, seed + 7)
        try:
            _run_steps(p2, o, 1, timing=False)
            ms, _, s, _ = _run_steps(p2, o, 1, timing=True)
        finally:
            p2.lib().qdrift_free(C.byref(o))
            p2.set_fp32_form(form0)
        ms = _max_over_ranks(ms, ws)
        elem = 16 if prec == p2.PREC_FP64 else 8
        arms[name] = {
            "value": ws * cmp_depth * namp / (ms / 1e3), "unit": UNIT,
            "rotations": cmp_depth,
            "passes": s["passes"],
            "kernel_gbs": (s["sweeps"] * 2 * namp * elem / 1e9) /
            (s["pass_ms"] / 1e3) if s["pass_ms"] else None}
    p2.set_precision(p2.PREC_FP64)
    if rank == 0 and not args.quick:
        ref_gpu = _reference_gpu(nqb)
        if ref_gpu:
            arms["reference_gpu_fp64"] = ref_gpu
    ratios = {}
    if arms.get("fp64_fused"):
        for name in ("fp32_fused_f32arith", "fp32_fused_f64arith",
                     "fp32_fused_mixed"):
            if arms.get(name):
                ratios[f"{name}_vs_fp64_fused"] = (
                    arms[name]["value"] / arms["fp64_fused"]["value"])
    if arms.get("fp64_plain"):
        ratios["headline_vs_fp64_plain"] = value / arms["fp64_plain"]["value"]

    peaks = _peaks()
    passes_per_step = st["passes"] / args.steps
    # one state round trip per pass kernel (or per sweep kernel when
    # sweeps are on): the unit the roofline bytes are counted in
    trips_per_step = st["sweeps"] / args.steps
    launch_ms = st_t["pass_ms"] / max(1, st_t["timed_sweeps"])
    bytes_per_launch = 2 * namp * 8
    achieved = bytes_per_launch / (launch_ms / 1e3) / 1e9
    hbm_gbs_step = trips_per_step * bytes_per_launch / (
        dev_ms / args.steps / 1e3) / 1e9
    kernel = _headline_kernel(p2, head_form)
    solo = ws == 1 and rank == 0 and not args.quick
    cpu = _cpu_reference(cfg, CPU_DEPTH, CPU_REPS, 1) if solo else None
    extra = {}
    if solo:
        t_studies = time.perf_counter()
        extra["fp32_error"] = {"headline_samples": qdrift_error_study(
            cfg, seed + 11, samples=4)}
        for fname, form in (("f32_arith", p2.FORM_LIFTED_F32),
                            ("f64_arith", p2.FORM_LIFTED),
                            ("mixed", p2.FORM_LIFTED_MIXED)):
            p2.set_fp32_form(form)
            try:
                extra["fp32_error"][fname] = fp32_error_study()
            finally:
                p2.set_fp32_form(form0)
        studies = args.studies.split(",") if args.studies else []
        for name in STUDY_ORDER:
            if name not in studies:
                continue
            left = args.study_budget - (time.perf_counter() - t_studies)
            need = STUDY_SECONDS.get(name, 60)
            if left < need:
                extra[name] = {"skipped": (
                    f"study budget: {left:.0f} s left of "
                    f"{args.study_budget:.0f} s, the study takes about "
                    f"{need:.0f} s (--study-budget)")}
                continue
            # a study that fails is reported in its slot; the bench line
            # itself still prints
            try:
                extra[name] = globals()[f"{name}_study"]()
            except Exception as e:  # noqa: BLE001
                extra[name] = {"error": f"{type(e).__name__}: {e}"}
        extra["study_seconds"] = time.perf_counter() - t_studies
    if rank != 0:
        return
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "storage": STORAGE[head_form],
        "data": "synthetic (seeded JW-like Hamiltonian, no dataset)",
        "config": _config(cfg),
        "fp32_form": FORM_NAME[head_form],
        "l2": f"inputs larger than L2 ({namp * 8 / 2**30:.1f} GiB state)",
        "parallelism": f"replicas x{ws} (independent samples)",
        "hbm_gbs": hbm_gbs_step,
        "passes_per_step": passes_per_step,
        "rotations_per_pass": depth / passes_per_step,
        "roofline": {"bound": "hbm", "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"],
                     "peak_source": peaks["source"],
                     "kernel": kernel,
                     "bytes_per_launch": bytes_per_launch,
                     "launch_ms": launch_ms,
                     "traffic": _traffic_per_launch(kernel)},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": st["h2d_bytes"] / args.steps,
                "d2h_bytes_per_step": st["d2h_bytes"] / args.steps},
        "gpu_launches": st["launches"],
        "clocks": clocks,
        "comparison": arms,
        "ratios": ratios,
        "overlaps": [[z.real, z.imag] for z in zs[:2]],
        **extra,
    }
    print(json.dumps(line), flush=True)


def qdrift_error_study(cfg: dict, seed: int, samples: int = 4) -> dict:
    """FP32 error on the headline workload itself: `samples` qDRIFT samples
    of the 30-qubit configuration run in FP64 and in each FP32 form from
    the same seed (the same draws), the error of every sample's overlap
    against the FP64 one (the FP64 path is bit-identical to the reference,
    tests/test_wide_parity_gpu.py)."""
    import numpy as np

    import phase2_b200 as p2
    t, d = cfg["terms"], cfg["dets"]
    form0 = p2.get_fp32_form()
    zs, secs = {}, {}
    try:
        for name, prec, form in (("fp64", p2.PREC_FP64, form0),
                                 ("f32_arith", p2.PREC_FP32,
                                  p2.FORM_LIFTED_F32),
                                 ("f64_arith", p2.PREC_FP32,
                                  p2.FORM_LIFTED),
                                 ("mixed", p2.PREC_FP32,
                                  p2.FORM_LIFTED_MIXED)):
            p2.set_precision(prec)
            p2.set_fp32_form(form)
            t0 = time.perf_counter()
            zs[name] = p2.qdrift(cfg["nqb"], t, d, samples, cfg["depth"],
                                 cfg["step_size"], seed)
            secs[name] = time.perf_counter() - t0
    finally:
        p2.set_fp32_form(form0)
        p2.set_precision(p2.PREC_FP64)
    out = {"workload": (f"qdrift {cfg['nqb']} qubits, {len(t.cf)} JW terms, "
                        f"{samples} samples x {cfg['depth']} draws, FP32 vs "
                        "FP64 on the same draws"),
           "overlaps_fp64": [[z.real, z.imag] for z in zs["fp64"]],
           "seconds": secs}
    for name in ("f32_arith", "f64_arith", "mixed"):
        err = np.abs(zs[name] - zs["fp64"])
        out[name] = {"abs_err_per_sample": [float(e) for e in err],
                     "max_abs_err": float(err.max())}
    return out


def fp32_error_study(nqb: int = 20, nterms: int = 300, steps: int = 1000,
                     delta: float = 0.05) -> dict:
    """Second-order Trotter with a JW Hamiltonian (lexicographic order, 4
    determinants), FP32 and FP64 states side by side; error of every
    step's overlap against the FP64 run, which is bit-identical to the CPU
    oracle (tests/test_parity_gpu.py)."""
    import numpy as np

    import phase2_b200 as p2
    from phase2_b200 import workloads
    t = workloads.jw_terms(nqb, nterms, seed=0xE220)
    d = workloads.hamming_dets(nqb, 4, nqb // 2, seed=0xE221)
    p2.set_precision(p2.PREC_FP64)
    t0 = time.perf_counter()
    z64 = p2.trott2(nqb, t, d, steps, delta)
    p2.set_precision(p2.PREC_FP32)
    try:
        z32 = p2.trott2(nqb, t, d, steps, delta)
    finally:
        p2.set_precision(p2.PREC_FP64)
    err = np.abs(z32 - z64)
    at = {str(s): float(err[s - 1]) for s in (1, 10, 100, 1000)
          if s <= steps}
    return {"workload": (f"trott2 {nqb} qubits, {nterms} JW terms, "
                         f"4 determinants, delta {delta}"),
            "steps": steps, "rotations": 2 * nterms * steps,
            "max_abs_err": float(err.max()), "err_at_step": at,
            "final_overlap_fp64": [float(z64[-1].real), float(z64[-1].imag)],
            "seconds": time.perf_counter() - t0}


def trott26_study(steps: int = 256, term_order: int = 2) -> dict:
    """Second-order Trotter at 26 qubits (20,000 JW terms in flip-mask
    order -- phase2_set_term_order(FLIP), not the reference's lexicographic
    sort, unless `term_order` says otherwise -- 16 determinants of weight
    13, delta 0.05), FP64 and FP32 states (the process's FP32 form) side by
    side on the same inputs, `steps` of its 256 steps: device rot.amp/s of
    each (CUDA events around the pass launches) and the FP32 overlap error
    against the FP64 run after every step (the FP64 path is bit-identical
    to the reference)."""
    import numpy as np

    import phase2_b200 as p2
    from phase2_b200 import workloads
    cfg = workloads.strang26(steps=steps)
    t, d = cfg["terms"], cfg["dets"]
    oname = {0: "the reference's lexicographic", 1: "given",
             2: "flip-mask"}[term_order]
    out = {"workload": (f"trott2 26 qubits, 20000 JW terms in {oname} "
                        f"order, 16 determinants, delta 0.05, {steps} of "
                        "256 steps"), "unit": UNIT}
    zs = {}
    order = p2.lib().phase2_get_term_order()
    for name, prec in (("fp64", p2.PREC_FP64), ("fp32", p2.PREC_FP32)):
        p2.set_precision(prec)
        p2.set_term_order(term_order)
        try:
            z, st = p2.trott2(26, t, d, steps, cfg["delta"], timing=True,
                              with_stats=True)
        finally:
            p2.set_precision(p2.PREC_FP64)
            p2.set_term_order(order)
        zs[name] = z
        rot = st["rotations"]
        out[name] = {"value": rot * (1 << 26) / (st["pass_ms"] / 1e3),
                     "rotations": int(rot), "passes": int(st["passes"]),
                     "rotations_per_pass": rot / max(1, st["passes"]),
                     "pass_seconds": st["pass_ms"] / 1e3,
                     "hbm_gbs": st["bytes"] / (st["pass_ms"] / 1e3) / 1e9}
    out["fp32_form"] = FORM_NAME.get(p2.get_fp32_form())
    out["fp32_vs_fp64"] = out["fp32"]["value"] / out["fp64"]["value"]
    err = np.abs(zs["fp32"] - zs["fp64"])
    out["fp32_max_abs_err"] = float(np.max(err))
    out["fp32_abs_err_per_step"] = [float(f"{e:.3g}") for e in err]
    out["final_overlap_fp64"] = [float(zs["fp64"][-1].real),
                                 float(zs["fp64"][-1].imag)]
    return out


def trott26lex_study(steps: int = 2) -> dict:
    """Config 2 in the reference's own term order (lexicographic, the
    drivers' default), 2 of its 256 steps: fewer rotations per pass than
    the flip-mask order (the pass kernels' memory-bound end)."""
    return trott26_study(steps=steps, term_order=0)


def sampling_study() -> dict:
    """qdrift and cmpsit on FP32 and FP64 registers of 10-24 qubits
    (JW-like terms, four determinants), the samples drawn, planned and run
    by the host loop and then on the device (device sampling): wall time of
    the driver call each way (after one untimed run of the same shape) and
    whether the overlaps agree bit for bit."""
    import time

    import numpy as np

    import phase2_b200 as p2
    from phase2_b200 import workloads
    cases = [("qdrift", 10, 251, (64, 300, 0.01, 7)),
             ("qdrift", 14, 400, (64, 1000, 0.01, 7)),
             ("qdrift", 20, 800, (16, 2000, 0.01, 7)),
             ("qdrift", 24, 1000, (8, 2000, 0.01, 7)),
             ("cmpsit", 10, 251, (16, 8, 60, 50, 0.05, 0.002, 9)),
             ("cmpsit", 14, 2000, (16, 4, 200, 800, 0.05, 0.002, 9)),
             ("cmpsit", 20, 2000, (4, 4, 200, 800, 0.05, 0.002, 9))]
    out = []
    try:
        for (kind, n, nt, args), prec in [(c, p) for p in (p2.PREC_FP32,
                                                            p2.PREC_FP64)
                                           for c in cases]:
            p2.set_precision(prec)
            t = workloads.jw_terms(n, nt, seed=n)
            d = workloads.hamming_dets(n, 4, n // 2, seed=n + 1)
            fn = getattr(p2, kind)
            res = {}
            for mode in (p2.DEVICE_SAMPLING_OFF, p2.DEVICE_SAMPLING_ON):
                p2.set_device_sampling(mode)
                fn(n, t, d, *args)
                t0 = time.perf_counter()
                z = fn(n, t, d, *args)
                res[mode] = (time.perf_counter() - t0, z)
            host, dev = res[p2.DEVICE_SAMPLING_OFF], res[p2.DEVICE_SAMPLING_ON]
            out.append({"driver": kind, "nqb": n, "terms": nt,
                        "precision": "fp64" if prec == p2.PREC_FP64
                        else "fp32",
                        "args": list(args), "host_ms": host[0] * 1e3,
                        "device_ms": dev[0] * 1e3,
                        "speedup": host[0] / dev[0],
                        "bit_identical": bool(np.array_equal(host[1],
                                                             dev[1]))})
    finally:
        p2.set_device_sampling(p2.DEVICE_SAMPLING_AUTO)
        p2.set_precision(p2.PREC_FP64)
    return {"workload": "qdrift/cmpsit, host vs device sampling",
            "cases": out}


def sweeps_study(nqb: int = 26) -> dict:
    """The bench's qDRIFT draws (100,000 JW terms, 4096 per sample, two
    samples) at `nqb` qubits, FP32, under several sweep shapes: each plan
    run with one kernel per sweep and with one kernel per pass, device
    rot.amp/s (CUDA events) and the HBM GB/s of the state round trips."""
    import phase2_b200 as p2
    from phase2_b200 import workloads
    cfg = workloads.qdrift30(nqb=nqb)
    t, d = cfg["terms"], cfg["dets"]
    rows = []
    old = p2.get_sweep()
    form = p2.get_fp32_form()
    p2.set_precision(p2.PREC_FP32)
    p2.set_fp32_form(p2.FORM_LIFTED_F32)  # the form sweeps run in
    p2.set_device_sampling(p2.DEVICE_SAMPLING_OFF)
    try:
        for shape in ((0, 5), (13, 5), (13, 4), (12, 4), (14, 5)):
            for kernel in ((True, False) if shape[0] else (True,)):
                p2.set_sweep(*shape)
                p2.set_sweep_kernel(kernel)
                p2.qdrift(nqb, t, d, 1, cfg["depth"], 1e-3, 11)
                z, st = p2.qdrift(nqb, t, d, 2, cfg["depth"], 1e-3, 12,
                                  with_stats=True, timing=True)
                sec = st["pass_ms"] / 1e3
                rows.append({"tile": shape[0], "low": shape[1],
                             "sweep_kernel": kernel,
                             "passes": int(st["passes"]),
                             "round_trips": int(st["sweeps"]),
                             "value": st["rotations"] * (1 << nqb) / sec,
                             "hbm_gbs": st["bytes"] / sec / 1e9})
    finally:
        p2.set_sweep(*old)
        p2.set_sweep_kernel(True)
        p2.set_device_sampling(p2.DEVICE_SAMPLING_AUTO)
        p2.set_precision(p2.PREC_FP64)
        p2.set_fp32_form(form)
    return {"workload": (f"qdrift {nqb} qubits, 100000 JW terms, 2 samples "
                         f"x {cfg['depth']} draws, FP32 (FP32 arithmetic)"),
            "unit": UNIT,
            "rows": rows}


def _sharded_c_timing(nqb, world, dets, samples):
    """The same samples on the C sharded layer (include/phase2_sharded.h,
    every rank held, in-place swaps): mean wall seconds per sample after
    the first, and swaps per sample."""
    import numpy as np
    import torch

    import phase2_b200 as p2
    torch.cuda.empty_cache()
    L = p2.lib()
    ranks = (C.c_uint32 * world)(*range(world))
    h = L.phase2_sharded_new(nqb, world, ranks, world, p2.PREC_FP32, None, 0)
    if not h:
        raise RuntimeError("phase2_sharded_new failed")
    u64 = C.POINTER(C.c_uint64)
    f64 = C.POINTER(C.c_double)
    idx = np.ascontiguousarray(dets.idx, dtype=np.uint64)
    cf = np.ascontiguousarray(dets.cf, dtype=np.complex128)
    sec = []
    sw0 = C.c_uint64()
    sw1 = C.c_uint64()
    try:
        L.phase2_sharded_counters(h, C.byref(sw0), None)
        for f, ph, phi in samples:
            f = np.ascontiguousarray(f, dtype=np.uint64)
            ph = np.ascontiguousarray(ph, dtype=np.uint64)
            phi = np.ascontiguousarray(phi, dtype=np.float64)
            L.phase2_sharded_prepst(h, idx.ctypes.data_as(u64),
                                    cf.ctypes.data_as(f64), len(idx))
            L.phase2_sharded_synchronize(h)
            t0 = time.perf_counter()
            if L.phase2_sharded_paulirot(h, f.ctypes.data_as(u64),
                                         ph.ctypes.data_as(u64),
                                         phi.ctypes.data_as(f64), len(phi)):
                raise RuntimeError("phase2_sharded_paulirot failed")
            L.phase2_sharded_synchronize(h)
            sec.append(time.perf_counter() - t0)
        L.phase2_sharded_counters(h, C.byref(sw1), None)
    finally:
        L.phase2_sharded_free(h)
    return (float(np.mean(sec[1:])),
            (sw1.value - sw0.value) / len(samples))


def sharded_study(nqb: int = 30, worlds=(2, 4, 8)) -> dict:
    """A register split by its high qubits over 2, 4, 8 ranks held by this
    process on one GPU (phase2_b200.sharded: qubit swaps through
    qreg_slab_get / qreg_slab_put), against one register, on 4096 qDRIFT
    draws from the bench's 100,000 JW terms (|c|-weighted numpy draws,
    angle asin(1e-3) sign(c)), FP32.  Wall clock per sample with the
    device synchronised (the sharded register's host waits for each
    exchange), swaps per sample (pairs in this process trade halves in
    place, qreg_slab_swap), the bandwidth of one in-place swap (4 x 8 B
    per half amplitude) and of the half-slab gather that exchanges between
    processes use (2 x 8 B per amplitude), from CUDA events on the
    register's stream; and the same samples on the C layer
    (include/phase2_sharded.h, `c_layer`)."""
    import numpy as np
    import torch

    import phase2_b200 as p2
    from phase2_b200 import sharded, workloads
    cfg = workloads.qdrift30(nqb=nqb)
    t, d = cfg["terms"], cfg["dets"]
    rng = np.random.Generator(np.random.PCG64(0x5A4D))
    w = np.abs(t.cf)
    om = math.asin(1e-3)

    def draws():
        k = rng.choice(len(t), size=cfg["depth"], p=w / w.sum())
        return t.flip[k], t.phase[k], om * np.sign(t.cf[k])

    samples = [draws() for _ in range(3)]

    def timed(reg, prep):
        out = []
        for f, ph, phi in samples:
            prep()
            reg.synchronize()
            t0 = time.perf_counter()
            reg.paulirot(f, ph, phi)
            reg.synchronize()
            out.append(time.perf_counter() - t0)
        return out[1:]  # the first sample warms plans and buffers

    p2.set_device_sampling(p2.DEVICE_SAMPLING_OFF)
    res = {"workload": (f"{nqb} qubits FP32, 3 samples x {cfg['depth']} "
                        "qDRIFT draws of 100000 JW terms, first sample "
                        "untimed"), "unit": UNIT}
    try:
        with p2.Register(nqb, p2.PREC_FP32) as one:
            def prep1():
                one.zero()
                one.setamps(d.idx, d.cf)
            sec = timed(one, prep1)
        res["one_register"] = {
            "sec_per_sample": float(np.mean(sec)),
            "value": cfg["depth"] * (1 << nqb) / float(np.mean(sec))}
        rows = []
        for world in worlds:
            torch.cuda.empty_cache()
            with sharded.ShardedRegister.on_one_gpu(nqb, world,
                                                    p2.PREC_FP32) as reg:
                s0 = reg.swaps
                sec = timed(reg, lambda: reg.prepst(d))
                swaps = (reg.swaps - s0) / len(samples)
                slab = reg.slabs[0]
                cnt = min(1 << (reg.nlocal - 1), sharded.CHUNK)
                buf = slab.buffer(cnt)
                stream = torch.cuda.ExternalStream(
                    p2.lib().qreg_stream(C.byref(slab.reg.reg)))
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                gbs = {}
                for bit in (reg.nlocal - 1, 5, 0):
                    ev[0].record(stream)
                    slab.slab_get(bit, 1, 0, cnt, buf)
                    ev[1].record(stream)
                    ev[1].synchronize()
                    gbs[f"bit{bit}"] = (2 * 8 * cnt /
                                        (ev[0].elapsed_time(ev[1]) * 1e-3)
                                        / 1e9)
                del buf
                # one in-place pair swap: both halves read and written
                nhalf = 1 << (reg.nlocal - 1)
                ev[0].record(stream)
                slab.swap_halves(reg.slabs[1], reg.nlocal - 1, 1, 0)
                ev[1].record(stream)
                ev[1].synchronize()
                swap_gbs = (4 * 8 * nhalf /
                            (ev[0].elapsed_time(ev[1]) * 1e-3) / 1e9)
            csec, cswaps = _sharded_c_timing(nqb, world, d, samples)
            rows.append({
                "world": world, "local_qubits": reg.nlocal,
                "sec_per_sample": float(np.mean(sec)),
                "value": cfg["depth"] * (1 << nqb) / float(np.mean(sec)),
                "swaps_per_sample": swaps, "in_place": reg.in_place,
                "swap_gbs": swap_gbs,
                "gather_gbs": gbs, "gather_amplitudes": cnt,
                "c_layer": {"sec_per_sample": csec,
                            "value": cfg["depth"] * (1 << nqb) / csec,
                            "swaps_per_sample": cswaps}})
        res["sharded"] = rows
    finally:
        p2.set_device_sampling(p2.DEVICE_SAMPLING_AUTO)
    return res


def cmpsit33_study(steps: int = 1) -> dict:
    """The composite driver at 33 qubits (200,000 JW terms, 2,000
    deterministic, 8,192 draws per half step, 32 determinants), `steps` of
    its 64 steps, FP32 state (64 GiB) and FP64 state (128 GiB) in turn:
    device rot.amp/s and the FP32 error (opt-in: several minutes)."""
    import numpy as np

    import phase2_b200 as p2
    from phase2_b200 import workloads
    cfg = workloads.cmpsit33(steps=steps)
    out = {"workload": (f"cmpsit 33 qubits, {steps} of 64 steps, "
                        "200000 JW terms, length 2000, depth 8192, "
                        "32 determinants"), "unit": UNIT}
    zs = {}
    for name, prec in (("fp32", p2.PREC_FP32), ("fp64", p2.PREC_FP64)):
        p2.set_precision(prec)
        try:
            z, st = p2.cmpsit(cfg["nqb"], cfg["terms"], cfg["dets"],
                              cfg["samples"], cfg["steps"], cfg["length"],
                              cfg["depth"], cfg["angle_det"],
                              cfg["angle_rand"], cfg["seed"], timing=True,
                              with_stats=True)
        finally:
            p2.set_precision(p2.PREC_FP64)
        zs[name] = z
        rot = st["rotations"]
        out[name] = {"value": rot * (1 << cfg["nqb"]) /
                     (st["pass_ms"] / 1e3), "rotations": int(rot),
                     "passes": int(st["passes"]),
                     "pass_seconds": st["pass_ms"] / 1e3,
                     "hbm_gbs": st["bytes"] / (st["pass_ms"] / 1e3) / 1e9}
    out["fp32_max_abs_err"] = float(np.max(np.abs(zs["fp32"] - zs["fp64"])))
    return out


def batch8_study(prec: int = 1, form: int | None = None) -> dict:
    """A small, L2-resident persistent batch (8 trott instances of 18-20
    qubits, 2,000 JW terms, 2 steps, FP32 in the process's form unless
    `form` is given), run twice: the case the persistent kernel's profile
    summaries capture (its second launch)."""
    import numpy as np

    import phase2_b200 as p2
    from phase2_b200 import workloads
    form0 = p2.get_fp32_form()
    if form is not None:
        p2.set_fp32_form(form)
    g = np.random.Generator(np.random.PCG64(5))
    probs = []
    for k in range(8):
        n = int(g.integers(18, 21))
        probs.append(dict(nqb=n, terms=workloads.jw_terms(n, 2000,
                                                          seed=100 + k),
                          dets=workloads.hamming_dets(n, 1, n // 2,
                                                      seed=200 + k),
                          steps=2, delta=0.05))
    p2.set_precision(prec)
    try:
        for _ in range(2):
            _, st = p2.batch("trott", probs, with_stats=True)
    finally:
        p2.set_precision(p2.PREC_FP64)
        p2.set_fp32_form(form0)
    return {"passes": int(sum(s["passes"] for s in st)),
            "kernel_ms": float(sum(s["pass_ms"] for s in st))}


def batch8f32_study() -> dict:
    """batch8 in the FP32-arithmetic form (the persistent kernel's FP32
    instance), for its profile summary."""
    import phase2_b200 as p2
    return batch8_study(prec=1, form=p2.FORM_LIFTED_F32)


def batch8fp64_study() -> dict:
    """batch8 with FP64 registers: the FP64 instance of the persistent
    kernel (exact pass arithmetic), for its profile summary."""
    return batch8_study(prec=0)


def batch4big_study() -> dict:
    """A small persistent batch of HBM-sized registers: 4 trott instances
    of 23-24 qubits (512 MiB of FP32 states in all, above L2), 2,000 JW
    terms, 1 step, FP32 in the process's form, run twice: the case the
    persistent kernel's profile summary for config-4-sized registers
    captures (its second launch).  Algorithmic bytes: 2 * 2^n * 8 per
    pass, summed."""
    import numpy as np

    import phase2_b200 as p2
    from phase2_b200 import workloads
    probs = []
    for k, n in enumerate((24, 23, 24, 23)):
        probs.append(dict(nqb=n, terms=workloads.jw_terms(n, 2000,
                                                          seed=500 + k),
                          dets=workloads.hamming_dets(n, 1, n // 2,
                                                      seed=600 + k),
                          steps=1, delta=0.05))
    p2.set_precision(p2.PREC_FP32)
    try:
        for _ in range(2):
            _, st = p2.batch("trott", probs, with_stats=True)
    finally:
        p2.set_precision(p2.PREC_FP64)
    ms = float(sum(s["pass_ms"] for s in st))
    nbytes = int(sum(s["bytes"] for s in st))
    return {"passes": int(sum(s["passes"] for s in st)), "kernel_ms": ms,
            "algorithmic_bytes": nbytes,
            "hbm_gbs_kernel": nbytes / (ms * 1e-3) / 1e9,
            "fp32_form": FORM_NAME.get(p2.get_fp32_form())}


def batched_study(ninst: int = 64, work_cap: float = 1.5e14,
                  seed: int = 0xBA7C4):
    """Independent trott problems of uneven size run together: qubits
    U{18..24}, JW terms log-uniform in [1e3, 5e4], steps U{16..512}, FP32
    state, one determinant each.  The drawn configuration totals about
    9e14 rot.amp; to bound the run, every instance's step count is scaled
    by the same factor so that the total is at most work_cap (at least 16
    steps each), which keeps the unevenness between instances.  Aggregate
    rot.amp/s over the batch (wall clock around the batch call,
    recording/planning and result download included), in one persistent
    launch and on per-instance streams; HBM GB/s counts 2 * 2^n * 8 bytes
    per pass, l2_fit_byte_share is the part of those bytes that belongs to
    instances whose state fits in L2 (n <= 23), which the L2 can serve
    instead of HBM, and hbm_gbs_kernel_non_l2 counts only the others.  The
    persistent launch also reports when each instance finished (device
    timer): the tail is the time between the median and the last
    finish."""
    import numpy as np

    import phase2_b200 as p2
    from phase2_b200 import workloads
    rng = np.random.Generator(np.random.PCG64(seed))
    shape = []
    for _ in range(ninst):
        n = int(rng.integers(18, 25))
        nt = int(round(10 ** rng.uniform(3, np.log10(5e4))))
        steps = int(rng.integers(16, 513))
        shape.append((n, nt, steps))
    drawn = sum(st * nt * (1 << n) for n, nt, st in shape)
    scale = min(1.0, work_cap / drawn)
    probs, work = [], 0
    for k, (n, nt, steps) in enumerate(shape):
        run = max(16, int(round(steps * scale)))
        t = workloads.jw_terms(n, nt, seed=seed + k)
        d = workloads.hamming_dets(n, 1, n // 2, seed=seed + 1000 + k)
        probs.append(dict(nqb=n, terms=t, dets=d, steps=run, delta=0.05))
        work += run * nt * (1 << n)
    out = {"workload": (f"{ninst} trott instances, 18-24 qubits, 1e3-5e4 "
                        "JW terms, steps drawn U{16..512} and scaled by "
                        f"{scale:.3f} (at least 16) to cap the batch at "
                        f"{work_cap:.1e} rot.amp, FP32 state"),
           "rot_amp": work, "rot_amp_drawn": drawn, "step_scale": scale,
           "steps_run": [p["steps"] for p in probs], "unit": UNIT,
           "fp32_form": FORM_NAME.get(p2.get_fp32_form())}
    p2.set_precision(p2.PREC_FP32)
    order = p2.lib().phase2_get_term_order()
    try:
        for mode, persistent in (("persistent", True), ("streams", False)):
            p2.set_term_order(0)
            p2.set_batch_persistent(persistent)
            p2.batch("trott", [dict(pr, steps=1) for pr in probs[:2]])
            t0 = time.perf_counter()
            _, stats = p2.batch("trott", probs, with_stats=True)
            wall = time.perf_counter() - t0
            hbm = sum(s["bytes"] for s in stats)
            kms = sum(s["pass_ms"] for s in stats)
            # bytes of instances whose FP32 state fits the 126 MB L2
            # (n <= 23: 64 MiB); their passes can be served from L2
            l2 = sum(s["bytes"] for s, pr in zip(stats, probs)
                     if (1 << pr["nqb"]) * 8 <= 126 * 10 ** 6)
            row = {
                "seconds": wall, "value": work / wall,
                "hbm_gbs_wall": hbm / wall / 1e9,
                "kernel_seconds": kms / 1e3 if persistent else None,
                "hbm_gbs_kernel": (hbm / (kms / 1e3) / 1e9
                                   if persistent and kms else None),
                "launches": int(sum(s["launches"] for s in stats)),
                "passes": int(sum(s["passes"] for s in stats)),
                "l2_fit_byte_share": l2 / hbm if hbm else None}
            if persistent and kms:
                row["hbm_gbs_kernel_non_l2"] = (hbm - l2) / (kms / 1e3) / 1e9
                fin = sorted(s["finish_ms"] for s in stats
                             if s.get("finish_ms") is not None)
                if fin:
                    row["finish_ms"] = {
                        "first": fin[0], "median": fin[len(fin) // 2],
                        "last": fin[-1],
                        "tail_after_median": fin[-1] - fin[len(fin) // 2]}
            out[mode] = row
    finally:
        p2.set_batch_persistent(True)
        p2.set_term_order(order)
        p2.set_precision(p2.PREC_FP64)
    out["value"] = out["persistent"]["value"]
    return out


# studies appended to the N=1 line, in this order, with their approximate
# B200 durations (for the study budget)
STUDY_ORDER = ("batched", "cmpsit33", "trott26", "sharded", "sampling",
               "sweeps")
STUDY_SECONDS = {"trott26": 600, "batched": 180, "cmpsit33": 300,
                 "sharded": 70, "sampling": 30, "sweeps": 60}


# ---- the reference arm -------------------------------------------------


def reference_arm(args) -> None:
    """The reference's own CPU implementation of the path on the host
    cores: its qdrift driver on the headline workload (same Hamiltonian,
    determinant, step size, seed) as R MPI ranks of one job, each step one
    sample truncated to CPU_DEPTH draws (the GPU arm's cpu_baseline is the
    same measurement); value = rot.amp/s of the fastest of the --steps
    samples after --warmup (the reference's min-of-K convention).  Under
    torchrun only rank 0 runs it."""
    ws, rank, _ = _dist()
    if rank != 0:
        return
    from phase2_b200 import workloads
    from oracle import REF_MPI
    if not REF_MPI.is_file():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/ref_mpi was not built (reference "
                          "sources absent at build time)"}), flush=True)
        return
    cfg = workloads.qdrift30(nqb=args.nqb, depth=args.depth)
    t0 = time.perf_counter()
    cb = _cpu_reference(cfg, CPU_DEPTH, args.steps, args.warmup)
    elapsed = time.perf_counter() - t0
    v = cb["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * cb["seconds_per_sample"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded JW-like Hamiltonian, no "
                                "dataset)",
        "config": _config(cfg),
        "sample": (f"each step is the workload's qDRIFT sample truncated "
                   f"to {CPU_DEPTH} of its {cfg['depth']} draws (a bounded "
                   "CPU sample; the metric is a rate)"),
        "parallelism": f"{cb['cores']} MPI ranks on host cores",
        "cpu_baseline": cb,
        "wall_seconds": elapsed,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nqb", type=int, default=30)
    ap.add_argument("--depth", type=int, default=4096)
    ap.add_argument("--cmp-depth", type=int, default=512)
    ap.add_argument("--fp32-form", default=None,
                    choices=["f32", "f64", "mixed"],
                    help="arithmetic of FP32 passes for the run: f32 (FP32 "
                         "FMAs), f64 (FP64 arithmetic, one rounding to "
                         "FP32 per pass) or mixed (FP32 FMAs, FP64 on "
                         "cosets holding an amplitude >= 2^-10); default: "
                         "the library's")
    ap.add_argument("--lift-kernel", default=None,
                    choices=["direct", "bulk", "staged", "staged2"],
                    help="kernel of FP64-arithmetic FP32 passes: direct "
                         "loads, or the next cosets staged by bulk copies "
                         "or by cp.async (staged2: two blocks per SM with "
                         "the whole register file)")
    ap.add_argument("--quick", action="store_true",
                    help="skip the CPU baseline and secondary arms")
    ap.add_argument("--studies", default="batched,cmpsit33,trott26,sharded",
                    help="comma list of studies to append (run at N=1, in "
                         "the order batched, cmpsit33, trott26, sharded, "
                         "sampling, sweeps, each only while the study "
                         "budget lasts)")
    ap.add_argument("--study-budget", type=float, default=1200.0,
                    help="seconds of studies at most (a study that would "
                         "not fit the remainder is skipped and reported)")
    ap.add_argument("--only-study", default=None,
                    help="run just this study (batched, trott26, cmpsit33, "
                         "batch8, batch8f32, batch8fp64, batch4big, "
                         "trott26lex, "
                         "sampling, sweeps, "
                         "sharded) "
                         "and print its JSON; --nqb, when given, sets the "
                         "sweeps or sharded study's width")
    args = ap.parse_args()
    if args.only_study:
        import inspect

        import phase2_b200 as p2
        p2.world_ensure()
        if args.fp32_form:
            p2.set_fp32_form({"f32": p2.FORM_LIFTED_F32,
                              "f64": p2.FORM_LIFTED,
                              "mixed": p2.FORM_LIFTED_MIXED}[args.fp32_form])
        fn = globals()[f"{args.only_study}_study"]
        kw = {}
        if "nqb" in inspect.signature(fn).parameters and \
                "--nqb" in sys.argv:
            kw["nqb"] = args.nqb
        print(json.dumps({args.only_study: fn(**kw)}), flush=True)
        return
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)
        # every rank has left its last collective when gpu_arm returns;
        # after an exception a peer may still be inside one, so the group
        # is left to process exit instead of a blocking teardown
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
