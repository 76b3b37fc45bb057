#!/usr/bin/env python
"""Benchmark: 256^3 pressure projections per second on B200.

Workload (the standalone-projection configuration): a 256^3 MAC grid whose fluid
mask is 32 seeded Gaussian blobs (sigma ~ U[0.03,0.12]) thresholded at 0.5, a
random box obstacle covering 10% of the volume, a solid border and U[-1,1] FP32
face velocities (xfluid_b200.scenes.blob_scene, seed 3).  The headline solves
xFluid's own matrix on it (no fractional face weights), the same computation
the reference arm times, so the two arms' figures compare like for like; the
same scene with the obstacle's fractional face weights is timed beside it
(forms.fractional_faces_mixed).  One step = one projection: layout + assembly,
MIC(0) factorisation, PCG to |r|_inf <= 1e-6 |b|_inf, pressure scatter and
velocity update.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm prints one JSON line whose `value` is device-resident throughput in the
mixed-precision form (inputs already in HBM, a distinct input copy per step so
inputs exceed L2), with `e2e` measured through the C ABI from pinned host
buffers, `roofline` for the dominant kernel (the MIC(0) triangular-solve sweeps,
timed with CUDA events on the launching stream), the plain FP32 and FP64 GPU
forms beside it, and the CPU baseline.  The reference arm (--impl reference)
times xFluid's own CPU solver (oracle/_ref, built from the reference sources;
the oracle's C port where that build is absent) on the same scene.

Multi-GPU: a single projection does not shard (the lexicographic MIC(0) is one
global wavefront), so N GPUs run N independent replicas; value = N * K / (max
over ranks of the timed region).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "256³ projections/s, mixed-prec vs plain GPU MIC(0)-PCG at rel-res 1e-6; HBM GB/s"
UNIT = "projections/s"
TOL = 1e-6
MAXIT = 2000
SEED = 3


def workload_config(n, rows=None, iters=None):
    cfg = {"workload": f"blob scene {n}^3 (32 Gaussian blobs, 10% box obstacle, U[-1,1] FP32 faces, seed {SEED}), "
                       f"xFluid's variational matrix (the obstacle's fractional face weights: "
                       f"forms.fractional_faces_mixed); tol 1e-6 relative inf-norm",
           "grid": [n, n, n], "tol": TOL, "l2": "inputs larger than L2: a distinct input copy per step"}
    if rows is not None:
        cfg["rows"] = rows
    if iters is not None:
        cfg["iterations"] = iters
    return cfg


# ---------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms (read-only)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.samples = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(s[1]) for s in self.samples if num(s[1]) is not None]
        mx = [num(s[2]) for s in self.samples if num(s[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for s in self.samples for q in range(4)
                          if len(s) > 5 + q and s[5 + q].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ---------------------------------------------------------------------------- CPU baseline
def cpu_project_seconds(sc, keep=False):
    """One projection of the scene (xFluid's matrix: no face weights) by
    xFluid's own CPU solver when it was built (oracle/_ref): its solve and its
    applyPressure, single-threaded; else by the oracle's C port.  Returns
    (seconds, kind), and with keep=True also the reference's result
    {p, iters, u, v, w}."""
    import oracle
    s64 = sc.astype(np.float64).reference_mode()
    if oracle.reference_available():
        R = oracle.Reference()
        before = R.set_threads(1)   # the single-core figure: applyPressure's OpenMP loop on one thread
        try:
            t = time.perf_counter()
            sol = R.solve(s64, tol=TOL, maxit=MAXIT)
            u, v, w = R.apply(s64, sol["p"])
            sec = time.perf_counter() - t
        finally:
            R.set_threads(before)
        out = {"p": sol["p"], "iters": sol["iters"], "u": u, "v": v, "w": w}
        return (sec, "reference", out) if keep else (sec, "reference")
    oracle.build_oracle()
    O = oracle.Oracle()
    t = time.perf_counter()
    res = O.project(s64, tol=TOL, maxit=MAXIT)
    sec = time.perf_counter() - t
    out = {"p": res["p"], "iters": res["iters"], "u": res["u"], "v": res["v"], "w": res["w"]}
    return (sec, "port", out) if keep else (sec, "port")


def cpu_apply_pressure(sc):
    """xFluid's own applyPressure (its OpenMP loop over i,
    variational_pressuresolver.cpp:120-220) on all host cores and on one,
    mean of 2 calls each on the scene with a zero pressure field (the work does
    not depend on the values).  None when the reference was not built."""
    import oracle
    if not oracle.reference_available():
        return None
    R = oracle.Reference()
    s64 = sc.astype(np.float64).reference_mode()
    p = np.zeros((sc.nk, sc.nj, sc.ni))
    cores = os.cpu_count() or 1
    ms_all = 1e3 * R.time_apply(s64, p, cores, 2)
    ms_one = 1e3 * R.time_apply(s64, p, 1, 2)
    return {"kind": "reference", "threads": cores, "ms_all_threads": ms_all, "ms_1_thread": ms_one,
            "sample": f"applyPressure alone on the {sc.ni}^3 scene, OpenMP on {cores} threads and on 1"}


def _ref_worker(conn, n):
    from xfluid_b200 import scenes
    sc = scenes.blob_scene(n, seed=SEED, dtype=np.float32)
    small = scenes.blob_scene(64, seed=SEED, dtype=np.float32)
    conn.send("ready")
    while True:
        msg = conn.recv()
        if msg == "stop":
            break
        sec, kind = cpu_project_seconds(small if msg == "warm" else sc)
        conn.send((sec, kind))


REF_PROC_BYTES = 4.5e9   # peak host memory of one 256^3 reference projection (measured 3.7 GB) plus margin


def reference_processes(n):
    """How many reference projections run at once: one per usable host core,
    unless host memory holds fewer (each 256^3 projection peaks near 3.7 GB:
    xFluid's row-list matrix spans every cell).  Returns (processes, cores,
    reason or None)."""
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    need = REF_PROC_BYTES * (n / 256.0) ** 3
    avail = None
    try:
        for line in Path("/proc/meminfo").read_text().splitlines():
            if line.startswith("MemAvailable:"):
                avail = float(line.split()[1]) * 1024
    except OSError:
        pass
    if avail is None:
        return cores, cores, None
    by_mem = max(1, int(0.8 * avail // need))
    if by_mem < cores:
        return by_mem, cores, (f"host memory: {avail / 1e9:.0f} GB available holds {by_mem} concurrent "
                               f"{n}^3 projections at ~{need / 1e9:.1f} GB each")
    return cores, cores, None


def reference_arm(args, rank, world):
    """xFluid's CPU solver on every usable host core: one process per core, each
    running whole projections.  A timed step is a round in which every process
    completes one projection; ceil(K / processes) rounds are timed, so the run
    stays within a few minutes on a many-core host while every core works.
    Warm-up rounds project the 64^3 scene (code and allocator warm-up; the
    reference has nothing to compile)."""
    import multiprocessing as mp
    if rank != 0:
        return
    nproc, cores, why = reference_processes(args.n)
    ctxmp = mp.get_context("spawn")
    pipes, procs = [], []
    for _ in range(nproc):
        a, b = ctxmp.Pipe()
        p = ctxmp.Process(target=_ref_worker, args=(b, args.n), daemon=True)
        p.start()
        pipes.append(a)
        procs.append(p)
    for a in pipes:
        a.recv()
    kinds = set()

    def step(msg="go"):
        for a in pipes:
            a.send(msg)
        res = [a.recv() for a in pipes]
        kinds.update(k for _, k in res)
        return [sec for sec, _ in res]

    for _ in range(max(1, args.warmup)):
        step("warm")
    rounds = max(1, -(-args.steps // nproc))
    t0 = time.perf_counter()
    per = []
    for _ in range(rounds):
        per += step()
    el = time.perf_counter() - t0
    for a in pipes:
        a.send("stop")
    for p in procs:
        p.join(timeout=30)
    done = nproc * rounds
    value = done / el
    kind = "reference" if kinds == {"reference"} else "port"
    sample = (f"{nproc} processes on {cores} usable host cores, {rounds} round(s) of one full {args.n}^3 "
              f"projection per process ({done} projections; assemble + MIC(0)-PCG to 1e-6 + applyPressure, "
              f"{statistics.median(per):.1f} s median each), same seeded scene as the GPU arm's headline "
              f"(xFluid's matrix: no fractional face weights)")
    cpu = {"value": value, "unit": UNIT, "cores": nproc, "host_cores": cores, "kind": kind, "sample": sample}
    if why:
        cpu["fewer_processes_than_cores"] = why
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": workload_config(args.n),
            "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------- our arm
def sweep_traffic_per_row():
    """DRAM bytes per unknown row of one sweep launch, from the committed ncu
    summary (profiles/sweep_traffic.txt); None when absent."""
    f = ROOT / "profiles" / "sweep_traffic.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("dram_bytes_per_row_per_sweep:"):
            try:
                return float(line.split(":", 1)[1])
            except ValueError:
                return None
    return None


FULL_FIXTURE = ROOT / "tests" / "golden" / "full_blob256.npz"


def stall_cases(args, stream, ctx_for, project_dev, mat, vel0):
    """Where the mixed form earns its keep: cases in which plain FP32 PCG needs
    many more iterations, or stalls, before reaching the accuracy the mixed
    form reaches.  Each case times one projection per form (after one
    untimed) -- plain FP32, mixed and plain FP64 at the case's tolerance --
    and reports iterations, status and the pressure's relative L2 error
    against an FP64 solve of the same system to tol 1e-12 (the FP64 path
    follows the reference's operation order), and the mixed form's speed over
    plain FP32.  Plain FP32 stops on its recursive residual, which drifts
    from the true one; the mixed form stops on the true FP64 residual, as the
    FP64 form does.
      blob_tol_1e-8  the headline scene at tol 1e-8;
      dam_256_tol_1e-6  the 256^3 dam break (fluid x < 0.4, y < 0.5, solid
                        border, the first step's gravity impulse), tol 1e-6
                        (the reference needs 125 iterations here)."""
    import torch
    from xfluid_b200 import scenes
    cases = {}
    dam = scenes.dam_break(args.n, seed=1, dtype=np.float32) if args.n >= 64 else None
    specs = [("blob_tol_1e-8", mat, vel0, 1e-8)]
    if dam is not None:
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
        specs.append(("dam_256_tol_1e-6" if args.n == 256 else f"dam_{args.n}_tol_1e-6",
                      torch.from_numpy(dam.mat).cuda(), [t(a) for a in (dam.u, dam.v, dam.w)], 1e-6))
    for name, m, v0, tol in specs:
        shape = tuple(m.shape)

        def run(prec, tol_, reps, maxit=MAXIT):
            c = ctx_for(prec, 1)
            o = c.opts
            o.tol, o.max_iter = tol_, maxit
            c.set_options(o)
            p = torch.zeros(shape, dtype=torch.float32, device="cuda")
            ms, st = None, None
            try:
                for k in range(reps):
                    vel = [a.clone() for a in v0]
                    torch.cuda.synchronize()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    _, st = project_dev(c, vel, p, m=m)
                    e1.record(stream)
                    torch.cuda.synchronize()
                    ms = e0.elapsed_time(e1)
            finally:
                c.close()
            return p.double(), ms, st

        pe, _, _ = run("f64", 1e-12, 1, maxit=20000)
        entry = {"tol": tol}
        for prec in ("f32", "mixed", "f64"):
            p, ms, st = run(prec, tol, 2)
            entry[{"f32": "plain_f32", "mixed": "mixed", "f64": "plain_f64"}[prec]] = {
                "projections_per_s": 1000.0 / ms, "iterations": int(st["iterations"]), "status": int(st["status"]),
                "refinements": int(st["refinements"]),
                "pressure_rel_l2_vs_fp64_exact": float(torch.linalg.norm(p - pe) / torch.linalg.norm(pe))}
        entry["mixed_over_plain_f32"] = entry["mixed"]["projections_per_s"] / entry["plain_f32"]["projections_per_s"]
        cases[name] = entry
    return cases





def parity_report(sc, kind, ref, gpu):
    """The GPU forms' results on the headline scene against xFluid's own solver
    run on the same scene at the same tolerance (the CPU-baseline leg's
    projection): pressure and projected-velocity relative L2, iterations, and
    both divergence figures after the projection -- the m-weighted one the
    projection drives to tol * |b|_inf (per cell it equals b - A p) and the
    reference's own unweighted diagnostic (variational_pressuresolver.cpp:
    526-597, which leaves solid faces out).  The convergence error against the
    exact solution (the reference solved to 1e-12, committed as a sample in
    tests/golden/full_blob256.npz for the 256^3 scene) is reported separately
    from the precision error."""
    import oracle
    from xfluid_b200 import scenes  # noqa: F401
    oracle.build_oracle()
    O = oracle.Oracle()
    s64 = sc.astype(np.float64).reference_mode()
    b_inf = float(np.abs(O.assemble(s64)["b"]).max())
    ref_vel = np.concatenate([a.ravel() for a in (ref["u"], ref["v"], ref["w"])])
    exact = None
    if FULL_FIXTURE.exists():
        import hashlib
        g = np.load(FULL_FIXTURE)
        h = hashlib.sha256()
        for a in (sc.mat, sc.u, sc.v, sc.w):
            h.update(np.ascontiguousarray(a).tobytes())
        if int(g["n"]) == sc.ni and h.hexdigest() == str(g["digest"]):
            exact = (g["idx_p"], g["pe"])

    def rl2(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    def divs(u, v, w):
        dw = O.weighted_divergence(s64, u, v, w)
        du = O.divergence_ref(s64, u, v, w)
        return {"weighted_div_inf_over_b_inf": float(np.abs(dw).max()) / b_inf,
                "unweighted_div_inf": float(np.abs(du).max())}

    out = {"scene": "the headline scene, xFluid's matrix", "tol": TOL,
           "reference": dict({"kind": kind, "iterations": int(ref["iters"])},
                             **divs(ref["u"], ref["v"], ref["w"]))}
    if exact is not None:
        idx, pe = exact
        out["reference"]["pressure_rel_l2_vs_exact_sample"] = rl2(ref["p"].ravel()[idx], pe)
    for name, r in gpu.items():
        p = r["p"].double().cpu().numpy()
        u, v, w = (a.double().cpu().numpy() for a in r["vel"])
        e = {"iterations": int(r["iterations"]),
             "iterations_vs_reference": int(r["iterations"]) - int(ref["iters"]),
             "pressure_rel_l2_vs_reference": rl2(p, ref["p"]),
             "velocity_rel_l2_vs_reference": rl2(np.concatenate([u.ravel(), v.ravel(), w.ravel()]), ref_vel),
             "rel_residual_reported": float(r["rel_residual"])}
        if exact is not None:
            e["pressure_rel_l2_vs_exact_sample"] = rl2(p.ravel()[idx], pe)
        e.update(divs(u, v, w))
        out[name] = e
    return out


def phases(st):
    """A projection's phases (CUDA events inside the library): layout + assembly
    (+ the FP32 copies in mixed precision), MIC(0) factorisation (+ its FP32
    copies), PCG, pressure scatter + velocity update."""
    return {k: round(float(st[k]), 4) for k in ("ms_setup", "ms_factor", "ms_solve", "ms_apply")}


def ours(args, rank, world):
    import ctypes as C
    import torch
    import torch.distributed as dist
    from xfluid_b200 import _lib, scenes

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    stream = torch.cuda.current_stream()

    sc = scenes.blob_scene(args.n, seed=SEED, dtype=np.float32)
    ni, nj, nk = sc.ni, sc.nj, sc.nk

    def ctx_for(prec, device_pointers, matrix="variational"):
        o = _lib.default_options()
        o.precision = _lib.PREC[prec]
        o.matrix = _lib.MATRIX[matrix]
        o.tol, o.max_iter = TOL, MAXIT
        o.device = dev
        o.device_pointers = device_pointers
        o.stream = C.c_void_p(stream.cuda_stream)
        return _lib.Context(o)

    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    mat = t(sc.mat)
    wts = [t(a) for a in (sc.wu, sc.wv, sc.ww)]   # the obstacle's fractional face weights (their own form)
    nsteps = args.steps + args.warmup
    vel0 = [t(a) for a in (sc.u, sc.v, sc.w)]
    copies = [[a.clone() for a in vel0] for _ in range(nsteps)]
    pres = torch.zeros((nk, nj, ni), dtype=torch.float32, device="cuda")
    P = lambda x: C.c_void_p(x.data_ptr())

    def project_dev(ctx, vel, p, weights=False, m=None):
        st = _lib.XfpStats()
        m = mat if m is None else m
        rc = ctx.lib.xfp_project_f32(ctx.ptr, ni, nj, nk, P(m), P(vel[0]), P(vel[1]), P(vel[2]),
                                     *(map(P, wts) if weights else (None, None, None)), P(p), C.byref(st))
        ctx.check(rc)
        return rc, st.as_dict()

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        tt = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    # ---------------- headline: mixed precision, device-resident inputs ----------------
    ctx = ctx_for("mixed", 1)
    stats = []
    for s in range(args.warmup):
        project_dev(ctx, copies[s], pres)
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        ev0.record(stream)
        for s in range(args.steps):
            rc, st = project_dev(ctx, copies[args.warmup + s], pres)
            stats.append((rc, st))
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms)
    value = world * args.steps / (ms_max / 1000.0)
    last = stats[-1][1]
    rows = int(last["rows"])
    iters = int(last["iterations"])
    launches = int(sum(s["launches"] for _, s in stats))
    sweep_ms = sum(s["ms_sweeps"] for _, s in stats)
    sweeps = sum(s["sweeps"] for _, s in stats)
    # algorithmic bytes of one sweep launch (mixed: FP32 vectors and L, the FP64
    # pivots streamed as FP32): forward r 4 + L 12 + invdiag 4 + y 4 = 24 B/row;
    # backward y 4 + L 12 + invdiag 4 + r 4 + z 4 = 28 B/row; launches
    # alternate -> 26 B/row average.  Only launches that did work are timed
    # (the PCG loop's launches after convergence return at once).
    bytes_per_launch = 26.0 * rows
    avg_launch_s = (sweep_ms / max(sweeps, 1)) / 1000.0
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = bytes_per_launch / avg_launch_s / 1e9 if avg_launch_s > 0 else None
    tr = sweep_traffic_per_row()
    roofline = {"bound": "hbm", "kernel": "MIC(0) triangular solves (solve_kernel fwd/bwd, lockstep wavefronts)",
                "achieved": achieved, "peak": peak, "unit": "GB/s",
                "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6650 GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": (tr * rows) if tr is not None else None,
                "algorithmic_bytes_per_launch": bytes_per_launch, "avg_launch_ms": avg_launch_s * 1000,
                # events sample every 16th iteration: the share scales the
                # average launch by the launches that did work (two per
                # iteration, the preconditioner's first pair included)
                "sweep_share_of_step": (avg_launch_s * 1000 * sum(2 * max(int(s["iterations"]), 1) for _, s in stats)
                                        / ms) if ms > 0 else None}
    # the PCG loop's vector kernels, event-timed the same way (launches after
    # convergence excluded): algorithmic bytes per unknown row (FP32 vectors
    # and coefficients) -- SpMV s + 4 coefficients + z = 24; x/r update x, s,
    # r, z read + x, r written = 24; s update z, s read + s written = 12
    vec_ms = [sum(s_["ms_vec"][k] for _, s_ in stats) for k in range(3)]
    vec_n = [sum(s_["vec_launches"][k] for _, s_ in stats) for k in range(3)]
    vk = {}
    for k, (name, bpr) in enumerate((("spmv_dot", 24.0), ("update_xr", 24.0), ("update_s", 12.0))):
        if vec_n[k] > 0 and vec_ms[k] > 0:
            avg = vec_ms[k] / vec_n[k]
            gbs = bpr * rows / (avg / 1000.0) / 1e9
            # launches that did work: one per iteration (the s update: all but the last)
            work = sum(max(int(s_["iterations"]) - (k == 2), 0) for _, s_ in stats)
            vk[name] = {"avg_launch_ms": avg, "launches_timed": vec_n[k], "algorithmic_bytes_per_row": bpr,
                        "achieved_gbs": gbs, "frac": gbs / peak, "share_of_step": avg * work / ms}
    roofline["vector_kernels"] = vk

    # ---------------- e2e: through the C ABI from pinned host buffers ----------------
    ctx_h = ctx_for("mixed", 0)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    hmat = pin(sc.mat)
    hvel0 = [pin(a) for a in (sc.u, sc.v, sc.w)]
    hp = torch.zeros((nk, nj, ni), dtype=torch.float32).pin_memory()
    e2e_steps = max(2, min(args.steps, 5))
    hcopies = [[a.clone().pin_memory() for a in hvel0] for _ in range(e2e_steps + 1)]

    moved = []

    def project_host(vel):
        st = _lib.XfpStats()
        rc = ctx_h.lib.xfp_project_f32(ctx_h.ptr, ni, nj, nk, P(hmat), P(vel[0]), P(vel[1]), P(vel[2]),
                                       None, None, None, P(hp), C.byref(st))
        ctx_h.check(rc)
        moved.append((st.h2d_bytes, st.d2h_bytes, st.host_faces))

    project_host(hcopies[0])
    barrier()
    torch.cuda.synchronize()
    moved.clear()
    t0 = time.perf_counter()
    for s in range(e2e_steps):
        project_host(hcopies[1 + s])
    torch.cuda.synchronize()
    el = max_over_ranks(time.perf_counter() - t0)
    # bytes the calls reported moving: the material and the pressure whole,
    # and of the velocities only the faces that border fluid (the arrays are
    # page-locked, so the library reads and writes them in place)
    h2d = sum(m[0] for m in moved) / len(moved)
    d2h = sum(m[1] for m in moved) / len(moved)
    sparse = all(m[2] == 1 for m in moved)
    e2e = {"value": world * e2e_steps / el, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h),
           "whole_array_bytes_per_step": int(sc.mat.nbytes + hp.numel() * 4 + 2 * sum(a.nbytes for a in (sc.u, sc.v, sc.w))),
           "path": "xfp_project_f32, host pointers (pinned)" + (", fluid-bordering faces only" if sparse else "")}

    # ---------------- the other forms on the same scene ----------------
    # plain FP32 and FP64 at the same tolerance (their pressures and projected
    # velocities are kept for the parity report), and the mixed form with the
    # obstacle's fractional face weights
    forms = {}
    gpu_results = {"mixed": {"p": pres, "vel": copies[args.warmup + args.steps - 1] if args.steps else None,
                             "iterations": iters, "rel_residual": last["rel_residual"],
                             "refinements": int(last["refinements"])}}
    for prec, weights, name in (("f32", False, "plain_f32"), ("f64", False, "plain_f64"),
                                ("mixed", True, "fractional_faces_mixed")):
        c2 = ctx_for(prec, 1)
        p2 = torch.zeros_like(pres)
        project_dev(c2, [a.clone() for a in vel0], p2, weights=weights)
        torch.cuda.synchronize()
        reps = 2
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        vs = [[a.clone() for a in vel0] for _ in range(reps)]
        e0.record(stream)
        for r_ in range(reps):
            rc2, st2 = project_dev(c2, vs[r_], p2, weights=weights)
        e1.record(stream)
        torch.cuda.synchronize()
        forms[name] = {"value": reps / (e0.elapsed_time(e1) / 1000.0), "unit": UNIT,
                       "iterations": int(st2["iterations"]), "rel_residual": st2["rel_residual"], "status": rc2,
                       "phases_ms": phases(st2)}
        if weights:
            forms[name]["note"] = ("the obstacle's fractional face weights (open fractions), an extension with no "
                                   "counterpart in xFluid")
        else:
            gpu_results[prec] = {"p": p2, "vel": vs[-1], "iterations": int(st2["iterations"]),
                                 "rel_residual": st2["rel_residual"]}
        c2.close()
    # xFluid's NormalPressureSolver matrix (classic Poisson, no face weights)
    # on the same scene and tolerance, mixed precision
    cn = ctx_for("mixed", 1, "normal")
    pn = torch.zeros_like(pres)
    project_dev(cn, [a.clone() for a in vel0], pn)
    torch.cuda.synchronize()
    reps = 2
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    vs = [[a.clone() for a in vel0] for _ in range(reps)]
    e0.record(stream)
    for r_ in range(reps):
        rcn, stn = project_dev(cn, vs[r_], pn)
    e1.record(stream)
    torch.cuda.synchronize()
    forms["normal_matrix_mixed"] = {"value": reps / (e0.elapsed_time(e1) / 1000.0), "unit": UNIT,
                                    "iterations": int(stn["iterations"]), "rel_residual": stn["rel_residual"],
                                    "status": rcn, "matrix": "NormalPressureSolver (pressuresolver.cpp)"}
    cn.close()
    # the simulator steps either side of the projection (body force before,
    # 6-layer velocity extrapolation after): fused into one call against the
    # force pass + projection + extrapolation as three calls, mixed precision
    cs = ctx_for("mixed", 1)
    f3 = (C.c_double * 3)(0.0, -9.8, 0.0)
    dt_s, layers = 1.0 / 30.0, 6

    def step_fused(vel, p):
        st = _lib.XfpStats()
        cs.check(cs.lib.xfp_project_step_f32(cs.ptr, ni, nj, nk, P(mat), P(vel[0]), P(vel[1]), P(vel[2]),
                                             None, None, None, P(p), f3, dt_s, layers, C.byref(st)))

    def step_separate(vel, p):
        cs.check(cs.lib.xfp_apply_forces_f32(cs.ptr, ni, nj, nk, P(mat), P(vel[0]), P(vel[1]), P(vel[2]), f3,
                                             dt_s))
        project_dev(cs, vel, p)
        cs.check(cs.lib.xfp_extrapolate_f32(cs.ptr, ni, nj, nk, P(mat), P(vel[0]), P(vel[1]), P(vel[2]), layers))

    ps = torch.zeros_like(pres)
    step_fused([a.clone() for a in vel0], ps)
    torch.cuda.synchronize()
    times = {}
    for name, fn in (("fused", step_fused), ("separate", step_separate)):
        vs = [[a.clone() for a in vel0] for _ in range(2)]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for r_ in range(2):
            fn(vs[r_], ps)
        e1.record(stream)
        torch.cuda.synchronize()
        times[name] = e0.elapsed_time(e1) / 2
    forms["sim_step_forces_project_extrapolate"] = {
        "ms_fused": times["fused"], "ms_separate": times["separate"], "layers": layers,
        "force": [0.0, -9.8, 0.0], "dt": dt_s, "unit": "ms per step"}
    cs.close()
    forms["mixed_phases_ms"] = phases(last)
    forms["mixed_over_plain_f32"] = value / world / forms["plain_f32"]["value"]
    forms["stall_cases"] = stall_cases(args, stream, ctx_for, project_dev, mat, vel0)
    forms["mixed_over_plain_f64"] = value / world / forms["plain_f64"]["value"]

    # ---------------- batched uneven scenes (C4) beside the headline ----------------
    batch = None if args.no_batch else batch_leg(args, rank, world, stream, barrier, max_over_ranks)

    # ---------------- differentiable rollout (C5) beside the headline ----------------
    rollout = None if args.no_batch else rollout_leg(stream, barrier, max_over_ranks)
    particles = None
    if not args.no_batch:
        if world == 1:
            # an extra beside the headline: at one rank, never lose the line over it
            # (with more ranks every rank must take the same barrier sequence)
            try:
                particles = particles_leg(stream, barrier, max_over_ranks, cpu=not args.no_cpu)
            except Exception as e:
                particles = {"error": repr(e)[:300]}
        else:
            particles = particles_leg(stream, barrier, max_over_ranks, cpu=(rank == 0 and not args.no_cpu))

    # ---------------- xFluid's whole time step on the device, beside the headline ----------------
    timestep = None
    if not args.no_batch:
        if world == 1:
            try:
                timestep = timestep_leg(stream, barrier, max_over_ranks)
            except Exception as e:
                timestep = {"error": repr(e)[:300]}
        else:
            timestep = timestep_leg(stream, barrier, max_over_ranks)

    # ---------------- CPU baseline and parity (rank 0, N=1 only) ----------------
    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sec, kind, ref = cpu_project_seconds(sc, keep=True)
        cpu = {"value": 1.0 / sec, "unit": UNIT, "cores": 1, "kind": kind,
               "sample": (f"one full {args.n}^3 projection ({sec:.1f} s): assemble + MIC(0)-PCG to 1e-6 + "
                          "applyPressure, single-threaded as xFluid's PCG is, on the headline's scene"
                          + ("" if kind == "reference" else " (oracle C port)"))}
        try:
            cpu["apply_pressure"] = cpu_apply_pressure(sc)
        except Exception as e:   # a reported extra: never lose the line over it
            cpu["apply_pressure"] = {"error": repr(e)[:200]}
        try:
            parity = parity_report(sc, kind, ref, gpu_results)
        except Exception as e:
            parity = {"error": repr(e)[:300]}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "mixed f32/f64",
            "data": "synthetic (seeded blob scene)",
            "config": dict(workload_config(args.n, rows, iters),
                           parallelism="replicas" if world > 1 else "single GPU",
                           tile_k=int(last.get("tile_k", 0))),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk.summary(), "parity": parity, "forms": forms, "batch": batch, "rollout": rollout, "particles": particles,
            "timestep": timestep}
    if rank == 0:
        print(json.dumps(line), flush=True)
    for c in (ctx, ctx_h):
        c.close()
    if world > 1:
        dist.destroy_process_group()


def batch_leg(args, rank, world, stream, barrier, max_over_ranks):
    """64 independent scenes, nx,ny,nz ~ U[32,160] (seed 4), blob masks, FP32
    faces, mixed precision to 1e-6: one batched call (xfp_project_batch_f32,
    tile height autotuned) against a loop of single-scene calls on the same
    inputs, both device-resident.  Across ranks the scenes are LPT-sharded
    (no collective on the data path); times are the max over ranks."""
    import ctypes as C
    import torch
    from xfluid_b200 import _lib, scenes
    from xfluid_b200.batch import BatchProjector, shard_scenes

    scs_all = scenes.batch_scenes(count=64, seed=4, lo=32, hi=160, dtype=np.float32)
    mine = shard_scenes([s.ncells for s in scs_all], world)[rank]
    scs = [scs_all[q] for q in mine]
    cells_all = sum(s.ncells for s in scs_all)
    T = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).cuda()
    base = [{"mat": T(s.mat), "u": T(s.u), "v": T(s.v), "w": T(s.w), "wu": T(s.wu), "wv": T(s.wv), "ww": T(s.ww)}
            for s in scs]

    def fresh():
        return [dict(b, u=b["u"].clone(), v=b["v"].clone(), w=b["w"].clone(),
                     pressure=torch.zeros((s.nk, s.nj, s.ni), device="cuda")) for b, s in zip(base, scs)]

    def timed(fn, reps):
        best = None
        for _ in range(reps):
            items = fresh()
            barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = fn(items)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = max_over_ranks(e0.elapsed_time(e1))
            best = ms if best is None else min(best, ms)
        return best, out

    o = _lib.default_options()
    # single solves with their tile height tuned per grid shape (cached by the warm-up loop)
    o.precision, o.tol, o.max_iter, o.device_pointers, o.tile_k = _lib.PREC["mixed"], TOL, MAXIT, 1, 0
    o.stream = C.c_void_p(stream.cuda_stream)
    ctx = _lib.Context(o)
    P = lambda x: None if x is None else C.c_void_p(x.data_ptr())

    def loop(items):
        iters = []
        for it, s in zip(items, scs):
            st = _lib.XfpStats()
            ctx.check(ctx.lib.xfp_project_f32(ctx.ptr, s.ni, s.nj, s.nk, P(it["mat"]), P(it["u"]), P(it["v"]),
                                              P(it["w"]), P(it["wu"]), P(it["wv"]), P(it["ww"]), P(it["pressure"]),
                                              C.byref(st)))
            iters.append(st.iterations)
        return iters

    bp = BatchProjector("mixed", tol=TOL, max_iter=MAXIT, tile_k=0, stream=stream.cuda_stream)

    def batched(items):
        ok = bp.project(items) if items else True
        return ok, [s["iterations"] for s in bp.stats], ((bp.stats[0]["tile_k"], bp.stats[0]["graph"])
                                                           if bp.stats else (None, None))

    loop(fresh())                       # warm-up
    ms_loop, it_loop = timed(loop, 2)
    batched(fresh())                    # warm-up: tile height timed and cached
    ms_batch, (ok, it_batch, (tile_k, graph)) = timed(batched, 3)
    ctx.close()
    bp.close()
    return {"workload": "64 scenes, nx,ny,nz ~ U[32,160] (seed 4), 32-blob masks, U[-1,1] FP32 faces, "
                        "mixed precision, tol 1e-6, device-resident",
            "metric": "cells/s", "value": cells_all / (ms_batch / 1000.0), "unit": "cells/s",
            "loop_value": cells_all / (ms_loop / 1000.0), "speedup_over_loop": ms_loop / ms_batch,
            "ms_batch": ms_batch, "ms_loop": ms_loop, "cells": cells_all, "n_scenes": len(scs_all),
            "all_converged": bool(ok), "iterations_equal_to_single": it_batch == it_loop, "tile_k": tile_k,
            "pcg_loop": "CUDA graph" if graph else "direct launches (graph capture refused)",
            "sharding": f"LPT over {world} rank(s)"}


def profile_case(n, tile_k=8):
    """Two mixed-precision projections of the n^3 blob scene, inputs on the device."""
    import ctypes as C
    import torch
    from xfluid_b200 import _lib, scenes
    sc = scenes.blob_scene(n, seed=SEED, dtype=np.float32)
    o = _lib.default_options()
    o.precision, o.tol, o.max_iter, o.device_pointers, o.tile_k = _lib.PREC["mixed"], TOL, MAXIT, 1, tile_k
    ctx = _lib.Context(o)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    P = lambda x: C.c_void_p(x.data_ptr())
    mat, wts = T(sc.mat), [T(a) for a in (sc.wu, sc.wv, sc.ww)]
    for _ in range(2):
        vel = [T(a) for a in (sc.u, sc.v, sc.w)]
        st = _lib.XfpStats()
        ctx.check(ctx.lib.xfp_project_f32(ctx.ptr, sc.ni, sc.nj, sc.nk, P(mat), *map(P, vel), *map(P, wts), None,
                                          C.byref(st)))
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": n, "rows": st.rows, "iterations": st.iterations,
                      "sweep_ms": st.ms_sweeps / max(1, st.sweeps)}))
    ctx.close()


ROLLOUT_BOXES = {"configured": ((0.6, 0.9), (0.6, 0.9), (0.6, 0.9)),
                 "inside_dam": ((0.1, 0.35), (0.1, 0.45), (0.2, 0.8))}


def rollout_leg(stream, barrier, max_over_ranks):
    """One gradient of the differentiable rollout at 128^3: 16 steps of
    (semi-Lagrangian advection -> projection) over the dam-break mask from
    u0 ~ U[-0.5,0.5] (seed 5), dt = 1/30, dx = 1/128, checkpoints every 4 steps,
    loss = sum of squared velocity in a box; mixed precision (FP32 fields).
    The gradient costs 16 forward, 16 recomputed and 16 adjoint projections.
    Two boxes: the configured [0.6,0.9]^3, which lies in air away from the dam
    (the adjoint projections' right-hand sides G^T g stay zero there, so their
    solves do nothing; reported), and a box inside the dam's fluid, where every
    adjoint projection solves a nonzero system."""
    import torch
    from xfluid_b200 import scenes
    from xfluid_b200.rollout import Rollout
    n = 128
    sc = scenes.dam_break(n, seed=1)
    rng = np.random.default_rng(5)
    u0 = [torch.from_numpy(rng.uniform(-0.5, 0.5, a.shape).astype(np.float32)).cuda() for a in (sc.u, sc.v, sc.w)]
    out = {}
    for name, box in ROLLOUT_BOXES.items():
        r = Rollout(torch.from_numpy(sc.mat).cuda(), steps=16, checkpoint_every=4, dt_over_dx=n / 30.0, box=box,
                    precision="mixed", tol=1e-6, max_iter=MAXIT)
        try:
            r.forward(*u0)
            r.backward()                         # warm-up
            barrier()
            torch.cuda.synchronize()
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            r.iterations = {"forward": 0, "backward": 0}
            e0.record(stream)
            loss = r.forward(*u0)
            e1.record(stream)
            g = r.backward()
            e2.record(stream)
            torch.cuda.synchronize()
            gn = float(sum(float((a.double() ** 2).sum()) for a in g) ** 0.5)
            rhs = r.adjoint_rhs_inf
            out[name] = {"box": [list(x) for x in box],
                         "forward_ms": max_over_ranks(e0.elapsed_time(e1)),
                         "gradient_ms": max_over_ranks(e0.elapsed_time(e2)), "projections_per_gradient": 48,
                         "pcg_iterations": dict(r.iterations), "loss": loss, "grad_norm": gn,
                         "adjoint_rhs_inf": {"max": max(rhs), "min": min(rhs),
                                             "zero_steps": sum(1 for x in rhs if x == 0.0)}}
        finally:
            r.close()
    return dict(out["configured"],
                workload="dam break 128^3, 16 advect+project steps, checkpoints every 4, u0 ~ U[-0.5,0.5] "
                         "(seed 5), box [0.6,0.9]^3, mixed precision, tol 1e-6",
                box_inside_dam=out["inside_dam"])


def timestep_leg(stream, barrier, max_over_ranks, n=128, warm=2, timed=4):
    """xFluid's whole time step on the device (xfluid_b200.simulation: field
    and material, forces + projection + extrapolation, particle advection and
    the particle-to-grid transfer) on the pool drop at n^3: pool y < 0.3 plus a
    fluid sphere (r 0.15 at (0.5,0.7,0.5)), a static solid sphere (r 0.1 at
    (0.3,0.2,0.5)) as solid cells, 8 particles per fluid cell seeded as
    xFluid seeds them, at rest; gravity -9.8, CFL 5, tol 1e-6, FP64 as the
    reference.  dt from the particles' speed (capped at 1/30).  Each step is
    blocking library calls; the steps are timed together with CUDA events."""
    import torch
    from xfluid_b200 import scenes
    from xfluid_b200.simulation import Simulation
    sc = scenes.pool_drop(n, seed=2)
    dx = 1.0 / n
    P = scenes.seed_particles(sc.mat, dx, seed=7, vel=np.zeros((int((sc.mat == 1).sum()) * 8, 3)))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    sim = Simulation(T(sc.mat), T(P), dx, force=(0.0, -9.8, 0.0), cfl=5.0, tol=TOL, max_iter=MAXIT)
    try:
        for _ in range(warm):
            sim.time_step(sim.step_dt(max_dt=1.0 / 30.0))
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        its = []
        e0.record(stream)
        for _ in range(timed):
            sim.time_step(sim.step_dt(max_dt=1.0 / 30.0))
            its.append(int(sim.stats.get("iterations", 0)))
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1)) / timed
        return {"workload": f"pool drop {n}^3, {len(P)} particles at rest, gravity -9.8, CFL 5, tol 1e-6, FP64; "
                            f"steps {warm + 1}-{warm + timed}",
                "particles": len(P), "ms_per_step": ms, "steps_per_s": 1000.0 / ms, "pcg_iterations": its,
                "stages": "distance field + material, save, forces + projection + extrapolation, advection, "
                          "particle-to-grid"}
    finally:
        sim.close()


def particles_leg(stream, barrier, max_over_ranks, cpu=True):
    """The particle steps around the projection on the 128^3 dam break: eight
    particles per fluid cell seeded as xFluid seeds them (jitter dx/5),
    velocities U[-1,1] (seed 11), the scene's faces (gravity impulse) with
    U[-0.5,0.5] noise on every face (particles move and hit the walls), saved
    faces perturbed,
    dt 0.01, ratio 0.95; the distance field at FluidSimulator's settings
    (subdivision 2, radius 3x the particle radius, threshold 0.4).  Device-
    resident FP64; each step is one blocking library call timed with CUDA
    events on the launching stream (mean of 5 after a warm-up, particles
    restored before each advection).  The CPU figure is the oracle (the
    reference's operation order, one thread) on the 64^3 version of the scene."""
    import ctypes as C
    import time

    import torch
    from xfluid_b200 import _lib, scenes

    def setup(n):
        sc = scenes.dam_break(n, seed=1, noise=0.5)
        dx = 1.0 / n
        P = scenes.seed_particles(sc.mat, dx, seed=11, jitter=0.2 * dx, vel_scale=1.0)
        rng = np.random.default_rng(11)
        saved = [a + 0.05 * rng.standard_normal(a.shape) for a in (sc.u, sc.v, sc.w)]
        return sc, dx, P, saved

    n = 128
    sc, dx, P, saved = setup(n)
    radius = 3.0 * (3 * (dx ** 3 / 8.0) / (4 * 3.141592653)) ** (1.0 / 3.0)
    o = _lib.default_options()
    o.device_pointers = 1
    o.stream = C.c_void_p(stream.cuda_stream)
    ctx = _lib.Context(o)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()   # noqa: E731
    P0, Pd = t(P), t(P)
    mat = t(np.asarray(sc.mat, np.uint8))
    uvw = [t(np.asarray(a, np.float64)) for a in (sc.u, sc.v, sc.w)]
    sv = [t(a) for a in saved]
    gf = [torch.zeros_like(a) for a in uvw]
    phi = torch.zeros((n * 2 + 1,) * 3, dtype=torch.float64, device="cuda")
    m2 = mat.clone()
    ptr = lambda a: C.c_void_p(a.data_ptr())   # noqa: E731
    L, N = ctx.lib, len(P)
    steps = {
        "advect": lambda: L.xfp_advect_particles_f64(ctx.ptr, n, n, n, dx, ptr(mat), *map(ptr, uvw), *map(ptr, sv),
                                                     0.95, 0.01, N, ptr(Pd)),
        "particles_to_grid": lambda: L.xfp_particles_to_grid_f64(ctx.ptr, n, n, n, dx, N, ptr(Pd), *map(ptr, gf)),
        "update_material": lambda: L.xfp_update_material(ctx.ptr, n, n, n, dx, N, ptr(Pd), ptr(m2)),
        "distance_field": lambda: L.xfp_distance_field_f64(ctx.ptr, n, n, n, dx, 2, radius, 0.4, N, ptr(Pd), ptr(phi),
                                                           ptr(m2)),
    }
    out = {"workload": f"dam break {n}^3, {N} particles (8 per fluid cell, xFluid's seeding, jitter dx/5), "
                       "velocities U[-1,1], faces with U[-0.5,0.5] noise, dt 0.01, ratio 0.95; field subdivision 2, radius 3x particle radius, "
                       "threshold 0.4; FP64, device-resident",
           "particles": N, "ms": {}, "particles_per_s": {}}
    try:
        for name, fn in steps.items():
            reps = []
            for rep in range(6):
                if name == "advect":
                    Pd.copy_(P0)
                barrier()
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ctx.check(fn())
                e1.record(stream)
                torch.cuda.synchronize()
                if rep > 0:
                    reps.append(e0.elapsed_time(e1))
            ms = max_over_ranks(float(np.mean(reps)))
            out["ms"][name] = ms
            out["particles_per_s"][name] = N / (ms * 1e-3)
        # algorithmic bytes of the advection: particles read + written (96 B),
        # the faces and material it samples are L2-resident at this size
        out["advect_gbs"] = N * 96 / (out["ms"]["advect"] * 1e-3) / 1e9
    finally:
        ctx.close()
    if cpu:
        import oracle   # the checker, timed here as the CPU baseline only
        scs, dxs, Ps, saveds = setup(64)
        O = oracle.Oracle()
        c = {}
        t0 = time.perf_counter()
        Pa = O.advect_particles(scs, saveds, Ps, 0.95, 0.01, dxs)
        c["advect"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        O.p2g((64, 64, 64), dxs, Pa)
        c["particles_to_grid"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        O.update_material(scs.mat, dxs, Pa)
        c["update_material"] = time.perf_counter() - t0
        rs = 3.0 * (3 * (dxs ** 3 / 8.0) / (4 * 3.141592653)) ** (1.0 / 3.0)
        t0 = time.perf_counter()
        O.distance_field(scs.mat, dxs, 2, rs, 0.4, Pa)
        c["distance_field"] = time.perf_counter() - t0
        out["cpu_baseline"] = {"kind": "port", "cores": 1, "sample": f"the 64^3 scene ({len(Ps)} particles)",
                               "particles_per_s": {k: len(Ps) / v for k, v in c.items()}}
    return out


def main():
    # The roofline's solve and vector-kernel durations come from CUDA events on
    # every 16th PCG iteration of the timed projections, the preconditioner's
    # first solve pair included (the library records none by default: an
    # event between two launches serialises them, and events on every launch
    # cost 6 % of a projection).
    os.environ.setdefault("XFP_KERNEL_EVENTS", "16")
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=25)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-scenes leg")
    ap.add_argument("--particles-case", action="store_true",
                    help="only run the particle-steps leg (128^3 dam break, no CPU baseline), print its JSON and "
                         "exit: the case the ncu captures of the particle kernels use")
    ap.add_argument("--profile-case", type=int, default=0, metavar="N",
                    help="only project the N^3 blob scene twice (mixed, device-resident) and exit: "
                         "the small case the ncu captures of the sweep kernels use")
    ap.add_argument("--tile-k", type=int, default=8, help="sweep tile height of --profile-case (8, 15 or 16)")
    args = ap.parse_args()
    if args.particles_case:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps(particles_leg(torch.cuda.current_stream(), lambda: None, lambda x: x, cpu=False)))
        return
    if args.profile_case:
        profile_case(args.profile_case, args.tile_k)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
    else:
        ours(args, rank, world)


if __name__ == "__main__":
    main()
