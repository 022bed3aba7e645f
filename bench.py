#!/usr/bin/env python
"""Frequency points per second of the periodic-MoM fill + solve sweep on B200.

Workload (the precision form of the meanderline polarizer): meander(a=5, b=10, h=6,
w1=w2=0.3 mm, ntri=3000) -> 2840 triangles, N = 3976 RWG unknowns, on a 1 mm eps_r=2.2
substrate between half-spaces, normal incidence, 101 frequencies 8..18 GHz.  One step =
the whole 101-point sweep of the sheet's partial GSM: modal tables, face-pair integrals,
fill, LU, basis transforms, solves (+ FP64 refinement) and modal projection.

value  = sweep points / s from the library's CUDA-event span of each step (inputs already
         on the device: mesh, topology and J/K cache resident);
e2e    = the same through the C ABI call with host buffers (per-point inputs copied in,
         dS copied out), CUDA events on the caller's stream around the call.
The FP64 form is timed too (fp64_value) and its results give max|dS| of the FP32 form.

Both arms compute the sheet's face-pair integrals (filljk!) once per 101-point sweep: the
GPU arm drops its cached integrals before every step, the CPU arm adds one J/K pass per
101 points.

At one GPU the line also carries the 6000-unknown targets (target_sweep: the meanderline at
ntri = 4000, N = 5610, 201 frequencies, FP32 + refinement against the FP64 form; grads: the
adjoint gradient of that sweep's objective in trace width, pitch and eps_r, grads/s), the
square patch (patch_sweep: N = 736, 11 frequencies) and the two-sheet oblique cascade
(cascade_sweep: Jerusalem cross on a lossy substrate, air gap, square aperture; 51
frequencies, theta = 30, phi = 45, so the face-pair integrals run at every point), both
through analyze in a child process of their own so that their outcome cannot touch this
line's other numbers.

--impl reference: the CPU oracle (C restatement + LAPACK) on the host cores, one point
per step with the sweep's J/K pass amortised over the 101 points.

Multi-GPU (torchrun): weak scaling, each rank runs its own 101-point sweep (frequency
band shifted by rank); no collectives on the data path; device time max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

# Worker streams beyond the default 8 hardware work queues would share queues (false
# dependencies); this process-local setting must precede CUDA context creation.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
NFREQ = 101
WORKLOAD = ("meanderline a=5 b=10 h=6 w1=w2=0.3 mm ntri=3000 (2840 faces, N=3976) on 1 mm eps_r=2.2, "
            "normal incidence, 101 freqs 8-18 GHz")
METRIC = "freq-points/sec fill+solve, FP32+refine vs FP64 on GPU at max|dS|<=1e-6; grads/s"
KERNELS = {  # profiled kernel kinds (PSS_PROF_*) -> name, roofline bound
    "tc_update": ("k_cgemm_tf32x3 (3xTF32 complex Schur update, tcgen05)", "tensor"),
    "panel": ("k_panel<FP32, 32> (cluster panel factorisation)", "hbm"),
    "simt_update": ("k_gemm32 (SIMT complex Schur update below the tensor-core size)", "tensor"),
}
# DRAM bytes (read + write) of one launch from an ncu capture of each kernel, with the
# algorithmic work of that same launch, so traffic scales to the average launch (the
# captures are summarised in profiles/); None where no capture exists.
TRAFFIC = {
    # trailing update of outer block 2 for a batch of 2 points (M = N = 3720, K = 128):
    # 252.7 MB read + 163.2 MB written, 2.834e10 algorithmic flops
    "tc_update": (252.7e6 + 163.2e6, 2.834e10),
    # FP32 panel of 2696 rows x 32 columns: 1.26 MB read, 0 written back to DRAM during the
    # launch (the rows stay in L2), 1.38 MB algorithmic
    "panel": (1.26e6, 2 * 2696 * 32 * 8.0),
    "simt_update": None,
}


CONFIG = {"workload": WORKLOAD, "points_per_sweep": NFREQ, "face_integrals": "once per sweep",
          "l2": "working set > L2 (Z is 253 MB FP64 + 126 MB FP32 per point)"}


def cpu_info():
    """Host CPU model and the thread counts the CPU legs run with (OpenMP of the oracle,
    BLAS of LAPACK's LU)."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    omp = blas = None
    try:
        from threadpoolctl import threadpool_info
        for t in threadpool_info():
            if t.get("user_api") == "openmp":
                omp = max(omp or 0, t["num_threads"])
            elif t.get("user_api") == "blas":
                blas = max(blas or 0, t["num_threads"])
    except Exception:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count(), "omp_threads": omp, "blas_threads": blas}


def load_package():
    import importlib.util
    if "pssfss_b200" in sys.modules:
        return sys.modules["pssfss_b200"]
    pkgdir = os.path.join(ROOT, "pssfss.jl_b200")
    spec = importlib.util.spec_from_file_location(
        "pssfss_b200", os.path.join(pkgdir, "__init__.py"), submodule_search_locations=[pkgdir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pssfss_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def build_case(rank=0, npts=NFREQ, ntri=3000, nfreq=NFREQ):
    pkg = load_package()
    from pssfss_b200.analyze import make_plan, sheet_gblocks, sheet_io
    sheet = pkg.meander(a=5, b=10, h=6, w1=0.3, w2=0.3, ntri=ntri, units=pkg.mm)
    strata = [pkg.Layer(), sheet, pkg.Layer(epsr=2.2, width=pkg.Length(1, pkg.mm)), pkg.Layer()]
    shift = 0.01 * rank
    freqs = np.linspace(8.0 + shift, 18.0 + shift, nfreq)[:npts]
    plan = make_plan(strata, freqs, {"θ": 0.0, "ϕ": 0.0})
    (ig, (i1, i2), isht, s), = sheet_gblocks(plan)
    rwg = plan.rwgdat[isht - 1]
    u = plan.uvec[isht - 1]
    ios = [sheet_io(pt.layers[i1 - 1:i2], sheet, s, pt.k0, pt.beta00) for pt in plan.points]
    return dict(plan=plan, sheet=sheet, rwg=rwg, rng=(i1, i2), s=s, u=u, ios=ios)


class ClockSampler:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def run_reference(args, rank, world):
    """CPU oracle on the host cores (bounded sample: one sweep point per step)."""
    if rank != 0:
        return
    sys.path.insert(0, ROOT)
    import oracle
    case = build_case(0)
    sheet, rwg, (i1, i2), s, u = case["sheet"], case["rwg"], case["rng"], case["s"], case["u"]
    pts = case["plan"].points
    t0 = time.perf_counter()
    io0 = case["ios"][0]
    jk = oracle.filljk(sheet, rwg, u / sheet.units.units_per_meter, io0.psi1, io0.psi2)
    oracle.prime_jk_cache(sheet, jk)
    t_jk = time.perf_counter() - t0
    times = []
    for step in range(args.warmup + args.steps):
        i = (step * 37) % len(pts)
        pt = pts[i]
        region = pt.layers[i1 - 1:i2]
        t = time.perf_counter()
        oracle.partial_dS(sheet, rwg, region, s, pt.k0, u, case["ios"][i])
        dt = time.perf_counter() - t
        if step >= args.warmup:
            times.append(dt)
    per_point = statistics.mean(times) + t_jk / NFREQ
    value = 1.0 / per_point
    ci = cpu_info()
    cores = max(ci["omp_threads"] or 0, ci["blas_threads"] or 0) or os.cpu_count()
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "freq-points/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_point * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic (structured meander mesh built from the reference's element recipe)",
            "config": dict(CONFIG),
            "cpu_baseline": {"value": value, "unit": "freq-points/s", "cores": cores, "kind": "port",
                             "sample": f"1 sweep point per step (fill+LU+solve+projection), {args.steps} points, "
                                       f"+ one J/K pass ({t_jk:.1f} s) amortised over {NFREQ} points", **ci},
            "e2e": {"value": value, "unit": "freq-points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(case):
    """Bounded CPU-oracle sample for the report line (~10-30 s on the host cores)."""
    sys.path.insert(0, ROOT)
    import oracle
    sheet, rwg, (i1, i2), s, u = case["sheet"], case["rwg"], case["rng"], case["s"], case["u"]
    pt = case["plan"].points[NFREQ // 2]
    io = case["ios"][NFREQ // 2]
    t0 = time.perf_counter()
    jk = oracle.filljk(sheet, rwg, u / sheet.units.units_per_meter, io.psi1, io.psi2)
    t_jk = time.perf_counter() - t0
    oracle.prime_jk_cache(sheet, jk)
    t1 = time.perf_counter()
    dS_ref, _, _ = oracle.partial_dS(sheet, rwg, pt.layers[i1 - 1:i2], s, pt.k0, u, io)
    t_pt = time.perf_counter() - t1
    ci = cpu_info()
    cores = max(ci["omp_threads"] or 0, ci["blas_threads"] or 0) or os.cpu_count()
    return {"value": 1.0 / (t_pt + t_jk / NFREQ), "unit": "freq-points/s", "cores": cores,
            "kind": "port", "sample": f"1 sweep point (fill+LU+solve+projection {t_pt:.2f} s) + J/K pass "
                                      f"({t_jk:.1f} s) amortised over {NFREQ} points", **ci}, NFREQ // 2, dS_ref


def patch_cpu_baseline():
    """The square-patch configuration (the one the reference itself runs on a CPU) whole
    through the CPU oracle's ``analyze`` on the host cores: every step of the 11-point sweep
    (J/K pass, fill, LAPACK LU and solves, projection, cascade), one warm-up run first."""
    sys.path.insert(0, ROOT)
    import oracle
    load_package()
    from pssfss_b200 import workloads
    strata, flist, steer = workloads.square_patch_sweep()
    oracle.analyze(strata, flist, steer)
    t = time.perf_counter()
    res = oracle.analyze(strata, flist, steer)
    sec = time.perf_counter() - t
    ci = cpu_info()
    cores = max(ci["omp_threads"] or 0, ci["blas_threads"] or 0) or os.cpu_count()
    return {"value": len(res) / sec, "unit": "freq-points/s", "cores": cores, "kind": "port",
            "sample": f"the whole {len(res)}-point sweep through the oracle's analyze ({sec:.2f} s)"}


def run_rings(args, rank, world=1, local=0):
    """Freq-points/s over the seeded batch of 64 ring problems (period 6-12 mm, 300-3000
    triangles, so unknown counts 480-4800; theta in {0, 15, 30, 45}; 21 frequencies each;
    1344 points), FP32 + refinement, with the batch size and LU tile shape of the stored
    autotuning table.  On one GPU all 64 problems go into ONE library call
    (analyze.analyze_many -> pss_partial_gsms_multi: a shared work list of like-N batches,
    largest first); under torchrun the problems are split across the ranks by estimated cost
    (sweep.analyze_many_sharded: one call per rank, one gather of the results), a fixed total
    workload (strong scaling).  value = points / device span of the ranks' calls (max over
    ranks); e2e = points / wall clock of analyze_many_sharded (host planning, transfers, the
    cascade and the gather included, max over ranks), device synchronised on both sides."""
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    load_package()
    from pssfss_b200 import autotune, workloads
    from pssfss_b200.sweep import analyze_many_sharded
    batch = workloads.ring_batch()
    npts = sum(len(f) for _, f, _ in batch)
    tuned = os.path.exists(autotune.TABLE) and not args.no_tuning
    tuning = autotune.lookup if tuned else None
    for _ in range(args.warmup):
        analyze_many_sharded(batch, precision="fp32r", tuning=tuning)
    walls, spans = [], []
    for _ in range(args.steps):
        st = {}
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t = time.perf_counter()
        analyze_many_sharded(batch, precision="fp32r", tuning=tuning, stats=st)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t
        span = st["timings_ms"]["total"] / 1e3 if "timings_ms" in st else 0.0
        if dist:
            m = torch.tensor([wall, span], dtype=torch.float64, device="cuda")
            dist.all_reduce(m, op=dist.ReduceOp.MAX)
            wall, span = float(m[0]), float(m[1])
        walls.append(wall)
        spans.append(span)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {"metric": "freq-points/sec over a batch of ring problems of differing size", "value": npts / statistics.mean(spans),
            "unit": "freq-points/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.mean(spans) * 1e3, "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak",
            "vs_baseline": None, "dtype": "c64+c128-refine",
            "data": "synthetic (seeded ring problems, own Delaunay meshes)",
            "e2e": {"value": npts / statistics.mean(walls), "unit": "freq-points/s",
                    "note": "wall clock of analyze_many_sharded: host planning, transfers, cascade, gather included"},
            "config": {"workload": f"64 ring problems (seed 0), {npts} points, N "
                                   f"{min(b[0][1].nface for b in batch)}..{max(b[0][1].nface for b in batch)} faces, "
                                   + ("one pss_partial_gsms_multi call" if world == 1 else
                                      f"problems split over {world} ranks by estimated cost, one call per rank"),
                       "parallelism": f"problems x{world}",
                       "tuning": autotune.TABLE.split(os.sep + "pssfss.jl_b200" + os.sep)[-1] if tuned else "defaults",
                       "table": [{k: b[k] for k in ("nmax", "n", "batch", "panel_w", "outer_nb")}
                                 for b in (json.load(open(autotune.TABLE))["buckets"] if tuned else [])]}}
    print(json.dumps(line), flush=True)


def run_autotune(args, rank):
    """Search the batch size and LU tile shape per unknown-count bucket and store the table."""
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(0)
    load_package()
    from pssfss_b200 import autotune
    tab = autotune.tune()
    print(json.dumps({"autotune": autotune.TABLE, "buckets": [{k: b[k] for k in ("nmax", "n", "batch", "panel_w",
                                                                                   "outer_nb", "ms_per_point",
                                                                                   "default_ms_per_point")}
                                                               for b in tab["buckets"]]}), flush=True)


def grads_sample(npts=None, warmup=1, steps=1, precision="fp32r"):
    """Adjoint gradient of Σ_f (|S21_TE|² − |S21_TM|²) in trace width, pitch and substrate
    eps_r of the meanderline at ntri = 4000 (3960 faces, N = 5610) over 201 frequencies
    8-18 GHz: per point one FP32 + refinement factorisation, forward and transposed solves on
    it, and per perturbed set (+/- step of each parameter) a fused assemble-and-contract pass
    (pss_partial_gsms_adj).  Wall clock per gradient, host planning included, device
    synchronised on both sides.  Returns (seconds per gradient, objective, gradient)."""
    import functools
    import torch
    load_package()
    from pssfss_b200 import engine, workloads
    from pssfss_b200.gradient import meander_linearized_gradient
    params, flist, ntri = workloads.meander_gradient_workload()
    if npts:
        flist = flist[:npts]
    part = functools.partial(engine.partial_gsms_adjoint, precision=precision)
    for _ in range(warmup):
        meander_linearized_gradient(params, flist, part, ntri=ntri)
    times = []
    for _ in range(steps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        f, g = meander_linearized_gradient(params, flist, part, ntri=ntri)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t)
    return statistics.mean(times), float(f), {k: float(v) for k, v in g.items()}, len(flist), ntri


def run_grads(args, rank):
    """The adjoint gradient alone (grads/s), one line."""
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(0)
    sec, f, g, nf, ntri = grads_sample(args.grad_npts or None, args.warmup, args.steps)
    line = {"metric": "grads/s (adjoint gradient of the meanderline sweep objective)", "value": 1.0 / sec,
            "unit": "grads/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64+c128-refine",
            "data": "synthetic (structured meander mesh built from the reference's element recipe)",
            "config": {"workload": f"meanderline w=0.3 a=5 mm ntri={ntri} on 1 mm eps_r=2.2, {nf} freqs 8-18 GHz, "
                                   "d/d(w, a, eps_r)", "objective": f, "gradient": g}}
    print(json.dumps(line), flush=True)


def _analyze_rates(strata, flist, steer):
    """Points/s of ``analyze`` on one workload (wall clock with the device synchronised on both
    sides: host planning, every sheet's sweep, the GSM cascade), FP64 and FP32 + refinement
    after one warm-up each, and the largest |S| difference between the two forms."""
    import torch
    from pssfss_b200.analyze import analyze

    def run(prec):
        torch.cuda.synchronize()
        t = time.perf_counter()
        res = analyze(strata, flist, steer, precision=prec)
        torch.cuda.synchronize()
        return res, time.perf_counter() - t

    out = {}
    for prec in ("fp64", "fp32r"):
        run(prec)  # warm-up: sheet uploads, buffers, kernels
        out[prec] = run(prec)
    (r64, t64), (r32, t32) = out["fp64"], out["fp32r"]
    npts = len(r64)
    dmax = max(float(np.max(np.abs(a.gsm[k] - b.gsm[k]))) for a, b in zip(r32, r64)
               for k in ((1, 1), (1, 2), (2, 1), (2, 2)))
    return {"fp64_value": npts / t64, "fp32r_value": npts / t32, "unit": "freq-points/s",
            "timed": "analyze() wall clock after one warm-up per form (host planning, sweeps, cascade)",
            "max_abs_S_fp32r_vs_fp64": dmax}


def config_sweeps():
    """The two smaller configurations through ``analyze``: the free-standing square patch
    (8 mm in a 10 mm cell, 512 triangles, N = 736; 11 frequencies 10-20 GHz, normal incidence)
    and the two-sheet cascade (workloads.jerusalem_aperture_cascade: a Jerusalem cross of about
    1500 triangles on 0.5 mm eps_r = 3, tan d = 0.002, a 2 mm air gap, a 6 mm square aperture of
    about 1200 triangles; 51 frequencies 5-25 GHz at theta = 30, phi = 45, so both sheets'
    face-pair integrals run at every point)."""
    load_package()
    from pssfss_b200 import workloads
    strata, flist, steer = workloads.square_patch_sweep()
    patch = dict(workload="square patch 8 mm in a 10 mm cell (%d faces), free-standing, 11 freqs 10-20 GHz, "
                          "normal incidence" % strata[1].nface, **_analyze_rates(strata, flist, steer))
    strata, flist, steer = workloads.jerusalem_aperture_cascade()
    casc = dict(workload="Jerusalem cross (%d faces) on 0.5 mm eps_r=3 tan d=0.002, 2 mm air gap, square "
                         "aperture (%d faces), 51 freqs 5-25 GHz, theta=30 phi=45" % (strata[1].nface, strata[4].nface),
                **_analyze_rates(strata, flist, steer))
    return {"patch_sweep": patch, "cascade_sweep": casc}


def target_sweep(fp64_steps=1):
    """The 6000-unknown sweep (meanderline ntri = 4000, N = 5610, 201 frequencies, normal
    incidence): points/s of the FP32 + refinement form and of the plain FP64 form (device span
    of the library, face integrals once per sweep), their ratio and max|dS| between them."""
    from pssfss_b200 import engine
    case = build_case(0, ntri=4000, nfreq=201)
    call = (case["sheet"], case["rwg"], case["plan"].points, case["rng"], case["s"], case["u"], case["ios"])
    npts = len(case["plan"].points)

    def sweep(prec):
        engine.clear_face_integrals(case["sheet"], case["rwg"])
        st = {}
        dS = engine.partial_gsms(*call, precision=prec, stats=st)
        return dS, st["timings_ms"]["total"], st["status"]

    sweep("fp32r")  # warm-up: buffers sized, kernels loaded
    d32, t32, s32 = sweep("fp32r")
    t64s = []
    for _ in range(max(1, fp64_steps)):
        d64, t64, _ = sweep("fp64")
        t64s.append(t64)
    t64 = statistics.mean(t64s)
    return {"workload": "meanderline a=5 b=10 h=6 w1=w2=0.3 mm ntri=4000 (3960 faces, N=%d) on 1 mm eps_r=2.2, "
                        "normal incidence, 201 freqs 8-18 GHz" % case["rwg"].nbf,
            "fp32r_value": npts / (t32 / 1e3), "fp64_value": npts / (t64 / 1e3), "unit": "freq-points/s",
            "fp32r_speedup_vs_fp64": t64 / t32,
            "max_abs_dS_fp32r_vs_fp64": float(max(np.max(np.abs(a - b)) for a, b in zip(d32, d64))),
            "refine_fallbacks": int(sum(1 for x in s32 if x & 32))}


def config_sweeps_child(timeout=240):
    """``config_sweeps`` in a child process (``bench.py --configs``): its two entries, or the
    reason there are none."""
    try:
        p = subprocess.run([sys.executable, os.path.abspath(__file__), "--configs"], capture_output=True,
                           text=True, timeout=timeout, cwd=ROOT)
        lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
        if p.returncode == 0 and lines:
            return json.loads(lines[-1])
        err = {"error": f"exit {p.returncode}: " + (p.stderr or p.stdout)[-300:]}
    except Exception as e:  # report, never fake
        err = {"error": str(e)[:200]}
    return {"patch_sweep": err, "cascade_sweep": err}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--npts", type=int, default=NFREQ,
                    help="sweep points per step (default: the full 101-point sweep; fewer only for profiling)")
    ap.add_argument("--grads", action="store_true",
                    help="time gradients of the meander gradient workload instead (grads/s)")
    ap.add_argument("--grad-npts", type=int, default=0,
                    help="frequencies of the gradient workload (default: all 201)")
    ap.add_argument("--rings", action="store_true",
                    help="time the seeded batch of 64 ring problems of differing size instead")
    ap.add_argument("--configs", action="store_true",
                    help="time the square patch and the two-sheet oblique cascade through analyze "
                         "(one JSON line; the default run adds both to its line)")
    ap.add_argument("--no-targets", action="store_true",
                    help="skip the 6000-unknown target sweep and the gradient (profiling runs)")
    ap.add_argument("--no-tuning", action="store_true", help="--rings with the library defaults")
    ap.add_argument("--autotune", action="store_true",
                    help="search batch size and LU tile shape per unknown count; write the table")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.grads:
        return run_grads(args, rank)
    if args.rings:
        return run_rings(args, rank, world, local)
    if args.configs:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(config_sweeps()), flush=True)
        return None
    if args.autotune:
        return run_autotune(args, rank)

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    pkg = load_package()
    from pssfss_b200 import engine
    case = build_case(rank, args.npts)
    dev = local
    call_args = (case["sheet"], case["rwg"], case["plan"].points, case["rng"], case["s"], case["u"], case["ios"])

    def step(precision):
        # face-pair integrals once per sweep, as the CPU arm pays them
        engine.clear_face_integrals(case["sheet"], case["rwg"], dev)
        st = {}
        dS = engine.partial_gsms(*call_args, precision=precision, device=dev, stats=st)
        return dS, st

    for _ in range(args.warmup):
        dS32, _ = step("fp32r")
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(dev)
    sampler.start()
    l0 = engine.lib().pss_kernel_launches()
    spans, e2e_ms, statuses = [], [], []
    prof = {k: {"launches": 0, "ms": 0.0, "work": 0.0} for k in KERNELS}
    phases = {}
    engine.set_profiling(True, device=dev)
    for _ in range(args.steps):
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record()
        dS32, st = step("fp32r")
        ev1.record()
        ev1.synchronize()
        e2e_ms.append(ev0.elapsed_time(ev1))
        spans.append(st["timings_ms"]["total"])
        statuses.extend(st["status"])
        g = engine.profile_result(device=dev)
        for kind in prof:
            for k in prof[kind]:
                prof[kind][k] += g[kind][k]
        for k, v in st["timings_ms"].items():
            phases[k] = phases.get(k, 0.0) + v / args.steps
    engine.set_profiling(False, device=dev)
    torch.cuda.synchronize()
    launches = engine.lib().pss_kernel_launches() - l0
    clocks = sampler.stop()
    if dist:
        dist.barrier()
    # FP64 form (same sweep) for the speed-up and the accuracy gate
    spans64 = []
    for _ in range(max(1, args.fp64_steps)):
        dS64, st64 = step("fp64")
        spans64.append(st64["timings_ms"]["total"])
    max_dS = float(max(np.max(np.abs(a - b)) for a, b in zip(dS32, dS64)))

    tot_ms = sum(spans)
    tot_e2e = sum(e2e_ms)
    if dist:
        t = torch.tensor([tot_ms, tot_e2e, float(np.mean(spans64)), max_dS], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_ms, tot_e2e, mean64, max_dS = t.tolist()
    else:
        mean64 = float(np.mean(spans64))
    npts = len(case["plan"].points)
    value = world * npts * args.steps / (tot_ms / 1e3)
    e2e = world * npts * args.steps / (tot_e2e / 1e3)
    fp64_value = world * npts / (mean64 / 1e3)
    nm = len(case["ios"][0].wobs)
    h2d = npts * (8 + 16 + nm * (16 + 32 + 16 + 16))
    d2h = npts * (nm * nm * 16 + 4)
    if rank == 0:
        pk, pk_kind = peaks()
        line = {"metric": METRIC, "value": value, "unit": "freq-points/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c64+c128-refine",
                "data": "synthetic (structured meander mesh built from the reference's element recipe)",
                "config": dict(CONFIG, points_per_sweep=npts),
                "precision": "fp32r", "parallelism": f"weak x{world}: independent sweeps per GPU",
                "fp64_value": fp64_value, "fp32r_speedup_vs_fp64": value / fp64_value / world * world,
                "max_abs_dS_fp32r_vs_fp64": max_dS,
                "refine_fallbacks": int(sum(1 for s in statuses if s & 32)),
                "e2e": {"value": e2e, "unit": "freq-points/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h},
                "gpu_launches": int(launches), "clocks": clocks,
                "phase_ms_per_step_worker0": phases, "peaks_source": pk_kind}
        # Roofline of the profiled kernels (CUDA events around every launch on its own
        # stream during the timed steps): achieved = algorithmic work / summed launch time.
        # The dominant one (largest summed time) is "roofline"; all are in "kernels".
        hbm = float(pk["hbm_gbs"])
        tens = float(pk.get("bf16_tflops_sustained", pk["bf16_tflops"]))
        roofs = {}
        for kind, (name, bound) in KERNELS.items():
            g = prof[kind]
            if g["launches"] == 0 or g["ms"] <= 0:
                continue
            per = g["work"] / g["launches"]
            if bound == "tensor":
                achieved, peak, unit = g["work"] / (g["ms"] / 1e3) / 1e12, tens, "TFLOP/s"
            else:
                achieved, peak, unit = g["work"] / (g["ms"] / 1e3) / 1e9, hbm, "GB/s"
            tr = TRAFFIC[kind]
            roofs[kind] = {"kernel": name, "bound": bound, "achieved": achieved, "peak": peak, "unit": unit,
                           "frac": achieved / peak,
                           "traffic": (tr[0] / tr[1] * per) if tr else None,
                           "launches": g["launches"], "avg_launch_us": 1e3 * g["ms"] / g["launches"],
                           "total_ms": g["ms"],
                           "peak_note": f"{pk_kind}: " + ("HBM copy GB/s" if bound == "hbm" else
                                                          "dense bf16 sustained TFLOP/s (TF32 dense is half; "
                                                          "3xTF32 executes 3 products per algorithmic one)")}
        if roofs:
            dom = max(roofs, key=lambda k: roofs[k]["total_ms"])
            line["roofline"] = roofs[dom]
            line["kernels"] = roofs
        else:
            line["roofline"] = None
        if not args.no_cpu_baseline:
            try:
                cb, ip, dref = cpu_baseline_sample(case)
                line["cpu_baseline"] = cb
                if ip < len(dS32):
                    # the FP64 oracle's dS at that point against both device forms
                    line["max_abs_dS_fp32r_vs_oracle"] = float(np.max(np.abs(dS32[ip] - dref)))
                    line["max_rel_dS_fp64_vs_oracle"] = float(np.max(np.abs(dS64[ip] - dref)) / np.max(np.abs(dref)))
                    line["oracle_check_point_ghz"] = float(case["plan"].points[ip].fghz)
            except Exception as e:  # report, never fake
                line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        if world == 1 and not args.no_targets:
            try:
                line["target_sweep"] = target_sweep(args.fp64_steps)
            except Exception as e:
                line["target_sweep"] = {"error": str(e)[:200]}
            try:
                sec, f, g, nf, ntri = grads_sample()
                line["grads"] = {"value": 1.0 / sec, "unit": "grads/s", "ms_per_grad": sec * 1e3,
                                 "workload": f"meanderline ntri={ntri} (N=5610), {nf} freqs, adjoint "
                                             "d/d(w, a, eps_r) of sum_f |S21_TE|^2 - |S21_TM|^2, FP32 + refinement",
                                 "objective": f, "gradient": g, "timed": "1 gradient after 1 warm-up, host "
                                 "planning included"}
            except Exception as e:
                line["grads"] = {"error": str(e)[:200]}
            line.update(config_sweeps_child())
            if not args.no_cpu_baseline and "error" not in line["patch_sweep"]:
                try:
                    line["patch_sweep"]["cpu_baseline"] = patch_cpu_baseline()
                except Exception as e:  # report, never fake
                    line["patch_sweep"]["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
