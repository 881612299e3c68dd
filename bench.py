#!/usr/bin/env python
"""Benchmark: bfps NSVEparticles step (IF-RK3 vorticity DNS + tracers) on B200.

Default workload (the configuration the headline metric is quoted on):
512^3 grid, FP32 fields, nu = 0.002, dt = 0.001, seeded k^4 exp(-2 (k/4)^2)
initial spectrum, linear band forcing on 1.5 <= |k| <= 3 (amplitude 0.5),
smooth dealiasing, 4e6 tracers with the (neighbours 3, smoothness 2) kernel
and AB3.  One step = NSVEparticles::step: velocity at t -> tracers advance ->
fluid IF-RK3 step.  Inputs are synthetic (seeded), generated on the host.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload C3]
    python bench.py --impl reference ...   # CPU restatement on host cores

Multi-GPU runs are independent replicas (one per rank, no data exchange;
scaling "weak"); timing is on the device (CUDA events on the engine's own
stream) and the max over ranks is reported.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # 512^3 FP32 + 4e6 tracers (n=3, m=2), AB3
    "C3": dict(n=512, precision="single", nu=0.002, dt=0.001, k0=4.0, ntracers=4_000_000,
               neighbours=3, smoothness=2, nsteps_ab=3, dealias=1, accuracy_steps=100),
    # the plain FP64 path at 512^3 (comparator of the precision form)
    "C3_fp64": dict(n=512, precision="double", nu=0.002, dt=0.001, k0=4.0,
                    ntracers=4_000_000, neighbours=3, smoothness=2, nsteps_ab=3, dealias=1),
    # 256^3 FP32 + 1e5 tracers (n=2, m=2), AB4
    "C2": dict(n=256, precision="single", nu=0.005, dt=0.002, k0=3.0, ntracers=100_000,
               neighbours=2, smoothness=2, nsteps_ab=4, dealias=1, accuracy_steps=200),
    # 32^3 FP64, 1024 tracers, 6-point Lagrange, AB2, 2/3 dealiasing
    "C1": dict(n=32, precision="double", nu=0.1, dt=0.01, k0=3.0, ntracers=1024,
               neighbours=2, smoothness=0, nsteps_ab=2, dealias=0),
    # batched ensemble: 40 x 32^3, 16 x 64^3, 8 x 128^3, FP32, 1e4 Lagrange-6 tracers
    # each, AB4, dt from CFL 0.5, 500-step solves
    "C4": dict(kind="ensemble", sizes=[32] * 40 + [64] * 16 + [128] * 8, precision="single",
               nu_range=(0.005, 0.05), ntracers=10_000, neighbours=2, smoothness=0, nsteps_ab=4,
               solve_steps=500),
    # serving: Poisson arrivals (20/s), N in {64: 0.6, 128: 0.3, 256: 0.1}, FP32,
    # 100..1000 steps, 0..1e5 cubic-spline tracers, HBM budget 150 GB
    "C5": dict(kind="serving", rate=20.0, requests=60, budget=150e9, precision="single"),
}
FORCING = dict(forcing_type="linear", fk0=1.5, fk1=3.0, famplitude=0.5)
KIND_NAMES = ["IZ", "IY", "X", "FY", "FZ", "kspace", "tracers", "stats"]


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def algorithmic_bytes(cfg):
    """Per-step and per-kernel-launch algorithmic bytes.

    U = N^2 (N+2) P is one scalar field (real padded or half-spectrum complex).
    Step model (2-pass fused): 105 U for the IF-RK3 step; tracers add
    n * 24 * (k+2) + 6 N^3 P (write real u once, read it once in the gather).
    Per launch of this engine's kernels (what each must move at least):
    IZ 9U, IY 12U, X 9U (+ 3 N^3 P when it also writes the real velocity),
    FY 6U, FZ 9U (stage 1) / 12U (stages 2, 3), tracers n*24*(k+2) + 3 N^3 P.
    """
    n = cfg["n"]
    P = 4 if cfg["precision"] == "single" else 8
    U = n * n * (n + 2) * P
    k = cfg["nsteps_ab"]
    nt = cfg["ntracers"]
    real3 = 3 * n ** 3 * P
    step = 105 * U + nt * 24 * (k + 2) + 2 * real3
    per_launch = {
        "IZ": 9 * U,
        "IY": 12 * U,
        "X": 9 * U + (real3 / 3.0 if nt else 0.0),
        "FY": 6 * U,
        "FZ": (9 * U + 12 * U + 12 * U) / 3.0,
        "kspace": 0.0,
        "tracers": nt * 24 * (k + 2) + real3,
        "stats": 0.0,
    }
    return step, per_launch, U


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one launch
# divided by its algorithmic bytes, from the ncu captures summarised under
# profiles/ (256^3 FP32 passes; tracer kernel at 4e6 tracers on 256^3).
# Traffic at another size is taken to scale with the algorithmic bytes.
TRAFFIC_RATIO = {"X": 0.951, "IZ": 0.93, "IY": 0.949, "FY": 0.878, "FZ": 0.989, "tracers": 0.983}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 9:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(ngpus):
    """Replica ranks (bfps_b200.replicas): NCCL over the GPUs of one node."""
    from bfps_b200 import replicas
    return replicas.setup("nccl")


def barrier(pg):
    from bfps_b200 import replicas
    replicas.barrier(pg)


def allmax(pg, v):
    from bfps_b200 import replicas
    return replicas.allmax(pg, v)


def make_inputs(cfg, seed):
    from bfps_b200 import ic
    n = cfg["n"]
    cdt = np.complex64 if cfg["precision"] == "single" else np.complex128
    w0 = ic.vorticity_ic(n, seed=seed, k0=cfg["k0"], dealias_type=cfg["dealias"], dtype=cdt)
    pos = ic.tracer_ic(cfg["ntracers"], seed=seed)
    return w0, pos


def build_solver(cfg, w0, pos, device):
    from bfps_b200.solver import vorticity_equation, particles_system
    ve = vorticity_equation(cfg["n"], precision=cfg["precision"], dealias_type=cfg["dealias"],
                            device=device)
    ve.nu = cfg["nu"]
    ve.forcing_type = FORCING["forcing_type"]
    ve.fk0, ve.fk1, ve.famplitude = FORCING["fk0"], FORCING["fk1"], FORCING["famplitude"]
    ve.set_cvorticity(w0)
    ps = particles_system(ve, pos, cfg["neighbours"], cfg["smoothness"], cfg["nsteps_ab"])
    return ve, ps


def acceleration_report(ve, ps, cfg, reps=3):
    """NSVEparticles::do_stats acceleration sampling (pressure, Lagrangian
    acceleration, inverse transform, tracer gather) on the current state:
    device time per call from per-launch CUDA events, and achieved bandwidth
    against its algorithmic bytes, 109 U + 48 n (19 launches: velocity to
    real space 18U, two products 12U, two forward transforms 36U, two
    pressure contractions 9U, velocity 6U, acceleration 7U, inverse
    transform 18U, gather 3U + 48 n)."""
    from bfps_b200 import _lib
    L = _lib.lib()
    out = np.empty((ps.n, 3))
    L.bfg_particles_sample_acceleration(ps.handle, _lib.ptr(out))
    L.bfg_profile(ve.handle, 1)
    for _ in range(reps):
        L.bfg_particles_sample_acceleration(ps.handle, _lib.ptr(out))
    tot, n = 0.0, 0
    for k in range(len(KIND_NAMES)):
        t, c = _lib.ctypes.c_double(), _lib.ctypes.c_int64()
        L.bfg_profile_read(ve.handle, k, _lib.ctypes.byref(t), _lib.ctypes.byref(c))
        tot += t.value
        n += c.value
    L.bfg_profile(ve.handle, 0)
    ms = tot / reps
    P = 4 if cfg["precision"] == "single" else 8
    U = cfg["n"] ** 2 * (cfg["n"] + 2) * P
    nbytes = 109 * U + 48 * ps.n
    peak, _ = peaks()
    return {"device_ms": round(ms, 3), "launches_per_call": n // reps,
            "algorithmic_bytes": int(nbytes), "achieved_gbs": round(nbytes / (ms / 1e3) / 1e9, 1),
            "frac_of_peak": round(nbytes / (ms / 1e3) / 1e9 / peak, 4)}


def precision_report(cfg, w0, pos, device, nsteps):
    """Precision form against FP64: the same initial field (the FP32-rounded
    one) and tracers stepped nsteps times in FP32 and in FP64; relative error
    of the energy spectrum E(k) = tr(spec_uu)/2 over the shells holding at
    least 1e-6 of the peak shell energy, of the total energy, of the
    dissipation eps = 2 nu Omega, and the largest tracer displacement error
    relative to the box (2 pi)."""
    from bfps_b200.solver import NSVEparticles_step
    res = {}
    for prec in ("single", "double"):
        c = dict(cfg, precision=prec)
        w = w0.astype(np.complex64).astype(np.complex128 if prec == "double" else np.complex64)
        ve, ps = build_solver(c, w, pos, device)
        NSVEparticles_step(ve, ps, cfg["dt"], nsteps)
        st = ve.do_stats()
        sv, sw = st["velocity"][0], st["vorticity"][0]
        ek = 0.5 * np.einsum("kii->k", sv)
        omega = 0.5 * np.einsum("kii->k", sw).sum()
        res[prec] = (ek, 2 * cfg["nu"] * omega, ps.state()[0])
        ps.close()
        ve.close()
    ek32, eps32, p32 = res["single"]
    ek64, eps64, p64 = res["double"]
    keep = ek64 >= 1e-6 * ek64.max()
    rel = np.abs(ek32[keep] - ek64[keep]) / ek64[keep]
    return {"steps": nsteps, "spectrum_max_rel": float(rel.max()),
            "spectrum_shells": int(keep.sum()),
            "energy_rel": float(abs(ek32.sum() - ek64.sum()) / ek64.sum()),
            "dissipation_rel": float(abs(eps32 - eps64) / eps64),
            "positions_max_abs_over_box": float(np.abs(p32 - p64).max() / (2 * np.pi)),
            "how": "same FP32-rounded initial field and tracers, stepped in FP32 and FP64 "
                   "with this engine; shells with E64(k) >= 1e-6 max"}


def run_ours(args, cfg):
    import torch
    from bfps_b200 import _lib
    from bfps_b200.solver import NSVEparticles_step
    world, rank, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = local
    w0, pos = make_inputs(cfg, seed=rank)
    ve, ps = build_solver(cfg, w0, pos, dev)
    L = _lib.lib()
    dt = cfg["dt"]
    # warm-up
    for _ in range(args.warmup):
        NSVEparticles_step(ve, ps, dt)
    torch.cuda.synchronize()
    # timed region: K steps in one engine call, device-timed on its stream,
    # per-kernel events on the same stream
    L.bfg_profile(ve.handle, 1)
    launches0 = ve.kernel_launches()
    clocks = ClockSampler(dev)
    clocks.start()
    barrier(pg)
    torch.cuda.synchronize()
    NSVEparticles_step(ve, ps, dt, args.steps)
    ms = ve.last_step_ms()
    torch.cuda.synchronize()
    barrier(pg)
    clk = clocks.stop()
    launches = ve.kernel_launches() - launches0
    kinds = {}
    for k, name in enumerate(KIND_NAMES):
        tot, cnt = _lib.ctypes.c_double(), _lib.ctypes.c_int64()
        L.bfg_profile_read(ve.handle, k, _lib.ctypes.byref(tot), _lib.ctypes.byref(cnt))
        if cnt.value:
            kinds[name] = (tot.value, cnt.value)
    L.bfg_profile(ve.handle, 0)
    ms_max = allmax(pg, ms)
    ms_per_step = ms_max / args.steps
    value = world * args.steps / (ms_max / 1e3)

    # end to end through the public API with host buffers: every step the
    # state (vorticity field + tracer positions and rhs history) is copied in
    # from pinned host memory and the result is read back
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    cdt = np.complex64 if cfg["precision"] == "single" else np.complex128
    h_w = torch.empty(ve.cshape[0] * ve.cshape[1] * ve.cshape[2] * 3,
                      dtype=torch.complex64 if cdt == np.complex64 else torch.complex128,
                      pin_memory=True).numpy().reshape(ve.cshape)
    h_w[...] = ve.get_cvorticity()
    h_pos = torch.empty(ps.n * 3, dtype=torch.float64, pin_memory=True).numpy().reshape(ps.n, 3)
    h_rhs = torch.empty(ps.nsteps * ps.n * 3, dtype=torch.float64,
                        pin_memory=True).numpy().reshape(ps.nsteps, ps.n, 3)
    p0, r0, _ = ps.state()
    h_pos[...] = p0
    h_rhs[...] = r0
    sidx = ps.step_idx
    barrier(pg)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ve.set_cvorticity(h_w)
        L.bfg_particles_upload(ps.handle, _lib.ptr(h_pos), _lib.ptr(h_rhs), sidx)
        NSVEparticles_step(ve, ps, dt)
        L.bfg_field_download(ve.handle, _lib.FIELD_VORTICITY, h_w.ctypes.data)
        L.bfg_particles_download(ps.handle, _lib.ptr(h_pos), _lib.ptr(h_rhs), None)
        sidx += 1
    t1 = time.perf_counter()
    e2e_s = allmax(pg, t1 - t0)
    e2e_value = world * e2e_steps / e2e_s
    h2d = h_w.nbytes + h_pos.nbytes + h_rhs.nbytes
    d2h = h2d

    step_bytes, per_launch, U = algorithmic_bytes(cfg)
    peak, peak_kind = peaks()
    kern = {}
    for name, (tot, cnt) in kinds.items():
        avg = tot / cnt
        b = per_launch.get(name, 0.0)
        kern[name] = {"launches": cnt, "total_ms": round(tot, 4), "avg_ms": round(avg, 5),
                      "share": None, "gbs": round(b / (avg / 1e3) / 1e9, 1) if b else None}
    tot_all = sum(v[0] for v in kinds.values()) or 1.0
    for name in kern:
        kern[name]["share"] = round(kinds[name][0] / tot_all, 4)
    dominant = max(kinds, key=lambda k: kinds[k][0]) if kinds else None
    roof = None
    if dominant:
        avg = kinds[dominant][0] / kinds[dominant][1]
        ach = per_launch[dominant] / (avg / 1e3) / 1e9
        roof = {"bound": "hbm", "kernel": dominant, "achieved": round(ach, 1), "peak": peak,
                "unit": "GB/s", "frac": round(ach / peak, 4),
                "traffic": (round(TRAFFIC_RATIO[dominant] * per_launch[dominant])
                            if dominant in TRAFFIC_RATIO else None),
                "traffic_source": "ncu dram bytes per launch / algorithmic bytes (profiles/), "
                                  "scaled to this size",
                "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind}
    step_ach = step_bytes / (ms_per_step / 1e3) / 1e9
    out = {
        "metric": "512^3 RK3 steps/s (% HBM peak)" if cfg["n"] == 512 else "%d^3 RK3 steps/s" % cfg["n"],
        "value": round(value, 4),
        "unit": "steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if cfg["precision"] == "single" else "f64",
        "data": "synthetic (seeded k^4 exp(-2(k/k0)^2) spectrum, uniform tracers)",
        "config": {"workload": args.workload + ": %d^3 %s, nu=%g, dt=%g, k0=%g, %d tracers "
                   "(n=%d, m=%d), AB%d, linear forcing 1.5<=|k|<=3" % (
                       cfg["n"], "fp32" if cfg["precision"] == "single" else "fp64",
                       cfg["nu"], cfg["dt"], cfg["k0"], cfg["ntracers"], cfg["neighbours"],
                       cfg["smoothness"], cfg["nsteps_ab"]),
                   "grid": cfg["n"], "tracers": cfg["ntracers"],
                   "parallelism": "replicas x%d" % world,
                   "l2": "inputs larger than L2 (one 3-vector field is %.2f GB)" % (3 * U / 1e9)},
        "roofline": roof,
        "step_roofline": {"bytes_per_step": step_bytes, "achieved": round(step_ach, 1),
                          "peak": peak, "unit": "GB/s", "frac": round(step_ach / peak, 4),
                          "model": "105 U per IF-RK3 step + tracers n*24*(k+2) + 6 N^3 P"},
        "kernels": kern,
        "e2e": {"value": round(e2e_value, 4), "unit": "steps/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": e2e_steps},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if ps.n > 0 and world == 1:
        out["acceleration_sampling"] = acceleration_report(ve, ps, cfg)
    ps.close()
    ve.close()
    if cfg.get("accuracy_steps") and cfg["precision"] == "single" and not args.no_precision:
        out["precision_error"] = precision_report(cfg, w0, pos, dev, cfg["accuracy_steps"])
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(cfg, args.cpu_budget)
    if pg is not None:
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


# ------------------------------------------------------ batched / served ---
def _ensemble_requests(cfg):
    from bfps_b200 import serve
    rng = np.random.default_rng(1000)
    reqs = []
    for i, n in enumerate(cfg["sizes"]):
        nu = float(np.exp(rng.uniform(np.log(cfg["nu_range"][0]), np.log(cfg["nu_range"][1]))))
        r = serve.Request(rid=i, n=n, nu=nu, steps=cfg["solve_steps"], ntracers=cfg["ntracers"],
                          arrival=0.0, seed=i, precision=cfg["precision"],
                          neighbours=cfg["neighbours"], smoothness=cfg["smoothness"],
                          nsteps_ab=cfg["nsteps_ab"])
        serve.prepare(r)
        reqs.append(r)
    return reqs


def _member(r, device=0):
    from bfps_b200.solver import vorticity_equation, particles_system
    fs = vorticity_equation(r.n, precision=r.precision, device=device)
    fs.nu = r.nu
    fs.forcing_type = FORCING["forcing_type"]
    fs.fk0, fs.fk1, fs.famplitude = FORCING["fk0"], FORCING["fk1"], FORCING["famplitude"]
    fs.set_cvorticity(r.w0)
    ps = particles_system(fs, r.pos, r.neighbours, r.smoothness, r.nsteps_ab) if r.ntracers else None
    return fs, ps


def ensemble_bytes(reqs):
    """105 U per instance step + n*24*(k+2) + 6 N^3 P per instance (tracers)."""
    tot = 0
    for r in reqs:
        P = 4 if r.precision == "single" else 8
        U = r.n * r.n * (r.n + 2) * P
        tot += 105 * U + r.ntracers * 24 * (r.nsteps_ab + 2) + 6 * r.n ** 3 * P
    return tot


def run_ensemble(args, cfg):
    import torch
    from bfps_b200.solver import ensemble, NSVEparticles_step
    world, rank, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    reqs = _ensemble_requests(cfg)
    members = [_member(r, local) for r in reqs]
    ens = ensemble(local)
    for (fs, ps), r in zip(members, reqs):
        ens.add(fs, r.dt, ps)
    ens.step(args.warmup)
    ens.last_ms()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(pg)
    launches0 = ens.kernel_launches()
    ens.step(args.steps)
    ms = ens.last_ms()
    launches = ens.kernel_launches() - launches0
    barrier(pg)
    clk = clocks.stop()
    ms = allmax(pg, ms)
    ms_step = ms / args.steps
    nsolve = len(reqs)
    solves_s = world * nsolve / (cfg["solve_steps"] * ms_step / 1e3)
    # the plain path one instance at a time: every member stepped alone with
    # the single-instance entry point (same kernels, one launch per pass each)
    seq_ms = 0.0
    timed = {}
    for (fs, ps), r in zip(members, reqs):
        key = r.n
        if key not in timed:
            NSVEparticles_step(fs, ps, r.dt, 2)
            fs.last_step_ms()
            NSVEparticles_step(fs, ps, r.dt, max(3, args.steps // 2))
            timed[key] = fs.last_step_ms() / max(3, args.steps // 2)
        seq_ms += timed[key]
    seq_solves_s = world * nsolve / (cfg["solve_steps"] * seq_ms / 1e3)
    # end to end: every step the states go host -> device -> host
    from bfps_b200 import _lib
    L = _lib.lib()
    host = []
    for (fs, ps), r in zip(members, reqs):
        w = torch.empty(int(np.prod(fs.cshape)), dtype=torch.complex64, pin_memory=True)
        w = w.numpy().reshape(fs.cshape)
        w[...] = fs.get_cvorticity()
        host.append(w)
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for (fs, ps), w in zip(members, host):
            L.bfg_field_upload(fs.handle, _lib.FIELD_VORTICITY, w.ctypes.data)
        ens.step(1)
        ens.last_ms()
        for (fs, ps), w in zip(members, host):
            L.bfg_field_download(fs.handle, _lib.FIELD_VORTICITY, w.ctypes.data)
    e2e_s = allmax(pg, time.perf_counter() - t0)
    nbytes = sum(w.nbytes for w in host)
    e2e_solves = world * nsolve / (cfg["solve_steps"] * e2e_s / e2e_steps)
    peak, peak_kind = peaks()
    step_bytes = ensemble_bytes(reqs)
    ach = step_bytes / (ms_step / 1e3) / 1e9
    out = {
        "metric": "batched solves/s (mixed 32^3/64^3/128^3 ensemble)",
        "value": round(solves_s, 4), "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if cfg["precision"] == "single" else "f64",
        "data": "synthetic (seeded fields per instance, uniform tracers)",
        "config": {"workload": "C4: 64 instances (40x32^3, 16x64^3, 8x128^3) fp32, nu log-uniform "
                               "[0.005, 0.05], CFL-0.5 dt, 1e4 Lagrange-6 tracers each, AB4, "
                               "500-step solves",
                   "instances": nsolve, "parallelism": "replicas x%d" % world,
                   "l2": "ensemble state 2.4 GB > L2"},
        "roofline": {"bound": "hbm", "kernel": "ensemble step (all passes)", "achieved": round(ach, 1),
                     "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4), "traffic": None},
        "sequential": {"solves_s": round(seq_solves_s, 4), "ms_per_ensemble_step": round(seq_ms, 4),
                       "speedup": round(solves_s / seq_solves_s, 3),
                       "how": "each instance stepped alone with the single-instance entry point"},
        "e2e": {"value": round(e2e_solves, 4), "unit": "solves/s", "h2d_bytes_per_step": int(nbytes),
                "d2h_bytes_per_step": int(nbytes), "steps": e2e_steps},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    ens.close()
    for fs, ps in members:
        if ps is not None:
            ps.close()
        fs.close()
    if pg is not None:
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_serving(args, cfg):
    import torch
    from bfps_b200 import serve
    from bfps_b200.solver import NSVEparticles_step
    world, rank, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    reqs = serve.poisson_stream(cfg["requests"], rate=cfg["rate"], seed=2000 + rank)
    for r in reqs:
        r.precision = cfg["precision"]
        serve.prepare(r)
    # warm-up: one small solve through the server (kernels, attributes)
    w = serve.Request(rid=-1, n=64, nu=0.01, steps=3, ntracers=10, arrival=0.0, seed=99,
                      precision=cfg["precision"])
    serve.prepare(w)
    srv = serve.Server(hbm_budget=cfg["budget"], device=local)
    srv.run([w])
    srv.done.clear()
    barrier(pg)
    launches0 = srv.ens.kernel_launches()
    t0 = time.perf_counter()
    done = srv.run(reqs)
    wall = time.perf_counter() - t0
    launches = srv.ens.kernel_launches() - launches0
    srv.close()
    ttc = np.array([r.finished - r.arrival for r in done])
    span = max(r.finished for r in done) - min(r.arrival for r in done)
    solves_s = len(done) / span
    # the plain path one request at a time: per-size single-instance step time
    step_ms = {}
    for n in sorted({r.n for r in reqs}):
        r0 = next(r for r in reqs if r.n == n)
        fs, ps = _member(r0, local)
        NSVEparticles_step(fs, ps, r0.dt, 2)
        fs.last_step_ms()
        NSVEparticles_step(fs, ps, r0.dt, 5)
        step_ms[n] = fs.last_step_ms() / 5
        if ps is not None:
            ps.close()
        fs.close()
    seq_s = sum(r.steps * step_ms[r.n] / 1e3 for r in reqs)
    seq_solves_s = len(reqs) / seq_s
    out = {
        "metric": "served solves/s, p50/p99 time-to-completion (Poisson stream)",
        "value": round(solves_s * world, 4), "unit": "solves/s", "n_gpus": world,
        "steps": None, "warmup": 1, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic request stream",
        "config": {"workload": "C5: %d requests, Poisson 20/s, N in {64:0.6,128:0.3,256:0.1}, nu "
                               "log-uniform [0.002,0.02], 100..1000 steps, 0..1e5 n2m2 tracers, "
                               "HBM budget 150 GB" % len(reqs),
                   "parallelism": "replicas x%d" % world},
        "p50_s": round(float(np.percentile(ttc, 50)), 4),
        "p99_s": round(float(np.percentile(ttc, 99)), 4),
        "completed": len(done), "wall_s": round(wall, 3),
        "sequential": {"solves_s": round(seq_solves_s, 4), "speedup": round(solves_s / seq_solves_s, 3),
                       "how": "sum of steps x single-instance step time per size"},
        "e2e": {"value": round(solves_s * world, 4), "unit": "solves/s",
                "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "note": "wall clock from arrival to read-back of every request"},
        "gpu_launches": int(launches),
    }
    if pg is not None:
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


# ------------------------------------------------------------------ CPU ---
class CpuSample:
    """Bounded sample of the step on the host cores with the CPU restatement
    of the reference (oracle/): one IF-RK3 stage (a third of the fluid work
    of a step, timed and multiplied by 3) and the tracer step for a fraction
    of the tracers (timed and scaled to all of them).  Inputs are built once."""

    def __init__(self, cfg, tracer_count):
        from oracle import nsve as O
        from oracle import particles as P
        from bfps_b200 import ic
        self.cfg = cfg
        n = cfg["n"]
        self.cores = os.cpu_count() or 1
        rd = np.float32 if cfg["precision"] == "single" else np.float64
        ve = O.VorticityEquation(n, dealias_type=cfg["dealias"], rdtype=rd, workers=self.cores)
        ve.nu = cfg["nu"]
        ve.forcing_type = FORCING["forcing_type"]
        ve.fk0, ve.fk1, ve.famplitude = FORCING["fk0"], FORCING["fk1"], FORCING["famplitude"]
        ve.cvorticity = ic.vorticity_ic(n, seed=0, k0=cfg["k0"], dealias_type=cfg["dealias"],
                                        dtype=np.complex64 if rd == np.float32 else np.complex128)
        self.ve = ve
        self.ur = ve.ift(ve.compute_velocity(ve.cvorticity))
        self.nt = max(1, min(cfg["ntracers"], tracer_count))
        self.frac = self.nt / max(cfg["ntracers"], 1)
        self.pos = ic.tracer_ic(self.nt, seed=0)
        self.P = P

    def run(self):
        """Seconds of one full step (extrapolated) and the two measured parts."""
        ve, cfg, P = self.ve, self.cfg, self.P
        t0 = time.perf_counter()
        Nl = ve.omega_nonlin(ve.cvorticity)  # velocity, 6 C2R, product, 3 R2C, k-space
        k2 = ve.kk.K2
        f0 = np.exp(-ve.nu * k2 * cfg["dt"])[..., None]
        _ = np.where((k2 <= ve.kk.kM2)[..., None], (ve.cvorticity + cfg["dt"] * Nl) * f0, 0)
        stage_s = time.perf_counter() - t0
        ps = P.ParticlesSystem(self.pos, np.zeros((cfg["nsteps_ab"], self.nt, 3)), cfg["neighbours"],
                               cfg["smoothness"], P.Geometry(cfg["n"], cfg["n"], cfg["n"]))
        t1 = time.perf_counter()
        ps.complete_loop(self.ur, cfg["dt"])
        tracer_s = (time.perf_counter() - t1) / self.frac
        return 3 * stage_s + tracer_s, stage_s, tracer_s


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_baseline(cfg, budget):
    smp = CpuSample(cfg, 20_000)
    step_s, stage_s, tracer_s = smp.run()
    return {"value": round(1.0 / step_s, 6), "unit": "steps/s", "cores": smp.cores, "kind": "port",
            "cpu_model": cpu_model(),
            "sample": ("CPU restatement (numpy + scipy.fft, %d workers): one IF-RK3 stage at "
                       "%d^3 timed (%.2f s, x3) + tracer step for %d of %d tracers (%.2f s "
                       "scaled)" % (smp.cores, cfg["n"], stage_s, smp.nt, cfg["ntracers"],
                                    tracer_s))}


def run_reference(args, cfg):
    """The reference's CPU path on the host cores (its own build is impossible
    without FFTW/HDF5/MPI, so this is the restatement in oracle/).  Each step
    is one bounded sample; samples stop once the time budget is spent (at
    least one is timed), so that the run ends within a few minutes."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if cfg.get("kind"):
        print(json.dumps({"impl": "reference", "unavailable":
                          "no CPU restatement of the batched/served forms (the reference has "
                          "neither); compare against the single-instance arm"}), flush=True)
        return
    budget = args.cpu_budget
    smp = CpuSample(cfg, 20_000)
    t_start = time.perf_counter()
    times = []
    for i in range(max(1, args.steps)):
        step_s, stage_s, tracer_s = smp.run()
        times.append(step_s)
        if time.perf_counter() - t_start > budget:
            break
    s = statistics.mean(times)
    out = {
        "metric": "512^3 RK3 steps/s (% HBM peak)" if cfg["n"] == 512 else "%d^3 RK3 steps/s" % cfg["n"],
        "value": round(1.0 / s, 6), "unit": "steps/s", "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(s * 1e3, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if cfg["precision"] == "single" else "f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": cfg["n"], "tracers": cfg["ntracers"]},
        "impl": "reference",
        "cpu_baseline": {"value": round(1.0 / s, 6), "unit": "steps/s", "cores": smp.cores,
                         "kind": "port", "cpu_model": cpu_model(),
                         "sample": "per step: one IF-RK3 stage at %d^3 (x3) + tracer step for %d "
                                   "of %d tracers (scaled); %d samples timed (warm-up skipped: "
                                   "the CPU path has no warm-up state) within a %d s budget" % (
                                       cfg["n"], smp.nt, cfg["ntracers"], len(times), budget)},
        "e2e": {"value": round(1.0 / s, 6), "unit": "steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="C3", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-budget", type=float, default=120.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-precision", action="store_true",
                    help="skip the FP32-vs-FP64 error report of the FP32 workloads")
    ap.add_argument("--grid", type=int, default=None,
                    help="override the workload's grid size N (profiling cases)")
    ap.add_argument("--tracers", type=int, default=None,
                    help="override the workload's tracer count (profiling cases)")
    args = ap.parse_args()
    cfg = dict(WORKLOADS[args.workload])
    if args.grid is not None:
        cfg["n"] = args.grid
    if args.tracers is not None:
        cfg["ntracers"] = args.tracers
    if args.impl == "reference":
        run_reference(args, cfg)
    elif cfg.get("kind") == "ensemble":
        run_ensemble(args, cfg)
    elif cfg.get("kind") == "serving":
        run_serving(args, cfg)
    else:
        run_ours(args, cfg)


if __name__ == "__main__":
    main()
