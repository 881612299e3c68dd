#!/usr/bin/env python
"""Benchmark: bfps NSVEparticles step (IF-RK3 vorticity DNS + tracers) on B200.

Default workload (the configuration the headline metric is quoted on):
512^3 grid, FP32 fields, nu = 0.002, dt = 0.001, seeded k^4 exp(-2 (k/4)^2)
initial spectrum, linear band forcing on 1.5 <= |k| <= 3 (amplitude 0.5),
smooth dealiasing, 4e6 tracers with the (neighbours 3, smoothness 2) kernel
and AB3.  One step = NSVEparticles::step: velocity at t -> tracers advance ->
fluid IF-RK3 step.  Inputs are synthetic (seeded), generated on the host.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload C3]
    python bench.py --impl reference ...   # C++/OpenMP restatement on the host cores

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
TRAFFIC_RATIO = {"X": 0.951, "IZ": 0.931, "IY": 0.948, "FY": 0.886, "FZ": 0.744, "tracers": 0.983}


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
    """Seeded initial field and tracers.  With BFPS_IC_CACHE set to a
    directory, the generated arrays are kept there as .npy files and reused
    by later runs of the same workload (generation takes ~40 s at 512^3)."""
    from bfps_b200 import ic
    n = cfg["n"]
    cdt = np.complex64 if cfg["precision"] == "single" else np.complex128
    cache = os.environ.get("BFPS_IC_CACHE")
    if cache:
        tag = "n%d_%s_k%g_d%d_s%d_t%d" % (n, cfg["precision"], cfg["k0"], cfg["dealias"], seed,
                                         cfg["ntracers"])
        fw, fp = os.path.join(cache, tag + "_w.npy"), os.path.join(cache, tag + "_p.npy")
        if os.path.exists(fw) and os.path.exists(fp):
            return np.load(fw), np.load(fp)
    w0 = ic.vorticity_ic(n, seed=seed, k0=cfg["k0"], dealias_type=cfg["dealias"], dtype=cdt)
    pos = ic.tracer_ic(cfg["ntracers"], seed=seed)
    if cache:
        os.makedirs(cache, exist_ok=True)
        np.save(fw, w0)
        np.save(fp, pos)
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
            "how": "same FP32-rounded initial field and tracers, stepped in FP32 and in FP64 "
                   "with this engine (its FP64 path agrees with the FP64 oracle to 1e-10 "
                   "at 256^3 over six steps); shells with E64(k) >= 1e-6 max"}


def run_ours(args, cfg):
    import torch
    from bfps_b200 import _lib
    from bfps_b200.solver import NSVEparticles_step
    world, rank, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = local
    w0, pos = make_inputs(cfg, seed=rank)
    ve, ps = build_solver(cfg, w0, pos, dev)
    # the column passes' schedules for this grid and precision (bfg_autotune)
    tuned = ve.autotune(reps=3) if not args.no_tune else ve.schedules()
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
        "config": workload_config(args, cfg, world),
        "roofline": roof,
        "step_roofline": {"bytes_per_step": step_bytes, "achieved": round(step_ach, 1),
                          "peak": peak, "unit": "GB/s", "frac": round(step_ach / peak, 4),
                          "model": "105 U per IF-RK3 step + tracers n*24*(k+2) + 6 N^3 P"},
        "kernels": kern,
        "e2e": {"value": round(e2e_value, 4), "unit": "steps/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": e2e_steps},
        "gpu_launches": int(launches),
        "clocks": clk,
        "schedules": {k: {"schedule": v[0], "ms": [round(v[1], 4), round(v[2], 4)]}
                      for k, v in tuned.items()},
    }
    if ps.n > 0 and world == 1:
        out["acceleration_sampling"] = acceleration_report(ve, ps, cfg)
    ps.close()
    ve.close()
    if cfg.get("accuracy_steps") and cfg["precision"] == "single" and not args.no_precision:
        out["precision_error"] = precision_report(cfg, w0, pos, dev, cfg["accuracy_steps"])
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"], cmp = cpu_baseline(cfg, w0, pos, dev)
        if "precision_error" in out:
            out["precision_error"]["vs_fp64_oracle"] = cmp
        else:
            out["vs_fp64_oracle"] = cmp
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
    # schedules of the column passes, timed on each size group as the
    # ensemble launches it (all members of a size in one launch)
    if args.no_tune:
        tuned = {}
        for fs, _ in members:
            k = sum(1 for g, _ in members if g.nx == fs.nx)
            tuned.setdefault(fs.nx, fs.schedules(members=k))
    else:
        tuned = ens.autotune(reps=3)
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
        "schedules": {str(n): {k: {"schedule": v[0], "ms": [round(v[1], 4), round(v[2], 4)]}
                               for k, v in t.items()} for n, t in tuned.items()},
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
    busy0, ticks0, host0 = srv.busy_ms, srv.ticks, dict(srv.host_s)
    t0 = time.perf_counter()
    done = srv.run(reqs)
    wall = time.perf_counter() - t0
    busy_s = (srv.busy_ms - busy0) / 1e3
    ticks = srv.ticks - ticks0
    srv_host = {k: v - host0[k] for k, v in srv.host_s.items()}
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
        "device_busy_s": round(busy_s, 3), "ticks": ticks,
        "host_phases_s": {k: round(v, 3) for k, v in srv_host.items()},
        "sequential": {"solves_s": round(seq_solves_s, 4), "speedup": round(solves_s / seq_solves_s, 3),
                       "device_s": round(seq_s, 3),
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
def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


class OracleRun:
    """Whole NSVEparticles steps of the workload on the host cores with the
    C++/OpenMP restatement of the reference (oracle/nsve_omp.cpp, FP64
    fields and tracers, all OpenMP threads): the fluid IF-RK3 step on the
    full grid and the tracer step for every tracer.  The same seeded inputs
    as the GPU arm (the FP32-rounded field where the workload is FP32)."""

    def __init__(self, cfg, w0=None, pos=None):
        from oracle import fast as F
        self.F = F
        self.cfg = cfg
        n = cfg["n"]
        if w0 is None:
            w0, pos = make_inputs(cfg, seed=0)
        self.ve = F.VorticityEquation(n, dealias_type=cfg["dealias"])
        self.ve.nu = cfg["nu"]
        self.ve.forcing_type = FORCING["forcing_type"]
        self.ve.fk0, self.ve.fk1, self.ve.famplitude = (FORCING["fk0"], FORCING["fk1"],
                                                         FORCING["famplitude"])
        self.ve.cvorticity = w0.astype(np.complex128)
        self.ps = F.ParticlesSystem(self.ve, pos, np.zeros((cfg["nsteps_ab"], pos.shape[0], 3)),
                                    cfg["neighbours"], cfg["smoothness"])
        self.threads = F.threads()

    def step(self):
        t0 = time.perf_counter()
        self.F.nsveparticles_step(self.ve, self.ps, self.cfg["dt"])
        return time.perf_counter() - t0

    def close(self):
        self.ps.close()
        self.ve.close()


def energy_spectrum(w, dk=1.0, kM=None):
    """E(k) = sum over the shell int(|k|/dk) of w_x |u_k|^2 / 2 with
    |u_k|^2 = |w_k|^2 / k^2 (divergence-free w), modes 0 < k^2 <= kM^2,
    w_x = 1 on kx = 0 and 2 elsewhere (kspace.cpp:521-598, the trace of the
    velocity co-spectrum over two); w in the state layout (ny, nz, nx/2+1, 3).
    Accumulated one ky plane at a time in FP64."""
    ny, nz, nxv = w.shape[:3]
    n = ny
    kx = np.arange(nxv) * dk
    kk = np.array([i if i <= n // 2 else i - n for i in range(n)], dtype=np.float64) * dk
    if kM is None:
        kM = dk * (n // 2 - 1)
    wx = np.where(np.arange(nxv) == 0, 1.0, 2.0)[None, :]
    nsh = int(kM / dk) + 2
    spec = np.zeros(nsh)
    for iy in range(ny):
        k2 = (kx[None, :] ** 2 + kk[iy] ** 2) + kk[:, None] ** 2
        a = w[iy].astype(np.complex128)
        e2 = (np.abs(a) ** 2).sum(axis=-1)
        m = (k2 > 0) & (k2 <= kM * kM)
        sh = (np.sqrt(k2[m]) / dk).astype(np.int64)
        spec += np.bincount(sh, weights=(wx * e2 / np.where(m, k2, 1.0))[m] * 0.5,
                            minlength=nsh)[:nsh]
    return spec


def oracle_comparison(cfg, w0, pos, device, orc_w, orc_pos):
    """One NSVEparticles step of the engine (the workload's precision) from
    the inputs the oracle step started from, against the FP64 oracle's step:
    relative error of the vorticity field (max over modes / max), of E(k)
    over the shells holding at least 1e-6 of the peak, of the total energy,
    and the largest tracer position error relative to the box."""
    from bfps_b200.solver import NSVEparticles_step
    ve, ps = build_solver(cfg, w0, pos, device)
    NSVEparticles_step(ve, ps, cfg["dt"])
    w = ve.get_cvorticity()
    p = ps.state()[0]
    ps.close()
    ve.close()
    e_gpu = energy_spectrum(w)
    e_orc = energy_spectrum(orc_w)
    keep = e_orc >= 1e-6 * e_orc.max()
    field_rel = float(np.abs(w - orc_w).max() / np.abs(orc_w).max())
    return {"steps": 1,
            "field_max_rel": field_rel,
            "spectrum_max_rel": float((np.abs(e_gpu[keep] - e_orc[keep]) / e_orc[keep]).max()),
            "spectrum_shells": int(keep.sum()),
            "energy_rel": float(abs(e_gpu.sum() - e_orc.sum()) / e_orc.sum()),
            "positions_max_abs_over_box": float(np.abs(p - orc_pos).max() / (2 * np.pi)),
            "how": "engine step from the same inputs as one FP64 oracle step "
                   "(oracle/nsve_omp.cpp); E(k) from the vorticity, shells with "
                   "E(k) >= 1e-6 max"}


def cpu_baseline(cfg, w0, pos, device):
    """The oracle timed over one whole step of the workload on rank 0, and
    the engine compared with that step (oracle_comparison)."""
    orc = OracleRun(cfg, w0.astype(np.complex64) if cfg["precision"] == "single" else w0, pos)
    s = orc.step()
    orc_w = orc.ve.cvorticity
    orc_pos = orc.ps.state()[0]
    threads = orc.threads
    orc.close()
    base = {"value": round(1.0 / s, 6), "unit": "steps/s", "cores": threads, "kind": "port",
            "cpu_model": cpu_model(),
            "sample": ("one whole step of the workload (%d^3 IF-RK3 step + %d tracers, n=%d m=%d, "
                       "AB%d) by the C++/OpenMP restatement of the reference (oracle/nsve_omp.cpp, "
                       "FP64, %d threads): %.2f s" % (cfg["n"], cfg["ntracers"], cfg["neighbours"],
                                                     cfg["smoothness"], cfg["nsteps_ab"], threads,
                                                     s))}
    cmp = oracle_comparison(cfg, w0, pos, device, orc_w, orc_pos)
    return base, cmp


def workload_config(args, cfg, world):
    """The `config` of a single-instance workload's line (both arms)."""
    U = cfg["n"] * cfg["n"] * (cfg["n"] + 2) * (4 if cfg["precision"] == "single" else 8)
    return {"workload": args.workload + ": %d^3 %s, nu=%g, dt=%g, k0=%g, %d tracers "
                        "(n=%d, m=%d), AB%d, linear forcing 1.5<=|k|<=3" % (
                            cfg["n"], "fp32" if cfg["precision"] == "single" else "fp64",
                            cfg["nu"], cfg["dt"], cfg["k0"], cfg["ntracers"], cfg["neighbours"],
                            cfg["smoothness"], cfg["nsteps_ab"]),
            "grid": cfg["n"], "tracers": cfg["ntracers"],
            "parallelism": "replicas x%d" % world,
            "l2": "inputs larger than L2 (one 3-vector field is %.2f GB)" % (3 * U / 1e9)}


def run_reference(args, cfg):
    """The reference's CPU path on the host cores.  Its own build needs
    FFTW3, HDF5 and MPI, absent here and on the GPU box, so this is the
    C++/OpenMP restatement in oracle/ (all OpenMP threads): min(1, W)
    untimed warm-up steps, then whole steps of the workload, at least three
    and at most K, until a time budget is spent; `steps` is the number timed."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if cfg.get("kind"):
        print(json.dumps({"impl": "reference", "unavailable":
                          "no CPU restatement of the batched/served forms (the reference has "
                          "neither); compare against the single-instance arm"}), flush=True)
        return
    budget = args.cpu_budget
    orc = OracleRun(cfg)
    for _ in range(min(1, args.warmup)):
        orc.step()
    t_start = time.perf_counter()
    times = []
    while len(times) < max(1, args.steps):
        times.append(orc.step())
        if len(times) >= min(3, max(1, args.steps)) and time.perf_counter() - t_start > budget:
            break
    threads = orc.threads
    orc.close()
    s = sum(times) / len(times)
    out = {
        "metric": "512^3 RK3 steps/s (% HBM peak)" if cfg["n"] == 512 else "%d^3 RK3 steps/s" % cfg["n"],
        "value": round(1.0 / s, 6), "unit": "steps/s", "n_gpus": 0, "steps": len(times),
        "warmup": min(1, args.warmup), "ms_per_step": round(s * 1e3, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded k^4 exp(-2(k/k0)^2) spectrum, uniform tracers)",
        "config": workload_config(args, cfg, 1),
        "impl": "reference",
        "cpu_baseline": {"value": round(1.0 / s, 6), "unit": "steps/s", "cores": threads,
                         "kind": "port", "cpu_model": cpu_model(),
                         "sample": "%d whole steps of the workload (%d^3 IF-RK3 step + all %d "
                                   "tracers) by the C++/OpenMP restatement of the reference "
                                   "(oracle/nsve_omp.cpp, FP64 fields and tracers, %d threads), "
                                   "after %d untimed warm-up step(s)" % (
                                       len(times), cfg["n"], cfg["ntracers"], threads,
                                       min(1, args.warmup))},
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
    ap.add_argument("--cpu-budget", type=float, default=90.0,
                    help="seconds of whole CPU steps the reference arm times (at least 3 steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default column-pass schedules (no bfg_autotune)")
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
