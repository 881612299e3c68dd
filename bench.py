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
               neighbours=3, smoothness=2, nsteps_ab=3, dealias=1),
    # the plain FP64 path at 512^3 (comparator of the precision form)
    "C3_fp64": dict(n=512, precision="double", nu=0.002, dt=0.001, k0=4.0,
                    ntracers=4_000_000, neighbours=3, smoothness=2, nsteps_ab=3, dealias=1),
    # 256^3 FP32 + 1e5 tracers (n=2, m=2), AB4
    "C2": dict(n=256, precision="single", nu=0.005, dt=0.002, k0=3.0, ntracers=100_000,
               neighbours=2, smoothness=2, nsteps_ab=4, dealias=1),
    # 32^3 FP64, 1024 tracers, 6-point Lagrange, AB2, 2/3 dealiasing
    "C1": dict(n=32, precision="double", nu=0.1, dt=0.01, k0=3.0, ntracers=1024,
               neighbours=2, smoothness=0, nsteps_ab=2, dealias=0),
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
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        import torch
        pg.barrier()
        torch.cuda.synchronize()


def allmax(pg, v):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


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
                "unit": "GB/s", "frac": round(ach / peak, 4), "traffic": None,
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
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(cfg, args.cpu_budget)
    ps.close()
    ve.close()
    if pg is not None:
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


# ------------------------------------------------------------------ CPU ---
def _cpu_sample(cfg, tracer_fraction):
    """One bounded sample of the step on the host cores, with the CPU
    restatement of the reference (oracle/): one IF-RK3 stage (a third of the
    fluid work of a step) and the tracer step for a fraction of the tracers.
    Returns the extrapolated seconds for one full step and the breakdown."""
    from oracle import nsve as O
    from oracle import particles as P
    from bfps_b200 import ic
    n = cfg["n"]
    cores = os.cpu_count() or 1
    rd = np.float32 if cfg["precision"] == "single" else np.float64
    ve = O.VorticityEquation(n, dealias_type=cfg["dealias"], rdtype=rd, workers=cores)
    ve.nu = cfg["nu"]
    ve.forcing_type = FORCING["forcing_type"]
    ve.fk0, ve.fk1, ve.famplitude = FORCING["fk0"], FORCING["fk1"], FORCING["famplitude"]
    w0 = ic.vorticity_ic(n, seed=0, k0=cfg["k0"], dealias_type=cfg["dealias"],
                         dtype=np.complex64 if rd == np.float32 else np.complex128)
    ve.cvorticity = w0
    t0 = time.perf_counter()
    Nl = ve.omega_nonlin(ve.cvorticity)  # one stage: velocity, 6 C2R, product, 3 R2C, k-space
    k2 = ve.kk.K2
    f0 = np.exp(-ve.nu * k2 * cfg["dt"])[..., None]
    _ = np.where((k2 <= ve.kk.kM2)[..., None], (w0 + cfg["dt"] * Nl) * f0, 0)
    t1 = time.perf_counter()
    stage_s = t1 - t0
    ur = ve.ift(ve.compute_velocity(ve.cvorticity))
    nt = max(1, int(cfg["ntracers"] * tracer_fraction))
    pos = ic.tracer_ic(nt, seed=0)
    geom = P.Geometry(n, n, n)
    ps = P.ParticlesSystem(pos, np.zeros((cfg["nsteps_ab"], nt, 3)), cfg["neighbours"],
                           cfg["smoothness"], geom)
    t2 = time.perf_counter()
    ps.complete_loop(ur, cfg["dt"])
    t3 = time.perf_counter()
    tracer_s = (t3 - t2) / tracer_fraction
    return 3 * stage_s + tracer_s, stage_s, tracer_s, nt, cores


def cpu_baseline(cfg, budget):
    frac = min(1.0, 2e5 / max(cfg["ntracers"], 1))
    step_s, stage_s, tracer_s, nt, cores = _cpu_sample(cfg, frac)
    return {"value": round(1.0 / step_s, 6), "unit": "steps/s", "cores": cores, "kind": "port",
            "sample": ("CPU restatement (numpy + scipy.fft, %d workers): one IF-RK3 stage at "
                       "%d^3 timed (%.2f s, x3) + tracer step for %d of %d tracers (%.2f s "
                       "scaled)" % (cores, cfg["n"], stage_s, nt, cfg["ntracers"], tracer_s))}


def run_reference(args, cfg):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    frac = min(1.0, 2e5 / max(cfg["ntracers"], 1))
    budget = args.cpu_budget
    times = []
    t_start = time.perf_counter()
    total = args.warmup + args.steps
    for i in range(total):
        step_s, stage_s, tracer_s, nt, cores = _cpu_sample(cfg, frac)
        if i >= args.warmup:
            times.append(step_s)
        if time.perf_counter() - t_start > budget and len(times) >= 1:
            break
        if i < args.warmup and time.perf_counter() - t_start > budget / 3:
            continue
    s = statistics.mean(times)
    out = {
        "metric": "512^3 RK3 steps/s (% HBM peak)" if cfg["n"] == 512 else "%d^3 RK3 steps/s" % cfg["n"],
        "value": round(1.0 / s, 6), "unit": "steps/s", "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(s * 1e3, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if cfg["precision"] == "single" else "f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": cfg["n"], "tracers": cfg["ntracers"]},
        "impl": "reference",
        "cpu_baseline": {"value": round(1.0 / s, 6), "unit": "steps/s", "cores": cores,
                         "kind": "port",
                         "sample": "per step: one IF-RK3 stage at %d^3 (x3) + tracer step "
                                   "for %d tracers (scaled); %d samples timed within a %d s "
                                   "budget" % (cfg["n"], nt, len(times), budget)},
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
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-budget", type=float, default=150.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    cfg = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, cfg)
    else:
        run_ours(args, cfg)


if __name__ == "__main__":
    main()
