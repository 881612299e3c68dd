"""Serving form: a request loop over the batched engine (continuous batching).

A request asks for one DNS solve: grid size N, viscosity, seed, number of
steps and tracers.  Requests are admitted while their device memory fits an
HBM budget; admitted requests become ensemble members (their state stays
resident on the GPU) and advance together, with the stages of all resident
requests of the same size batched into one launch per pass.  A tick runs the
ensemble up to the next event (a resident request reaching its step count,
or the next arrival as estimated from the measured step time) and
synchronises once; while it runs, the host polls it (bfg_ens_wait) and
prepares the inputs of requests that have arrived.  A request that reaches its step count is read back and
retired, freeing its memory for waiting requests.  Requests that arrive
while others are running join at the next tick.

Nothing here computes on the host: every step is bfg_ens_step.
"""
import dataclasses
import math
import time

import numpy as np

from . import ic
from .solver import ensemble, particles_system, vorticity_equation


@dataclasses.dataclass
class Request:
    rid: int
    n: int
    nu: float
    steps: int
    ntracers: int
    arrival: float            # seconds after the start of the stream
    seed: int = 0
    precision: str = "single"
    neighbours: int = 2
    smoothness: int = 2
    nsteps_ab: int = 4
    fk0: float = 1.5
    fk1: float = 3.0
    famplitude: float = 0.5
    # inputs (generated from the seed by prepare() when absent)
    w0: object = None          # vorticity, (n, n, n/2+1, 3) complex
    pos: object = None         # tracer positions, (ntracers, 3)
    # filled in by prepare() / the server
    dt: float = 0.0
    admitted: float = math.nan
    finished: float = math.nan
    result: object = None


def request_bytes(n, precision, ntracers, nsteps_ab):
    """Device memory of one resident request (five complex buffers, the real
    velocity, tracer state and its sort buffers)."""
    rb = 4 if precision == "single" else 8
    field = n * n * (n // 2 + 4) * 3 * 2 * rb
    ru = n ** 3 * 3 * rb
    tracers = ntracers * (2 * 24 * (1 + nsteps_ab) + 16 + 8 + 24) + 2 * n * n * 4
    return 5 * field + ru + tracers + (1 << 20)


def poisson_stream(nreq, rate=20.0, seed=2000, sizes=((64, 0.6), (128, 0.3), (256, 0.1)),
                   nu_range=(0.002, 0.02), steps_range=(100, 1000), tracer_max=100_000):
    """Seeded synthetic request stream: Poisson arrivals, mixed sizes."""
    rng = np.random.default_rng(seed)
    t = 0.0
    ns = [s for s, _ in sizes]
    ps = np.array([p for _, p in sizes])
    out = []
    for i in range(nreq):
        t += rng.exponential(1.0 / rate)
        n = int(rng.choice(ns, p=ps / ps.sum()))
        nu = float(np.exp(rng.uniform(np.log(nu_range[0]), np.log(nu_range[1]))))
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        nt = int(rng.integers(0, tracer_max + 1))
        out.append(Request(rid=i, n=n, nu=nu, steps=steps, ntracers=nt, arrival=t, seed=i))
    return out


def prepare(req):
    """Inputs of a request from its seed (the initial vorticity, tracer
    positions) and its fixed time step dt = 0.5 dx / max|u| (CFL 0.5 on the
    initial field; Adams-Bashforth needs a constant dt)."""
    cdt = np.complex64 if req.precision == "single" else np.complex128
    w0, u = ic.vorticity_ic(req.n, seed=req.seed, dtype=cdt, return_velocity=True)
    req.w0 = w0
    ur = np.fft.irfftn(np.swapaxes(u.astype(np.complex128), 0, 1), s=(req.n,) * 3,
                       axes=(0, 1, 2), norm="forward")
    umax = float(np.sqrt((ur ** 2).sum(axis=-1)).max())
    req.dt = ic.cfl_dt(umax, req.n)
    req.pos = ic.tracer_ic(req.ntracers, seed=req.seed) if req.ntracers else None
    return req


class Server:
    def __init__(self, hbm_budget=150e9, device=0, use_graphs=False, max_tick=64):
        self.budget = hbm_budget
        self.used = 0
        self.device = device
        self.max_tick = max_tick   # most ensemble steps between two synchronisations
        self.step_ms = 0.0         # device time of one ensemble step, last tick
        self.ens = ensemble(device)
        self.ens.use_graphs(use_graphs)
        self.running = {}   # rid -> (request, fs, ps, steps_done)
        self.done = []

    def _start(self, req, now):
        fs = vorticity_equation(req.n, precision=req.precision, device=self.device)
        fs.nu = req.nu
        fs.forcing_type = "linear"
        fs.famplitude, fs.fk0, fs.fk1 = req.famplitude, req.fk0, req.fk1
        if req.w0 is None:
            prepare(req)
        fs.set_cvorticity(req.w0)
        ps = None
        if req.ntracers > 0:
            ps = particles_system(fs, req.pos, req.neighbours, req.smoothness, req.nsteps_ab)
        self.ens.add(fs, req.dt, ps)
        req.admitted = now
        self.running[req.rid] = [req, fs, ps, 0]
        self.used += request_bytes(req.n, req.precision, req.ntracers, req.nsteps_ab)

    def _finish(self, rid, now):
        req, fs, ps, _ = self.running.pop(rid)
        self.ens.remove(fs)
        # the final state's statistics (NSVE::do_stats): the energy spectrum
        # E(k) = tr(spec_uu) / 2, summed in a fixed order on the device, so a
        # request gives the same bits alone and in the mix
        spec_uu = fs.do_stats()["velocity"][0]
        req.result = {"vorticity_checksum": float(np.abs(fs.get_cvorticity()).sum()),
                      "iteration": fs.iteration,
                      "energy_spectrum": 0.5 * np.einsum("kii->k", spec_uu)}
        if ps is not None:
            req.result["tracers"] = ps.state()[0]
            ps.close()
        fs.close()
        req.finished = now
        self.used -= request_bytes(req.n, req.precision, req.ntracers, req.nsteps_ab)
        self.done.append(req)

    def run(self, requests, clock=time.perf_counter, max_wall=None):
        """Serve a stream (arrival times relative to the call).  Returns the
        finished requests; time-to-completion is finished - arrival."""
        pending = sorted(requests, key=lambda r: r.arrival)
        t0 = clock()
        qi = 0
        waiting = []
        while qi < len(pending) or waiting or self.running:
            now = clock() - t0
            if max_wall is not None and now > max_wall:
                break
            while qi < len(pending) and pending[qi].arrival <= now:
                waiting.append(pending[qi])
                qi += 1
            # admission by HBM budget, in arrival order
            still = []
            for req in waiting:
                need = request_bytes(req.n, req.precision, req.ntracers, req.nsteps_ab)
                if self.used + need <= self.budget:
                    self._start(req, clock() - t0)
                else:
                    still.append(req)
            waiting = still
            if not self.running:
                if qi < len(pending):
                    time.sleep(max(0.0, min(0.01, pending[qi].arrival - (clock() - t0))))
                continue
            # one tick: ensemble steps up to the next event -- the first resident
            # request reaching its step count, or (by the measured step time)
            # the next arrival -- then one synchronisation
            k = min(r[0].steps - r[3] for r in self.running.values())
            if qi < len(pending) and self.step_ms > 0.0:
                until = pending[qi].arrival - (clock() - t0)
                k = min(k, max(1, int(until * 1e3 / self.step_ms)))
            k = max(1, min(k, self.max_tick))
            self.ens.step(k)
            # while the tick runs, prepare the inputs of arrived requests
            # that still need them (host work off the GPU's critical path)
            while not self.ens.wait(0.002):
                now = clock() - t0
                todo = [r for r in waiting + pending[qi:] if r.arrival <= now and r.w0 is None]
                if not todo:
                    self.ens.wait()
                    break
                prepare(todo[0])
            self.step_ms = self.ens.last_ms() / k
            for rid in list(self.running):
                self.running[rid][3] += k
                if self.running[rid][3] >= self.running[rid][0].steps:
                    self._finish(rid, clock() - t0)
        return self.done

    def close(self):
        for rid in list(self.running):
            req, fs, ps, _ = self.running.pop(rid)
            self.ens.remove(fs)
            if ps is not None:
                ps.close()
            fs.close()
        self.ens.close()
