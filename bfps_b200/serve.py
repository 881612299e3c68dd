"""Serving form: a request loop over the batched engine (continuous batching).

A request asks for one DNS solve: grid size N, viscosity, seed, number of
steps and tracers.  Requests are admitted while their device memory fits an
HBM budget; admitted requests become ensemble members (their state stays
resident on the GPU) and advance together, with the stages of all resident
requests of the same size batched into one launch per pass.  A tick runs the
ensemble up to the next event (a resident request reaching its step count,
or the next arrival as estimated from the measured step time) and
synchronises once; while it runs, the host reads back the requests that
finished in the previous tick, stages the requests that have arrived (a
context of their size from a pool of finished ones, reset by
bfg_ctx_reset, or a new one) and prepares the inputs of later arrivals,
polling the tick with bfg_ens_wait.  Staged requests join the ensemble at
the next tick; the memory of finished ones serves later requests of the
same size, or is freed between ticks for others.

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
    """Continuous batching over one ensemble.

    The GPU runs ticks (bfg_ens_step over the resident requests) while the
    host does everything else: reading back the requests that finished in
    the previous tick (statistics and field downloads on their own
    contexts' streams), staging newly arrived requests (a context of their
    size from the pool, or a new one; upload of the initial field; tracers)
    and preparing the inputs of requests that have arrived.  Membership
    changes (adding staged requests, removing finished ones) and the release
    of device memory happen between ticks, when the GPU is idle:
    cudaFree waits for the whole device.  Memory is reclaimed lazily: the
    contexts of finished requests serve later requests of their size, and
    their tracer systems (a few tens of MB; freeing one took 10-30 ms even
    on an idle GPU) stay allocated, counted in the budget, until memory is
    needed or the server closes.
    """

    def __init__(self, hbm_budget=150e9, device=0, use_graphs=False, max_tick=64, pool=True):
        self.budget = hbm_budget
        self.used = 0              # bytes of running, staged, finishing and pooled requests
        self.device = device
        self.max_tick = max_tick   # most ensemble steps between two synchronisations
        self.step_ms = 0.0         # device time of one ensemble step, last tick
        self.busy_ms = 0.0         # device time of all ticks
        self.ticks = 0
        self.ens = ensemble(device)
        self.ens.use_graphs(use_graphs)
        self.running = {}   # rid -> [request, fs, ps, steps_done]
        self.staged = []    # [request, fs, ps] not yet in the ensemble
        self.finishing = [] # [request, fs, ps] out of the ensemble, results not yet read
        self.pool = {} if pool else None   # (n, precision) -> idle contexts
        self.retired = []   # [particles_system, bytes] of finished requests, not yet freed
        self.done = []
        # host seconds per phase of run(): step (the bfg_ens_step call:
        # membership rebuild and launches), collect, admit, wait (the tick
        # still running), between (memory release, staging and membership
        # changes while the GPU is idle)
        self.host_s = dict(step=0.0, collect=0.0, admit=0.0, wait=0.0, between=0.0)

    @staticmethod
    def _ctx_bytes(n, precision):
        return request_bytes(n, precision, 0, 0)

    @staticmethod
    def _tracer_bytes(req):
        return (request_bytes(req.n, req.precision, req.ntracers, req.nsteps_ab)
                - request_bytes(req.n, req.precision, 0, 0))

    def _context(self, req):
        key = (req.n, req.precision)
        if self.pool is not None and self.pool.get(key):
            fs = self.pool[key].pop()
            fs.reset()
            return fs, False
        return vorticity_equation(req.n, precision=req.precision, device=self.device), True

    def _stage(self, req, now):
        fs, fresh = self._context(req)
        fs.nu = req.nu
        fs.forcing_type = "linear"
        fs.famplitude, fs.fk0, fs.fk1 = req.famplitude, req.fk0, req.fk1
        if req.w0 is None:
            prepare(req)
        fs.set_cvorticity(req.w0)
        ps = None
        if req.ntracers > 0:
            ps = particles_system(fs, req.pos, req.neighbours, req.smoothness, req.nsteps_ab)
        req.admitted = now
        if fresh:
            self.used += self._ctx_bytes(req.n, req.precision)
        self.used += self._tracer_bytes(req)
        self.staged.append([req, fs, ps])

    def _admit(self, waiting, now):
        """Stage waiting requests in arrival order while they fit the budget
        (a pooled context of the right size costs nothing new)."""
        still = []
        for req in waiting:
            key = (req.n, req.precision)
            pooled = self.pool is not None and bool(self.pool.get(key))
            need = self._tracer_bytes(req) + (0 if pooled else self._ctx_bytes(req.n, req.precision))
            if self.used + need <= self.budget:
                self._stage(req, now)
            else:
                still.append(req)
        return still

    def _free_tracers(self, fs=None):
        """Free retired tracer systems (all of them, or those of context fs)."""
        keep = []
        for ps, nbytes in self.retired:
            if fs is None or ps.fs is fs:
                ps.close()
                self.used -= nbytes
            else:
                keep.append([ps, nbytes])
        self.retired = keep

    def _release(self, req):
        """Between ticks: free retired tracer systems, then idle contexts of
        other sizes, until `req` fits (a pooled context of its own size is
        kept for it).  A context is freed only after the tracer systems that
        still refer to it."""
        key = (req.n, req.precision)
        pooled = self.pool is not None and bool(self.pool.get(key))
        need = self._tracer_bytes(req) + (0 if pooled else self._ctx_bytes(*key))
        if self.used + need <= self.budget:
            return
        self._free_tracers()
        if not self.pool:
            return
        for other in list(self.pool):
            if other == key:
                continue
            while self.pool[other] and self.used + need > self.budget:
                fs = self.pool[other].pop()
                fs.close()
                self.used -= self._ctx_bytes(*other)

    def _collect(self, entry, now):
        """Results of a request out of the ensemble (its own streams), then
        its context to the pool; its tracers are freed between ticks."""
        req, fs, ps = entry
        # the final state's statistics (NSVE::do_stats): the energy spectrum
        # E(k) = tr(spec_uu) / 2, summed in a fixed order on the device, so a
        # request gives the same bits alone and in the mix
        spec_uu = fs.do_stats()["velocity"][0]
        req.result = {"vorticity_checksum": float(np.abs(fs.get_cvorticity()).sum()),
                      "iteration": fs.iteration,
                      "energy_spectrum": 0.5 * np.einsum("kii->k", spec_uu)}
        if ps is not None:
            req.result["tracers"] = ps.state()[0]
            self.retired.append([ps, self._tracer_bytes(req)])
        else:
            self.used -= self._tracer_bytes(req)
        if self.pool is not None:
            self.pool.setdefault((req.n, req.precision), []).append(fs)
        else:
            if ps is not None:
                self._free_tracers(fs)
            fs.close()
            self.used -= self._ctx_bytes(req.n, req.precision)
        req.finished = now
        self.done.append(req)

    def _between_ticks(self):
        for req, fs, ps in self.staged:
            self.ens.add(fs, req.dt, ps)
            self.running[req.rid] = [req, fs, ps, 0]
        self.staged = []

    def run(self, requests, clock=time.perf_counter, max_wall=None):
        """Serve a stream (arrival times relative to the call).  Returns the
        finished requests; time-to-completion is finished - arrival (the
        results read back on the host)."""
        pending = sorted(requests, key=lambda r: r.arrival)
        t0 = clock()
        qi = 0
        waiting = []
        while qi < len(pending) or waiting or self.running or self.staged or self.finishing:
            now = clock() - t0
            if max_wall is not None and now > max_wall:
                break
            while qi < len(pending) and pending[qi].arrival <= now:
                waiting.append(pending[qi])
                qi += 1
            # between ticks (the GPU is idle): release what waits for it
            tb = clock()
            if waiting:
                self._release(waiting[0])
            waiting = self._admit(waiting, clock() - t0)
            self._between_ticks()
            self.host_s["between"] += clock() - tb
            if not self.running:
                for entry in self.finishing:
                    self._collect(entry, clock() - t0)
                self.finishing = []
                if qi < len(pending) and not waiting:
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
            tb = clock()
            self.ens.step(k)
            tc = clock()
            self.host_s["step"] += tc - tb
            # while the tick runs: the previous tick's finished requests,
            # newly arrived requests (staged for the next tick) and the
            # inputs of arrived requests
            for entry in self.finishing:
                self._collect(entry, clock() - t0)
            self.finishing = []
            td = clock()
            self.host_s["collect"] += td - tc
            while qi < len(pending) and pending[qi].arrival <= clock() - t0:
                waiting.append(pending[qi])
                qi += 1
            waiting = self._admit(waiting, clock() - t0)
            te = clock()
            self.host_s["admit"] += te - td
            while not self.ens.wait(0.002):
                now = clock() - t0
                todo = [r for r in waiting + pending[qi:] if r.arrival <= now and r.w0 is None]
                if not todo:
                    self.ens.wait()
                    break
                prepare(todo[0])
            tick_ms = self.ens.last_ms()
            self.host_s["wait"] += clock() - te
            self.busy_ms += tick_ms
            self.ticks += 1
            self.step_ms = tick_ms / k
            for rid in list(self.running):
                self.running[rid][3] += k
                if self.running[rid][3] >= self.running[rid][0].steps:
                    req, fs, ps, _ = self.running.pop(rid)
                    self.ens.remove(fs)
                    self.finishing.append([req, fs, ps])
        return self.done

    def close(self):
        # retired tracer systems first: their contexts may since have been
        # reused by running or staged requests, and are freed below
        self._free_tracers()
        for rid in list(self.running):
            req, fs, ps, _ = self.running.pop(rid)
            self.ens.remove(fs)
            if ps is not None:
                ps.close()
            fs.close()
        for req, fs, ps in self.staged + self.finishing:
            if ps is not None:
                ps.close()
            fs.close()
        self.staged, self.finishing = [], []
        if self.pool:
            for fss in self.pool.values():
                for fs in fss:
                    fs.close()
            self.pool = {}
        self.ens.close()
