"""The serving loop's bookkeeping on the host (bfps_b200.serve.Server), with
stand-ins for the engine objects: every request finishes with its own step
count; contexts of finished requests are reused for later requests of their
size; tracer systems are reclaimed lazily and always before the context they
refer to is freed; the budget accounting returns to what is still held; and
close() frees everything.  The device path of the same loop is tested on the
GPU (tests/test_gpu_ensemble.py::test_serving_results_equal_alone)."""
import numpy as np
import pytest

from bfps_b200 import serve

EVENTS = []


class FakeContext:
    made = 0

    def __init__(self, n, precision="single", device=0):
        FakeContext.made += 1
        self.nx = n
        self.iteration = 0
        self.closed = False
        self.nu = self.famplitude = self.fk0 = self.fk1 = 0.0
        self.forcing_type = "none"

    def _live(self):
        assert not self.closed, "context used after it was freed"

    def set_cvorticity(self, w):
        self._live()

    def reset(self):
        self._live()
        self.iteration = 0
        EVENTS.append(("reset", id(self)))

    def do_stats(self):
        self._live()
        return {"velocity": (np.zeros((4, 3, 3)), None, None)}

    def get_cvorticity(self):
        self._live()
        return np.zeros((2, 2, 2, 3), np.complex64)

    def close(self):
        self._live()
        self.closed = True
        EVENTS.append(("close_ctx", id(self)))


class FakeTracers:
    def __init__(self, fs, pos, neighbours, smoothness, nsteps):
        fs._live()
        self.fs = fs
        self.n = len(pos)
        self.closed = False

    def state(self):
        assert not self.closed
        return (np.zeros((self.n, 3)), None, None)

    def close(self):
        assert not self.closed
        # a tracer system is freed while its context still exists
        assert not self.fs.closed, "tracer system freed after its context"
        self.closed = True
        EVENTS.append(("close_tracers", id(self)))


class FakeEnsemble:
    def __init__(self, device=0):
        self.members = []

    def use_graphs(self, enable):
        pass

    def add(self, fs, dt, ps):
        fs._live()
        assert fs not in self.members
        self.members.append(fs)

    def remove(self, fs):
        self.members.remove(fs)

    def step(self, k):
        for fs in self.members:
            fs._live()
            fs.iteration += k

    def wait(self, timeout_s=None):
        return True

    def last_ms(self):
        return 1.0

    def close(self):
        pass


@pytest.fixture
def fakes(monkeypatch):
    EVENTS.clear()
    FakeContext.made = 0
    monkeypatch.setattr(serve, "vorticity_equation", FakeContext)
    monkeypatch.setattr(serve, "particles_system", FakeTracers)
    monkeypatch.setattr(serve, "ensemble", FakeEnsemble)


def _stream():
    spec = [(16, 5, 20, 0.0), (16, 3, 0, 0.0), (32, 4, 10, 0.0), (16, 6, 30, 0.02),
            (32, 2, 0, 0.03), (16, 2, 5, 0.04)]
    reqs = []
    for i, (n, steps, nt, arr) in enumerate(spec):
        r = serve.Request(rid=i, n=n, nu=0.01, steps=steps, ntracers=nt, arrival=arr, seed=i)
        r.w0 = np.zeros((n, n, n // 2 + 1, 3), np.complex64)
        r.pos = np.zeros((nt, 3)) if nt else None
        r.dt = 0.01
        reqs.append(r)
    return reqs


def test_every_request_finishes_with_its_step_count(fakes):
    srv = serve.Server(hbm_budget=1e12)
    done = srv.run(_stream())
    assert sorted(r.rid for r in done) == list(range(6))
    for r in done:
        assert r.result["iteration"] == r.steps
        assert r.finished >= r.admitted >= r.arrival
    srv.close()


def test_contexts_are_reused_and_memory_accounted(fakes):
    reqs = _stream()
    srv = serve.Server(hbm_budget=1e12)
    srv.run(reqs)
    # the later 16^3 requests reuse contexts of finished ones (reset first)
    assert FakeContext.made < len(reqs)
    assert any(e[0] == "reset" for e in EVENTS)
    # what is still held: pooled contexts and retired tracer systems
    pooled = sum(serve.Server._ctx_bytes(n, p) * len(v) for (n, p), v in srv.pool.items())
    retired = sum(b for _, b in srv.retired)
    assert srv.used == pooled + retired
    srv.close()
    assert not srv.retired and not srv.pool


def test_tight_budget_frees_retired_tracers_and_reuses_the_context(fakes):
    """Four 16^3 requests with 1e4 tracers each (about twice a 16^3 context)
    under a budget that holds one at a time: each finished request's tracer
    system is freed during the run to make room for the next, whose context
    is the finished one's, reset."""
    reqs = []
    for i in range(4):
        r = serve.Request(rid=i, n=16, nu=0.01, steps=3 + i, ntracers=10000, arrival=0.0, seed=i)
        r.w0 = np.zeros((16, 16, 9, 3), np.complex64)
        r.pos = np.zeros((10000, 3))
        r.dt = 0.01
        reqs.append(r)
    one = serve.request_bytes(16, "single", 10000, 4)
    srv = serve.Server(hbm_budget=one + one // 4)
    done = srv.run(reqs, max_wall=30.0)
    assert sorted(r.rid for r in done) == [0, 1, 2, 3]
    assert all(r.result["iteration"] == r.steps for r in done)
    assert srv.used <= srv.budget
    assert FakeContext.made == 1
    kinds = [e[0] for e in EVENTS]
    assert kinds.count("close_tracers") >= 3 and kinds.count("reset") == 3
    assert "close_ctx" not in kinds
    srv.close()


def test_tight_budget_frees_contexts_of_other_sizes(fakes):
    """A budget with room for one 32^3 and one 16^3 request: idle contexts
    of one size are freed for requests of another, never while a retired
    tracer system still refers to them (the stand-ins assert that order)."""
    reqs = _stream()
    budget = (serve.request_bytes(32, "single", 10, 4) + serve.request_bytes(16, "single", 30, 4)
              + (1 << 20))
    srv = serve.Server(hbm_budget=budget)
    done = srv.run(reqs, max_wall=30.0)
    assert sorted(r.rid for r in done) == list(range(6))
    assert srv.used <= budget
    srv.close()
