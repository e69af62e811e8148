"""Host logic of the serving loop: the open-loop driver submits every request
at its arrival time whatever the completions, and latency percentiles.  A
fake clock and a fake server stand in for the native engine."""
from hashgraph_b200.serve import Request, latency_summary, run_open_loop


class _Clock:
    def __init__(self):
        self.t = 100.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += dt


class _FakeServer:
    """Completes each request 5 ms after its submission."""

    def __init__(self, clock):
        self.clock = clock
        self.pending = []
        self.submitted = []

    def submit(self, r):
        self.submitted.append((r, self.clock()))
        self.pending.append((r, self.clock() + 0.005))

    def poll(self, block=False):
        done = [r for r, t in self.pending if t <= self.clock()]
        self.pending = [(r, t) for r, t in self.pending if t > self.clock()]
        for r in done:
            r.latency_s = 0.005
        return done

    def drain(self):
        out = [r for r, _ in self.pending]
        for r in out:
            r.latency_s = 0.005
        self.pending = []
        return out


def test_open_loop_submits_at_arrival_times():
    clock = _Clock()
    srv = _FakeServer(clock)
    reqs = [Request("intersect", 0, 10.0 + 0.001 * k) for k in range(20)]
    makespan = run_open_loop(srv, reqs, clock=clock, sleep=clock.sleep)
    assert len(srv.submitted) == 20
    # each request goes in no earlier than its arrival, and not long after it
    for r, t in srv.submitted:
        assert r.arrival - 1e-12 <= t <= r.arrival + 0.0006
    # arrivals were re-stamped relative to the first one
    assert abs(reqs[0].arrival - 100.0) < 1e-9 and abs(reqs[-1].arrival - reqs[0].arrival - 0.019) < 1e-9
    assert makespan >= 0.019
    assert all(r.latency_s == 0.005 for r in reqs)


def test_latency_percentiles():
    reqs = [Request("build", 0, 0.0, latency_s=k / 1000.0) for k in range(1, 101)]
    s = latency_summary(reqs)
    assert abs(s["p50_ms"] - 51.0) < 1e-9 and abs(s["p99_ms"] - 100.0) < 1e-9
    assert abs(s["mean_ms"] - 50.5) < 1e-9 and s["max_ms"] == 100.0
    assert latency_summary([]) == {}
