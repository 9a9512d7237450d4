"""Host logic of the serving loop (no GPU): admission against the HBM budget,
co-batching by lattice size, the DSF phases and latency bookkeeping, driven
by a fake lane engine that records what the device would be asked to do."""
import numpy as np

from pned_b200 import serve


class FakeLane:
    log = []

    def __init__(self, n, R, max_steps):
        self.n, self.R, self.dim = n, R, 2 ** n
        self.vec_bytes = 16 * self.dim
        self.bytes = 56 * self.dim * R + 32 * self.dim
        self.pool = [object()]
        self.occ = [None] * R
        self.done = [0] * R
        self.max_occupied = 0
        FakeLane.log.append(("open", n, R))

    def load(self, slot, ch):
        assert self.occ[slot] is None
        assert ch.steps <= 512
        self.occ[slot] = ch
        self.done[slot] = 0
        FakeLane.log.append(("load", self.n, slot, ch.job.req.rid, ch.kind, ch.index))

    def take_vector(self):
        return self.pool.pop() if self.pool else None

    def give_vector(self, x):
        self.pool.append(x)

    def release(self, slot):
        self.occ[slot] = None

    def step(self, k):
        assert k >= 1
        self.max_occupied = max(self.max_occupied, sum(o is not None for o in self.occ))
        for s, ch in enumerate(self.occ):
            if ch is not None:
                self.done[s] = min(ch.steps, self.done[s] + k)

    def query(self):
        return True

    def last_step_ms(self):
        return 0.5

    def read(self, slot):
        ch = self.occ[slot]
        k = self.done[slot]
        assert k == ch.steps, "a slot is read only when its chain has finished"
        a = -1.0 - 0.01 * np.arange(k) - ch.job.req.rid * 1e-3
        b = 0.5 + 0.001 * np.arange(k)
        return {"kind": ch.kind, "steps": k, "status": 0, "alpha": a, "beta": b, "coef": np.ones((k, 5)),
                "cnorm": 0.25}

    def close(self):
        FakeLane.log.append(("close", self.n))


def make(budget, **kw):
    FakeLane.log = []
    lanes = []

    def factory(n, R, ms):
        lane = FakeLane(n, R, ms)
        lanes.append(lane)
        return lane

    return serve.Server(budget, lane_factory=factory, sleep=lambda s: None, **kw), lanes


def small_stream(n=60, seed=5):
    return serve.make_stream(n, rate=1e6, seed=seed, sizes=(10, 12, 14), p30=0.0, lanczos_steps=30, tpq_steps=40,
                             dsf_steps=20, dsf_gs_steps=25)


def test_all_requests_complete_with_their_phases():
    reqs = small_stream()
    srv, lanes = make(budget=1 << 40, lane_slots=lambda n: 4, max_lanes=lambda n: 1)
    st = srv.run(reqs, realtime=False)
    assert sorted(r["rid"] for r in st.results) == [q.rid for q in reqs]
    by = {r["rid"]: r for r in st.results}
    for q in reqs:
        r = by[q.rid]
        assert r["latency"] >= 0 and r["finished"] >= r["admitted"]
        if q.kind == "lanczos":
            assert np.isfinite(r["e0"])
        elif q.kind == "tpq":
            assert r["coef"].shape == (q.steps, q.nvec, 5)
        else:
            assert len(r["salpha"]) == q.nq and len(r["sbeta"][0]) == q.steps + 1
            kinds = [e[4] for e in FakeLane.log if e[0] == "load" and e[3] == q.rid]
            assert kinds == ["lanczos", "vector"] + ["szq"] * q.nq
    # requests of one size share a lane and run side by side
    assert {e[1] for e in FakeLane.log if e[0] == "open"} == {q.n for q in reqs}
    assert max(l.max_occupied for l in lanes) > 1
    assert st.slot_steps >= st.occupied_slot_steps > 0


def test_budget_bounds_the_lanes_held():
    reqs = small_stream(40, seed=9)
    one_lane = 56 * 2 ** 14 * 2 + 32 * 2 ** 14
    srv, lanes = make(budget=one_lane, lane_slots=lambda n: 2, max_lanes=lambda n: 1)
    st = srv.run(reqs, realtime=False)
    assert len(st.results) == len(reqs)
    assert st.peak_bytes <= one_lane
    # the lanes held at any time fit the budget; the N = 14 lane holds all of it
    held, sizes = 0, {}
    for e in FakeLane.log:
        if e[0] == "open":
            sizes[e[1]] = 56 * 2 ** e[1] * e[2] + 32 * 2 ** e[1]
            held += sizes[e[1]]
            assert held <= one_lane
        elif e[0] == "close":
            held -= sizes[e[1]]
    assert any(e[0] == "close" for e in FakeLane.log)


def test_stream_statistics():
    reqs = serve.make_stream(2000, rate=50.0, seed=20261203)
    kinds = np.array([r.kind for r in reqs])
    ns = np.array([r.n for r in reqs])
    assert abs(np.mean(kinds == "lanczos") - 0.80) < 0.03
    assert abs(np.mean(kinds == "tpq") - 0.15) < 0.03
    assert abs(np.mean(ns == 30) - 0.02) < 0.01
    assert set(ns) <= {18, 20, 22, 24, 26, 30}
    gaps = np.diff([r.arrival for r in reqs])
    assert abs(np.mean(gaps) - 1 / 50.0) < 0.003
    assert all(-0.2 <= r.gamma <= 0.2 and 0 <= r.h <= 0.1 for r in reqs)
    assert len({r.seed for r in reqs}) == len(reqs)


def test_summary_percentiles():
    reqs = small_stream(20, seed=3)
    srv, _ = make(budget=1 << 40, lane_slots=lambda n: 4)
    st = srv.run(reqs, realtime=False)
    s = serve.summarize(st, reqs)
    assert s["requests"] == 20 and s["p99_latency_s"] >= s["p50_latency_s"] >= 0


def test_several_lanes_per_size_run_side_by_side():
    reqs = small_stream(40, seed=21)
    srv, lanes = make(budget=1 << 40, lane_slots=lambda n: 1, max_lanes=lambda n: 3)
    st = srv.run(reqs, realtime=False)
    assert len(st.results) == len(reqs)
    per_n = {}
    for e in FakeLane.log:
        if e[0] == "open":
            per_n[e[1]] = per_n.get(e[1], 0) + 1
    assert max(per_n.values()) == 3 and all(v <= 3 for v in per_n.values())


def test_short_stream_holds_the_requested_n30_requests():
    """A short sample of the serving mix (2 % at N = 30) that drew no N = 30
    request has one moved there, a Lanczos request from the middle; the rest of
    the stream is unchanged."""
    base = serve.make_stream(40, rate=1.0, seed=20261203)
    got = serve.make_stream(40, rate=1.0, seed=20261203, min_n30=1)
    n30 = [q for q in got if q.n == 30]
    assert len(n30) >= 1
    moved = [(a, b) for a, b in zip(base, got) if a.n != b.n]
    assert len(moved) == max(0, 1 - sum(1 for q in base if q.n == 30))
    for a, b in moved:
        assert b.kind == "lanczos" and b.n == 30 and (a.rid, a.arrival, a.seed) == (b.rid, b.arrival, b.seed)
    assert serve.make_stream(40, rate=1.0, seed=20261203, min_n30=3)[20].n in (18, 20, 22, 24, 26, 30)
    assert sum(1 for q in serve.make_stream(40, rate=1.0, seed=20261203, min_n30=3) if q.n == 30) >= 3
