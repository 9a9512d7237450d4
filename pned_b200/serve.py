"""Serving loop: continuous batching of Lanczos, mTPQ and DSF solves.

Requests for S = 1/2 honeycomb clusters of different N and couplings arrive
over time.  Each lattice size N has a *lane*: a slot batch (R slots over the
N-site lattice, libpned_gpu's pned_slots_*) on its own CUDA stream, so lanes
of different N run concurrently on the device.  A request is split into
*chains*, each occupying one slot:

  lanczos  one Lanczos chain (parallelized_lnc1z); result E0 by bisec
  tpq      nvec TPS chains with L = N l (parallelized_TPSz); per-step coefficients
  dsf      a Lanczos chain (E0, tridiagonal eigenvector by vec12), the
           eigenvector pass (parallelized_lncv1z) into a device vector x, then
           nq momentum chains from S^z_q x (intalv_zz, parallelized_dsflnc1z);
           spectra by exec_renbun

A chain is admitted when its lane has a free slot (an eigenvector pass also
needs the lane's eigenvector buffer); a lane is created when the HBM budget,
counted as 16 dim bytes per vector held (3 per slot, a start-vector buffer
and an eigenvector buffer per lane, plus the diagonal at 8 dim bytes per
slot), allows.  Lanes
advance in chunks of steps; between chunks finished chains are read and
released and waiting chains are loaded, so new requests join while others
run.  Latency of a request = completion time - arrival time.
"""
from __future__ import annotations

import collections
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import api
from . import couplings as CP
from .lattice import cluster_for_sites


# --------------------------------------------------------------------------- requests

@dataclass
class Request:
    rid: int
    kind: str                 # "lanczos" | "tpq" | "dsf"
    n: int
    phi: float                # J = cos(phi), K = 2 sin(phi)
    gamma: float
    h: float                  # field magnitude along [111]
    arrival: float            # seconds after the start of the stream
    steps: int                # Lanczos / TPS / DSF-chain steps
    nvec: int = 1             # TPQ vectors
    nq: int = 4               # DSF momenta
    gs_steps: int = 100       # DSF ground-state Lanczos steps
    l: float = 2.0            # TPQ: L = n l
    seed: int = 0

    def couplings(self):
        return (CP.kitaev_heisenberg(math.cos(self.phi), 2.0 * math.sin(self.phi), gamma=self.gamma),
                CP.field_111(self.h))


def make_stream(n_requests: int, rate: float, seed: int = 20261203, sizes=(18, 20, 22, 24, 26), p30: float = 0.02,
                mix=(0.80, 0.15, 0.05), lanczos_steps: int = 300, tpq_steps: int = 500, tpq_vectors: int = 4,
                dsf_steps: int = 100, dsf_momenta: int = 4, dsf_gs_steps: int = 100, min_n30: int = 0) -> list:
    """Poisson arrivals (rate per second) of the mixed request stream: N uniform over
    `sizes` plus a fraction p30 at N = 30; phi ~ U[0, 2 pi), Gamma ~ U[-0.2, 0.2],
    |h| ~ U[0, 0.1] along [111]; one seed per request id.  min_n30: a short
    sample that drew fewer N = 30 requests has its middle ones moved to N = 30
    (Lanczos requests first), so that the sample holds at least that many."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for rid in range(n_requests):
        t += rng.exponential(1.0 / rate) if rate > 0 else 0.0
        u = rng.random()
        kind = "lanczos" if u < mix[0] else ("tpq" if u < mix[0] + mix[1] else "dsf")
        n = 30 if rng.random() < p30 else int(rng.choice(sizes))
        phi, gamma, h = rng.uniform(0, 2 * math.pi), rng.uniform(-0.2, 0.2), rng.uniform(0, 0.1)
        steps = {"lanczos": lanczos_steps, "tpq": tpq_steps, "dsf": dsf_steps}[kind]
        out.append(Request(rid=rid, kind=kind, n=n, phi=phi, gamma=gamma, h=h, arrival=t, steps=steps,
                           nvec=tpq_vectors if kind == "tpq" else 1, nq=dsf_momenta, gs_steps=dsf_gs_steps,
                           seed=seed * 7919 + rid))
    short = min_n30 - sum(1 for q in out if q.n == 30)
    order = sorted(range(len(out)), key=lambda i: (out[i].kind != "lanczos", abs(i - len(out) // 2)))
    for i in order:
        if short <= 0:
            break
        if out[i].n != 30:
            out[i].n = 30
            short -= 1
    return out


# --------------------------------------------------------------------------- jobs and chains

@dataclass
class Chain:
    job: "Job"
    kind: str                 # "lanczos" | "tps" | "vector" | "szq"
    steps: int
    index: int = 0            # vector / momentum index within the job
    L: float = 0.0


class Job:
    """Request-level state machine: hands out chains, collects their results."""

    def __init__(self, req: Request, cluster):
        self.req = req
        self.cluster = cluster
        cpl, fld = req.couplings()
        self.couplings = api.ModelInput.from_couplings(cluster, cpl, field=fld)
        self.result: dict = {"rid": req.rid, "kind": req.kind, "n": req.n, "arrival": req.arrival}
        self.pending = 0
        self.x = None             # DSF eigenvector handle
        self.done = False
        self.parts: dict = {}

    def first_chains(self) -> list:
        r = self.req
        if r.kind == "lanczos":
            return self._issue([Chain(self, "lanczos", r.steps)])
        if r.kind == "tpq":
            L = r.n * r.l
            return self._issue([Chain(self, "tps", r.steps, index=k, L=L) for k in range(r.nvec)])
        return self._issue([Chain(self, "lanczos", r.gs_steps)])

    def _issue(self, chains):
        self.pending += len(chains)
        return chains

    def chain_done(self, ch: Chain, out: dict, engine) -> list:
        """Records a finished chain; returns the chains of the next phase (if any)."""
        self.pending -= 1
        r = self.req
        if out["status"]:
            self.result["status"] = "breakdown"
        if r.kind == "lanczos":
            self.result["e0"] = float(api.bisec(out["alpha"], out["beta"], out["steps"], 1)[0])
            self.result["alpha"], self.result["beta"] = out["alpha"], out["beta"]
        elif r.kind == "tpq":
            self.parts[ch.index] = out["coef"]
            if self.pending == 0:
                self.result["coef"] = np.stack([self.parts[k] for k in range(r.nvec)], axis=1)
                self.result["L"] = r.n * r.l
        elif ch.kind == "lanczos":          # DSF ground-state pass
            k = out["steps"]
            E = api.bisec(out["alpha"], out["beta"], k, 1)
            self.result["e0"] = float(E[0])
            c = api.vec12(out["alpha"], out["beta"], E, k, 1)[0]
            self.parts["gs"] = (out["alpha"], out["beta"], c)
            return self._issue([Chain(self, "vector", k)])
        elif ch.kind == "vector":
            return self._issue([Chain(self, "szq", r.steps, index=q) for q in range(r.nq)])
        else:                               # DSF momentum chain
            self.parts[("q", ch.index)] = (out["alpha"], np.concatenate([[out["cnorm"]], out["beta"]]))
            if self.pending == 0:
                self.result["salpha"] = [self.parts[("q", q)][0] for q in range(r.nq)]
                self.result["sbeta"] = [self.parts[("q", q)][1] for q in range(r.nq)]
        if self.pending == 0 and not (r.kind == "dsf" and "salpha" not in self.result):
            self.done = True
        return []


def dsf_spectra(result: dict, i_range: int = 2000, omega_max: float = 3.0, eta: float = 0.05):
    """S(q, w) of a finished DSF request on i_range points of [0, omega_max] (exec_renbun)."""
    split = omega_max / (i_range - 1)
    out = []
    for sa, sb in zip(result["salpha"], result["sbeta"]):
        _, _, d = api.exec_renbun(i_range, len(sa) + 2, split, result["e0"], eta, sa, sb)
        out.append(d)
    return np.array(out)


# --------------------------------------------------------------------------- device engine of a lane

class GpuLane:
    """Slot batch of one lattice size on its own CUDA stream."""

    def __init__(self, n: int, R: int, max_steps: int, budget: int = 0, n_vectors: int = 1, tune: bool = True):
        import torch
        self.torch = torch
        self.n = n
        self.cluster = cluster_for_sites(n)
        self.stream = torch.cuda.Stream()
        structure = api.ModelInput.structure(self.cluster)
        self.batch = api.SlotBatch(structure, R, max_steps, hbm_budget=budget, stream=self.stream)
        self.tuning = None
        if tune:
            from .tune import autotune_slots
            self.tuning = autotune_slots(self.batch, structure)
        self.R, self.dim = self.batch.R, self.batch.dim
        with torch.cuda.stream(self.stream):
            self.tmp = torch.empty(self.dim, dtype=torch.complex128, device="cuda")
            # eigenvectors of DSF requests between their eigenvector pass and the
            # loads of their momentum chains
            self.xpool = [torch.zeros(self.dim, dtype=torch.complex128, device="cuda") for _ in range(n_vectors)]
        self.vec_bytes = 16 * self.dim
        self.bytes = self.batch.bytes + self.vec_bytes * (1 + n_vectors)
        self._ev = None

    def load(self, slot: int, ch: Chain):
        job, r = ch.job, ch.job.req
        if ch.kind in ("lanczos", "vector", "tps"):
            nsrc = r.nvec if ch.kind == "tps" else 1
            api.gaussian_column(self.dim, nsrc, ch.index if ch.kind == "tps" else 0, r.seed, self.tmp, self.stream)
        if ch.kind == "lanczos":
            self.batch.load(slot, "lanczos", job.couplings, self.tmp, ch.steps)
        elif ch.kind == "tps":
            self.batch.load(slot, "tps", job.couplings, self.tmp, ch.steps, L=ch.L)
        elif ch.kind == "vector":
            a, b, c = job.parts["gs"]
            self.batch.load_vector(slot, job.couplings, self.tmp, a, b, c, job.x)
        else:
            self.batch.load_szq(slot, job.couplings, job.x, self.cluster.qr(ch.index), ch.steps)

    def take_vector(self):
        return self.xpool.pop() if self.xpool else None

    def give_vector(self, x):
        self.xpool.append(x)

    def release(self, slot: int):
        self.batch.release(slot)

    def step(self, k: int):
        t = self.torch
        e0, e1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        self.batch.step(k)
        e1.record(self.stream)
        self._ev = (e0, e1, k)

    def query(self) -> bool:
        return self.batch.query()

    def last_step_ms(self):
        if not self._ev:
            return None
        e0, e1, k = self._ev
        return e0.elapsed_time(e1) / k

    def read(self, slot: int) -> dict:
        return self.batch.read(slot)

    def close(self):
        self.batch.close()
        self.tmp = None
        self.xpool = []


# --------------------------------------------------------------------------- scheduler

def default_lane_slots(n: int) -> int:
    """Slots per lane.  Measured on B200: a step of R slots costs R times the
    single-vector step or more from N = 20 up (the partner-tile reads that
    bound the H.V scale with R), so larger lattices get single-slot lanes and
    run side by side instead; at N <= 18 four slots cost 0.7x per slot."""
    return 4 if n <= 18 else 1


def default_max_lanes(n: int) -> int:
    """Lanes per lattice size that may run side by side (small lattices leave
    most of the device idle, large ones fill it)."""
    if n <= 20:
        return 8
    if n <= 22:
        return 4
    if n <= 24:
        return 2
    return 1


@dataclass
class _LaneState:
    n: int
    eng: object
    occ: list
    left: list
    busy: bool = False
    idle_since: float = 0.0
    step_ms: float = 0.0
    steps_run: int = 0


@dataclass
class ServeStats:
    results: list = field(default_factory=list)
    makespan_s: float = 0.0
    lanes_created: int = 0
    peak_bytes: int = 0
    chunks: int = 0
    slot_steps: int = 0
    occupied_slot_steps: int = 0


class Server:
    """Continuous-batching request loop over lanes (see the module docstring).

    lane_factory(n, R, max_steps) builds a lane engine (GpuLane on the device);
    budget is the HBM budget in bytes; chunk_ms bounds the device time of one
    chunk, so that arrivals wait at most about that long for admission."""

    def __init__(self, budget: int, lane_factory=None, lane_slots=default_lane_slots, max_steps: int = 512,
                 chunk_ms: float = 30.0, clock=time.perf_counter, sleep=time.sleep, max_lanes=default_max_lanes,
                 exclusive_n: int = 24):
        self.budget = int(budget)
        # lanes of exclusive_n sites and more run their chunks one at a time: their H.V
        # holds a window of the vector in L2, which a second such kernel beside it evicts
        self.exclusive_n = exclusive_n
        self.lane_factory = lane_factory or (lambda n, R, ms: GpuLane(n, R, ms))
        self.lane_slots = lane_slots
        self.max_lanes = max_lanes
        self.max_steps = max_steps
        self.chunk_ms = chunk_ms
        self.clock, self.sleep = clock, sleep
        self.lanes: list = []
        self.used = 0
        self.clusters: dict = {}

    def _cluster(self, n):
        if n not in self.clusters:
            self.clusters[n] = cluster_for_sites(n)
        return self.clusters[n]

    def _lane_bytes(self, n, R):
        dim = 2 ** n
        return 56 * dim * R + 32 * dim

    def _open_lane(self, n, now, stats) -> bool:
        R = self.lane_slots(n)
        need = self._lane_bytes(n, R)
        if self.used + need > self.budget:
            # free idle lanes (nothing loaded, nothing waiting for their size), oldest first
            for ls in sorted(self.lanes, key=lambda x: x.idle_since):
                if self.used + need <= self.budget:
                    break
                if not ls.busy and all(o is None for o in ls.occ) and not self.waiting[ls.n]:
                    self._close_lane(ls)
            if self.used + need > self.budget:
                return False
        eng = self.lane_factory(n, R, self.max_steps)
        self.lanes.append(_LaneState(n=n, eng=eng, occ=[None] * eng.R, left=[0] * eng.R, idle_since=now))
        self.used += eng.bytes
        stats.lanes_created += 1
        stats.peak_bytes = max(stats.peak_bytes, self.used)
        return True

    def warm(self, sizes):
        """Plans (autotunes) the lanes of these lattice sizes ahead of the requests,
        as a server does at start-up: each lane is opened once and closed again,
        so that requests do not wait for the tuner (its choice is cached)."""
        for n in sorted(set(sizes)):
            eng = self.lane_factory(n, self.lane_slots(n), self.max_steps)
            eng.close()

    def _close_lane(self, ls):
        self.lanes.remove(ls)
        self.used -= ls.eng.bytes
        ls.eng.close()

    def run(self, requests, realtime: bool = True) -> ServeStats:
        """Serves `requests` (sorted by arrival); realtime=False admits each
        request as soon as the previous ones are admitted (arrival times are
        then only used for latency)."""
        stats = ServeStats()
        reqs = sorted(requests, key=lambda r: r.arrival)
        self.waiting = collections.defaultdict(collections.deque)
        jobs_open = 0
        i = 0
        t0 = self.clock()
        while i < len(reqs) or jobs_open:
            now = self.clock() - t0
            while i < len(reqs) and (not realtime or reqs[i].arrival <= now):
                job = Job(reqs[i], self._cluster(reqs[i].n))
                job.result["admitted"] = now
                self.waiting[job.req.n].extend(job.first_chains())
                jobs_open += 1
                i += 1
            progressed = False
            for ls in list(self.lanes):
                n = ls.n
                if ls.busy:
                    if not ls.eng.query():
                        continue
                    ls.busy = False
                    ms = ls.eng.last_step_ms()
                    if ms:
                        ls.step_ms = ms if ls.step_ms == 0 else 0.7 * ls.step_ms + 0.3 * ms
                # harvest
                for s in range(len(ls.occ)):
                    ch = ls.occ[s]
                    if ch is not None and ls.left[s] == 0:
                        out = ls.eng.read(s)
                        ls.eng.release(s)
                        ls.occ[s] = None
                        nxt = ch.job.chain_done(ch, out, ls.eng)
                        for c in reversed(nxt):        # a request's next phase goes first
                            self.waiting[n].appendleft(c)
                        if ch.job.done:
                            ch.job.result["finished"] = self.clock() - t0
                            ch.job.result["latency"] = ch.job.result["finished"] - ch.job.req.arrival
                            stats.results.append(ch.job.result)
                            jobs_open -= 1
                # admit waiting chains of this N into free slots, in order; an
                # eigenvector pass also needs room for its vector x
                q = self.waiting[n]
                free = [s for s in range(len(ls.occ)) if ls.occ[s] is None]
                skipped = []
                while free and q:
                    ch = q.popleft()
                    if ch.kind == "vector" and ch.job.x is None:
                        ch.job.x = ls.eng.take_vector()
                        if ch.job.x is None:
                            skipped.append(ch)
                            continue
                    s = free.pop(0)
                    ls.eng.load(s, ch)
                    ls.occ[s] = ch
                    ls.left[s] = ch.steps
                    if ch.kind == "szq" and ch.index == ch.job.req.nq - 1:
                        ls.eng.give_vector(ch.job.x)   # S^z_q x is formed at load; x is free after the last
                        ch.job.x = None
                q.extendleft(reversed(skipped))
                active = [s for s in range(len(ls.occ)) if ls.occ[s] is not None]
                if not active:
                    continue
                if n >= self.exclusive_n and any(o is not ls and o.busy and o.n >= self.exclusive_n
                                                 for o in self.lanes):
                    continue
                k = min(ls.left[s] for s in active)
                if ls.step_ms > 0:
                    k = max(1, min(k, int(self.chunk_ms / ls.step_ms)))
                else:
                    k = min(k, 3)
                ls.eng.step(k)
                ls.busy = True
                ls.idle_since = now
                ls.steps_run += k
                stats.chunks += 1
                stats.slot_steps += k * len(ls.occ)
                stats.occupied_slot_steps += k * len(active)
                for s in active:
                    ls.left[s] -= k
                progressed = True
            # more lanes for sizes whose waiting chains outnumber their free slots
            for n, q in self.waiting.items():
                if not q:
                    continue
                mine = [ls for ls in self.lanes if ls.n == n]
                free = sum(o is None for ls in mine for o in ls.occ)
                if len(q) > free and len(mine) < self.max_lanes(n):
                    if self._open_lane(n, now, stats):
                        progressed = True
            if not progressed:
                nxt = reqs[i].arrival - (self.clock() - t0) if i < len(reqs) and realtime else 0.0
                self.sleep(min(max(nxt, 0.0), 2e-4) if nxt > 0 else 5e-5)
        stats.makespan_s = self.clock() - t0
        return stats

    def close(self):
        for ls in list(self.lanes):
            self._close_lane(ls)


def summarize(stats: ServeStats, requests) -> dict:
    lat = np.array([r["latency"] for r in stats.results])
    first = min(r.arrival for r in requests)
    span = max(r["finished"] for r in stats.results) - first
    return {
        "requests": len(stats.results),
        "solves_per_s": len(stats.results) / span if span > 0 else float("inf"),
        "p50_latency_s": float(np.percentile(lat, 50)),
        "p99_latency_s": float(np.percentile(lat, 99)),
        "makespan_s": stats.makespan_s,
        "lanes_created": stats.lanes_created,
        "peak_bytes": stats.peak_bytes,
        "slot_occupancy": stats.occupied_slot_steps / max(1, stats.slot_steps),
    }


# --------------------------------------------------------------------------- plain one-at-a-time path

def warm_plain(requests):
    """Tunes the plain path's plans for every (size, vector count) the requests
    use, once (the autotuner caches per lattice, terms and R)."""
    from .tune import autotune
    seen = set()
    for r in requests:
        widths = {"lanczos": (1,), "tpq": (r.nvec,), "dsf": (1, r.nq)}[r.kind]
        for R in widths:
            key = (r.n, R, r.kind == "tpq")
            if key in seen:
                continue
            seen.add(key)
            cl = cluster_for_sites(r.n)
            cpl, fld = r.couplings()
            m = api.Model.from_couplings(cl, cpl, field=fld, tps_L=r.n * r.l if r.kind == "tpq" else None)
            autotune(m, R)
            m.close()


def run_plain(req: Request) -> dict:
    """One request alone through the plain path (model, context and whole-run
    driver per request, as a caller without the serving loop would), with the
    autotuner's plan for its lattice and vector count (cached after the first)."""
    import torch
    cl = cluster_for_sites(req.n)
    cpl, fld = req.couplings()
    out = {"rid": req.rid, "kind": req.kind, "n": req.n}
    from .tune import autotune
    if req.kind == "lanczos":
        m = api.Model.from_couplings(cl, cpl, field=fld)
        autotune(m, 1)
        ctx = api.Context(m, R=1)
        v = torch.empty(m.dim, dtype=torch.complex128, device="cuda")
        ctx.fill_gaussian(req.seed, v)
        r = ctx.lanczos(v, req.steps)
        out["e0"] = float(api.bisec(r["alpha"][:, 0], r["beta"][:, 0], req.steps, 1)[0])
    elif req.kind == "tpq":
        L = req.n * req.l
        m = api.Model.from_couplings(cl, cpl, field=fld, tps_L=L)
        autotune(m, req.nvec)
        ctx = api.Context(m, R=req.nvec)
        v = torch.empty(m.dim * req.nvec, dtype=torch.complex128, device="cuda")
        ctx.fill_gaussian(req.seed, v)
        r = ctx.tps(L, v, req.steps)
        out["coef"] = r["coef"]
    else:
        m = api.Model.from_couplings(cl, cpl, field=fld)
        autotune(m, 1)
        autotune(m, req.nq)
        ctx = api.Context(m, R=1)
        v = torch.empty(m.dim, dtype=torch.complex128, device="cuda")
        ctx.fill_gaussian(req.seed, v)
        r = ctx.lanczos(v, req.gs_steps)
        a, b = r["alpha"][:, 0], r["beta"][:, 0]
        E = api.bisec(a, b, req.gs_steps, 1)
        e0 = float(E[0])
        c = api.vec12(a, b, E, req.gs_steps, 1)[0]
        x = ctx.lanczos_vector(v, a, b, c)
        ctx.close()
        ctxq = api.Context(m, R=req.nq)
        qrs = np.stack([cl.qr(q) for q in range(req.nq)])
        d = ctxq.dsf(x, qrs, req.steps)
        out["e0"] = e0
        out["salpha"] = [d["salpha"][:, q] for q in range(req.nq)]
        out["sbeta"] = [d["sbeta"][:, q] for q in range(req.nq)]
        ctxq.close()
    ctx.close()
    m.close()
    torch.cuda.synchronize()
    return out
