"""Benchmark: Lanczos steps/s on the N = 30 S = 1/2 Kitaev-Heisenberg honeycomb.

Workload (default): 3x5 periodic honeycomb, 30 sites, 45 bonds, full basis of
2^30 states, complex128; J = cos(0.3 pi), K = 2 sin(0.3 pi), no Gamma / field;
one Lanczos chain from a seeded complex-Gaussian vector.  A step is one
Lanczos iteration (H.v with the fused <v|Hv>, the residual with beta, and the
scalar update) over the whole 2^30 basis.

Prints one JSON line (rank 0).  `--impl reference` times the reference's CPU
algorithm (the oracle restatement of pNED's single-rank path, OpenMP on all host
cores) on a bounded sample of the same workload instead.

Inputs are larger than L2 (each vector is 17.2 GB), so no L2 flush is needed
between steps.  Multi-GPU (--gpus N under torchrun): independent replicas, one
per GPU, no collective on the data path; value = steps of all ranks / max time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "lanczos_steps_per_s_N30"
UNIT = "steps/s"
SEED = 20261203


def workload_config(n_sites=30):
    return {
        "workload": f"S=1/2 Kitaev-Heisenberg honeycomb N={n_sites} (3x5 periodic, 45 bonds), full basis "
                    f"D=2^{n_sites}, complex128, 1 Lanczos chain, J=cos(0.3pi), K=2sin(0.3pi)",
        "n_sites": n_sites, "dim": 2 ** n_sites, "R": 1, "parallelism": "replicas",
        "l2": "inputs larger than L2 (17.2 GB per vector), no flush",
        "seed": SEED,
    }


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_bench_{os.getpid()}.csv")

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            return out
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for nm, val in zip(names, r[5:9]):
                    if val.strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                continue
        if sm:
            out.update(sm_mhz=statistics.median(sm), sm_max_mhz=max(mx), reasons=sorted(reasons), samples=len(sm))
        return out


def build_model(n_sites=30, R=1):
    import pned_b200 as P
    from pned_b200 import couplings as CP
    from pned_b200.lattice import cluster_for_sites
    cl = cluster_for_sites(n_sites)
    cpl = CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi))
    return P.Model.from_couplings(cl, cpl), cl


class CpuSample:
    """Reference CPU algorithm on a bounded sample of the workload: one Lanczos
    step's p_mltply_v3 restricted to 2^slice_log2 output states (all bond x
    element passes, gathering from a full-size input vector) plus the step's
    vector updates on the same slice; a sample's time is scaled to the whole
    basis."""

    def __init__(self, n_sites: int, threads: int, slice_log2: int = 24):
        import numpy as np
        from oracle import oracle as O
        from pned_b200 import couplings as CP
        from pned_b200.lattice import cluster_for_sites
        self.O = O
        O.set_num_threads(threads)
        cl = cluster_for_sites(n_sites)
        cpl = CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi))
        X = O.xlocal(2, 0, cpl)
        skip, _, pt = O.parity_skip(2, 0, X)
        self.om = O.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
        self.D = self.om.ldim
        self.v1 = O.gaussian(SEED, self.D)          # full-size gather source
        self.hi = 1 << min(slice_log2, n_sites)
        self.v0 = np.zeros(self.hi, dtype=np.complex128)
        self.scale = self.D / self.hi
        self.desc = (f"p_mltply_v3 (all {self.om.nbond * 4} bond x element passes) + the step's vector updates "
                     f"over 2^{int(math.log2(self.hi))} of the 2^{n_sites} output states, full-size input vector, "
                     f"time scaled x{int(self.scale)}")

    def step_seconds(self) -> float:
        O = self.O
        self.v0[:] = 0
        t0 = time.perf_counter()
        self.om.p_mltply_v3_slice(self.v1, self.v0, 0, self.hi)
        # swap (4 vector passes) + calc_beta (2 passes) on the slice
        a = self.v1[:self.hi]
        tmp = (self.v0 - 0.5 * a) / 1.5
        self.v0[:] = -1.5 * a
        O.inprdct(tmp, tmp)
        return (time.perf_counter() - t0) * self.scale


def run_reference(args, rank, world):
    """--impl reference: the reference CPU algorithm, timed on the host cores."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    cs = CpuSample(args.n_sites, threads, slice_log2=args.ref_slice_log2)
    for _ in range(args.warmup):
        cs.step_seconds()
    secs = [cs.step_seconds() for _ in range(args.steps)]
    value = args.steps / sum(secs)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 / value, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128", "data": "synthetic (seeded complex Gaussian)", "impl": "reference",
        "config": workload_config(args.n_sites),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": cs.desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import pned_b200 as P

    torch.cuda.set_device(local_rank)
    P.lib().pned_set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    model, cl = build_model(args.n_sites)
    D = model.dim
    stream = torch.cuda.Stream(device=dev)
    ctx = P.Context(model, R=1, stream=stream)   # every kernel of the context runs on `stream`
    v = torch.empty(D, dtype=torch.complex128, device=dev)
    ctx.fill_gaussian(SEED, v, normalise=True)
    total_steps = args.warmup + args.steps + args.profile_steps + 1
    ctx.session_begin("lanczos", v, total_steps)
    ctx.session_step(args.warmup)
    ctx.synchronize()
    # --- timed region: exactly K steps
    import torch.distributed as dist
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        time.sleep(0.3)
        torch.cuda.synchronize()
        start.record(stream)
        ctx.session_step(args.steps)
        end.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    res = ctx.session_read()
    # --- per-kernel timing for the roofline (CUDA events on the context's stream)
    hv_ms, step_ms = ctx.session_profile(args.profile_steps)
    ctx.session_end()
    alpha = res["alpha"][:, 0]
    beta = res["beta"][:, 0]
    e0 = float(P.bisec(alpha, beta, len(alpha), 1)[0])

    # --- end to end through the public API: host vector in, alpha/beta out
    e2e = None
    if args.e2e:
        try:
            host = torch.empty(D, dtype=torch.complex128, pin_memory=True)
            host.copy_(v)
            hv = host.numpy()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = ctx.lanczos(hv, args.steps)
            t1 = time.perf_counter()
            e2e = {"value": args.steps / (t1 - t0), "unit": UNIT, "h2d_bytes_per_step": 16 * D / args.steps,
                   "d2h_bytes_per_step": 16, "e0": float(out["ene"][0])}
            del host, hv
        except Exception as exc:  # pinned allocation can fail on small hosts
            e2e = {"value": None, "unit": UNIT, "error": str(exc)[:200]}

    peak, peak_kind = load_peaks()
    plan = model.plan()
    # algorithmic bytes of the H.v in a Lanczos step (all flip masks resolved on
    # chip): read C, read P, write W (16 B each) + real diagonal (8 B)
    bytes_hv = (16 + 16 + 16 + 8) * D
    achieved = bytes_hv / (hv_ms * 1e-3) / 1e9
    # kernels per step: the H.v launches (one per tile pass), finish, residual, finish, epilogue
    launches_per_step = max(1, plan["tile_passes"]) + 4
    value = world * args.steps / (ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded complex Gaussian start vector)",
        "config": workload_config(args.n_sites),
        "e0_after_warmup_plus_steps": e0,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "kernel": (f"hv_tile_kernel x{plan['tile_passes']} passes (K=1)" if plan["tile_passes"]
                                else "hv_xor_kernel (K=1)"),
                     "hv_ms": hv_ms, "step_ms_profiled": step_ms, "algorithmic_bytes_per_hv": bytes_hv,
                     "plan": plan, "traffic": args.traffic},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk.summary(),
        "e2e": e2e,
    }
    if rank == 0 and args.cpu_baseline:
        try:
            cs = CpuSample(args.n_sites, os.cpu_count() or 1, slice_log2=args.ref_slice_log2)
            cs.step_seconds()
            secs = [cs.step_seconds() for _ in range(3)]
            line["cpu_baseline"] = {"value": 3 / sum(secs), "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                    "sample": cs.desc + "; mean of 3 samples after 1 warm-up"}
            del cs
        except Exception as exc:
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "error": str(exc)[:200]}
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n-sites", type=int, default=30)
    ap.add_argument("--profile-steps", type=int, default=3)
    ap.add_argument("--ref-slice-log2", type=int, default=24)
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--traffic", type=float, default=None, help="DRAM bytes per H.v launch from an ncu capture")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if args.impl == "ours":
            torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo",
                                timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
