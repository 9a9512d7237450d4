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
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "lanczos_steps_per_s_N30"
LOAD_FRACTION = 0.7   # the served latency run's arrival rate, as a fraction of the measured capacity
UNIT = "steps/s"
SEED = 20261203


def workload_config(n_sites=30):
    from pned_b200.lattice import cluster_for_sites
    cl = cluster_for_sites(n_sites)
    gb = 16 * 2 ** n_sites / 1e9
    l2 = (f"inputs larger than L2 ({gb:.1f} GB per vector), no flush" if gb > 0.126 else
          f"vectors of {gb * 1e3:.0f} MB, below L2 (no flush)")
    return {
        "workload": f"S=1/2 Kitaev-Heisenberg honeycomb N={n_sites} ({cl.L1}x{cl.L2} periodic, {cl.nbond} bonds), "
                    f"full basis D=2^{n_sites}, complex128, 1 Lanczos chain, J=cos(0.3pi), K=2sin(0.3pi)",
        "n_sites": n_sites, "dim": 2 ** n_sites, "R": 1, "parallelism": "replicas",
        "l2": l2,
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
        self.path = os.path.join(tempfile.gettempdir(), f"pned_clocks_{os.getpid()}.csv")

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


# single-vector tile kernel by partner-tile staging mode of the plan
TILE_KERNELS = {0: "hv_tile_kernel", 1: "hv_tile_stage_kernel", 2: "hv_tile_bulk_kernel", 3: "hv_tile_tma_kernel"}


def cpu_step_timing(n_sites: int, threads: int, samples: int, warmup: int, full: int, slice_log2: int) -> dict:
    """The reference CPU algorithm (the oracle port of parallelized_lnc1z's step)
    timed by oracle/cpu_step.py in a process of its own, so that torch's OpenMP
    threads do not share the cores with the oracle's: `samples` bounded samples
    (one step on 2^slice_log2 output states, scaled) and `full` whole steps."""
    cmd = [sys.executable, "-m", "oracle.cpu_step", "--n-sites", str(n_sites), "--threads", str(threads),
           "--samples", str(samples), "--warmup", str(warmup), "--full", str(full), "--slice-log2", str(slice_log2)]
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    out = subprocess.run(cmd, cwd=os.path.dirname(os.path.abspath(__file__)), env=env, capture_output=True, text=True,
                         check=True)
    return json.loads(out.stdout.strip().splitlines()[-1])


def replica_aggregate(ms_local: float, steps: int, world: int, device="cuda"):
    """Whole-job figure of independent replicas: the slowest rank's time (max
    over ranks, after a barrier) and all ranks' steps over it."""
    ms = float(ms_local)
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    return ms, world * steps / (ms * 1e-3)


def run_reference(args, rank, world):
    """--impl reference: the reference CPU algorithm, timed on the host cores --
    args.steps bounded samples (after args.warmup) and one whole step."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    t = cpu_step_timing(args.n_sites, threads, args.steps, args.warmup, args.ref_full_steps, args.ref_slice_log2)
    sampled = len(t["sample_step_s"]) / sum(t["sample_step_s"])
    full = len(t["full_step_s"]) / sum(t["full_step_s"]) if t["full_step_s"] else None
    value = full if full is not None else sampled
    sample = (f"{len(t['full_step_s'])} whole Lanczos step(s) over all 2^{args.n_sites} states timed as they are "
              f"(value); beside them {len(t['sample_step_s'])} bounded samples: {t['sample']}")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 / value, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128", "data": "synthetic (seeded complex Gaussian)", "impl": "reference",
        "config": workload_config(args.n_sites),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                         "cpu": t["cpu"], "full_steps_executed": len(t["full_step_s"]),
                         "full_step_s": t["full_step_s"], "sampled_steps_executed": len(t["sample_step_s"]),
                         "sampled_value": sampled, "sample_step_s": t["sample_step_s"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def dense_check(n_sites: int = 12):
    """E0 of the headline couplings on a small cluster: the library's Lanczos
    against full FP64 diagonalisation (numpy eigvalsh, LAPACK zheevd) of the
    dense matrix assembled column by column from the library's own H.v.
    Reports the Lanczos error only; the H.v itself is held to the oracle by the
    parity tests."""
    import numpy as np
    import torch
    import pned_b200 as P
    model, cl = build_model(n_sites)
    D, R = model.dim, 16
    ctx = P.Context(model, R=R)
    Ht = np.zeros((D, D), dtype=np.complex128)   # rows: H^T e_k (p_mltply_v3 applies H^T)
    eye = torch.zeros(D * R, dtype=torch.complex128, device="cuda")
    out = torch.zeros_like(eye)
    for k0 in range(0, D, R):
        eye.zero_()
        out.zero_()
        idx = torch.arange(R, device="cuda")
        eye[(k0 + idx) * R + idx] = 1.0
        ctx.p_mltply_v3(eye, out)
        Ht[k0:k0 + R] = out.view(D, R).t().cpu().numpy()
    ctx.close()
    e_dense = float(np.linalg.eigvalsh(Ht.T)[0])
    ctx1 = P.Context(model, R=1)
    v = torch.empty(D, dtype=torch.complex128, device="cuda")
    ctx1.fill_gaussian(SEED, v, normalise=True)
    run = ctx1.lanczos(v, 300, check_conv=True)
    ctx1.close()
    model.close()
    e_lz = float(run["ene"][0])
    return {"n_sites": n_sites, "dim": D, "e0_lanczos": e_lz, "e0_dense_zheevd": e_dense,
            "rel_err": abs(e_lz - e_dense) / abs(e_dense), "lanczos_steps": int(run["itr"])}


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import pned_b200 as P

    torch.cuda.set_device(local_rank)
    P.lib().pned_set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    model, cl = build_model(args.n_sites)
    D = model.dim
    tuning = None
    if args.plan:
        plan = [int(x) for x in args.plan.split(",")]
        model.set_plan(1, *plan)
        tuning = {"plan": plan, "tried": []}
    elif args.tune:
        from pned_b200.tune import autotune
        tuning = autotune(model, 1)
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
    ms, value = replica_aggregate(start.elapsed_time(end), args.steps, world, device=dev)
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
    # DRAM traffic of the tiled H.v per state, from the ncu capture of the same
    # kernel and plan shape at N=26 (6.92 GB per H.v over 2^26 states), scaled
    # to this basis; an ncu figure passed with --traffic replaces it
    traffic = args.traffic if args.traffic is not None else (6.92e9 / 2 ** 26 * D if plan["tile_passes"] else None)
    # algorithmic bytes of the H.v in a Lanczos step (all flip masks resolved on
    # chip): read C, read P, write W (16 B each) + real diagonal (8 B)
    bytes_hv = (16 + 16 + 16 + 8) * D
    achieved = bytes_hv / (hv_ms * 1e-3) / 1e9
    # kernels per step: the H.v launches (one per tile pass), the finish of the per-tile
    # sums (a second level above 2048 of them), residual, finish, epilogue
    n_sums = plan["tile_passes"] * D // max(1, plan["tile_states"]) if plan["tile_passes"] else 0
    launches_per_step = max(1, plan["tile_passes"]) + 4 + (1 if n_sums > 2048 else 0)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded complex Gaussian start vector)",
        "config": workload_config(args.n_sites),
        "e0_after_warmup_plus_steps": e0,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "kernel": (f"{TILE_KERNELS.get(plan.get('staging', 0), 'hv_tile_kernel')} "
                                f"x{plan['tile_passes']} passes (K=1)" if plan["tile_passes"]
                                else "hv_xor_kernel (K=1)"),
                     "hv_ms": hv_ms, "step_ms_profiled": step_ms, "algorithmic_bytes_per_hv": bytes_hv,
                     "plan": plan, "traffic": traffic,
                     "traffic_source": ("--traffic" if args.traffic is not None else
                                        "scaled from the N=26 ncu capture (103 B/state)"),
                     # the accounting that counts every partner-tile read (m of them) as a vector read
                     "partner_read_accounting": {
                         "m": plan["partner_tiles"],
                         "bytes_per_hv": 16 * D * (1 + plan["partner_tiles"]) + 16 * D,
                         "GBs": (16 * D * (2 + plan["partner_tiles"])) / (hv_ms * 1e-3) / 1e9,
                         "frac": (16 * D * (2 + plan["partner_tiles"])) / (hv_ms * 1e-3) / 1e9 / peak,
                         "note": "partner tiles are read from L2, not HBM, so this fraction can exceed 1"}},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk.summary(),
        "e2e": e2e,
    }
    # the bound that holds this gather in practice: every flip term moves a 16-byte
    # operand per state through the SM's load/store data path (128 B per clock per
    # SM), whether it comes from shared memory or from L1/L2; the own-row and
    # epilogue accesses come on top, so the fraction is a lower bound
    clk_sum = line["clocks"]
    if plan["tile_passes"] and clk_sum.get("sm_mhz"):
        nsm = torch.cuda.get_device_properties(dev).multi_processor_count
        lsu_bytes = 16 * model.n_terms * D
        lsu_peak = 128 * nsm * clk_sum["sm_mhz"] * 1e6 / 1e12
        lsu_ach = lsu_bytes / (hv_ms * 1e-3) / 1e12
        line["roofline"]["data_path"] = {
            "bound": "l1_data_path", "unit": "TB/s", "flip_terms": model.n_terms,
            "bytes_per_hv": lsu_bytes, "achieved": lsu_ach, "peak": lsu_peak, "frac": lsu_ach / lsu_peak,
            "note": "flip-term operands only (16 B per term and state) against 128 B per clock per SM at the "
                    "median SM clock of the timed region; own-row and epilogue accesses are not counted"}
    if tuning is not None:
        pl = list(tuning["plan"]) + [-1] * (4 - len(tuning["plan"]))
        line["roofline"]["tuned_plan"] = {"row_fixed_bits": pl[0], "window_bits": pl[1], "max_passes": pl[2],
                                          "j_bits": pl[3] if len(pl) > 3 else -1,
                                          "blocks_per_sm": pl[6] if len(pl) > 6 else -1,
                                          "objective": pl[7] if len(pl) > 7 else 0,
                                          "terms_in_flight": pl[8] if len(pl) > 8 else -1,
                                          "plan_arg": ",".join(str(x) for x in pl),
                                          "candidates": len(tuning.get("tried", []))}
    if rank == 0 and args.dense_check:
        try:
            line["dense_check"] = dense_check(12)
        except Exception as exc:  # reported, not fatal: the headline line stands without it
            line["dense_check"] = {"error": str(exc)}
    if rank == 0 and args.cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            t = cpu_step_timing(args.n_sites, threads, 3, 1, 0, args.ref_slice_log2)
            line["cpu_baseline"] = {"value": len(t["sample_step_s"]) / sum(t["sample_step_s"]), "unit": UNIT,
                                    "cores": threads, "kind": "port", "cpu": t["cpu"],
                                    "sample": t["sample"] + "; mean of 3 samples after 1 warm-up, in a process "
                                              "without torch"}
        except Exception as exc:
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "error": str(exc)[:200]}
    # the batched and served workloads are one-GPU measurements beside the headline
    if world == 1 and (args.batched or args.served or args.configs):
        del v
        ctx.close()
        model.close()
        torch.cuda.empty_cache()
        if args.batched:
            line["batched"] = {"tpq": batched_tpq(dev, args), "dsf": batched_dsf(dev, args),
                               "by_size": batch_table(dev, args)}
        if args.configs:
            line["configs"] = configs_section(dev, args)
        if args.served:
            line["served"] = served_section(args, local_rank, args.served_requests, args.served_rate)
    if rank == 0:
        print(json.dumps(line), flush=True)


def _kh(gamma=0.0):
    from pned_b200 import couplings as CP
    return CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi), gamma=gamma)


def _timed_session(ctx, st, kind, v, warm, steps, L=0.0):
    """Times `steps` session steps on the context's stream `st` (CUDA events)."""
    import torch
    ctx.session_begin(kind, v, warm + steps + 1, L=L)
    if warm > 0:
        ctx.session_step(warm)
    ctx.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    ctx.session_step(steps)
    e1.record(st)
    torch.cuda.synchronize()
    res = ctx.session_read()
    ctx.session_end()
    return e0.elapsed_time(e1) / steps, res


def batched_tpq(dev, args):
    """mTPQ with R = 16 vectors, S=1/2 N=24 honeycomb (3x4), KH + Gamma 0.1 + h 0.05 [111], l = 2:
    batched steps against the same vectors advanced one at a time."""
    import torch
    import pned_b200 as P
    from pned_b200 import couplings as CP
    from pned_b200.lattice import cluster_for_sites
    from pned_b200.tune import autotune
    cl = cluster_for_sites(24)
    L = 2.0 * cl.n
    m = P.Model.from_couplings(cl, _kh(0.1), field=CP.field_111(0.05), tps_L=L)
    out = {"workload": "mTPQ R=16, S=1/2 KH+Gamma=0.1+h=0.05[111] honeycomb N=24 (3x4), D=2^24, l=2.0 (L=48), "
                       "complex128, interleaved [2^24][16]", "steps_timed": args.batch_steps}
    for R in (16, 1):
        autotune(m, R)
        st = torch.cuda.Stream(device=dev)
        ctx = P.Context(m, R=R, stream=st)
        v = torch.empty(m.dim * R, dtype=torch.complex128, device=dev)
        ctx.fill_gaussian(SEED, v)
        ms, res = _timed_session(ctx, st, "tps", v, 3, args.batch_steps, L=L)
        if R == 16:
            out.update(ms_per_step=ms, steps_per_s=1000.0 / ms, vector_steps_per_s=16000.0 / ms,
                       plan=m.plan(16))
            # E(T) of the first step, averaged over R (coefficient 3 of eval_phys_val: L - alpha1)
            out["energy_first_step_mean"] = float(res["coef"][0, :, 3].mean())
        else:
            out.update(plain_ms_per_vector_step=ms, plain_vector_steps_per_s=1000.0 / ms)
        ctx.close()
        del v
        torch.cuda.empty_cache()
    out["vs_plain"] = out["vector_steps_per_s"] / out["plain_vector_steps_per_s"]
    m.close()
    return out


def batch_table(dev, args, sizes=(18, 20, 22, 24, 26), widths=(1, 4, 16), steps=None):
    """mTPQ steps (KH + Gamma 0.1 + h 0.05 [111], l = 2) per lattice size N and
    batch width R: vector-steps/s of R interleaved vectors in one session
    against R = 1 (the plain path, one vector at a time)."""
    import torch
    import pned_b200 as P
    from pned_b200 import couplings as CP
    from pned_b200.lattice import cluster_for_sites
    from pned_b200.tune import autotune
    rows = []
    for n in sizes:
        cl = cluster_for_sites(n)
        L = 2.0 * cl.n
        m = P.Model.from_couplings(cl, _kh(0.1), field=CP.field_111(0.05), tps_L=L)
        plain = None
        for R in widths:
            autotune(m, R)
            st = torch.cuda.Stream(device=dev)
            ctx = P.Context(m, R=R, stream=st)
            v = torch.empty(m.dim * R, dtype=torch.complex128, device=dev)
            ctx.fill_gaussian(SEED, v)
            k = steps or max(10, min(200, int(2 ** 26 / (m.dim * R)) * 4))
            ms, _ = _timed_session(ctx, st, "tps", v, 3, k, L=L)
            vps = 1000.0 * R / ms
            if R == 1:
                plain = vps
            rows.append({"n_sites": n, "R": R, "ms_per_step": ms, "vector_steps_per_s": vps,
                         "vs_plain": vps / plain if plain else None, "steps_timed": k, "plan": m.plan(R)})
            ctx.close()
            del v
            torch.cuda.empty_cache()
        m.close()
    return {"workload": "mTPQ steps, S=1/2 KH+Gamma=0.1+h=0.05[111] honeycomb, l=2.0, complex128, R interleaved "
                        "vectors [D][R] in one session; R=1 is the plain path", "rows": rows}


def configs_section(dev, args):
    """The other configurations as they are stated: config 0 (N=24 Lanczos, 300
    steps, E0 and the eigenvector's residual), config 1 (N=24 mTPQ, R=16, 2000
    steps, E(T) and C(T) of eval_mpi over the 16 seeds) and config 3 (S=1 N=18:
    a 300-step Lanczos E0 and mTPQ with R=4; of its 1500 steps a bounded number
    is timed, the rest projected)."""
    import numpy as np
    import torch
    import pned_b200 as P
    from pned_b200 import couplings as CP
    from pned_b200.lattice import cluster_for_sites
    from pned_b200.tune import autotune
    out = {}
    # config 0
    cl = cluster_for_sites(24)
    m = P.Model.from_couplings(cl, _kh())
    autotune(m, 1)
    st = torch.cuda.Stream(device=dev)
    ctx = P.Context(m, R=1, stream=st)
    v = torch.empty(m.dim, dtype=torch.complex128, device=dev)
    ctx.fill_gaussian(SEED, v)
    ms, res = _timed_session(ctx, st, "lanczos", v, 0, 300)
    a, b = res["alpha"][:, 0], res["beta"][:, 0]
    E = P.bisec(a, b, 300, 1)
    c = P.vec12(a, b, E, 300, 1)[0]
    t0 = time.perf_counter()
    x = ctx.lanczos_vector(v, a, b, c)
    t_vec = time.perf_counter() - t0
    hx = torch.zeros_like(x)
    ctx.p_mltply_v3(x, hx)
    out["config0"] = {"workload": "Lanczos ground state, S=1/2 KH honeycomb N=24 (3x4), D=2^24, complex128, "
                                  "300 steps from the seeded Gaussian",
                      "steps": 300, "ms_per_step": ms, "e0": float(E[0]),
                      "residual": float(torch.linalg.vector_norm(hx - float(E[0]) * x).item()),
                      "eigenvector_pass_s": t_vec}
    ctx.close()
    m.close()
    del v, x, hx
    torch.cuda.empty_cache()
    # config 1
    L = 2.0 * cl.n
    R = 16
    m = P.Model.from_couplings(cl, _kh(0.1), field=CP.field_111(0.05), tps_L=L)
    autotune(m, R)
    ctx = P.Context(m, R=R, stream=st)
    v = torch.empty(m.dim * R, dtype=torch.complex128, device=dev)
    ctx.fill_gaussian(SEED, v)
    ms, res = _timed_session(ctx, st, "tps", v, 0, args.cfg1_steps, L=L)
    beta = res["beta"].T
    energy = res["coef"][:, :, 3].T
    hmix = res["coef"][:, :, 4].T
    th = P.api.tpq_thermo(beta, energy, hmix, 0.05, 10.0, 12)
    out["config1"] = {"workload": "mTPQ R=16, S=1/2 KH+Gamma=0.1+h=0.05[111] honeycomb N=24, l=2.0 (L=48), "
                                  f"{args.cfg1_steps} steps, E(T) and C(T) of eval_mpi averaged over the 16 seeds",
                      "steps": args.cfg1_steps, "ms_per_step": ms, "run_s": ms * args.cfg1_steps / 1000.0,
                      "T": th[:, 0].tolist(), "E": th[:, 1].tolist(), "C": th[:, 2].tolist()}
    ctx.close()
    m.close()
    del v
    torch.cuda.empty_cache()
    # config 3
    cl = cluster_for_sites(18)
    cpl = CP.kitaev_heisenberg(0.2, -1.0)
    L3 = 3.0 * cl.n
    m = P.Model.from_couplings(cl, cpl, q=3, tree=1)
    ctx = P.Context(m, R=1, stream=st)
    v = torch.empty(m.dim, dtype=torch.complex128, device=dev)
    ctx.fill_gaussian(SEED, v)
    ms_l, res = _timed_session(ctx, st, "lanczos", v, 0, 300)
    a, b = res["alpha"][:, 0], res["beta"][:, 0]
    e0 = float(P.bisec(a, b, 300, 1)[0])
    ctx.close()
    m.close()
    del v
    torch.cuda.empty_cache()
    m = P.Model.from_couplings(cl, cpl, q=3, tree=1, tps_L=L3)
    ctx = P.Context(m, R=4, stream=st)
    v = torch.empty(m.dim * 4, dtype=torch.complex128, device=dev)
    ctx.fill_gaussian(SEED, v)
    ms_t, res = _timed_session(ctx, st, "tps", v, 3, args.cfg3_tpq_steps, L=L3)
    out["config3"] = {"workload": "S=1 KH honeycomb N=18 (3x3), K=-1, J=0.2, D=3^18, complex128: 300-step Lanczos "
                                  "E0 and mTPQ R=4, l=3.0 (L=54)",
                      "lanczos": {"steps": 300, "ms_per_step": ms_l, "e0": e0},
                      "tpq": {"steps_timed": args.cfg3_tpq_steps, "ms_per_step": ms_t,
                              "projected_1500_steps_s": ms_t * 1.5,
                              "vector_steps_per_s": 4000.0 / ms_t}}
    ctx.close()
    m.close()
    del v
    torch.cuda.empty_cache()
    return out


def batched_dsf(dev, args):
    """DSF: ground state of the N=24 KH cluster, S^z_q at all 12 momenta, 150-step
    chains for the 12 q in one batched run against one momentum at a time."""
    import numpy as np
    import torch
    import pned_b200 as P
    from pned_b200.lattice import cluster_for_sites
    from pned_b200.tune import autotune
    cl = cluster_for_sites(24)
    m = P.Model.from_couplings(cl, _kh())
    ctx1 = P.Context(m, R=1)
    v = torch.empty(m.dim, dtype=torch.complex128, device=dev)
    ctx1.fill_gaussian(SEED, v)
    gs_steps = 120
    r = ctx1.lanczos(v, gs_steps)
    a, b = r["alpha"][:, 0], r["beta"][:, 0]
    E = P.bisec(a, b, gs_steps, 1)
    c = P.vec12(a, b, E, gs_steps, 1)[0]
    x = ctx1.lanczos_vector(v, a, b, c)
    nq = len(cl.q_list)
    qrs = np.stack([cl.qr(i) for i in range(nq)])
    steps = 150
    out = {"workload": f"DSF S^z_q chains, {nq} momenta of the N=24 KH honeycomb (3x4), 150 steps each, "
                       "from the Lanczos ground state; S(q,w) on 2000 w in [0,3], eta=0.05",
           "e0": float(E[0]), "momenta": nq}
    autotune(m, nq)
    ctxq = P.Context(m, R=nq)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    d = ctxq.dsf(x, qrs, steps)
    t1 = time.perf_counter()
    out.update(batched_s=t1 - t0, chains_per_s=nq / (t1 - t0), plan=m.plan(nq))
    sp = [P.exec_renbun(2000, steps + 2, 3.0 / 1999, float(E[0]), 0.05, d["salpha"][:, i], d["sbeta"][:, i])[2]
          for i in range(nq)]
    out["spectral_weight_q0"] = float(np.sum(sp[0]) * 3.0 / 1999)
    ctxq.close()
    t0 = time.perf_counter()
    d1 = ctx1.dsf(x, qrs[:1], steps)
    t1 = time.perf_counter()
    out.update(plain_chain_s=t1 - t0, plain_chains_per_s=1.0 / (t1 - t0))
    out["vs_plain"] = out["chains_per_s"] / out["plain_chains_per_s"]
    out["max_rel_diff_alpha_q0"] = float(np.max(np.abs(d1["salpha"][:12, 0] - d["salpha"][:12, 0]) /
                                                np.abs(d["salpha"][:12, 0])))
    ctx1.close()
    m.close()
    del x, v
    torch.cuda.empty_cache()
    return out


def run_sector(args, rank, world, local_rank):
    """--workload sector: pure Heisenberg (J = 1) on the N-site honeycomb in the
    Sz = 0 sector (parity_type 0: mk_list12 order, Lin-table partner lookup),
    one Lanczos chain: K timed steps after W warm-up steps."""
    import math
    import torch
    import pned_b200 as P
    from pned_b200 import couplings as CP
    from pned_b200.lattice import cluster_for_sites
    if rank != 0:
        return
    torch.cuda.set_device(local_rank)
    P.lib().pned_set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = args.sector_sites
    cl = cluster_for_sites(n)
    with ClockSampler(local_rank) as clk:
        m = P.Model.from_couplings(cl, CP.kitaev_heisenberg(1.0, 0.0))
        D = m.dim
        st = torch.cuda.Stream(device=dev)
        ctx = P.Context(m, R=1, stream=st)
        v = torch.empty(D, dtype=torch.complex128, device=dev)
        ctx.fill_gaussian(SEED, v)
        ctx.session_begin("lanczos", v, args.warmup + args.steps + args.profile_steps + 1)
        ctx.session_step(args.warmup)
        ctx.synchronize()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        ctx.session_step(args.steps)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        hv_ms, step_ms = ctx.session_profile(args.profile_steps)
        res = ctx.session_read()
        ctx.session_end()
        # the segment kernel against the flat gather on one vector: W bit for bit, H.v time
        seg = {"active": m.sector_segments()}
        if seg["active"]:
            x = torch.empty(D, dtype=torch.complex128, device=dev)
            ctx.fill_gaussian(SEED + 1, x)
            ws = {}
            for on in (True, False):
                m.sector_segments(on)
                w = torch.zeros_like(x)
                ctx.p_mltply_v3(x, w)
                ctx.synchronize()
                ws[on] = w.clone()
                t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                t0.record(st)
                for _ in range(3):
                    ctx.p_mltply_v3(x, w)
                t1.record(st)
                torch.cuda.synchronize()
                seg["hv_ms" if on else "flat_hv_ms"] = t0.elapsed_time(t1) / 3
            m.sector_segments(True)
            seg["w_bit_identical"] = bool(torch.equal(ws[True], ws[False]))
            del x, w, ws
        ctx.close()
        m.close()
    peak, peak_kind = load_peaks()
    kernel = "hv_sector_kernel (segments, K=1)" if seg["active"] else "hv_xor_kernel (sector, K=1)"
    # per sector state: C 16 + P 16 + W 16 + real diagonal 8 = 56 B (as the full basis), plus the
    # state list entry (8 B); the Lin tables (2 x 2^ceil(n/2) entries) stay in L2
    bytes_hv = 64 * D
    line = {
        "metric": f"sector_lanczos_steps_per_s_N{n}", "value": 1000.0 / ms, "unit": "steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded complex Gaussian start vector)",
        "config": {"workload": f"S=1/2 Heisenberg (J=1) honeycomb N={n} ({cl.L1}x{cl.L2}), Sz=0 sector "
                               f"D={D} (mk_list12 order), complex128, 1 Lanczos chain", "dim": D, "R": 1},
        "e0_per_site": float(P.bisec(res["alpha"][:, 0], res["beta"][:, 0], res["alpha"].shape[0], 1)[0]) / n,
        "roofline": {"bound": "hbm", "kernel": kernel, "achieved": bytes_hv / (hv_ms * 1e-3) / 1e9,
                     "peak": peak, "unit": "GB/s", "frac": bytes_hv / (hv_ms * 1e-3) / 1e9 / peak,
                     "peak_kind": peak_kind, "hv_ms": hv_ms, "algorithmic_bytes_per_hv": bytes_hv},
        "segments": seg,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def run_s1(args, rank, world, local_rank):
    """--workload s1: S=1 Kitaev-Heisenberg (mixed radix, base 3) on the 18-site honeycomb
    (3x3), K=-1, J=0.2, D=3^18: batched mTPQ with R=4 vectors (l=3.0, L=54) and a
    Lanczos E0 run; K timed steps of each after W warm-up steps."""
    import torch
    import pned_b200 as P
    from pned_b200 import couplings as CP
    from pned_b200.lattice import cluster_for_sites
    if rank != 0:
        return
    torch.cuda.set_device(local_rank)
    P.lib().pned_set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    cl = cluster_for_sites(args.s1_sites)
    cpl = CP.kitaev_heisenberg(0.2, -1.0)
    L = 3.0 * cl.n
    R = args.s1_vectors
    out = {}
    with ClockSampler(local_rank) as clk:
        m = P.Model.from_couplings(cl, cpl, q=3, tree=1, tps_L=L)
        st = torch.cuda.Stream(device=dev)
        ctx = P.Context(m, R=R, stream=st)
        v = torch.empty(m.dim * R, dtype=torch.complex128, device=dev)
        ctx.fill_gaussian(SEED, v)
        ms_tpq, res = _timed_session(ctx, st, "tps", v, args.warmup, args.steps, L=L)
        out["tpq"] = {"ms_per_step": ms_tpq, "steps_per_s": 1000.0 / ms_tpq,
                      "vector_steps_per_s": R * 1000.0 / ms_tpq,
                      "energy_first_step_mean": float(res["coef"][0, :, 3].mean())}
        ctx.close()
        m.close()
        del v
        torch.cuda.empty_cache()
        m = P.Model.from_couplings(cl, cpl, q=3, tree=1)
        ctx = P.Context(m, R=1, stream=st)
        v = torch.empty(m.dim, dtype=torch.complex128, device=dev)
        ctx.fill_gaussian(SEED, v)
        ms_l, res = _timed_session(ctx, st, "lanczos", v, args.warmup, args.steps)
        a, b = res["alpha"][:, 0], res["beta"][:, 0]
        out["lanczos"] = {"ms_per_step": ms_l, "steps_per_s": 1000.0 / ms_l,
                          "e0_after_steps": float(P.bisec(a, b, len(a), 1)[0])}
        D = m.dim
        ctx.close()
        m.close()
    line = {
        "metric": f"s1_tpq_steps_per_s_N{cl.n}", "value": out["tpq"]["steps_per_s"], "unit": "steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": out["tpq"]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (seeded complex Gaussian start vectors)",
        "config": {"workload": f"S=1 KH honeycomb N={cl.n}, K=-1, J=0.2, base-3 basis D=3^{cl.n}, complex128; "
                               f"mTPQ R={R}, l=3.0 (L={L:g}), and a Lanczos E0 chain", "dim": D, "R": R},
        "tpq": out["tpq"], "lanczos": out["lanczos"],
        "roofline": {"bound": "hbm", "kernel": "hv_radix_kernel",
                     "achieved": 56 * D * R / (out["tpq"]["ms_per_step"] * 1e-3) / 1e9,
                     "unit": "GB/s", "note": "whole TPS step over 56 B per state and vector"},
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def served_section(args, local_rank, n_requests, rate, sweep=()):
    """Serving stream (continuous batching) against the plain one-at-a-time path:
    capacity (all requests queued at once), p50/p99 latency at `rate` (and at
    each rate of `sweep`: the same requests with arrival times rescaled), and the
    same requests run alone through the plain path.  rate None: a load the
    server sustains, LOAD_FRACTION of the capacity just measured (above the
    capacity the queue grows with the length of the stream and so does every
    latency figure)."""
    import torch
    from pned_b200 import serve
    auto_rate = rate is None
    reqs = serve.make_stream(n_requests, rate=1.0 if auto_rate else rate, seed=SEED, p30=args.p30,
                             min_n30=args.min_n30)
    free, _ = torch.cuda.mem_get_info()
    budget = int(0.85 * free)
    cap_reqs = [serve.Request(**{**q.__dict__, "arrival": 0.0}) for q in reqs]
    srv = serve.Server(budget=budget, max_steps=512)
    # plans tuned ahead, as a server and a plain caller do once per lattice size:
    # the lanes of each size, and the plain path's plans for each (size, vectors)
    t_warm = time.perf_counter()
    srv.warm({q.n for q in reqs})
    serve.warm_plain(reqs)
    t_warm = time.perf_counter() - t_warm
    swept = []
    with ClockSampler(local_rank) as clk:
        cap = srv.run(cap_reqs, realtime=True)
        if auto_rate:   # the stream was drawn at 1 request/s: rescale its arrival times
            rate = LOAD_FRACTION * len(cap.results) / cap.makespan_s
            reqs = [serve.Request(**{**q.__dict__, "arrival": q.arrival / rate}) for q in reqs]
        st = srv.run(reqs, realtime=True)
        for r in sweep:
            reqs_r = [serve.Request(**{**q.__dict__, "arrival": q.arrival * rate / r}) for q in reqs]
            sr = serve.summarize(srv.run(reqs_r, realtime=True), reqs_r)
            swept.append({"rate_per_s": r, "solves_per_s": sr["solves_per_s"], "p50_s": sr["p50_latency_s"],
                          "p99_s": sr["p99_latency_s"], "makespan_s": sr["makespan_s"]})
    srv.close()
    torch.cuda.empty_cache()
    capacity = len(cap.results) / cap.makespan_s
    s = serve.summarize(st, reqs)
    by = {r["rid"]: r for r in cap.results}
    k = min(len(reqs), args.plain_sample)
    tp, diffs = 0.0, []
    for q in reqs[:k]:
        t0 = time.perf_counter()
        p = serve.run_plain(q)
        tp += time.perf_counter() - t0
        if "e0" in p:
            diffs.append(abs(by[q.rid]["e0"] - p["e0"]) / abs(p["e0"]))
    plain = k / tp
    return {
        "workload": "Poisson stream of Lanczos E0 (300 steps), mTPQ (R=4, 500 steps), DSF (4 momenta, 100 steps) "
                    "requests, S=1/2 honeycomb N uniform in {18..26} + p30 at N=30, random phi, Gamma, h[111]; "
                    "HBM-budget admission, co-batching by N",
        "requests": len(reqs), "of_config_requests": 2000,
        "sample_note": f"{len(reqs)} of the configuration's 2000 requests (same mix and arrival law); at least "
                       f"{args.min_n30} at N=30 in the sample",
        "kinds": {kd: sum(1 for q in reqs if q.kind == kd) for kd in ("lanczos", "tpq", "dsf")},
        "sizes": {str(n): sum(1 for q in reqs if q.n == n) for n in sorted({q.n for q in reqs})},
        "hbm_budget_bytes": budget, "tuning_before_timing_s": t_warm,
        "solves_per_s": capacity,
        "capacity": {"makespan_s": cap.makespan_s, "lanes_created": cap.lanes_created,
                     "slot_occupancy": cap.occupied_slot_steps / max(1, cap.slot_steps), "peak_bytes": cap.peak_bytes,
                     "note": "all requests queued at t=0"},
        "latency": {"rate_per_s": rate, "solves_per_s": s["solves_per_s"], "p50_s": s["p50_latency_s"],
                    "p99_s": s["p99_latency_s"], "makespan_s": s["makespan_s"],
                    **({"rate_rule": f"{LOAD_FRACTION} x the measured capacity"} if auto_rate else {})},
        **({"latency_sweep": swept} if swept else {}),
        "plain": {"solves_per_s": plain, "sample": k, "mean_s": tp / k,
                  "max_rel_e0_diff_served_vs_plain": max(diffs) if diffs else None},
        "vs_plain": capacity / plain,
        "clocks": clk.summary(),
    }


def run_serve(args, rank, world, local_rank):
    """--workload serve: the serving stream as its own JSON line."""
    import torch
    import pned_b200 as P
    if rank != 0:
        return
    torch.cuda.set_device(local_rank)
    P.lib().pned_set_device(local_rank)
    sweep = [float(x) for x in args.rates.split(",")] if args.rates else []
    sv = served_section(args, local_rank, args.requests, args.rate, sweep)
    line = {
        "metric": "served_solves_per_s", "value": sv["solves_per_s"], "unit": "solves/s", "n_gpus": 1,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic request stream (seeded)",
        "config": {"workload": sv["workload"], "requests": sv["requests"], "rate_per_s": args.rate,
                   "p30": args.p30, "kinds": sv["kinds"], "sizes": sv["sizes"]},
        "p50_latency_s": sv["latency"]["p50_s"], "p99_latency_s": sv["latency"]["p99_s"],
        "served": sv, "vs_plain": sv["vs_plain"], "clocks": sv["clocks"],
        "e2e": {"value": sv["solves_per_s"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "note": "requests enter and results leave through host memory; start vectors are generated on "
                        "the device from each request's seed"},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n-sites", type=int, default=30)
    ap.add_argument("--profile-steps", type=int, default=3)
    ap.add_argument("--ref-slice-log2", type=int, default=24)
    ap.add_argument("--ref-full-steps", type=int, default=1, help="--impl reference: whole steps timed")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--traffic", type=float, default=None, help="DRAM bytes per H.v launch from an ncu capture")
    ap.add_argument("--workload", default="lanczos", choices=["lanczos", "serve", "s1", "sector", "batch", "configs"])
    ap.add_argument("--sector-sites", type=int, default=30)
    ap.add_argument("--no-tune", dest="tune", action="store_false")
    ap.add_argument("--plan", default=None, help="fixed tile plan 'row_fixed_bits,window_bits,max_passes,j_bits[,l1_carveout[,stage]]' "
                                                 "instead of autotuning (profiling runs)")
    ap.add_argument("--no-batched", dest="batched", action="store_false")
    ap.add_argument("--batch-steps", type=int, default=40)
    ap.add_argument("--requests", type=int, default=200)
    ap.add_argument("--rate", type=float, default=4.0)
    ap.add_argument("--rates", default=None, help="serve workload: further arrival rates, comma-separated "
                                                  "(the same requests, arrival times rescaled)")
    ap.add_argument("--p30", type=float, default=0.02)
    ap.add_argument("--min-n30", type=int, default=1, help="served sample: at least this many N=30 requests")
    ap.add_argument("--no-configs", dest="configs", action="store_false")
    ap.add_argument("--cfg1-steps", type=int, default=2000)
    ap.add_argument("--cfg3-tpq-steps", type=int, default=30)
    ap.add_argument("--plain-sample", type=int, default=200)
    ap.add_argument("--no-served", dest="served", action="store_false")
    ap.add_argument("--no-dense-check", dest="dense_check", action="store_false")
    ap.add_argument("--s1-sites", type=int, default=18)
    ap.add_argument("--s1-vectors", type=int, default=4)
    ap.add_argument("--served-requests", type=int, default=40)
    ap.add_argument("--served-rate", type=float, default=None,
                    help="arrival rate of the served section's latency run (default: 0.7 x its measured capacity)")
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
        elif args.workload == "serve":
            run_serve(args, rank, world, local_rank)
        elif args.workload == "s1":
            run_s1(args, rank, world, local_rank)
        elif args.workload == "sector":
            run_sector(args, rank, world, local_rank)
        elif args.workload == "configs":
            if rank == 0:
                import torch
                torch.cuda.set_device(local_rank)
                print(json.dumps({"configs": configs_section(torch.device("cuda", local_rank), args)}), flush=True)
        elif args.workload == "batch":
            if rank == 0:
                import torch
                torch.cuda.set_device(local_rank)
                print(json.dumps({"batched": {"by_size": batch_table(torch.device("cuda", local_rank), args)}}),
                      flush=True)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
