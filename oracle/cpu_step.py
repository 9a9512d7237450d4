"""CPU timing of the reference's Lanczos step on the headline workload, with the
oracle (the restatement of the reference's lnp = 1 path in oracle/pned_oracle.c)
as the thing timed.  Test and measurement infrastructure: bench.py runs it as a
separate process, so that no other OpenMP runtime (torch ships its own) spins
on the same host cores while the oracle's threads run.

    python -m oracle.cpu_step --n-sites 30 --threads 16 --samples 3 --warmup 1 --full 1

A step is parallelized_lnc1z's loop body (S_one_half/Hybrid_TPS_Lanczos.f90:
111-122): the swap of v1/v0 with the previous alpha and beta, p_mltply_v3 (all
bond x element passes, S_one_half/Hybrid_TPS_parallel.f90:190-263) and
calc_beta (:161-188).  Two measurements:

  samples  the step restricted to the output states [0, 2^slice_log2) --
           swap and calc_beta on that slice, p_mltply_v3 on it gathering from
           the full-size v1 -- each timed and scaled by 2^n / 2^slice_log2;
  full     whole steps over all 2^n states (34 GB of host vectors at N = 30),
           timed as they are.

Prints one JSON line with both, the thread count, and the host's CPU model.
"""
import argparse
import json
import math
import os
import platform
import time

import numpy as np

from oracle import oracle as O
from pned_b200 import couplings as CP
from pned_b200.lattice import cluster_for_sites

SEED = 20261203


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-sites", type=int, default=30)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--samples", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--slice-log2", type=int, default=24)
    ap.add_argument("--full", type=int, default=0, help="whole steps to time after the samples")
    args = ap.parse_args()
    O.set_num_threads(args.threads)
    cl = cluster_for_sites(args.n_sites)
    cpl = CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi))
    X = O.xlocal(2, 0, cpl)
    skip, _, pt = O.parity_skip(2, 0, X)
    om = O.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    D = om.ldim
    t0 = time.perf_counter()
    v1 = O.gaussian(SEED, D)
    v1 /= np.linalg.norm(v1)
    setup_s = time.perf_counter() - t0
    hi = 1 << min(args.slice_log2, args.n_sites)
    scale = D / hi
    # with alpha = 0, beta = 1 and v0 = v1 the first swap keeps v1 (and sets v0 = -v1)
    v0s = v1[:hi].copy()
    a, b = 0.0, 1.0
    samples = []
    for i in range(args.warmup + args.samples):
        t0 = time.perf_counter()
        a, b = om.lanczos_step_slice(v1, v0s, 0, hi, a, max(b, 1e-3))
        dt = (time.perf_counter() - t0) * scale
        if i >= args.warmup:
            samples.append(dt)
    full = []
    if args.full > 0:
        del v0s
        v1 /= np.linalg.norm(v1)
        v0 = v1.copy()
        a, b = 0.0, 1.0
        for _ in range(args.full):
            t0 = time.perf_counter()
            a, b = om.lanczos_step(v1, v0, a, max(b, 1e-3))
            full.append(time.perf_counter() - t0)
    print(json.dumps({
        "n_sites": args.n_sites, "dim": D, "threads": args.threads, "cpu": cpu_model(), "nproc": os.cpu_count(),
        "slice_log2": int(math.log2(hi)), "sample_scale": scale, "sample_step_s": samples, "full_step_s": full,
        "setup_s": setup_s,
        "sample": (f"one Lanczos step (swap, p_mltply_v3 over all {om.nbond * 4} bond x element passes, calc_beta) "
                   f"on 2^{int(math.log2(hi))} of the 2^{args.n_sites} output states, full-size input vector, time "
                   f"scaled x{int(scale)}"),
    }), flush=True)


if __name__ == "__main__":
    main()
