"""Comparison of Lanczos-type chains (DSF continued-fraction coefficients) with
the oracle, at the level the reference algorithm itself reproduces them.

Past a few dozen steps a Lanczos chain in finite precision is chaotic: its late
coefficients depend on the rounding of every step.  The reference's own results
move with its reduction order (OpenMP thread count, MPI ranks), its compiler's
rounding and the order in which p_mltply_v3 sums its items.  So a GPU chain is
compared with the oracle's in two parts: its coefficients over the prefix where
all oracle variants agree with one another within 1e-10, and its spectrum
S(q, w); each within 1e-10 or, where larger, ten times the largest spread among
the oracle variants over the same part.  The variants: another OpenMP thread count (1), the
start vector perturbed at the rounding level, the oracle built with fused
multiply-adds (PNED_ORACLE_BUILD=fma) and each H.v's items summed in reverse
order (PNED_ORACLE_ITEM_ORDER=reverse); the last two run as separate processes
(oracle/dsf_chains.py).
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

import pned_b200 as P
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def spread_bound(spread):
    """The stated 1e-10, or ten times the oracle's own run-to-run spread where larger."""
    return max(1e-10, 10.0 * spread)


def stable_prefix(a, b, tol=1e-10):
    """Length of the longest prefix over which two chains agree within tol
    (relative 2-norm of the prefix)."""
    k = 0
    for i in range(1, len(a) + 1):
        if rel(a[:i], b[:i]) <= tol:
            k = i
        else:
            break
    return k


def spectra(sa, sb, e0, steps, i_range=2000, w_max=3.0, eta=0.05, lib=P):
    """S(q, w) of exec_renbun on i_range points in [0, w_max]."""
    return lib.exec_renbun(i_range, steps + 2, w_max / (i_range - 1), e0, eta, sa, sb)[2]


def check_chain(got_a, got_b, ref, others, e0, steps, min_prefix=10, **spec):
    """GPU chain (salpha, sbeta) against the oracle's (ref), with the oracle's
    variant runs (others) as the measure of its spread; returns (prefix, spread)."""
    sa, sb = ref
    k = min(stable_prefix(sa, o[0]) for o in others)
    assert k >= min_prefix, k
    # over the prefix: 1e-10, or ten times the variants' own spread there where larger
    sp_a = max(rel(o[0][:k], sa[:k]) for o in others)
    sp_b = max(rel(o[1][:k], sb[:k]) for o in others)
    assert rel(got_a[:k], sa[:k]) <= spread_bound(sp_a), (k, rel(got_a[:k], sa[:k]), sp_a)
    assert rel(got_b[:k], sb[:k]) <= spread_bound(sp_b), (k, rel(got_b[:k], sb[:k]), sp_b)
    d_ref = spectra(sa, sb, e0, steps, lib=O, **spec)
    spread = max(rel(spectra(o[0], o[1], e0, steps, lib=O, **spec), d_ref) for o in others)
    d_gpu = spectra(got_a, got_b, e0, steps, **spec)
    assert rel(d_gpu, d_ref) <= spread_bound(spread), (rel(d_gpu, d_ref), spread)
    return k, spread


def perturbed(x, seed, eps):
    """x with each element times 1 + eps g (g seeded standard normal), normalised."""
    g = np.random.default_rng(seed).standard_normal(x.shape[0])
    y = x * (1.0 + eps * g)
    return y / np.linalg.norm(y)


def variant_oracle_chains(cl, X, skip, pt, x, qrs, steps, threads, env):
    """DSF chains (intalv_zz + parallelized_dsflnc1z) of an oracle variant chosen by
    environment variables, in a process of its own; [(salpha, sbeta)] per momentum."""
    with tempfile.TemporaryDirectory() as td:
        src, dst = os.path.join(td, "in.npz"), os.path.join(td, "out.npz")
        np.savez(src, n=cl.n, q=2, tree=0, ipair=cl.ipair, ibond_type=cl.ibond_type, X=X, skip=skip,
                 parity_type=pt, x=np.asarray(x), qr=np.asarray(qrs), steps=steps, threads=threads)
        subprocess.run([sys.executable, "-m", "oracle.dsf_chains", src, dst], check=True, cwd=ROOT,
                       env=dict(os.environ, **env))
        r = np.load(dst)
        return [(r["salpha"][k], r["sbeta"][k]) for k in range(len(qrs))]


def oracle_chain_variants(cl, cpl, x, qrs, steps, fld=None):
    """The oracle's DSF chains for each momentum (all threads) and its variant runs:
    returns [(ref, [variants...])] per momentum."""
    X = O.xlocal(2, 0, cpl, field=fld)
    skip, _, pt = O.parity_skip(2, 0, X)
    om = O.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    nth = O.num_threads()
    xp = perturbed(np.asarray(x), 1, 1e-15)
    runs = []
    try:
        for th, xx in ((max(2, nth), x), (1, x), (max(2, nth), xp)):
            O.set_num_threads(th)
            runs.append([om.dsf_chain(*om.intalv_zz(qr, xx), steps) for qr in qrs])
    finally:
        O.set_num_threads(nth)
    for env in ({"PNED_ORACLE_BUILD": "fma"}, {"PNED_ORACLE_ITEM_ORDER": "reverse"}):
        runs.append(variant_oracle_chains(cl, X, skip, pt, x, qrs, steps, max(2, nth), env))
    return [(runs[0][r], [runs[k][r] for k in range(1, len(runs))]) for r in range(len(qrs))]
