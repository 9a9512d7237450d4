"""Generates tests/golden/configs.npz: oracle results at the sizes of the
benchmark configurations, where the oracle takes minutes per run and cannot
run inside a test.

    python -m tests.golden.make_config_golden      (from the repository root)

The oracle (oracle/pned_oracle.c, the restatement of the reference's lnp = 1
path) computes every value here; the start vectors are the seeded complex
Gaussians of oracle.gaussian, which the GPU tests upload unchanged, so both
sides start from the same bits.

  cfg0   S = 1/2 Kitaev-Heisenberg honeycomb N = 24 (3x4), J = cos 0.3pi,
         K = 2 sin 0.3pi, full basis 2^24: 300 Lanczos steps
         (parallelized_lnc1z, S_one_half/Hybrid_TPS_Lanczos.f90:97-157) from
         gaussian(20261203) normalised -- alpha, beta, the 8 lowest Ritz values
         (bisec) -- then the eigenvector pass (parallelized_lncv1z,
         Lanczos.f90:183-329) with the vec12 coefficients of E0 and the
         residual ||H x - E0 x||.
  cfg2   DSF chains (intalv_zz + parallelized_dsflnc1z, S_one_half/
         Hybrid_TPS_DSF.f90:18-87, 195-261) of 150 steps at two momenta of the
         same cluster, from x = gaussian(3) normalised, run twice with
         different OpenMP thread counts (8, 3 and 1: only the reduction order
         differs),
         once more from x perturbed at the rounding level (each element times
         1 + 1e-15 g, g seeded standard normal, then normalised), once with the
         oracle built with fused multiply-adds (oracle/Makefile: other rounding
         in every vector element, as an optimised build for a current host
         has), and once with each H.v's items summed in reverse order (as
         another MPI rank decomposition of the reference orders them): these
         runs give the spread of the reference algorithm itself, against which
         the GPU's chains and spectra are held.
  cfg1   mTPQ (parallelized_TPSz, S_one_half/Hybrid_TPS_TPS.f90:325-409) on the
         16-site cluster (2x4) with Gamma = 0.1 and h = 0.05 along [111],
         l = 2.0 (L = 32), R = 4 seeds of gaussian(5) normalised, 2000 steps:
         the norms, coef(:,4) (energy) and coef(:,5) (Re<k-1|H|k>) per seed.
"""
import math
import os
import sys
import time

import numpy as np

from oracle import oracle as O
from pned_b200 import couplings as CP
from pned_b200.lattice import honeycomb

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "configs.npz")

KH = CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi))
KHGH = CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi), gamma=0.1)
FIELD = CP.field_111(0.05)

CFG0_SEED = 20261203
CFG0_STEPS = 300
CFG2_SEED = 3
CFG2_STEPS = 150
CFG2_MOMENTA = (1, 5)
CFG2_THREADS = (8, 3)
CFG2_PERTURB = 1e-15
CFG1_SEED = 5
CFG1_R = 4
CFG1_STEPS = 2000


def oracle_model(cl, cpl, fld=None, tps_L=None):
    X = O.xlocal(2, 0, cpl, field=fld)
    skip, _, pt = O.parity_skip(2, 0, X)
    if tps_L is not None:
        X = O.tps_explicit(2, cl.nbond, tps_L, X)
    return O.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)


def log(msg):
    print(f"[{time.strftime('%H:%M:%S')}] {msg}", flush=True)


def cfg0(out):
    cl = honeycomb(3, 4)
    om = oracle_model(cl, KH)
    v = O.gaussian(CFG0_SEED, om.ldim)
    v /= np.linalg.norm(v)
    run = om.lanczos(v, CFG0_STEPS)
    log(f"cfg0 lanczos: E0 {run['ene'][0]!r}")
    al, be = run["alpha"], run["beta"]
    E = O.bisec(al, be, CFG0_STEPS, 1)
    c = O.vec12(al, be, E, CFG0_STEPS, 1)[0]
    x = om.lanczos_vector(v, al, be, c)
    hx = np.zeros_like(x)
    om.p_mltply_v3(x, hx)
    res = np.linalg.norm(hx - E[0] * x)
    log(f"cfg0 eigenvector: residual {res:.3e}")
    out["cfg0/alpha"] = al
    out["cfg0/beta"] = be
    out["cfg0/ene"] = run["ene"]
    out["cfg0/E_bisec"] = E
    out["cfg0/coef"] = c
    out["cfg0/residual"] = np.array([res])
    out["cfg0/x_energy"] = np.array([np.vdot(x, hx).real])


def cfg2(out):
    cl = honeycomb(3, 4)
    om = oracle_model(cl, KH)
    x = O.gaussian(CFG2_SEED, om.ldim)
    x /= np.linalg.norm(x)
    for th in CFG2_THREADS:
        O.set_num_threads(th)
        for iq in CFG2_MOMENTA:
            vq, cn = om.intalv_zz(cl.qr(iq), x)
            sa, sb = om.dsf_chain(vq, cn, CFG2_STEPS)
            out[f"cfg2/t{th}/q{iq}/cnorm"] = np.array([cn.real])
            out[f"cfg2/t{th}/q{iq}/salpha"] = sa
            out[f"cfg2/t{th}/q{iq}/sbeta"] = sb
            log(f"cfg2 threads {th} q{iq} done")
    O.set_num_threads(os.cpu_count() or 1)


def cfg2p(out):
    cl = honeycomb(3, 4)
    om = oracle_model(cl, KH)
    x = O.gaussian(CFG2_SEED, om.ldim)
    x /= np.linalg.norm(x)
    g = np.random.default_rng(CFG2_SEED).standard_normal(om.ldim)
    x = x * (1.0 + CFG2_PERTURB * g)
    x /= np.linalg.norm(x)
    O.set_num_threads(CFG2_THREADS[0])
    for iq in CFG2_MOMENTA:
        vq, cn = om.intalv_zz(cl.qr(iq), x)
        sa, sb = om.dsf_chain(vq, cn, CFG2_STEPS)
        out[f"cfg2/perturbed/q{iq}/salpha"] = sa
        out[f"cfg2/perturbed/q{iq}/sbeta"] = sb
        log(f"cfg2 perturbed q{iq} done")
    O.set_num_threads(os.cpu_count() or 1)


def _chains_in_subprocess(out, env_extra, key):
    """The chains of cfg2 (8 threads) from an oracle variant chosen by environment
    variables, in a process of its own (the variant is fixed when the oracle loads)."""
    import subprocess
    import tempfile
    cl = honeycomb(3, 4)
    X = O.xlocal(2, 0, KH)
    skip, _, pt = O.parity_skip(2, 0, X)
    x = O.gaussian(CFG2_SEED, 1 << cl.n)
    x /= np.linalg.norm(x)
    with tempfile.TemporaryDirectory() as td:
        src, dst = os.path.join(td, "in.npz"), os.path.join(td, "out.npz")
        np.savez(src, n=cl.n, q=2, tree=0, ipair=cl.ipair, ibond_type=cl.ibond_type, X=X, skip=skip,
                 parity_type=pt, x=x, qr=np.stack([cl.qr(iq) for iq in CFG2_MOMENTA]), steps=CFG2_STEPS,
                 threads=CFG2_THREADS[0])
        subprocess.run([sys.executable, "-m", "oracle.dsf_chains", src, dst], env=dict(os.environ, **env_extra),
                       check=True, cwd=os.path.dirname(os.path.dirname(HERE)))
        r = np.load(dst)
        for k, iq in enumerate(CFG2_MOMENTA):
            out[f"cfg2/{key}/q{iq}/salpha"] = r["salpha"][k]
            out[f"cfg2/{key}/q{iq}/sbeta"] = r["sbeta"][k]
    log(f"cfg2 {key} done")


def cfg2t1(out):
    """The chains of cfg2 with one OpenMP thread (sequential sums), one process per
    momentum, side by side."""
    import subprocess
    import tempfile
    cl = honeycomb(3, 4)
    X = O.xlocal(2, 0, KH)
    skip, _, pt = O.parity_skip(2, 0, X)
    x = O.gaussian(CFG2_SEED, 1 << cl.n)
    x /= np.linalg.norm(x)
    root = os.path.dirname(os.path.dirname(HERE))
    with tempfile.TemporaryDirectory() as td:
        procs = []
        for iq in CFG2_MOMENTA:
            src, dst = os.path.join(td, f"in{iq}.npz"), os.path.join(td, f"out{iq}.npz")
            np.savez(src, n=cl.n, q=2, tree=0, ipair=cl.ipair, ibond_type=cl.ibond_type, X=X, skip=skip,
                     parity_type=pt, x=x, qr=cl.qr(iq)[None, :], steps=CFG2_STEPS, threads=1)
            procs.append((iq, dst, subprocess.Popen([sys.executable, "-m", "oracle.dsf_chains", src, dst], cwd=root)))
        for iq, dst, pr in procs:
            if pr.wait() != 0:
                raise RuntimeError("oracle.dsf_chains failed")
            r = np.load(dst)
            out[f"cfg2/t1/q{iq}/salpha"] = r["salpha"][0]
            out[f"cfg2/t1/q{iq}/sbeta"] = r["sbeta"][0]
    log("cfg2 t1 done")


def cfg2fma(out):
    """The oracle built with fused multiply-adds (oracle/Makefile)."""
    _chains_in_subprocess(out, {"PNED_ORACLE_BUILD": "fma"}, "fma")


def cfg2rev(out):
    """The oracle summing each H.v's items in reverse order (as another rank
    decomposition of the reference orders them differently)."""
    _chains_in_subprocess(out, {"PNED_ORACLE_ITEM_ORDER": "reverse"}, "reverse")


def cfg1(out):
    cl = honeycomb(2, 4)
    L = 2.0 * cl.n
    om = oracle_model(cl, KHGH, FIELD, tps_L=L)
    V = O.gaussian(CFG1_SEED, om.ldim, CFG1_R).reshape(om.ldim, CFG1_R)
    V /= np.linalg.norm(V, axis=0)
    beta, energy, hmix = [], [], []
    for r in range(CFG1_R):
        run = om.tps(L, np.ascontiguousarray(V[:, r]), CFG1_STEPS)
        beta.append(run["beta"])
        energy.append(run["coef"][:, 3])
        hmix.append(run["coef"][:, 4])
    out["cfg1/beta"] = np.stack(beta)
    out["cfg1/energy"] = np.stack(energy)
    out["cfg1/hmix"] = np.stack(hmix)
    log("cfg1 done")


def main(parts):
    out = dict(np.load(OUT)) if os.path.exists(OUT) else {}
    O.set_num_threads(os.cpu_count() or 1)
    for name in parts:
        {"cfg0": cfg0, "cfg1": cfg1, "cfg2": cfg2, "cfg2p": cfg2p, "cfg2fma": cfg2fma, "cfg2rev": cfg2rev,
         "cfg2t1": cfg2t1}[name](out)
        np.savez_compressed(OUT, **out)


if __name__ == "__main__":
    main(sys.argv[1:] or ["cfg1", "cfg0", "cfg2", "cfg2p", "cfg2fma", "cfg2rev", "cfg2t1"])
