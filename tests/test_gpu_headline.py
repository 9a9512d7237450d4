"""Parity of the tiled single-vector H.v at the headline sizes (N = 28, 30).

The measured workload is the S = 1/2 Kitaev-Heisenberg honeycomb at N = 30
(3x5, 45 bonds, D = 2^30, 17.2 GB per vector).  At that size the planner's
tiles keep a 12-bit L2 window and split the 45 flip masks over two passes,
structure that the 16- and 24-site clusters of the other parity tests never
reach.  Each plan the autotuner chooses between at these sizes (8- and 16-row
tiles, two or three resident blocks per SM, partner tiles streamed by the
bulk-copy engine, own rows brought in by tensor copies, tiles that hold the
most flip terms) and the plan it
actually picks run one H.v through the C ABI on device vectors; the oracle (p_mltply_v3 of the reference's lnp = 1 path,
S_one_half/Hybrid_TPS_parallel.f90:190-263, 415-440) gathers from the same
full input vector and computes three output slices of 2^20 states -- the
lowest, one in the middle and the highest.  Bound: relative 2-norm <= 1e-12 on
every slice.  The fused <v|Hv> is checked against an independent device
reduction of the returned vector (relative to the sum of |v||Hv|, since the
2^30 terms cancel).
"""
import math

import numpy as np
import pytest

import pned_b200 as P
from oracle import oracle as O
from pned_b200 import couplings as CP
from pned_b200.lattice import cluster_for_sites

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

KH = CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi))
SLICE = 1 << 20
EPERBD = 0.0625

# (row_fixed_bits, window_bits, max_passes, j_bits[, l1_carveout, stage_partner_tiles, blocks_per_sm,
#  objective, terms_in_flight]); objective 1 picks tiles that hold the most flip terms
PLANS = {
    30: [(5, 12, 2, 3), (5, 12, 2, 3, 1, 0, 3), (5, 11, 2, 4), (5, 10, 2, 3, 1, 2),
         (5, 10, 2, 3, 1, 0, -1, 1), (5, 10, 2, 4, 1, 0, -1, 1), (5, 8, 2, 3, 1, 3, -1, 1),
         (5, 8, 2, 3, 1, 3, -1, 1, 2)],
    28: [(5, 12, 2, 3), (5, 10, 2, 3, 1, 0, 3), (5, 11, 2, 4), (5, 10, 2, 3, 1, 2),
         (5, 10, 2, 3, 1, 0, -1, 1), (5, 9, 2, 4, 1, 0, -1, 1), (5, 8, 2, 3, 1, 3, -1, 1),
         (5, 8, 2, 3, 1, 3, -1, 1, 2)],
}


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("n_sites", [28, 30])
def test_headline_hv_slices_match_oracle(n_sites):
    from pned_b200 import tune
    cl = cluster_for_sites(n_sites)
    gm = P.Model.from_couplings(cl, KH)
    X = O.xlocal(2, 0, KH)
    skip, _, pt = O.parity_skip(2, 0, X)
    om = O.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    D = gm.dim
    assert D == 1 << n_sites
    ctx = P.Context(gm, R=1)
    v1 = torch.empty(D, dtype=torch.complex128, device="cuda")
    ctx.fill_gaussian(20261203, v1, normalise=False)
    torch.cuda.synchronize()
    v1h = v1.cpu().numpy()
    ctx.close()
    # oracle output slices, gathering from the full input vector
    slices = [0, (D // 2) + 3 * SLICE // 4, D - SLICE]
    ref = []
    for lo in slices:
        w = np.zeros(SLICE, dtype=np.complex128)
        om.p_mltply_v3_slice(v1h, w, lo, lo + SLICE, EPERBD)
        ref.append(w)
    del v1h
    # the default plan of this size first (no plan set: the tensor-copy kernel), then
    # the candidates and the plan the autotuner picks
    assert gm.plan(1)["staging"] == 3
    tuned = tune.autotune(gm, 1)
    plans = [()] + list(PLANS[n_sites])
    if tuple(tuned["plan"]) not in plans:
        plans.append(tuple(tuned["plan"]))
    w = torch.empty_like(v1)
    for plan in plans:
        got = gm.set_plan(1, *plan)
        assert got["tile_passes"] >= 2, plan
        if not plan:
            assert got["staging"] == 3
        if len(plan) > 5 and plan[5] in (2, 3):
            assert got["staging"] == plan[5], plan
        ctx = P.Context(gm, R=1)
        w.zero_()
        torch.cuda.synchronize()
        pr = ctx.p_mltply_v3(v1, w, EPERBD)[0]
        torch.cuda.synchronize()
        for lo, r in zip(slices, ref):
            g = w[lo:lo + SLICE].cpu().numpy()
            assert rel(g, r) <= 1e-12, (plan, lo, rel(g, r))
        dot = complex(torch.vdot(v1, w).item())
        scale = float(torch.sum(torch.abs(v1) * torch.abs(w)).item())
        assert abs(pr - dot) <= 1e-12 * scale, (plan, pr, dot)
        ctx.close()
    gm.set_plan(1)
    del v1, w
    torch.cuda.empty_cache()
