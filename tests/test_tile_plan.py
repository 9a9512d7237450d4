"""Host-side checks of the tile plans (no GPU): the single-vector S = 1/2 tiles
and the mixed-radix (S >= 1) tiles.

The tile kernel (pned_b200/csrc/device.cu, hv_tile_kernel) stages a tile of
256 x 2^jb states: thread t holds row t (its 8 bits on the global bits rowpos)
and j-th state base | jexp[j] (the j bits on jpos); the other (outer) bits
number the tiles.  An in-tile term gathers element (t ^ mask_lo) + 256 (j ^
mask_hi) of the staged tile, an out-of-tile term the state (base ^ mask) ^
jexp[j]; the coefficient index takes the dependency bits of `base` and, for
terms with a dependency on a j bit, the 4-bit field j of `jtab`.  These tests
replay that arithmetic in numpy for every state of the basis and compare it
with the direct global computation (partner s ^ xmask, index = the dependency
bits of s), and check that the passes cover every flip term exactly once.
The mixed-radix replay (check_qplan) does the same for hv_qtile_kernel's
base-q tile offsets and partner offsets.
"""
import numpy as np
import pytest

import pned_b200 as P
from pned_b200 import api
from pned_b200 import couplings as CP
from pned_b200.lattice import honeycomb


def bits_to(values, positions):
    """Scatter bit k of each value to global bit positions[k]."""
    out = np.zeros_like(values)
    for k, p in enumerate(positions):
        out |= ((values >> k) & 1) << p
    return out


def gather_bits(states, positions):
    """Bit k of the result = bit positions[k] of the state."""
    out = np.zeros_like(states)
    for k, p in enumerate(positions):
        out |= ((states >> p) & 1) << k
    return out


def check_plan(n, plan, fixed):
    want = sorted((t["xmask"], t["pos4"], t["tab"], t["nb"]) for t in plan["xterms"])
    got = []
    states = np.arange(1 << n, dtype=np.int64)
    for ps in plan["passes"]:
        tb, jb = ps["tbits"], ps["jb"]
        rowpos, jpos, outer = ps["rowpos"], ps["jpos"], ps["outer"]
        assert sorted(rowpos + jpos + outer) == list(range(n))
        assert rowpos[:fixed] == list(range(fixed))
        rowmask = sum(1 << b for b in rowpos)
        jmask = sum(1 << b for b in jpos)
        tilemask = rowmask | jmask
        tid = gather_bits(states, rowpos)
        j = gather_bits(states, jpos)
        jexp = bits_to(np.arange(1 << jb, dtype=np.int64), jpos)
        base = states & ~jmask
        terms = ps["terms"]
        for ti, T in enumerate(terms):
            inner = ti < ps["nin"]
            deps = [(T["pos4"] >> (8 * d)) & 0xFF for d in range(T["nb"])]
            if inner:
                tmask = (1 << tb) - 1
                gmask = int(bits_to(np.array([T["mask"] & tmask]), rowpos)[0]) | \
                    int(bits_to(np.array([T["mask"] >> tb]), jpos)[0])
                assert gmask & ~tilemask == 0
                lt, lj = tid ^ (T["mask"] & tmask), j ^ (T["mask"] >> tb)
                partner = (states & ~tilemask) | bits_to(lt, rowpos) | jexp[lj]
            else:
                gmask = T["mask"]
                assert gmask & ~tilemask != 0
                assert T["lmask"] == int(gather_bits(np.array([gmask & rowmask]), rowpos)[0]) | \
                    (int(gather_bits(np.array([gmask & jmask]), jpos)[0]) << tb)
                partner = (base ^ gmask) ^ jexp[j]
            assert np.array_equal(partner, states ^ gmask)
            got.append((gmask, T["pos4"], T["tab"], T["nb"]))
            assert T["hasj"] == int(any(p in jpos for p in deps))
            ib = gather_bits(base, deps)
            jt = np.array([(T["jtab"] >> (4 * jj)) & 15 for jj in range(1 << jb)], dtype=np.int64)
            kidx = ib | jt[j] if T["hasj"] else ib
            assert np.array_equal(kidx, gather_bits(states, deps))
        assert ps["gstart"][0] == ps["nin"] and ps["gstart"][-1] == len(terms)
        assert len(set(ps["gxor"])) == len(ps["gxor"])
        for g, gx in enumerate(ps["gxor"]):
            for ti in range(ps["gstart"][g], ps["gstart"][g + 1]):
                assert terms[ti]["mask"] & ~tilemask == gx
    assert sorted(got) == want


MODELS = [
    ("KH", CP.kitaev_heisenberg(0.3, -1.0), None),
    ("KHG-h111", CP.kitaev_heisenberg(0.3, -1.0, gamma=0.1), CP.field_111(0.05)),
    ("slots", CP.slots(J1=0.4, K1=-0.3, I11=0.2, I12=-0.1, J1p=0.7, K1p=1.1, J1pp=-0.5, I11p=0.05, I12p=0.3,
                       I12pp=-0.2, J2=0.15, K2=0.25, I21=0.01, I22=0.02, J3=0.3, ratio_l=0.8), [0.01, 0.02, 0.03]),
]
# (row_fixed_bits, window_bits, max_passes, j_bits[, objective]); objective 1: tiles that hold the most terms
PLANS = [(8, 10, 4, 3), (5, 8, 2, 4), (3, 6, 1, 4), (5, 12, 2, 2), (5, 4, 3, 1), (0, 6, 3, 4), (8, 2, 4, 3),
         (5, 6, 2, 3, 1), (5, 4, 3, 4, 1), (8, 6, 2, 3, 1), (3, 8, 2, 2, 1)]


@pytest.mark.parametrize("plan", PLANS, ids=[",".join(map(str, p)) for p in PLANS])
@pytest.mark.parametrize("name,cpl,fld", MODELS, ids=[m[0] for m in MODELS])
def test_tile_plan_index_arithmetic(name, cpl, fld, plan):
    cl = honeycomb(2, 4)
    X, skip, pt = P.build_xlocal(2, 0, cpl, field=fld)
    d = P.ModelInput(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    out = api.tile_plan_export(d, *plan[:4], objective=plan[4] if len(plan) > 4 else -1)
    assert 1 <= len(out["passes"]) <= plan[2]
    assert all(ps["jb"] == plan[3] for ps in out["passes"])
    check_plan(cl.n, out, plan[0])


def test_tile_plan_eighteen_sites_default_plan():
    """N = 18 (3x3) with the default plan and the 16-row tiles."""
    cl = honeycomb(3, 3)
    X, skip, pt = P.build_xlocal(2, 0, CP.kitaev_heisenberg(0.3, -1.0, gamma=0.1), field=CP.field_111(0.05))
    d = P.ModelInput(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    check_plan(cl.n, api.tile_plan_export(d), 8)
    check_plan(cl.n, api.tile_plan_export(d, 5, 10, 2, 4), 5)


# the multi-vector kernel: G = R / VPT threads a state, 256 / G state rows, SPT = 2^jb rows a thread
RV_SHAPES = [(16, 5, 2), (8, 6, 2), (4, 7, 2), (12, 5, 1), (6, 6, 1), (3, 7, 1)]   # (R, row bits, jb)


@pytest.mark.parametrize("R,tbits,jb", RV_SHAPES, ids=[f"R{r}" for r, _, _ in RV_SHAPES])
@pytest.mark.parametrize("fixed,window,passes", [(-1, 6, 2), (0, 10, 2), (2, 4, 3)])
def test_multi_vector_tile_plan_index_arithmetic(R, tbits, jb, fixed, window, passes):
    """The planner at the multi-vector kernel's tile shapes (hv_tile_rv_kernel:
    row l = thread / G on rowpos, in-tile partner row l ^ (mask & (2^tbits - 1)),
    j ^ (mask >> tbits))."""
    cl = honeycomb(2, 4)
    X, skip, pt = P.build_xlocal(2, 0, CP.kitaev_heisenberg(0.3, -1.0, gamma=0.1), field=CP.field_111(0.05))
    d = P.ModelInput(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    out = api.tile_plan_export(d, fixed, window, passes, jb, row_bits=tbits)
    assert all(ps["tbits"] == tbits and ps["jb"] == jb for ps in out["passes"])
    check_plan(cl.n, out, tbits if fixed < 0 else min(fixed, tbits))


def test_tile_plan_export_refuses_what_is_not_tiled():
    cl = honeycomb(2, 4)
    X, skip, pt = P.build_xlocal(2, 0, CP.kitaev_heisenberg(1.0, 0.0))
    assert pt == 0   # Sz sector: not tiled
    with pytest.raises(P.PnedError):
        api.tile_plan_export(P.ModelInput(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt))
    X, skip, pt = P.build_xlocal(2, 0, CP.kitaev_heisenberg(0.3, -1.0))
    with pytest.raises(P.PnedError):
        api.tile_plan_export(P.ModelInput(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt), 5, 8, 2, 5)


def check_qplan(r, low):
    """Replays the tiled mixed-radix kernel's index arithmetic (hv_qtile.cu):
    tile base from the outer digits, local index l from the tile sites' digits,
    state = base + goff[l], pair state from the local digits ls1/ls2, partner =
    base + goff[l + loff]; compared with the program's flat radix terms."""
    q, n = r["q"], r["n"]
    rt = {t["tab"]: t for t in r["rterms"]}
    assert len(rt) == len(r["rterms"])
    nonzero = np.array(r["nonzero"], dtype=bool)
    states = np.arange(q ** n, dtype=np.int64)
    digits = [(states // q ** i) % q for i in range(n)]
    covered = []
    for ps in r["passes"]:
        sites, outer = ps["sites"], ps["outer"]
        nt = q ** len(sites)
        assert sites == sorted(sites) and outer == sorted(outer) and sorted(sites + outer) == list(range(n))
        assert sites[:low] == list(range(low))
        loc = sum(digits[x] * q ** i for i, x in enumerate(sites))
        base = sum(digits[x] * q ** x for x in outer)
        lidx = np.arange(nt, dtype=np.int64)
        goff = sum(((lidx // q ** i) % q) * q ** x for i, x in enumerate(sites))
        assert np.array_equal(base + goff[loc], states)
        for T in ps["terms"]:
            R = rt[T["tab"]]
            covered.append(T["tab"])
            assert (sites[T["ls1"]], sites[T["ls2"]]) == (R["s1"], R["s2"])
            pair = (loc // q ** T["ls1"]) % q + q * ((loc // q ** T["ls2"]) % q)
            assert np.array_equal(pair, digits[R["s1"]] + q * digits[R["s2"]])
            nz = nonzero[R["tab"] + pair]
            pl = loc[nz] + T["loff"]
            assert np.all((pl >= 0) & (pl < nt))
            assert np.array_equal(base[nz] + goff[pl], states[nz] + R["offset"])
    assert sorted(covered) == sorted(rt)


QMODELS = [
    ("S1-KH", 3, CP.kitaev_heisenberg(0.2, -1.0), None, 2, 2),
    ("S1-KHG-h111", 3, CP.kitaev_heisenberg(0.2, -1.0, gamma=0.1), CP.field_111(0.05), 2, 2),
    ("S3/2-KHG", 4, CP.kitaev_heisenberg(-0.3, 0.6, gamma=0.2), None, 3, 1),
]


@pytest.mark.parametrize("k,low", [(3, 0), (4, 1), (5, 1), (6, 0)])
@pytest.mark.parametrize("name,q,cpl,fld,L1,L2", QMODELS, ids=[m[0] for m in QMODELS])
def test_qtile_plan_index_arithmetic(name, q, cpl, fld, L1, L2, k, low):
    cl = honeycomb(L1, L2)
    if k > cl.n - 2:
        pytest.skip("tiles leave at least two outer sites")
    X, skip, pt = P.build_xlocal(q, 1, cpl, field=fld)
    d = P.ModelInput(cl.n, q, 1, cl.ipair, cl.ibond_type, X, skip, pt)
    check_qplan(api.qtile_plan_export(d, k, low), low)


def test_headline_plan_structure_n30():
    """The N = 30 Kitaev-Heisenberg plans the measurements quote: the tuned plan
    (5 fixed row bits, 12 window bits, 2 passes, 8 rows a thread) has 2 passes and
    17 partner tiles; the 16-row tiles 14 (window 11) and 15 (window 10)."""
    import math
    from pned_b200.lattice import cluster_for_sites
    cl = cluster_for_sites(30)
    X, skip, pt = P.build_xlocal(2, 0, CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi)))
    d = P.ModelInput(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    for plan, groups in (((5, 12, 2, 3), 17), ((5, 11, 2, 4), 14), ((5, 10, 2, 4), 15)):
        r = api.tile_plan_export(d, *plan)
        assert len(r["xterms"]) == 45 and len(r["passes"]) == 2
        assert sum(len(ps["gxor"]) for ps in r["passes"]) == groups
        assert sum(len(ps["terms"]) for ps in r["passes"]) == 45


def test_every_tuner_candidate_plans_the_n30_model():
    """Each single-vector candidate of the autotuner yields a plan for the N = 30
    Kitaev-Heisenberg model within its pass limit (a candidate the planner
    refuses would be skipped silently while tuning)."""
    import math
    from pned_b200 import tune
    from pned_b200.lattice import cluster_for_sites
    cl = cluster_for_sites(30)
    X, skip, pt = P.build_xlocal(2, 0, CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi)))
    d = P.ModelInput(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    for c in tune.CANDIDATES_1:
        jb = c[3] if len(c) > 3 else -1
        r = api.tile_plan_export(d, c[0], c[1], c[2], jb, objective=c[7] if len(c) > 7 else -1)
        assert 1 <= len(r["passes"]) <= c[2]
        assert sum(len(ps["terms"]) for ps in r["passes"]) == 45


def test_most_terms_objective_n30():
    """Objective 1 at N = 30 (the measured Kitaev-Heisenberg model): the tiles
    take the rings of low sites, so more of the 45 flip terms gather from
    shared memory -- 13 + 9 with 8 rows a thread, 15 + 10 with 16 -- than the
    fewest-partner-tile plan's 6 + 0, and the terms left to gather through
    L1/L2 drop from 39 to 23 and 20; every term still in exactly one pass (the
    index arithmetic is checked for every state, here on an 18-site copy of the
    plan shape)."""
    import math
    from pned_b200.lattice import cluster_for_sites
    cl = cluster_for_sites(30)
    X, skip, pt = P.build_xlocal(2, 0, CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi)))
    d = P.ModelInput(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    base = api.tile_plan_export(d, 5, 12, 2, 3)
    assert [ps["nin"] for ps in base["passes"]] == [6, 0]
    for plan, nin in (((5, 10, 2, 3), [13, 9]), ((5, 10, 2, 4), [15, 10])):
        r = api.tile_plan_export(d, *plan, objective=1)
        assert [ps["nin"] for ps in r["passes"]] == nin
        assert sum(len(ps["terms"]) for ps in r["passes"]) == 45
        assert r["passes"][0]["rowpos"][:5] == [0, 1, 2, 3, 4]
    c18 = cluster_for_sites(18)
    d18 = P.ModelInput(c18.n, 2, 0, c18.ipair, c18.ibond_type, X, skip, pt)
    check_plan(c18.n, api.tile_plan_export(d18, 5, 6, 2, 3, objective=1), 5)


def tma_copy_dims(n, ps):
    """Copy dimensions of one pass's tile for the tensor-copy kernel
    (pned_b200/csrc/hv_staged.cu, tile_tma_geometry): the tile's bits in
    ascending order must be the 8 row bits, then the 3 j bits, from bit 0; runs
    of tile bits (the first at most 7 bits, later ones 8) and runs of outer bits
    (at most 31) each take one dimension.  None where the tile does not qualify."""
    tb = sorted(ps["rowpos"] + ps["jpos"])
    if len(ps["rowpos"]) != 8 or len(ps["jpos"]) != 3 or tb != ps["rowpos"] + ps["jpos"] or tb[0] != 0:
        return None
    tset, dims, b = set(tb), 0, 0
    while b < n:
        inside = b in tset
        e = b
        while e < n and (e in tset) == inside:
            e += 1
        s = b
        while s < e:
            s += min((7 if dims == 0 else 8) if inside else 31, e - s)
            dims += 1
        b = e
    return dims


@pytest.mark.parametrize("n", [26, 28, 30])
def test_default_plan_from_26_sites_is_the_tensor_copy_plan(n):
    """With no plan set, from 26 sites on the model plans 5 fixed row bits, a
    7-bit window, 2 passes and the most-terms objective (the autotuned plan of
    the tensor-copy kernel): the exporter gives the same plan, every pass's
    tile maps onto at most 5 copy dimensions (else the kernel would fall back
    to the gather), and every flip term is in exactly one pass.  At N = 30 the
    passes have 10 + 12 partner tiles and 13 + 9 terms inside the tile."""
    import math
    from pned_b200.lattice import cluster_for_sites
    cl = cluster_for_sites(n)
    X, skip, pt = P.build_xlocal(2, 0, CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi)))
    d = P.ModelInput(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    r = api.tile_plan_export(d)
    assert r == api.tile_plan_export(d, 5, 7, 2, 3, objective=1)
    assert len(r["passes"]) == 2
    assert sorted(t["tab"] for ps in r["passes"] for t in ps["terms"]) == sorted(x["tab"] for x in r["xterms"])
    assert len(r["xterms"]) == 3 * n // 2
    for ps in r["passes"]:
        dims = tma_copy_dims(n, ps)
        assert dims is not None and dims <= 5
    if n == 30:
        assert [len(ps["gxor"]) for ps in r["passes"]] == [10, 12]
        assert [ps["nin"] for ps in r["passes"]] == [13, 9]


def test_default_plan_below_26_sites_is_the_gather_plan():
    """Below 26 sites the default stays the fewest-partner-tile plan with a
    10-bit window (the gather kernel's): the exporter without a plan gives the
    plan of explicit defaults."""
    from pned_b200.lattice import cluster_for_sites
    cl = cluster_for_sites(24)
    X, skip, pt = P.build_xlocal(2, 0, CP.kitaev_heisenberg(0.6, 1.6))
    d = P.ModelInput(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    assert api.tile_plan_export(d) == api.tile_plan_export(d, 8, 10, -1, 3, objective=0)
