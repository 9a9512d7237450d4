"""Slot batches (continuous batching of chains with different couplings) against
the CPU oracle, and the alone-versus-in-the-mix property of the serving path.

Tolerances (FP64 complex): per-slot Lanczos alpha/beta (first 15 steps) and
E0, TPS alpha/beta/coef, DSF cnorm and chain coefficients relative <= 1e-10;
a chain run alone and in a mix of other slots (same batch width) agrees bit
for bit."""
import math

import numpy as np
import pytest

import pned_b200 as P
from oracle import oracle as O
from pned_b200 import couplings as CP
from pned_b200.lattice import cluster_for_sites, honeycomb

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from tests.chains import check_chain, oracle_chain_variants  # noqa: E402


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


def request_couplings(phi, gamma, h):
    return CP.kitaev_heisenberg(math.cos(phi), 2 * math.sin(phi), gamma=gamma), CP.field_111(h)


REQS = [(0.3 * math.pi, 0.1, 0.05), (1.1, -0.15, 0.02), (4.0, 0.05, 0.09), (2.5, -0.2, 0.0)]


def inputs(cl, cpl, fld, tps_L=None):
    slot_in = P.ModelInput.from_couplings(cl, cpl, field=fld)
    X, skip, pt = P.build_xlocal(2, 0, cpl, field=fld)
    if tps_L is not None:
        X, _ = P.tps_transform(2, 0, cl.nbond, X, L=tps_L)
    om = O.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    return slot_in, om


@pytest.mark.parametrize("R,plan", [(1, None), (4, None), (1, (5, 0, 2, 3, 1, 3, -1, 1, 2))])
def test_slots_lanczos_tps_parity(R, plan):
    """Each slot carries its own couplings; Lanczos and TPS slots share one H.V
    (also with a two-pass plan whose tile rows arrive by tensor copies)."""
    cl = honeycomb(3, 2)
    L = 2.0 * cl.n
    steps = 40
    sb = P.SlotBatch(P.ModelInput.structure(cl), R, steps)
    if plan is not None:
        assert sb.set_plan(*plan)["tile_passes"] == 2
    kinds = ["lanczos", "tps", "lanczos", "tps"][:max(R, 2)]
    runs = []
    for r, kind in enumerate(kinds):
        cpl, fld = request_couplings(*REQS[r])
        slot_in, om = inputs(cl, cpl, fld, tps_L=L if kind == "tps" else None)
        v = O.gaussian(100 + r, sb.dim)
        v /= np.linalg.norm(v)
        runs.append((r % R, kind, slot_in, om, v))
    # R = 1 runs the two kinds one after the other in the same slot
    groups = [runs] if R > 1 else [[x] for x in runs]
    for grp in groups:
        for slot, kind, slot_in, om, v in grp:
            sb.load(slot, kind, slot_in, v, steps, L=L)
        sb.step(steps + 2)
        for slot, kind, slot_in, om, v in grp:
            out = sb.read(slot)
            assert out["steps"] == steps and out["status"] == 0
            if kind == "lanczos":
                ref = om.lanczos(v, steps)
                assert rel(out["alpha"][:15], ref["alpha"][:15]) <= 1e-10
                assert rel(out["beta"][:15], ref["beta"][:15]) <= 1e-10
                e0 = P.bisec(out["alpha"], out["beta"], steps, 1)[0]
                assert abs(e0 - ref["ene"][0]) <= 1e-10 * abs(ref["ene"][0])
            else:
                ref = om.tps(L, v, steps)
                assert rel(out["alpha"], ref["alpha"]) <= 1e-10
                assert rel(out["beta"], ref["beta"]) <= 1e-10
                for j in range(5):
                    assert rel(out["coef"][:, j], ref["coef"][:, j]) <= 1e-10, j
            sb.release(slot)
    sb.close()


def test_slots_eigenvector_and_dsf_chains():
    """Lanczos E0 pass, eigenvector pass (stored alpha/beta) and S^z_q chains in slots."""
    cl = honeycomb(3, 2)
    cpl, fld = request_couplings(*REQS[0])
    slot_in, om = inputs(cl, cpl, fld)
    M = 90
    sb = P.SlotBatch(P.ModelInput.structure(cl), 4, M)
    v = O.gaussian(21, sb.dim)
    v /= np.linalg.norm(v)
    sb.load(2, "lanczos", slot_in, v, M)
    sb.step(M)
    first = sb.read(2)
    E = P.bisec(first["alpha"], first["beta"], M, 1)
    c = P.vec12(first["alpha"], first["beta"], E, M, 1)[0]
    x = torch.zeros(sb.dim, dtype=torch.complex128, device="cuda")
    sb.load_vector(1, slot_in, v, first["alpha"], first["beta"], c, x)
    sb.step(M)
    sb.synchronize()
    xh = x.cpu().numpy()
    xh /= np.linalg.norm(xh)
    hx = np.zeros_like(xh)
    om.p_mltply_v3(xh, hx, 0.0)
    assert np.linalg.norm(hx - E[0] * xh) <= 1e-6
    b = O.gaussian(22, sb.dim)
    xr, _, _ = om.inverse_iteration(E[0] - 1e-9, b / np.linalg.norm(b), inv_max=30)
    assert abs(abs(np.vdot(xr, xh)) - 1.0) <= 1e-9
    steps = 12
    for r in range(4):
        sb.load_szq(r, slot_in, x, cl.qr(r), steps)
    sb.step(steps)
    for r in range(4):
        out = sb.read(r)
        vq, cn = om.intalv_zz(cl.qr(r), xh)
        sa, sbeta = om.dsf_chain(vq, cn, steps)
        assert abs(out["cnorm"] - cn.real) <= 1e-10 * abs(cn)
        assert rel(out["alpha"], sa) <= 1e-10
        assert rel(out["beta"], sbeta[1:steps + 1]) <= 1e-10
    sb.close()


def test_slots_alone_equals_in_the_mix():
    """A chain loaded while other slots run (and are released and reloaded
    around it) gives the same coefficients as the chain alone."""
    cl = honeycomb(2, 4)
    structure = P.ModelInput.structure(cl)
    steps = 30
    cpl, fld = request_couplings(*REQS[1])
    a_in, om = inputs(cl, cpl, fld)
    va = O.gaussian(31, 2 ** cl.n)
    alone = P.SlotBatch(structure, 4, 64)
    alone.load(0, "lanczos", a_in, va, steps)
    alone.step(steps)
    ra = alone.read(0)
    alone.close()

    mix = P.SlotBatch(structure, 4, 64)
    others = []
    for k in (0, 2, 3):
        c, f = request_couplings(*REQS[k])
        others.append(P.ModelInput.from_couplings(cl, c, field=f))
    mix.load(0, "tps", others[0], O.gaussian(32, 2 ** cl.n), 50, L=2.0 * cl.n)
    mix.load(2, "lanczos", others[1], O.gaussian(33, 2 ** cl.n), 9)
    mix.step(7)
    mix.load(3, "lanczos", a_in, va, steps)       # joins mid-stream
    mix.step(5)
    mix.release(2)                                 # finished at step 9
    mix.load(2, "tps", others[2], O.gaussian(34, 2 ** cl.n), 40, L=2.0 * cl.n)
    mix.step(steps - 5)
    rm = mix.read(3)
    mix.close()
    assert rm["steps"] == steps and ra["steps"] == steps
    assert np.array_equal(rm["alpha"], ra["alpha"]) and np.array_equal(rm["beta"], ra["beta"])
    ref = om.lanczos(va / np.linalg.norm(va), steps)
    assert rel(ra["alpha"][:15], ref["alpha"][:15]) <= 1e-10
    e0 = P.bisec(ra["alpha"], ra["beta"], steps, 1)[0]
    assert abs(e0 - ref["ene"][0]) <= 1e-10 * abs(ref["ene"][0])


def test_slots_reject_bad_input():
    cl = honeycomb(2, 2)
    sb = P.SlotBatch(P.ModelInput.structure(cl), 2, 8)
    other = honeycomb(3, 2)
    v = np.ones(sb.dim, dtype=np.complex128)
    with pytest.raises(P.PnedError):
        sb.load(0, "lanczos", P.ModelInput.from_couplings(other, CP.kitaev_heisenberg(1.0, 0.5)), v, 4)
    with pytest.raises(P.PnedError):
        sb.load(2, "lanczos", P.ModelInput.from_couplings(cl, CP.kitaev_heisenberg(1.0, 0.5)), v, 4)
    with pytest.raises(P.PnedError):
        sb.load(0, "lanczos", P.ModelInput.from_couplings(cl, CP.kitaev_heisenberg(1.0, 0.5)), v, 9)
    with pytest.raises(P.PnedError):
        P.SlotBatch(P.ModelInput.structure(cl), 5, 8)
    sb.close()


def test_gaussian_column_matches_interleaved_fill():
    cl = honeycomb(2, 2)
    m = P.Model.from_couplings(cl, CP.kitaev_heisenberg(1.0, 0.5))
    R = 4
    ctx = P.Context(m, R=R)
    full = torch.empty(m.dim * R, dtype=torch.complex128, device="cuda")
    ctx.fill_gaussian(77, full, normalise=False)
    col = torch.empty(m.dim, dtype=torch.complex128, device="cuda")
    for r in range(R):
        P.api.gaussian_column(m.dim, R, r, 77, col)
        torch.cuda.synchronize()
        assert torch.equal(col, full.view(m.dim, R)[:, r].contiguous())
    ref = O.gaussian(77, m.dim, R).reshape(m.dim, R)
    assert np.max(np.abs(full.view(m.dim, R).cpu().numpy() - ref)) <= 1e-14


def oracle_dsf(q):
    """The oracle's run of a DSF request: the ground state from its seeded start
    vector (gs_steps Lanczos steps, vec12, the eigenvector pass), then the
    momentum chains with the variant runs that measure the oracle's own spread
    (tests/chains.py); returns (E0, [(ref, [variants])] per momentum)."""
    cl = cluster_for_sites(q.n)
    cpl, fld = q.couplings()
    X = O.xlocal(2, 0, cpl, field=fld)
    skip, _, pt = O.parity_skip(2, 0, X)
    om = O.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    v = O.gaussian(q.seed, om.ldim)
    v /= np.linalg.norm(v)
    run = om.lanczos(v, q.gs_steps)
    E = O.bisec(run["alpha"], run["beta"], q.gs_steps, 1)
    c = O.vec12(run["alpha"], run["beta"], E, q.gs_steps, 1)[0]
    x = om.lanczos_vector(v, run["alpha"], run["beta"], c)
    qrs = np.stack([cl.qr(k) for k in range(q.nq)])
    return E[0], oracle_chain_variants(cl, cpl, x, qrs, q.steps, fld=fld)


def test_serving_results_alone_and_in_the_mix():
    """Requests served in a mixed stream (lanes of N = 10, 12, 14, co-batched,
    joining while others run) give the same results as each request served
    alone (bit for bit) and as the plain path (E0 and TPQ coefficients 1e-10).
    DSF: both take the ground state from a 40-step Lanczos eigenvector pass,
    through different H.V kernels, so their chains are compared with the
    oracle's run of the same request instead, each within 1e-10 or ten times
    the oracle's own spread (coefficients over the prefix the oracle's variant
    runs agree on, and S(q, w)), as the configuration tests do."""
    from pned_b200 import serve
    reqs = serve.make_stream(14, rate=1e6, seed=11, sizes=(10, 12, 14), p30=0.0, mix=(0.5, 0.3, 0.2),
                             lanczos_steps=60, tpq_steps=40, dsf_steps=20, dsf_gs_steps=40)
    srv = serve.Server(budget=8 << 30, lane_slots=lambda n: 4, max_steps=128)
    st = srv.run(reqs, realtime=False)
    srv.close()
    assert len(st.results) == len(reqs)
    by = {r["rid"]: r for r in st.results}
    assert {r.kind for r in reqs} == {"lanczos", "tpq", "dsf"}
    for q in reqs:
        r = by[q.rid]
        assert "status" not in r
        alone_srv = serve.Server(budget=8 << 30, lane_slots=lambda n: 4, max_steps=128)
        a = alone_srv.run([q], realtime=False).results[0]
        alone_srv.close()
        p = serve.run_plain(q)
        if q.kind == "lanczos":
            assert np.array_equal(r["alpha"], a["alpha"]) and np.array_equal(r["beta"], a["beta"])
            assert abs(r["e0"] - p["e0"]) <= 1e-10 * abs(p["e0"])
        elif q.kind == "tpq":
            assert np.array_equal(r["coef"], a["coef"])
            for k in range(q.nvec):
                for j in range(5):
                    assert rel(r["coef"][:, k, j], p["coef"][:, k, j]) <= 1e-10, (k, j)
        else:
            for k in range(q.nq):
                assert np.array_equal(r["salpha"][k], a["salpha"][k])
            assert abs(r["e0"] - p["e0"]) <= 1e-10 * abs(p["e0"])
            e0, chains = oracle_dsf(q)
            assert abs(r["e0"] - e0) <= 1e-10 * abs(e0)
            for k, (ref, others) in enumerate(chains):
                for got in (r, p):
                    check_chain(np.asarray(got["salpha"][k]), np.asarray(got["sbeta"][k]), ref, others, e0, q.steps,
                                min_prefix=10)
