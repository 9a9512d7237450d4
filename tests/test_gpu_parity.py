"""GPU parity of the CUDA path (through the C ABI) against the CPU oracle.

Tolerances (FP64 complex throughout):
  H.v           relative 2-norm <= 1e-12, prdct relative <= 1e-12
  Lanczos E0    relative <= 1e-10; first alpha/beta relative <= 1e-10
  TPS           alpha, beta, coef relative <= 1e-10
  DSF           cnorm, chain coefficients and spectra relative <= 1e-10
"""
import math

import numpy as np
import pytest

import pned_b200 as P
from oracle import oracle as O
from pned_b200 import couplings as CP
from pned_b200.lattice import honeycomb

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

KH = CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi))
KHGH = CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi), gamma=0.1)
FIELD = CP.field_111(0.05)


def models(cl, q, tree, cpl, fld=None, tps_L=None):
    X, skip, pt = P.build_xlocal(q, tree, cpl, field=fld)
    if tps_L is not None:
        X, _ = P.tps_transform(q, tree, cl.nbond, X, L=tps_L)
    gm = P.Model(cl.n, q, tree, cl.ipair, cl.ibond_type, X, skip, pt)
    om = O.Model(cl.n, q, tree, cl.ipair, cl.ibond_type, X, skip, pt)
    return gm, om


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


HV_CASES = [
    # (L1, L2, q, tree, couplings, field, R)
    (2, 2, 2, 0, KH, None, 1),
    (3, 2, 2, 0, KHGH, FIELD, 1),
    (3, 2, 2, 0, KHGH, FIELD, 3),
    (2, 4, 2, 0, KH, None, 4),
    (2, 4, 2, 0, KHGH, FIELD, 12),
    (3, 2, 2, 0, KH, None, 16),
    (3, 2, 2, 1, KHGH, FIELD, 2),
    (3, 1, 3, 1, CP.kitaev_heisenberg(0.2, -1.0), None, 1),
    (3, 1, 3, 1, CP.kitaev_heisenberg(0.2, -1.0, gamma=0.1), FIELD, 4),
    (2, 2, 3, 1, CP.kitaev_heisenberg(0.2, -1.0), None, 6),
    (3, 1, 4, 1, CP.kitaev_heisenberg(0.5, 0.3, gamma=-0.2), FIELD, 8),
]


@pytest.mark.parametrize("case", HV_CASES, ids=[f"{c[0]}x{c[1]}q{c[2]}t{c[3]}R{c[6]}" for c in HV_CASES])
def test_hv_parity(case):
    L1, L2, q, tree, cpl, fld, R = case
    cl = honeycomb(L1, L2)
    gm, om = models(cl, q, tree, cpl, fld)
    ctx = P.Context(gm, R=R)
    rng = np.random.default_rng(17)
    D = gm.dim
    v1 = (rng.standard_normal((D, R)) + 1j * rng.standard_normal((D, R))).astype(np.complex128)
    v0 = (0.2 * rng.standard_normal((D, R)) + 0.1j * rng.standard_normal((D, R))).astype(np.complex128)
    eperbd = 0.0625
    w = np.ascontiguousarray(v0).reshape(-1).copy()
    pr = ctx.p_mltply_v3(np.ascontiguousarray(v1).reshape(-1), w, eperbd)
    w = w.reshape(D, R)
    for r in range(R):
        ref = np.ascontiguousarray(v0[:, r]).copy()
        prr = om.p_mltply_v3(np.ascontiguousarray(v1[:, r]), ref, eperbd)
        assert rel(w[:, r], ref) <= 1e-12
        assert abs(pr[r] - prr) <= 1e-12 * abs(prr)


QTILE_CASES = [
    # (L1, L2, q, tree, couplings, field, R): 12 and 8 sites, tiled mixed-radix passes
    (3, 2, 3, 1, CP.kitaev_heisenberg(0.2, -1.0), None, 1),
    (3, 2, 3, 1, CP.kitaev_heisenberg(0.2, -1.0, gamma=0.1), FIELD, 4),
    (3, 2, 3, 1, CP.kitaev_heisenberg(0.2, -1.0), FIELD, 16),
    (2, 2, 4, 1, CP.kitaev_heisenberg(0.5, 0.3, gamma=-0.2), FIELD, 2),
]


@pytest.mark.parametrize("case", QTILE_CASES, ids=[f"{c[0]}x{c[1]}q{c[2]}R{c[6]}" for c in QTILE_CASES])
def test_radix_tiles_parity(case):
    """S >= 1 on 8-12 sites runs the tiled mixed-radix kernel (several passes of
    q^k-state tiles in shared memory); H.V and prdct match the oracle."""
    L1, L2, q, tree, cpl, fld, R = case
    cl = honeycomb(L1, L2)
    gm, om = models(cl, q, tree, cpl, fld)
    ctx = P.Context(gm, R=R)
    plan = gm.plan(R)
    assert plan["tile_passes"] >= 2 and plan["tile_states"] >= q ** 4
    rng = np.random.default_rng(29)
    D = gm.dim
    v1 = (rng.standard_normal((D, R)) + 1j * rng.standard_normal((D, R))).astype(np.complex128)
    v0 = (0.2 * rng.standard_normal((D, R)) + 0.1j * rng.standard_normal((D, R))).astype(np.complex128)
    w = np.ascontiguousarray(v0).reshape(-1).copy()
    pr = ctx.p_mltply_v3(np.ascontiguousarray(v1).reshape(-1), w, 0.0625)
    w = w.reshape(D, R)
    for r in range(R):
        ref = np.ascontiguousarray(v0[:, r]).copy()
        prr = om.p_mltply_v3(np.ascontiguousarray(v1[:, r]), ref, 0.0625)
        assert rel(w[:, r], ref) <= 1e-12
        assert abs(pr[r] - prr) <= 1e-12 * abs(prr)


def test_radix_tiles_tps_and_lanczos():
    """S = 1, 12 sites: the TPS loop (K = 4 sums in the last pass) and a Lanczos
    chain through the tiled mixed-radix passes follow the oracle."""
    cl = honeycomb(3, 2)
    cpl = CP.kitaev_heisenberg(0.2, -1.0, gamma=0.1)
    L = 3.0 * cl.n
    gm, om = models(cl, 3, 1, cpl, FIELD, tps_L=L)
    R = 4
    V = O.gaussian(11, gm.dim, R).reshape(gm.dim, R)
    V /= np.linalg.norm(V, axis=0)
    out = P.Context(gm, R=R).tps(L, np.ascontiguousarray(V).reshape(-1), 25)
    for r in range(R):
        ref = om.tps(L, np.ascontiguousarray(V[:, r]), 25)
        assert rel(out["alpha"][:, r], ref["alpha"]) <= 1e-10
        assert rel(out["beta"][:, r], ref["beta"]) <= 1e-10
        assert rel(out["coef"][:, r, :5], ref["coef"][:, :5]) <= 1e-10
    gl, ol = models(cl, 3, 1, cpl, FIELD)
    v = np.ascontiguousarray(V[:, 0])
    run = P.Context(gl, R=1).lanczos(v, 30)
    refl = ol.lanczos(v, 30)
    assert rel(run["alpha"][:12, 0], refl["alpha"][:12]) <= 1e-10


def test_hv_device_pointers_and_dots():
    cl = honeycomb(2, 4)
    gm, om = models(cl, 2, 0, KHGH, FIELD)
    ctx = P.Context(gm, R=4)
    rng = np.random.default_rng(3)
    n = gm.dim * 4
    a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    pr = ctx.p_mltply_v3(ta, tb)
    b2 = b.copy()
    pr2 = ctx.p_mltply_v3(a, b2)
    assert np.array_equal(pr, pr2)
    assert np.array_equal(tb.cpu().numpy(), b2)
    d = ctx.calc_vec_inprdct(a, b2)
    for r in range(4):
        ref = O.inprdct(np.ascontiguousarray(a.reshape(-1, 4)[:, r]), np.ascontiguousarray(b2.reshape(-1, 4)[:, r]))
        assert abs(d[r] - ref) <= 1e-12 * abs(ref)
    al = np.array([0.3 + 0.01j, -1.0, 2.0 - 0.5j, 0.0])
    cb = ctx.calc_beta(al, a, b2)
    for r in range(4):
        x1 = a.reshape(-1, 4)[:, r]
        x2 = b2.reshape(-1, 4)[:, r]
        ref = np.sum(np.abs(x2 - al[r] * x1) ** 2)
        assert abs(cb[r] - ref) <= 1e-12 * ref


def test_gaussian_matches_oracle():
    cl = honeycomb(2, 4)
    gm, _ = models(cl, 2, 0, KH)
    for R in (1, 3, 16):
        ctx = P.Context(gm, R=R)
        t = torch.empty(gm.dim * R, dtype=torch.complex128, device="cuda")
        ctx.fill_gaussian(20261203, t, normalise=False)
        ref = O.gaussian(20261203, gm.dim, R)
        assert np.max(np.abs(t.cpu().numpy() - ref)) <= 1e-14
        ctx.fill_gaussian(20261203, t, normalise=True)
        nrm = np.linalg.norm(t.cpu().numpy().reshape(-1, R), axis=0)
        assert np.allclose(nrm, 1.0, atol=1e-14)


@pytest.mark.parametrize("L1,L2,q,tree,cpl,fld,steps", [
    (3, 2, 2, 0, KH, None, 90),
    (2, 4, 2, 0, KHGH, FIELD, 120),
    (3, 1, 3, 1, CP.kitaev_heisenberg(0.2, -1.0), None, 80),
])
def test_lanczos_parity(L1, L2, q, tree, cpl, fld, steps):
    cl = honeycomb(L1, L2)
    gm, om = models(cl, q, tree, cpl, fld)
    v = O.gaussian(7, gm.dim)
    v /= np.linalg.norm(v)
    ref = om.lanczos(v, steps)
    ctx = P.Context(gm, R=1)
    out = ctx.lanczos(v, steps)
    assert out["itr"] == steps
    assert abs(out["ene"][0] - ref["ene"][0]) <= 1e-10 * abs(ref["ene"][0])
    k = 15
    assert rel(out["alpha"][:k, 0], ref["alpha"][:k]) <= 1e-10
    assert rel(out["beta"][:k, 0], ref["beta"][:k]) <= 1e-10


def test_lanczos_batched_chains_are_independent():
    cl = honeycomb(2, 4)
    gm, om = models(cl, 2, 0, KHGH, FIELD)
    R = 4
    V = O.gaussian(11, gm.dim, R).reshape(gm.dim, R)
    V /= np.linalg.norm(V, axis=0)
    ctx = P.Context(gm, R=R)
    out = ctx.lanczos(np.ascontiguousarray(V).reshape(-1), 40)
    for r in range(R):
        ref = om.lanczos(np.ascontiguousarray(V[:, r]), 40)
        assert rel(out["alpha"][:12, r], ref["alpha"][:12]) <= 1e-10
        e0 = P.bisec(out["alpha"][:, r], out["beta"][:, r], 40, 1)[0]
        assert abs(e0 - ref["ene"][0]) <= 1e-10 * abs(ref["ene"][0])


def test_lanczos_convergence_stop_matches_oracle():
    cl = honeycomb(2, 2)
    gm, om = models(cl, 2, 0, KH)
    v = O.gaussian(11, gm.dim)
    v /= np.linalg.norm(v)
    ref = om.lanczos(v, 1024, check_conv=True)
    out = P.Context(gm, R=1).lanczos(v, 1024, check_conv=True)
    assert abs(out["ene"][0] - ref["ene"][0]) <= 1e-12 * abs(ref["ene"][0])
    assert out["itr"] % 5 == 0 and out["itr"] < 1024


@pytest.mark.parametrize("R", [1, 4])
def test_tps_parity(R):
    cl = honeycomb(2, 4)
    L = 2.0 * cl.n
    gm, om = models(cl, 2, 0, KHGH, FIELD, tps_L=L)
    V = O.gaussian(5, gm.dim, R).reshape(gm.dim, R)
    V /= np.linalg.norm(V, axis=0)
    # observables as the reference evaluates them: z-bond SzSz (1-based ipair
    # values as bit shifts) and S^zS^z(q), S^+S^-(q) at one momentum
    zb = [(int(cl.ipair[2 * i]), int(cl.ipair[2 * i + 1])) for i in range(cl.nbond) if cl.ibond_type[i] == 3]
    T_zz = np.array([[0.25, -0.25], [-0.25, 0.25]], dtype=complex)
    qr = cl.qr(1)
    T_pp = np.array([[0, 0.25], [0.25, 0]], dtype=complex)
    obs = [
        ([(a, b, 1.0) for a, b in zb], T_zz),
        ([(j, 0, np.exp(1j * qr[j])) for j in range(cl.n)], T_zz),
        ([(j, 0, np.exp(1j * qr[j])) for j in range(cl.n)], T_pp),
    ]
    specs = [P.ObservableSpec(a=np.array([t[0] for t in o[0]]), b=np.array([t[1] for t in o[0]]),
                              c=np.array([t[2] for t in o[0]], dtype=complex), T=o[1]) for o in obs]
    steps = 40
    out = P.Context(gm, R=R).tps(L, np.ascontiguousarray(V).reshape(-1), steps, specs)
    for r in range(R):
        ref = om.tps(L, np.ascontiguousarray(V[:, r]), steps, obs)
        assert rel(out["alpha"][:, r], ref["alpha"]) <= 1e-10
        assert rel(out["beta"][:, r], ref["beta"]) <= 1e-10
        for j in range(ref["coef"].shape[1]):
            assert rel(out["coef"][:, r, j], ref["coef"][:, j]) <= 1e-10, j


def test_dsf_parity():
    """DSF chains and spectra (12 sites, 4 momenta).

    While a chain is well conditioned (here its first 12 steps) coefficients
    agree to 1e-12 and the continued-fraction spectra to 1e-10.  For 30-step
    chains the coefficients are held to 1e-10 over the prefix where the
    oracle's own variants agree, and the spectra to the oracle's own spread
    (tests/chains.py)."""
    from tests.chains import check_chain, oracle_chain_variants
    cl = honeycomb(3, 2)
    gm, om = models(cl, 2, 0, KH)
    v = O.gaussian(3, gm.dim)
    v /= np.linalg.norm(v)
    e0 = om.lanczos(v, 120)["ene"][0]
    b = O.gaussian(4, gm.dim)
    b /= np.linalg.norm(b)
    x, _, _ = om.inverse_iteration(e0 - 1e-9, b, inv_max=30)
    R = 4
    qrs = np.stack([cl.qr(i) for i in range(R)])
    ctx = P.Context(gm, R=R)
    out = ctx.dsf(x, qrs, 12)
    for r in range(R):
        vq, cn = om.intalv_zz(qrs[r], x)
        sa, sb = om.dsf_chain(vq, cn, 12)
        assert abs(out["cnorm"][r] - cn.real) <= 1e-12 * abs(cn)
        assert rel(out["salpha"][:, r], sa) <= 1e-12
        assert rel(out["sbeta"][:, r], sb) <= 1e-12
        _, _, d1 = P.exec_renbun(400, 14, 3.0 / 399, e0, 0.05, out["salpha"][:, r], out["sbeta"][:, r])
        _, _, d2 = O.exec_renbun(400, 14, 3.0 / 399, e0, 0.05, sa, sb)
        assert rel(d1, d2) <= 1e-10
    out = ctx.dsf(x, qrs, 30)
    for r, (ref, others) in enumerate(oracle_chain_variants(cl, KH, x, qrs, 30)):
        check_chain(out["salpha"][:, r], out["sbeta"][:, r], ref, others, e0, 30, min_prefix=10,
                    i_range=400)


def test_lanczos_vector_parity():
    """parallelized_lncv1z: the eigenvector pass replays the chain with the stored
    alpha/beta; x agrees with the oracle to 1e-10 and is an eigenvector."""
    cl = honeycomb(3, 2)
    gm, om = models(cl, 2, 0, KHGH, FIELD)
    v = O.gaussian(3, gm.dim)
    v /= np.linalg.norm(v)
    M = 60
    ref = om.lanczos(v, M)
    E = P.bisec(ref["alpha"], ref["beta"], M, 1)
    c = P.vec12(ref["alpha"], ref["beta"], E, M, 1)[0]
    xr = om.lanczos_vector(v, ref["alpha"], ref["beta"], c)
    ctx = P.Context(gm, R=1)
    x = ctx.lanczos_vector(v, ref["alpha"], ref["beta"], c)
    assert rel(x, xr) <= 1e-10
    hx = np.zeros_like(x)
    om.p_mltply_v3(x, hx, 0.0)
    assert np.linalg.norm(hx - E[0] * x) <= 1e-10
    xd = ctx.lanczos_vector(torch.from_numpy(v).cuda(), ref["alpha"], ref["beta"], c)
    assert rel(xd.cpu().numpy(), xr) <= 1e-10


SECTOR_CASES = [
    # (L1, L2, q, tree, R): pure Heisenberg (Sz conserved, parity_type == 0), Sz = 0 sector
    (3, 2, 2, 0, 1),
    (3, 2, 2, 0, 4),
    (2, 4, 2, 1, 2),
    (3, 1, 3, 1, 1),
    (2, 2, 3, 1, 3),
]


@pytest.mark.parametrize("case", SECTOR_CASES, ids=[f"{c[0]}x{c[1]}q{c[2]}t{c[3]}R{c[4]}" for c in SECTOR_CASES])
def test_sector_hv_and_lanczos(case):
    """Sz-sector basis (mk_list12 order, Lin-table partner lookup): H.v to 1e-12 against
    the oracle's sector p_mltply_v3; Lanczos E0 equals the sector's oracle E0 and the
    full-basis ground-state energy (the Heisenberg ground state has Sz = 0)."""
    L1, L2, q, tree, R = case
    cl = honeycomb(L1, L2)
    cpl = CP.kitaev_heisenberg(1.0, 0.0)
    X, skip, pt = P.build_xlocal(q, tree, cpl)
    assert pt == 0
    gm = P.Model(cl.n, q, tree, cl.ipair, cl.ibond_type, X, skip, pt)
    om = O.Model(cl.n, q, tree, cl.ipair, cl.ibond_type, X, skip, pt)
    assert gm.dim == om.ldim and gm.dim < q ** cl.n
    list1, _, _ = P.mk_list12(cl.n, q, 0, cl.n // 2 * (q - 1))
    assert len(list1) == gm.dim
    ctx = P.Context(gm, R=R)
    rng = np.random.default_rng(5)
    D = gm.dim
    v1 = (rng.standard_normal((D, R)) + 1j * rng.standard_normal((D, R))).astype(np.complex128)
    v0 = (0.3 * rng.standard_normal((D, R))).astype(np.complex128)
    w = np.ascontiguousarray(v0).reshape(-1).copy()
    pr = ctx.p_mltply_v3(np.ascontiguousarray(v1).reshape(-1), w, 0.03125)
    w = w.reshape(D, R)
    for r in range(R):
        ref = np.ascontiguousarray(v0[:, r]).copy()
        prr = om.p_mltply_v3(np.ascontiguousarray(v1[:, r]), ref, 0.03125)
        assert rel(w[:, r], ref) <= 1e-12
        assert abs(pr[r] - prr) <= 1e-12 * abs(prr)
    v = O.gaussian(7, D)
    v /= np.linalg.norm(v)
    steps = min(60, D - 1)
    out = P.Context(gm, R=1).lanczos(v, steps)
    ref = om.lanczos(v, steps)
    assert abs(out["ene"][0] - ref["ene"][0]) <= 1e-10 * abs(ref["ene"][0])
    full = P.Model(cl.n, q, tree, cl.ipair, cl.ibond_type, X, skip, 1)
    vf = O.gaussian(8, full.dim)
    vf /= np.linalg.norm(vf)
    ef = P.Context(full, R=1).lanczos(vf, 120)["ene"][0]
    assert abs(out["ene"][0] - ef) <= 1e-8 * abs(ef)


@pytest.mark.parametrize("kind", ["lanczos", "tps"])
def test_session_checkpoint_resumes_exactly(kind, tmp_path):
    """A session saved after 9 steps and loaded into a fresh context continues
    exactly as the uninterrupted run (the role of interval_dump / _read)."""
    cl = honeycomb(3, 2)
    L = 2.0 * cl.n
    R = 2
    gm, _ = models(cl, 2, 0, KHGH, FIELD, tps_L=L if kind == "tps" else None)
    V = O.gaussian(41, gm.dim, R).reshape(gm.dim, R)
    V /= np.linalg.norm(V, axis=0)
    v = np.ascontiguousarray(V).reshape(-1)
    a = P.Context(gm, R=R)
    a.session_begin(kind, v, 25, L=L)
    a.session_step(20)
    full = a.session_read()
    a.session_end()
    b = P.Context(gm, R=R)
    b.session_begin(kind, v, 25, L=L)
    b.session_step(9)
    path = str(tmp_path / "session.ckpt")
    b.session_save(path)
    b.session_end()
    c = P.Context(gm, R=R)
    c.session_load(path, 25)
    c.session_step(11)
    resumed = c.session_read()
    assert np.array_equal(resumed["alpha"], full["alpha"]) and np.array_equal(resumed["beta"], full["beta"])
    if kind == "tps":
        assert np.array_equal(resumed["coef"], full["coef"])
    with pytest.raises(P.PnedError):
        P.Context(gm, R=1).session_load(path, 25)


@pytest.mark.parametrize("plan", [(8, 10, 4, 3, 1, 1), (5, 10, 2, 3, 1, 1), (3, 8, 1, 3, 1, 1), (5, 12, 2, 2, 1, 0),
                                  (5, 12, 2, 1, 0, 0), (8, 10, 4, 3, 1, 2), (5, 10, 2, 3, 1, 2), (3, 8, 1, 3, 1, 2),
                                  (5, 6, 3, 3, 1, 2), (8, 8, 2, 3, 1, 0, 3), (5, 10, 2, 3, 1, 0, 3),
                                  (5, 8, 2, 4, 1, 0), (8, 10, 4, 4, 1, 0), (3, 6, 1, 4, 0, 0),
                                  (5, 6, 2, 3, 1, 0, -1, 1), (5, 4, 2, 4, 1, 0, -1, 1), (5, 6, 2, 3, 1, 0, 3, 1),
                                  (5, 6, 2, 3, 1, 3, -1, 1), (5, 8, 2, 3, 1, 3, -1, 1), (5, 6, 3, 3, 0, 3, -1, 1),
                                  (5, 6, 2, 3, 1, 3, -1, 1, 2)])
def test_tile_plans_agree_with_oracle(plan):
    """Every tile plan the autotuner may pick (rows kept, window, passes, rows per
    thread, carveout, staged or bulk-streamed partner tiles, own rows by tensor
    copies, tiles that hold the most terms) gives the oracle's H.v to 1e-12."""
    cl = honeycomb(2, 4)
    gm, om = models(cl, 2, 0, KHGH, FIELD)
    got = gm.set_plan(1, *plan)
    assert got["tile_passes"] >= 1
    if plan[5] == 2:
        assert got["staging"] == 2 and got["ring_stages"] >= 2
    if plan[5] == 3:
        assert got["staging"] == 3
    ctx = P.Context(gm, R=1)
    rng = np.random.default_rng(23)
    v1 = rng.standard_normal(gm.dim) + 1j * rng.standard_normal(gm.dim)
    v0 = 0.1 * rng.standard_normal(gm.dim) + 0j
    w = v0.copy()
    pr = ctx.p_mltply_v3(v1, w, 0.0625)
    ref = v0.copy()
    prr = om.p_mltply_v3(v1, ref, 0.0625)
    assert rel(w, ref) <= 1e-12 and abs(pr[0] - prr) <= 1e-12 * abs(prr)
    v = O.gaussian(9, gm.dim)
    v /= np.linalg.norm(v)
    out = ctx.lanczos(v, 30)
    refl = om.lanczos(v, 30)
    assert rel(out["alpha"][:12, 0], refl["alpha"][:12]) <= 1e-10


@pytest.mark.parametrize("plan", [(5, 10, 2, 3), (8, 12, 1, 3), (3, 8, 3, 3)])
def test_bulk_streamed_tiles_match_gathered_tiles(plan):
    """N = 24 (8192 tiles, many per block, so the stage ring wraps across tiles):
    streaming the tiles with bulk copies gives the same W bit for bit as
    gathering the partner rows through L1/L2 with the same plan, and the same
    Lanczos coefficients to the summation order of the block sums."""
    cl = honeycomb(3, 4)
    gm, _ = models(cl, 2, 0, KHGH, FIELD)
    rng = np.random.default_rng(77)
    v1 = rng.standard_normal(gm.dim) + 1j * rng.standard_normal(gm.dim)
    v0 = 0.1 * (rng.standard_normal(gm.dim) + 1j * rng.standard_normal(gm.dim))
    v = O.gaussian(5, gm.dim)
    v /= np.linalg.norm(v)
    out = {}
    for stage in (0, 2):
        got = gm.set_plan(1, *plan, 1, stage)
        assert got["staging"] == stage
        ctx = P.Context(gm, R=1)
        w = v0.copy()
        pr = ctx.p_mltply_v3(v1, w, 0.0625)
        run = ctx.lanczos(v, 20)
        out[stage] = (w, pr, run["alpha"][:, 0], run["beta"][:, 0])
        ctx.close()
    assert np.array_equal(out[0][0], out[2][0])
    assert abs(out[0][1][0] - out[2][1][0]) <= 1e-12 * abs(out[0][1][0])
    assert rel(out[0][2], out[2][2]) <= 1e-12 and rel(out[0][3], out[2][3]) <= 1e-12
    gm.set_plan(1)


@pytest.mark.parametrize("plan", [(5, 6, 2, 3, 1, 3, -1, 1), (5, 8, 2, 3, 1, 3, -1, 1), (5, 4, 2, 3, 1, 3, -1, 1),
                                  (5, 6, 2, 3, 1, 3, -1, 1, 2)])
def test_tensor_copied_tiles_lanczos_tps_and_noalloc(plan):
    """N = 24, two passes: the tile kernel whose own rows, epilogue rows and
    diagonal arrive by tensor copies (stage 3) gives the oracle's H.v to 1e-12
    (and the gather kernel's with the same tiles; one or two out-of-tile terms
    in flight), the oracle's Lanczos and
    one-vector TPS coefficients to 1e-10 (the TPS pass forms the K = 4 sums),
    and the same H.v through the allocation-free entry point (static tile order)."""
    cl = honeycomb(3, 4)
    gm, om = models(cl, 2, 0, KHGH, FIELD)
    got = gm.set_plan(1, *plan)
    assert got["staging"] == 3 and got["tile_passes"] == 2
    rng = np.random.default_rng(31)
    v1 = rng.standard_normal(gm.dim) + 1j * rng.standard_normal(gm.dim)
    v0 = 0.1 * (rng.standard_normal(gm.dim) + 1j * rng.standard_normal(gm.dim))
    ctx = P.Context(gm, R=1)
    w = v0.copy()
    pr = ctx.p_mltply_v3(v1, w, 0.0625)
    ref = v0.copy()
    prr = om.p_mltply_v3(v1, ref, 0.0625)
    assert rel(w, ref) <= 1e-12 and abs(pr[0] - prr) <= 1e-12 * abs(prr)
    t1 = torch.from_numpy(v1).cuda()
    t0 = torch.from_numpy(v0).cuda()
    prn = P.hv_noalloc(gm, 1, t1, t0, 0.0625)
    torch.cuda.synchronize()
    assert rel(t0.cpu().numpy(), ref) <= 1e-12 and abs(prn[0] - prr) <= 1e-12 * abs(prr)
    v = O.gaussian(5, gm.dim)
    v /= np.linalg.norm(v)
    out = ctx.lanczos(v, 30)
    refl = om.lanczos(v, 30)
    assert rel(out["alpha"][:20, 0], refl["alpha"][:20]) <= 1e-10
    assert abs(out["ene"][0] - refl["ene"][0]) <= 1e-10 * abs(refl["ene"][0])
    ctx.close()
    gm.set_plan(1, *plan[:5], 0, *plan[6:])   # the same tiles gathered through L1/L2
    assert gm.plan(1)["staging"] == 0
    w0 = v0.copy()
    P.Context(gm, R=1).p_mltply_v3(v1, w0, 0.0625)
    assert rel(w, w0) <= 1e-13
    L = 2.0 * cl.n
    gt, ot = models(cl, 2, 0, KHGH, FIELD, tps_L=L)
    assert gt.set_plan(1, *plan)["staging"] == 3
    out = P.Context(gt, R=1).tps(L, v, 25)
    reft = ot.tps(L, v, 25)
    assert rel(out["beta"][:, 0], reft["beta"]) <= 1e-10
    assert rel(out["coef"][:, 0, :5], reft["coef"][:, :5]) <= 1e-10


@pytest.mark.parametrize("plan", [(5, 11, 2, 4), (8, 10, 3, 4)])
def test_sixteen_row_tiles_match_eight_row_tiles(plan):
    """N = 24 (4096 tiles of 4096 states): tiles of 16 rows a thread (two row
    chunks per gather) give the H.v of the default 8-row tiles to 1e-12 and the
    same Lanczos coefficients."""
    cl = honeycomb(3, 4)
    gm, _ = models(cl, 2, 0, KHGH, FIELD)
    rng = np.random.default_rng(31)
    v1 = rng.standard_normal(gm.dim) + 1j * rng.standard_normal(gm.dim)
    v0 = 0.1 * (rng.standard_normal(gm.dim) + 1j * rng.standard_normal(gm.dim))
    v = O.gaussian(3, gm.dim)
    v /= np.linalg.norm(v)
    out = []
    for pl in ((5, 12, 2, 3), plan):
        got = gm.set_plan(1, *pl)
        assert got["tile_states"] == 256 << pl[3]
        ctx = P.Context(gm, R=1)
        w = v0.copy()
        pr = ctx.p_mltply_v3(v1, w, 0.0625)
        run = ctx.lanczos(v, 20)
        out.append((w, pr[0], run["alpha"][:, 0], run["beta"][:, 0]))
        ctx.close()
    assert rel(out[1][0], out[0][0]) <= 1e-12
    assert abs(out[1][1] - out[0][1]) <= 1e-12 * abs(out[0][1])
    assert rel(out[1][2], out[0][2]) <= 1e-10 and rel(out[1][3], out[0][3]) <= 1e-10
    gm.set_plan(1)


def test_torch_tensors_written_just_before_the_call_are_ready():
    """The context runs on its own stream; a CUDA tensor that torch is still
    writing on its current stream (here behind a 10 ms GPU sleep) must be
    complete before the library reads or accumulates into it."""
    cl = honeycomb(3, 4)
    gm, _ = models(cl, 2, 0, KHGH, FIELD)
    ctx = P.Context(gm, R=1)
    rng = np.random.default_rng(5)
    v1h = rng.standard_normal(gm.dim) + 1j * rng.standard_normal(gm.dim)
    wh = np.full(gm.dim, 0.5 + 0.25j)
    ctx.p_mltply_v3(v1h, wh)
    v1 = torch.from_numpy(v1h).cuda()
    torch.cuda.synchronize()
    for _ in range(2):
        torch.cuda._sleep(20_000_000)
        w = torch.full_like(v1, 0.5 + 0.25j)
        ctx.p_mltply_v3(v1, w)
        assert np.array_equal(w.cpu().numpy(), wh)
    ctx.close()


@pytest.mark.parametrize("L1,L2", [(3, 4), (4, 3)])
def test_sector_segments_match_flat_gather(L1, L2):
    """S = 1/2 Heisenberg N = 24, Sz = 0 (2,704,156 states, segments of up to 924
    states): the per-segment H.v gives the flat gather's W bit for bit, the
    oracle's H.v to 1e-12, and Lanczos coefficients equal to the flat path's to
    the summation order of the block sums."""
    cl = honeycomb(L1, L2)
    X, skip, pt = P.build_xlocal(2, 0, CP.kitaev_heisenberg(1.0, 0.0))
    gm = P.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    assert gm.sector_segments() is True
    rng = np.random.default_rng(13)
    D = gm.dim
    v1 = rng.standard_normal(D) + 1j * rng.standard_normal(D)
    v0 = 0.2 * (rng.standard_normal(D) + 1j * rng.standard_normal(D))
    v = O.gaussian(11, D)
    v /= np.linalg.norm(v)
    out = {}
    for seg in (True, False):
        assert gm.sector_segments(seg) is seg
        ctx = P.Context(gm, R=1)
        w = v0.copy()
        pr = ctx.p_mltply_v3(v1, w, 0.0625)
        run = ctx.lanczos(v, 20)
        out[seg] = (w, pr[0], run["alpha"][:, 0], run["beta"][:, 0])
        ctx.close()
    gm.sector_segments(True)
    assert np.array_equal(out[True][0], out[False][0])
    assert abs(out[True][1] - out[False][1]) <= 1e-12 * abs(out[False][1])
    assert rel(out[True][2], out[False][2]) <= 1e-12 and rel(out[True][3], out[False][3]) <= 1e-12
    om = O.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    ref = v0.copy()
    prr = om.p_mltply_v3(v1, ref, 0.0625)
    assert rel(out[True][0], ref) <= 1e-12 and abs(out[True][1] - prr) <= 1e-12 * abs(prr)


def test_sector_segments_only_where_they_fill_a_block():
    """Segments shorter than one block (N = 12: at most 20 states) keep the flat gather."""
    cl = honeycomb(3, 2)
    X, skip, pt = P.build_xlocal(2, 0, CP.kitaev_heisenberg(1.0, 0.0))
    gm = P.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    assert gm.sector_segments() is False and gm.sector_segments(True) is False


XY_CASES = [
    # (L1, L2, q, tree, ipm, R, sector): S^{ipm}_q start vectors and DSF chains
    (3, 2, 2, 0, 1, 2, True),
    (3, 1, 3, 1, 1, 1, True),
    (3, 1, 3, 1, -1, 2, True),
    (2, 2, 2, 0, 1, 1, False),
]


@pytest.mark.parametrize("case", XY_CASES, ids=[f"{c[0]}x{c[1]}q{c[2]}ipm{c[4]}R{c[5]}{'s' if c[6] else 'f'}"
                                                 for c in XY_CASES])
def test_dsf_xy_chains(case):
    """DSF chains from S^{ipm}_q x (intalv_xy): x on the source sector, chains on the
    target sector (or both on the full basis); cnorm, salpha, sbeta follow the
    oracle's intalv_xy + parallelized_dsflnc1z."""
    L1, L2, q, tree, ipm, R, sector = case
    cl = honeycomb(L1, L2)
    n = cl.n
    cpl = CP.kitaev_heisenberg(1.0, 0.0) if sector else KH
    X, skip, pt = P.build_xlocal(q, tree, cpl)
    assert (pt == 0) == sector
    s0 = n // 2 * (q - 1)
    st = s0 + ipm if sector else s0
    gs = P.Model(n, q, tree, cl.ipair, cl.ibond_type, X, skip, pt, s0)
    gt = P.Model(n, q, tree, cl.ipair, cl.ibond_type, X, skip, pt, st)
    os_ = O.Model(n, q, tree, cl.ipair, cl.ibond_type, X, skip, pt, s0)
    ot = O.Model(n, q, tree, cl.ipair, cl.ibond_type, X, skip, pt, st)
    x = O.gaussian(13, gs.dim)
    x /= np.linalg.norm(x)
    qr = np.stack([cl.qr(r + 1) for r in range(R)])
    steps = 25
    out = P.Context(gt, R=R).dsf_xy(gs, x, qr, steps, ipm=ipm)
    if sector:   # a target that is not the neighbouring sector is refused before any kernel runs
        with pytest.raises(P.PnedError):
            P.Context(gs, R=R).dsf_xy(gs, x, qr, steps, ipm=ipm)
    for r in range(R):
        v, cn = ot.intalv_xy(os_, ipm, qr[r], x)
        sa, sb = ot.dsf_chain(v, cn, steps)
        assert abs(out["cnorm"][r] - cn.real) <= 1e-12 * cn.real
        assert rel(out["salpha"][:12, r], sa[:12]) <= 1e-10
        assert rel(out["sbeta"][:12, r], sb[:12]) <= 1e-10


def test_lanczos_breakdown_is_reported():
    """A start vector that is an eigenvector makes beta vanish after one step: the
    run returns PNED_EBREAKDOWN (the reference stops with #(E07), Lanczos.f90:126-130)."""
    X, skip, _ = P.build_xlocal(2, 0, CP.kitaev_heisenberg(1.0, 0.0))
    m = P.Model(2, 2, 0, np.array([1, 2]), np.array([3]), X, skip, 1)
    singlet = np.array([0, 1, -1, 0], dtype=np.complex128) / np.sqrt(2.0)
    with pytest.raises(P.PnedError) as ei:
        P.Context(m, R=1).lanczos(singlet, 5)
    assert ei.value.code == 4


def test_cg_inverse_iteration():
    cl = honeycomb(2, 2)
    gm, om = models(cl, 2, 0, KH)
    v = O.gaussian(3, gm.dim)
    v /= np.linalg.norm(v)
    e0 = om.lanczos(v, 100)["ene"][0]
    b = O.gaussian(8, gm.dim)
    b /= np.linalg.norm(b)
    ctx = P.Context(gm, R=1)
    x, ni, nc = ctx.cg(e0 - 1e-9, b, inv_max=30, cg_max=500)
    xr, _, _ = om.inverse_iteration(e0 - 1e-9, b, inv_max=30, cg_max=500)
    assert abs(abs(np.vdot(xr, x)) - 1) < 1e-9
    # residual of the eigenpair
    hx = np.zeros_like(x)
    om.p_mltply_v3(x, hx)
    assert np.linalg.norm(hx - e0 * x) < 1e-6


def test_larger_hv_parity_n24():
    cl = honeycomb(3, 4)
    gm, om = models(cl, 2, 0, KHGH, FIELD)
    v1 = O.gaussian(1, gm.dim)
    v0 = np.zeros(gm.dim, dtype=np.complex128)
    w = v0.copy()
    pr = P.Context(gm, R=1).p_mltply_v3(v1, w)
    prr = om.p_mltply_v3(v1, v0)
    assert rel(w, v0) <= 1e-12
    # prdct sums 2^24 terms with cancellation: bound the error by the absolute sum
    scale = np.sum(np.abs(v1) * np.abs(v0))
    assert abs(pr[0] - prr) <= 1e-12 * scale


@pytest.mark.parametrize("name", ["s12_kh_n8", "s12_khg_h111_n12", "s1_kh_n6", "s1_khg_h111_n8",
                                  "s12_heis_sz0_n12", "s12_heis_sz0_n16", "s1_heis_sz0_n8"])
def test_cuda_path_against_golden_fixtures(name):
    """The CUDA path, through the C ABI, reproduces the committed fixtures of
    tests/golden (H^T v and the ground-state energy from the independent dense
    construction)."""
    from tests.test_oracle import golden_case
    c = golden_case(name)
    X, skip, pt = P.build_xlocal(c["q"], c["tree"], c["cpl"], field=c["field"])
    m = P.Model(c["n"], c["q"], c["tree"], c["ipair"], c["btype"], X, skip, pt)
    ctx = P.Context(m, R=1)
    if "v" in c:
        w = np.zeros_like(c["v"])
        ctx.p_mltply_v3(np.ascontiguousarray(c["v"]), w)
        assert np.linalg.norm(w - c["w"]) <= 1e-12 * np.linalg.norm(c["w"])
    v = O.gaussian(3, m.dim)
    v /= np.linalg.norm(v)
    run = ctx.lanczos(v, 250, check_conv=True)
    assert abs(run["ene"][0] - c["e"][0]) <= 1e-10 * abs(c["e"][0])


@pytest.mark.parametrize("R", [2, 4, 12, 16])
@pytest.mark.parametrize("plan", [(0, 6, 2, -1, 1, 0, -1, 1), (1, 8, 2, -1, 1, 0, -1, 1), (0, 4, 3, -1, 1, 0, -1, 1)])
def test_multi_vector_plans_agree_with_oracle(plan, R):
    """The multi-vector kernel with tiles on the bits that hold the most flip terms
    (rows on any bits: a state's R values are one contiguous run) gives each
    column the oracle's H.v to 1e-12, and its TPS coefficients to 1e-10."""
    cl = honeycomb(2, 4)
    gm, om = models(cl, 2, 0, KHGH, FIELD)
    got = gm.set_plan(R, *plan)
    assert got["tile_passes"] >= 1
    ctx = P.Context(gm, R=R)
    rng = np.random.default_rng(41)
    D = gm.dim
    v1 = (rng.standard_normal((D, R)) + 1j * rng.standard_normal((D, R))).astype(np.complex128)
    v0 = (0.2 * rng.standard_normal((D, R)) + 0.1j * rng.standard_normal((D, R))).astype(np.complex128)
    w = np.ascontiguousarray(v0).reshape(-1).copy()
    pr = ctx.p_mltply_v3(np.ascontiguousarray(v1).reshape(-1), w, 0.0625)
    w = w.reshape(D, R)
    for r in range(R):
        ref = np.ascontiguousarray(v0[:, r]).copy()
        prr = om.p_mltply_v3(np.ascontiguousarray(v1[:, r]), ref, 0.0625)
        assert rel(w[:, r], ref) <= 1e-12
        assert abs(pr[r] - prr) <= 1e-12 * abs(prr)
    L = 2.0 * cl.n
    gt, ot = models(cl, 2, 0, KHGH, FIELD, tps_L=L)
    gt.set_plan(R, *plan)
    V = O.gaussian(13, gt.dim, R).reshape(gt.dim, R)
    V /= np.linalg.norm(V, axis=0)
    out = P.Context(gt, R=R).tps(L, np.ascontiguousarray(V).reshape(-1), 20)
    for r in (0, R - 1):
        ref = ot.tps(L, np.ascontiguousarray(V[:, r]), 20)
        assert rel(out["beta"][:, r], ref["beta"]) <= 1e-10
        assert rel(out["coef"][:, r, :5], ref["coef"][:, :5]) <= 1e-10


@pytest.mark.parametrize("plan", [(8, 10, 4, 3), (5, 6, 2, 3, 1, 0, -1, 1), (5, 6, 2, 3, 1, 3, -1, 1),
                                  (5, 6, 2, 3, 1, 3, -1, 1, 2)])
def test_complex_diagonal_tile_kernels(plan):
    """Local matrices with an imaginary part on their diagonal (the kernels'
    complex-diagonal form, which the Hermitian models of the configurations never
    reach) give the oracle's H.v to 1e-12, through the gather and the
    tensor-copy tile kernels, N = 24 (two passes)."""
    cl = honeycomb(3, 4)
    X, skip, pt = P.build_xlocal(2, 0, KHGH, field=FIELD)
    X = X.copy()
    for t in range(9):
        for i in range(4):
            X[t, i, i] += 0.01j * (i + 1) * (t + 1)
    gm = P.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    om = O.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    got = gm.set_plan(1, *plan)
    if len(plan) > 5 and plan[5] == 3:
        assert got["staging"] == 3
    rng = np.random.default_rng(41)
    v1 = rng.standard_normal(gm.dim) + 1j * rng.standard_normal(gm.dim)
    v0 = 0.1 * (rng.standard_normal(gm.dim) + 1j * rng.standard_normal(gm.dim))
    ctx = P.Context(gm, R=1)
    w = v0.copy()
    pr = ctx.p_mltply_v3(v1, w, 0.0625)
    ref = v0.copy()
    prr = om.p_mltply_v3(v1, ref, 0.0625)
    assert rel(w, ref) <= 1e-12 and abs(pr[0] - prr) <= 1e-12 * abs(prr)
