"""Pins the CPU oracle (oracle/pned_oracle.c) against independent checks.

The reference ships no tests or golden vectors and cannot be compiled here (no
Fortran compiler), so these checks stand in: an independent dense Kronecker
construction of H, known analytic answers, and numpy/scipy for the
tridiagonal and continued-fraction routines.
"""
import math
import os

import numpy as np
import pytest

from oracle import oracle as O
from pned_b200 import couplings as CP
from pned_b200.lattice import honeycomb
from tests import dense


def _model(cl, q, tree_sa, cpl, field=None, tps_L=None):
    X = O.xlocal(q, tree_sa, cpl, field=field)
    skip, _, pt = O.parity_skip(q, tree_sa, X)
    if tps_L is not None:
        X = O.tps_explicit(q, cl.nbond, tps_L, X)
    return O.Model(cl.n, q, tree_sa, cl.ipair, cl.ibond_type, X, skip, pt), X, skip, pt


CASES = [
    # (L1, L2, q, tree_sa, couplings, field)
    (2, 2, 2, 0, CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi)), None),
    (2, 2, 2, 0, CP.kitaev_heisenberg(0.3, -1.0, gamma=0.1), CP.field_111(0.05)),
    (3, 2, 2, 0, CP.kitaev_heisenberg(-0.4, 0.7, gamma=0.25, gamma_p=-0.05), np.array([0.02, -0.03, 0.07])),
    (3, 1, 3, 1, CP.kitaev_heisenberg(0.2, -1.0), None),
    (3, 1, 3, 1, CP.kitaev_heisenberg(0.2, -1.0, gamma=0.1), CP.field_111(0.05)),
    (2, 1, 2, 1, CP.kitaev_heisenberg(0.5, 1.0, gamma=0.2), CP.field_111(0.1)),
]


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}x{c[1]}q{c[2]}t{c[3]}" for c in CASES])
def test_hv_is_dense_transpose(case):
    L1, L2, q, tree_sa, cpl, field = case
    cl = honeycomb(L1, L2)
    m, X, skip, pt = _model(cl, q, tree_sa, cpl, field)
    assert pt != 0 and m.ldim == q ** cl.n
    H = dense.sparse_h(cl.n, q, tree_sa, cl.ipair, cl.ibond_type, cpl, field)
    assert abs(H - H.conj().T).max() < 1e-14
    rng = np.random.default_rng(7)
    v = rng.standard_normal(m.ldim) + 1j * rng.standard_normal(m.ldim)
    w = 0.3 * rng.standard_normal(m.ldim) + 0j
    w0 = w.copy()
    pr = m.p_mltply_v3(v, w, eperbd=0.125)
    hv = H.T @ v - 0.125 * cl.nbond * v
    ref = w0 + hv
    assert np.linalg.norm(w - ref) <= 1e-13 * np.linalg.norm(ref)
    assert abs(pr - np.vdot(v, hv)) <= 1e-12 * abs(np.vdot(v, hv))


def test_lanczos_e0_vs_dense():
    cl = honeycomb(3, 2)
    cpl = CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi))
    m, X, skip, pt = _model(cl, 2, 0, cpl)
    H = dense.sparse_h(cl.n, 2, 0, cl.ipair, cl.ibond_type, cpl)
    import scipy.sparse.linalg as sla_s
    e = sla_s.eigsh(H, k=1, which="SA", tol=1e-14)[0]
    v = O.gaussian(3, m.ldim)
    v /= np.linalg.norm(v)
    r = m.lanczos(v, 150)
    assert r["rc"] == 0
    assert abs(r["ene"][0] - e[0]) < 1e-10 * abs(e[0])


def test_lanczos_convergence_stop():
    cl = honeycomb(2, 2)
    m, X, skip, pt = _model(cl, 2, 0, CP.model20(54.0))
    v = O.gaussian(11, m.ldim)
    v /= np.linalg.norm(v)
    r = m.lanczos(v, 1024, check_conv=True)
    H = dense.dense_h(cl.n, 2, 0, cl.ipair, cl.ibond_type, CP.model20(54.0))
    e = np.linalg.eigvalsh(H)
    assert r["itr"] < 1024 and r["itr"] % 5 == 0
    assert abs(r["ene"][0] - e[0]) < 1e-11 * abs(e[0])


def test_known_answers_dimer():
    # two sites joined by one z-bond: Heisenberg dimer E0 = -3/4 J (S=1/2), -2 J (S=1)
    ipair = np.array([1, 2], dtype=np.int32)
    bt = np.array([3], dtype=np.int32)
    for q, tree, e0 in [(2, 0, -0.75), (3, 1, -2.0), (2, 1, -0.75)]:
        cpl = CP.kitaev_heisenberg(1.0, 0.0)
        X = O.xlocal(q, tree, cpl)
        skip, _, pt = O.parity_skip(q, tree, X)
        # pure Heisenberg conserves Sz: parity 0 -> Sz sector total_sz = n/2*(q-1)
        assert pt == 0
        m = O.Model(2, q, tree, ipair, bt, X, skip, pt)
        Hc = np.zeros((m.ldim, m.ldim), dtype=complex)
        for k in range(m.ldim):
            e = np.zeros(m.ldim, dtype=complex)
            e[k] = 1
            w = np.zeros(m.ldim, dtype=complex)
            m.p_mltply_v3(e, w)
            Hc[:, k] = w
        ev = np.linalg.eigvalsh(Hc.T)
        assert abs(ev[0] - e0) < 1e-14


def test_kitaev_single_bond():
    ipair = np.array([1, 2], dtype=np.int32)
    bt = np.array([3], dtype=np.int32)
    cpl = CP.kitaev_heisenberg(0.0, 1.0)    # K S^z S^z only
    X = O.xlocal(2, 0, cpl)
    assert np.allclose(np.diag(X[2].T), [0.25, -0.25, -0.25, 0.25])


def test_sz_sector_lists():
    for n, q in [(8, 2), (9, 2), (6, 3), (5, 3)]:
        tot = n // 2 * (q - 1)
        list1, l3a, l3b = O.mk_list12(n, q, 0, tot)
        states = np.arange(q ** n)
        digsum = sum((states // q ** j) % q for j in range(n))
        want = states[digsum == tot]
        assert np.array_equal(list1, want)
        # Lin index round trip: list3(1,lo) + list3(2,hi) - 1 == position
        ihf = (n + 1) // 2
        lo = list1 % q ** ihf
        hi = list1 // q ** ihf
        assert np.array_equal(l3a[lo] + l3b[hi] - 1, np.arange(len(list1)))


def test_sz_sector_hv():
    cl = honeycomb(2, 2)
    cpl = CP.kitaev_heisenberg(1.0, 0.0)   # Heisenberg -> parity 0 -> Sz sector
    X = O.xlocal(2, 0, cpl)
    skip, _, pt = O.parity_skip(2, 0, X)
    assert pt == 0
    m = O.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    H = dense.dense_h(cl.n, 2, 0, cl.ipair, cl.ibond_type, cpl)
    list1, _, _ = O.mk_list12(cl.n, 2, 0, cl.n // 2)
    Hs = H[np.ix_(list1, list1)]
    rng = np.random.default_rng(1)
    v = rng.standard_normal(m.ldim) + 1j * rng.standard_normal(m.ldim)
    w = np.zeros(m.ldim, dtype=complex)
    m.p_mltply_v3(v, w)
    assert np.linalg.norm(w - Hs.T @ v) < 1e-13 * np.linalg.norm(w)


@pytest.mark.parametrize("q,tree,ipm", [(2, 0, 1), (3, 1, 1), (3, 1, -1), (4, 1, 1)])
def test_intalv_xy_vs_explicit_ladder(q, tree, ipm):
    """S^{ipm}_q x between Sz sectors (the DSF 'xx'/'uu'/'dd' start vector): the
    oracle equals the ladder operator applied state by state, with the
    spin-ladder factor sqrt((S -+ m)(S +- m + 1)) (1 for S = 1/2), summed over
    sites, then normalised; cnorm = ||v||^2 / n."""
    cl = honeycomb(2, 2) if q == 2 else honeycomb(3, 1)
    n = cl.n
    X = O.xlocal(q, tree, CP.kitaev_heisenberg(1.0, 0.0))
    skip, _, pt = O.parity_skip(q, tree, X)
    assert pt == 0
    s0 = n // 2 * (q - 1)
    ms = O.Model(n, q, tree, cl.ipair, cl.ibond_type, X, skip, pt, s0)
    mt = O.Model(n, q, tree, cl.ipair, cl.ibond_type, X, skip, pt, s0 + ipm)
    src, _, _ = O.mk_list12(n, q, 0, s0)
    tgt, _, _ = O.mk_list12(n, q, 0, s0 + ipm)
    where = {int(t): i for i, t in enumerate(tgt)}
    rng = np.random.default_rng(3)
    x = rng.standard_normal(ms.ldim) + 1j * rng.standard_normal(ms.ldim)
    qr = rng.uniform(-math.pi, math.pi, n)
    S = 0.5 * (q - 1)
    ref = np.zeros(mt.ldim, dtype=complex)
    for j in range(n):
        for i, st in enumerate(src):
            d = (int(st) // q ** j) % q
            if not 0 <= d + ipm < q:
                continue
            m_ = d - S
            fac = math.sqrt((S - m_) * (S + m_ + 1)) if ipm == 1 else math.sqrt((S + m_) * (S - m_ + 1))
            ref[where[int(st) + ipm * q ** j]] += fac * np.exp(1j * qr[j]) * x[i]
    raw = np.vdot(ref, ref).real
    v, cn = mt.intalv_xy(ms, ipm, qr, x)
    assert np.linalg.norm(v - ref / math.sqrt(raw)) <= 1e-13
    assert abs(cn - raw / n) <= 1e-12 * raw / n


def test_bisec_vec12_vs_numpy():
    rng = np.random.default_rng(3)
    for nd in [5, 40, 300]:
        a = rng.standard_normal(nd)
        b = np.abs(rng.standard_normal(nd)) + 0.1
        T = np.diag(a) + np.diag(b[:-1], 1) + np.diag(b[:-1], -1)
        ev, evec = np.linalg.eigh(T)
        ne = min(8, nd)
        E = O.bisec(a, b, nd, ne)
        assert np.allclose(E, ev[:ne], atol=1e-12 * max(1, abs(ev).max()))
        V = O.vec12(a, b, E, nd, 1)
        assert abs(abs(V[0] @ evec[:, 0]) - 1) < 1e-10


def test_renbun_vs_direct_fraction():
    rng = np.random.default_rng(5)
    M = 30
    sa = rng.standard_normal(M)
    sb = np.abs(rng.standard_normal(M + 1)) + 0.2
    e0, eta, split, nw = -1.3, 0.05, 3.0 / 1999, 2000
    w, conv, dsf = O.exec_renbun(nw, 4096, split, e0, eta, sa, sb)
    # The reference arrays are zero padded, so the fraction runs one level past
    # the chain (alpha = 0, beta = sb[M]) and stops where beta = 0:
    #   f = a1/(b1 + a2/(b2 + ... a_{M+1}/b_{M+1})), a_m = -sb[m-1]^2,
    #   b_m = omega + e0 - sa[m-1] + i eta.
    for j in [0, 100, 999, 1999]:
        z = w[j] + e0 + 1j * eta
        f = 0j
        for m in range(M + 1, 1, -1):
            am = -(sb[m - 1] ** 2)
            bm = z - (sa[m - 1] if m - 1 < M else 0.0)
            f = am / (bm + f)
        direct = -(sb[0] ** 2) / (z - sa[0] + f)
        assert abs(dsf[j] - direct.imag) < 1e-9 * max(1.0, abs(direct.imag))
        assert 0 < conv[j] <= M + 2


def test_gaussian_stats():
    v = O.gaussian(20261203, 1 << 16)
    assert abs(np.mean(np.abs(v) ** 2) - 1) < 0.02
    assert abs(np.mean(v)) < 0.02
    v2 = O.gaussian(20261203, 1 << 16)
    assert np.array_equal(v, v2)
    assert not np.array_equal(v, O.gaussian(1, 1 << 16))


def test_tps_vs_dense_recurrence():
    cl = honeycomb(2, 2)
    cpl = CP.kitaev_heisenberg(0.3, -1.0, gamma=0.1)
    fld = CP.field_111(0.05)
    L = 2.0 * cl.n
    m, X, skip, pt = _model(cl, 2, 0, cpl, fld, tps_L=L)
    H = dense.dense_h(cl.n, 2, 0, cl.ipair, cl.ibond_type, cpl, fld)
    A = (L * np.eye(m.ldim) - H).T          # the reference applies (L - H)^T
    v = O.gaussian(9, m.ldim)
    v /= np.linalg.norm(v)
    r = m.tps(L, v, 20)
    x = v.copy()
    for i in range(20):
        y = A @ x
        alpha1 = np.vdot(x, y).real
        beta1 = np.linalg.norm(y)
        assert abs(r["alpha"][i] - (L - alpha1)) < 1e-11 * L
        assert abs(r["beta"][i] - beta1) < 1e-11 * beta1
        assert abs(r["coef"][i, 0] - 2 * (i + 1) / alpha1) < 1e-11
        x = y / beta1


def test_dsf_chain_vs_dense():
    cl = honeycomb(2, 2)
    cpl = CP.model20(54.0)
    m, X, skip, pt = _model(cl, 2, 0, cpl)
    H = dense.dense_h(cl.n, 2, 0, cl.ipair, cl.ibond_type, cpl)
    ev, evec = np.linalg.eigh(H)
    gs = evec[:, 0].conj()  # ground state of H^T = conj(H)
    qr = cl.qr(1)
    v, cn = m.intalv_zz(qr, gs)
    # dense S^z_q: bit 1 -> +1/2 in intalv_zz (S1/2 tree)
    states = np.arange(m.ldim)
    w = np.zeros(m.ldim, dtype=complex)
    for j in range(cl.n):
        w += (((states >> j) & 1) - 0.5) * np.exp(1j * qr[j])
    raw = w * gs
    assert abs(cn - np.vdot(raw, raw) / cl.n) < 1e-13
    assert np.allclose(v, raw / np.linalg.norm(raw), atol=1e-14)
    sa, sb = m.dsf_chain(v, cn, 12)
    # plain Lanczos with the same recurrence on dense H^T
    A = H.T
    v1, v0p, beta_prev = v.copy(), np.zeros_like(v), 0.0
    for i in range(12):
        y = A @ v1 - beta_prev * v0p
        a = np.vdot(v1, A @ v1).real
        y = y
        rr = y - a * v1
        b = np.linalg.norm(rr)
        assert abs(sa[i] - a) < 1e-11 * max(1, abs(a))
        assert abs(sb[i + 1] - b) < 1e-10 * max(1, b)
        v0p, v1, beta_prev = v1, rr / b, b


def test_inverse_iteration_ground_state():
    cl = honeycomb(2, 2)
    cpl = CP.model20(54.0)
    m, X, skip, pt = _model(cl, 2, 0, cpl)
    H = dense.dense_h(cl.n, 2, 0, cl.ipair, cl.ibond_type, cpl)
    ev, evec = np.linalg.eigh(H.T)
    b = O.gaussian(5, m.ldim)
    b /= np.linalg.norm(b)
    # the reference shifts by the Lanczos E0; a tiny offset keeps (H - E) regular
    x, ni, nc = m.inverse_iteration(ev[0] - 1e-9, b, inv_max=50, cg_max=500)
    assert abs(abs(np.vdot(evec[:, 0], x)) - 1) < 1e-8


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")
GOLDEN_CASES = ["s12_kh_n8", "s12_khg_h111_n12", "s1_kh_n6", "s1_khg_h111_n8",
                "s12_heis_sz0_n12", "s12_heis_sz0_n16", "s1_heis_sz0_n8"]


def golden_case(name):
    g = np.load(GOLDEN)
    q, tree, n = (int(x) for x in g[f"{name}/q"])
    fld = g[f"{name}/field"] if bool(g[f"{name}/has_field"][0]) else None
    case = dict(q=q, tree=tree, n=n, ipair=g[f"{name}/ipair"], btype=g[f"{name}/btype"],
                cpl=g[f"{name}/couplings"], field=fld, e=g[f"{name}/e"])
    if f"{name}/v" in g:
        case["v"], case["w"] = g[f"{name}/v"], g[f"{name}/w"]
    return case


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_against_golden_fixtures(name):
    """The oracle reproduces the committed fixtures of tests/golden (H^T v and the
    ground-state energy from the independent dense construction)."""
    c = golden_case(name)
    X = O.xlocal(c["q"], c["tree"], c["cpl"], field=c["field"])
    skip, _, pt = O.parity_skip(c["q"], c["tree"], X)
    m = O.Model(c["n"], c["q"], c["tree"], c["ipair"], c["btype"], X, skip, pt)
    if "v" in c:
        w = np.zeros_like(c["v"])
        m.p_mltply_v3(np.ascontiguousarray(c["v"]), w)
        assert np.linalg.norm(w - c["w"]) <= 1e-12 * np.linalg.norm(c["w"])
    v = O.gaussian(3, m.ldim)
    v /= np.linalg.norm(v)
    run = m.lanczos(v, 250, check_conv=True)
    assert abs(run["ene"][0] - c["e"][0]) <= 1e-10 * abs(c["e"][0])
