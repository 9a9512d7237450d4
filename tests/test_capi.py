"""CPU-side checks of the C ABI: the library loads, exports every symbol that
include/pned_gpu.h declares, and its host routines agree bit for bit with the
oracle's restatement of the reference."""
import math
import os
import re

import numpy as np
import pytest

import pned_b200 as P
from oracle import oracle as O
from pned_b200 import couplings as CP
from pned_b200.lattice import honeycomb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "pned_gpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(pned_\w+)\s*\(", src, flags=re.M)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = P.lib()
    names = _declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.pned_abi_version() == 1


COUPLINGS = [
    (2, 0, CP.kitaev_heisenberg(0.3, -1.0, gamma=0.1), CP.field_111(0.05)),
    (2, 0, CP.model20(54.0), None),
    (2, 0, CP.slots(J1=0.4, K1=-0.3, I11=0.2, I12=-0.1, J1p=0.7, K1p=1.1, J1pp=-0.5, I11p=0.05, I12p=0.3,
                    I12pp=-0.2, J2=0.15, K2=0.25, I21=0.01, I22=0.02, J3=0.3, ratio_l=0.8), [0.01, 0.02, 0.03]),
    (3, 1, CP.kitaev_heisenberg(0.2, -1.0), None),
    (3, 1, CP.kitaev_heisenberg(0.2, -1.0, gamma=0.1), CP.field_111(0.05)),
    (4, 1, CP.kitaev_heisenberg(-0.3, 0.6, gamma=0.2), None),
    (2, 1, CP.model0(0.2), None),
]


@pytest.mark.parametrize("q,tree,cpl,fld", COUPLINGS)
@pytest.mark.parametrize("simple", [0, 3])
def test_build_xlocal_matches_oracle(q, tree, cpl, fld, simple):
    X, skip, pt = P.build_xlocal(q, tree, cpl, simple=simple, field=fld)
    Xo = O.xlocal(q, tree, cpl, simple=simple, field=fld)
    so, _, pto = O.parity_skip(q, tree, Xo)
    assert np.array_equal(X, Xo)
    assert np.array_equal(skip, so)
    assert pt == pto
    for L in (None, 48.0):
        Xt, Lt = P.tps_transform(q, tree, 36, X, L=L)
        if L is None:
            Xto, Lto = O.tps_reference(q, tree, 36, Xo)
            assert Lt == Lto
        else:
            Xto = O.tps_explicit(q, 36, L, Xo)
        assert np.array_equal(Xt, Xto)


def test_tridiagonal_and_fraction_match_oracle():
    rng = np.random.default_rng(2)
    for nd in (1, 2, 7, 64, 700):
        a = rng.standard_normal(nd)
        b = np.abs(rng.standard_normal(nd)) + 0.05
        ne = min(8, nd)
        E = P.bisec(a, b, nd, ne)
        assert np.array_equal(E, O.bisec(a, b, nd, ne))
        assert np.array_equal(P.vec12(a, b, E, nd, min(3, nd)), O.vec12(a, b, E, nd, min(3, nd)))
    sa = rng.standard_normal(150)
    sb = np.abs(rng.standard_normal(151)) + 0.1
    for s_max in (152, 4096):
        w, c, d = P.exec_renbun(2000, s_max, 3.0 / 1999, -2.5, 0.05, sa, sb)
        w2, c2, d2 = O.exec_renbun(2000, s_max, 3.0 / 1999, -2.5, 0.05, sa, sb)
        assert np.array_equal(d, d2) and np.array_equal(c, c2) and np.array_equal(w, w2)
    dn = P.normalize_dsf(2000, 3.0 / 1999, 0.37, d)
    assert np.array_equal(dn, O.normalization_dsf(2000, 3.0 / 1999, 0.37, d))


@pytest.mark.parametrize("n,q", [(8, 2), (9, 2), (6, 3), (7, 3), (5, 4)])
def test_mk_list12_matches_oracle(n, q):
    tot = n // 2 * (q - 1)
    l1, lo, hi = P.mk_list12(n, q, 0, tot)
    o1, olo, ohi = O.mk_list12(n, q, 0, tot)
    assert np.array_equal(l1, o1)
    assert np.array_equal(lo[:len(olo)], olo) and np.array_equal(hi[:len(ohi)], ohi)


@pytest.mark.parametrize("n,tot", [(12, 6), (15, 7), (16, 5), (22, 11)])
def test_sector_segments_layout(n, tot):
    """The layout the S = 1/2 segment H.v relies on: the sector states sharing a
    high half form one contiguous segment, in ascending order, of C(ihf, tot -
    popcount(hi)) states; a state's index is lin_hi[hi] + rank with rank =
    lin_lo[lo] - 1; and for every Sz-conserving two-site flip the segment
    formulas (high-half flips: same rank in segment hi ^ mh; low-half or cross
    flips: rank of lo ^ ml) give the flat Lin index of the flipped state."""
    l1, lo_t, hi_t = P.mk_list12(n, 2, 0, tot)
    ihf = (n + 1) // 2
    lo = l1 & ((1 << ihf) - 1)
    hi = l1 >> ihf
    idx = np.arange(len(l1))
    assert np.all(np.diff(l1) > 0)
    starts = np.flatnonzero(np.r_[True, np.diff(hi) != 0])
    assert np.array_equal(hi[starts], np.unique(hi))
    lens = np.diff(np.r_[starts, len(l1)])
    pc = np.array([bin(int(h)).count("1") for h in hi[starts]])
    assert np.array_equal(lens, [math.comb(ihf, tot - p) for p in pc])
    assert np.array_equal(hi_t[hi[starts]], starts)
    rank = lo_t[lo] - 1
    assert np.array_equal(idx, hi_t[hi] + rank)
    assert np.array_equal(rank, idx - np.repeat(starts, lens))
    pos = {int(s): i for i, s in enumerate(l1)}
    rng = np.random.default_rng(n)
    for a, b in rng.integers(0, n, size=(40, 2)):
        if a == b:
            continue
        m = (1 << int(a)) | (1 << int(b))
        ml, mh = m & ((1 << ihf) - 1), m >> ihf
        ok = ((l1 >> a) & 1) != ((l1 >> b) & 1)          # the flip keeps Sz
        part = np.array([pos[int(s) ^ m] for s in l1[ok]])
        r = np.where(ml == 0, rank[ok], lo_t[lo[ok] ^ ml] - 1)
        base = hi_t[hi[ok] ^ mh]
        assert np.array_equal(base + r, part)


def test_errors_are_reported_not_fatal():
    with pytest.raises(P.PnedError):
        P.build_xlocal(3, 0, CP.model20(10.0))         # tree 0 needs q = 2
    with pytest.raises(P.PnedError):
        P.bisec(np.zeros(3), np.zeros(3), 3, 5)         # ne > ndim
    with pytest.raises(ValueError):
        P.build_xlocal(2, 0, np.zeros(5))


# --------------------------------------------------------------------------- mTPQ output chain

def test_salphasbeta_file_layout_and_round_trip(tmp_path):
    import struct
    n1, n2 = 7, 5
    rng = np.random.default_rng(3)
    a, b = rng.standard_normal(n1), rng.standard_normal(n1)
    c = rng.standard_normal((n1, n2))
    path = str(tmp_path / "SalphaSbeta_me00000seed00001zz")
    P.api.write_salphasbeta(path, a, b, c)

    def rec(payload):
        return struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload))
    expect = (rec(struct.pack("<i", n1)) + rec(struct.pack("<i", n2)) + rec(a.astype("<f8").tobytes()) +
              rec(b.astype("<f8").tobytes()) + rec(np.asfortranarray(c).T.astype("<f8").tobytes()))
    assert open(path, "rb").read() == expect
    a2, b2, c2 = P.api.read_salphasbeta(path)
    assert np.array_equal(a2, a) and np.array_equal(b2, b) and np.array_equal(c2, c)
    with open(path, "r+b") as f:
        f.seek(4 + 4 + 4 + 4 + 4 + 4)   # corrupt the first alpha record's length
        f.write(struct.pack("<i", 3))
    with pytest.raises(P.PnedError):
        P.api.read_salphasbeta(path)


def test_tpq_thermo_matches_oracle():
    """eval_mpi on oracle mTPQ runs: the library equals the numpy restatement to
    1e-12; its E(T) rises with T and tends to the exact ground-state energy at
    low T.  (Its weights carry bt/(2i) per factor, eval_mpi.f90:249, so at finite
    T it does not reproduce the exact canonical energy; mirrored as it is.)"""
    from dense import dense_h
    cl = honeycomb(3, 2)
    cpl = CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi))
    L = 2.0 * cl.n
    X = O.xlocal(2, 0, cpl)
    skip, _, pt = O.parity_skip(2, 0, X)
    Xt = O.tps_explicit(2, cl.nbond, L, X)
    om = O.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, Xt, skip, pt)
    steps = 150
    runs = []
    for seed in (1, 2):
        v = O.gaussian(seed, om.ldim)
        v /= np.linalg.norm(v)
        runs.append(om.tps(L, v, steps))
    beta = np.stack([r["beta"] for r in runs])
    energy = np.stack([r["coef"][:, 3] for r in runs])
    hmix = np.stack([r["coef"][:, 4] for r in runs])
    got = P.api.tpq_thermo(beta, energy, hmix, 0.05, 10.0, 12)
    ref = O.tpq_thermo(beta, energy, hmix, 0.05, 10.0, 12)
    assert np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)) <= 1e-12
    assert np.allclose(got[:, 0], np.exp(np.linspace(math.log(0.05), math.log(10.0), 13)), rtol=1e-12)
    assert np.all(np.diff(got[:, 1]) > 0) and np.all(got[:, 2] > 0) and np.all(got[:, 3] >= -1e-12)
    e0 = np.linalg.eigvalsh(dense_h(cl.n, 2, 0, cl.ipair, cl.ibond_type, cpl))[0]
    assert abs(got[0, 1] - e0) <= 0.02 * abs(e0)


def test_vector_and_dsf_files_layout(tmp_path):
    import struct

    def rec(payload):
        return struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload))
    rng = np.random.default_rng(8)
    x = rng.standard_normal(37) + 1j * rng.standard_normal(37)
    p = str(tmp_path / "basisme00000")
    P.api.write_vec_data(p, -3.25, x)
    assert open(p, "rb").read() == rec(struct.pack("<d", -3.25)) + rec(x.astype("<c16").tobytes())
    e, x2 = P.api.read_vec_data(p, 37)
    assert e == -3.25 and np.array_equal(x2, x)
    with pytest.raises(P.PnedError):
        P.api.read_vec_data(p, 36)
    sa, sb = rng.standard_normal(12), rng.standard_normal(12)
    q = str(tmp_path / "SalphaSbeta_q00003me00000zz")
    P.api.write_dsf_alpha_beta(q, 0.5 - 0.25j, sa, sb)
    assert open(q, "rb").read() == (rec(struct.pack("<dd", 0.5, -0.25)) + rec(sa.astype("<f8").tobytes()) +
                                    rec(sb.astype("<f8").tobytes()))
    sq, sa2, sb2 = P.api.read_dsf_alpha_beta(q, 12)
    assert sq == 0.5 - 0.25j and np.array_equal(sa2, sa) and np.array_equal(sb2, sb)


def test_long_records_are_written_as_fortran_subrecords(tmp_path):
    """Records longer than one subrecord (from N = 27 on, a vector is above
    gfortran's 2^31 - 9 bytes) are split as gfortran splits them: each
    subrecord framed by its length, the leading marker negative when another
    follows, the trailing marker negative when one precedes.  A small limit
    stands in for 2^31 - 9 bytes here."""
    import struct

    def subrecords(payload, limit):
        out, off, n = b"", 0, len(payload)
        while True:
            k = min(limit, n - off)
            lead = -k if off + k < n else k
            tail = k if off == 0 else -k
            out += struct.pack("<i", lead) + payload[off:off + k] + struct.pack("<i", tail)
            off += k
            if off >= n:
                return out
    rng = np.random.default_rng(21)
    x = rng.standard_normal(10) + 1j * rng.standard_normal(10)
    v2 = rng.standard_normal(10) + 1j * rng.standard_normal(10)
    try:
        for limit in (48, 40, 160, 7):
            P.api.set_max_subrecord(limit)
            p = str(tmp_path / f"basisme{limit:05d}")
            P.api.write_vec_data(p, 1.5, x)
            want = subrecords(struct.pack("<d", 1.5), limit) + subrecords(x.astype("<c16").tobytes(), limit)
            assert open(p, "rb").read() == want, limit
            P.api.set_max_subrecord()
            e, x2 = P.api.read_vec_data(p, 10)   # readers take any split
            assert e == 1.5 and np.array_equal(x2, x)
            with pytest.raises(P.PnedError):
                P.api.read_vec_data(p, 9)
        P.api.set_max_subrecord(64)
        q = str(tmp_path / "vec_q00001me00000zz")
        P.api.write_dsf_vectors(q, 7, x, v2)
        assert open(q, "rb").read() == (subrecords(struct.pack("<i", 7), 64) + subrecords(x.astype("<c16").tobytes(), 64)
                                        + subrecords(v2.astype("<c16").tobytes(), 64))
        i, a, b = P.api.read_dsf_vectors(q, 10)
        assert i == 7 and np.array_equal(a, x) and np.array_equal(b, v2)
        # a trailing marker whose sign disagrees with the split is refused
        raw = bytearray(open(q, "rb").read())
        off = 12 + (4 + 64 + 4) + 4 + 64   # record 1, then the trailing marker of record 2's second subrecord
        struct.pack_into("<i", raw, off, 64)
        open(q, "wb").write(bytes(raw))
        with pytest.raises(P.PnedError):
            P.api.read_dsf_vectors(q, 10)
        with pytest.raises(P.PnedError):
            P.api.set_max_subrecord(0)
    finally:
        P.api.set_max_subrecord()


def test_dsf_vectors_file_and_sq_line(tmp_path):
    import struct

    def rec(payload):
        return struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload))
    rng = np.random.default_rng(12)
    v1 = rng.standard_normal(19) + 1j * rng.standard_normal(19)
    v2 = rng.standard_normal(19) + 1j * rng.standard_normal(19)
    p = str(tmp_path / "vec_q00002me00000xx")
    P.api.write_dsf_vectors(p, 41, v1, v2)
    assert open(p, "rb").read() == (rec(struct.pack("<i", 41)) + rec(v1.astype("<c16").tobytes()) +
                                    rec(v2.astype("<c16").tobytes()))
    i, a, b = P.api.read_dsf_vectors(p, 19)
    assert i == 41 and np.array_equal(a, v1) and np.array_equal(b, v2)
    with pytest.raises(P.PnedError):
        P.api.read_dsf_vectors(p, 18)
    s = str(tmp_path / "sq.txt")
    P.api.append_sq(s, 3, [0.5, -2.25], 0.0625)
    P.api.append_sq(s, 12, [-1.0, 3.0], 1.5)
    # '(A,I3,2F12.6,F25.18)' as the DSF driver writes it
    assert open(s).read().split("\n")[:2] == [" q =   3    0.500000   -2.250000     0.062500000000000000",
                                               " q =  12   -1.000000    3.000000     1.500000000000000000"]


def test_dsf_res_text_block(tmp_path):
    p = str(tmp_path / "dsf_res_zz")
    P.api.append_dsf_res(p, 0.75, [0.5, -1.25], [0.0, 1.5], [2.0, 0.125], [3, 4])
    P.api.append_dsf_res(p, 0.5, [0.0, 0.0], [0.25], [1.0], [1])
    lines = open(p).read().split("\n")
    assert lines[0] == "#        " + "%25.18f" % 0.75
    assert lines[1] == "%18.10f%18.10f%25.16f%25.16f%5d" % (0.5, -1.25, 0.0, 2.0, 3)
    assert lines[2] == "%18.10f%18.10f%25.16f%25.16f%5d" % (0.5, -1.25, 1.5, 0.125, 4)
    assert lines[3:7] == [" "] * 4 and lines[7].startswith("#")


def test_sector_model_must_conserve_sz():
    """parity_type 0 (Sz sector basis, Lin-table partners) is refused for a model
    whose nonzero elements change Sz; the refusal comes before any device work."""
    from pned_b200.lattice import honeycomb
    cl = honeycomb(2, 2)
    for q, tree in ((2, 0), (3, 1)):
        X, skip, pt = P.build_xlocal(q, tree, CP.kitaev_heisenberg(0.3, -1.0))
        assert pt != 0
        with pytest.raises(P.PnedError, match="changes Sz"):
            P.Model(cl.n, q, tree, cl.ipair, cl.ibond_type, X, skip, 0)


def test_rejects_bad_arguments():
    with pytest.raises(ValueError):
        P.build_xlocal(2, 0, np.zeros(5))
    with pytest.raises(P.PnedError):
        P.api.tpq_thermo(np.ones((1, 4)), np.ones((1, 4)), np.ones((1, 4)), -1.0, 2.0, 4)
    with pytest.raises(P.PnedError):
        P.api.read_salphasbeta("/nonexistent/file")
    with pytest.raises(P.PnedError):
        P.mk_list12(0, 2, 0, 0)
    with pytest.raises(P.PnedError):
        P.bisec(np.ones(3), np.ones(3), 0, 1)
