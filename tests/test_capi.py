"""CPU-side checks of the C ABI: the library loads, exports every symbol that
include/pned_gpu.h declares, and its host routines agree bit for bit with the
oracle's restatement of the reference."""
import os
import re

import numpy as np
import pytest

import pned_b200 as P
from oracle import oracle as O
from pned_b200 import couplings as CP

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


def test_errors_are_reported_not_fatal():
    with pytest.raises(P.PnedError):
        P.build_xlocal(3, 0, CP.model20(10.0))         # tree 0 needs q = 2
    with pytest.raises(P.PnedError):
        P.bisec(np.zeros(3), np.zeros(3), 3, 5)         # ne > ndim
    with pytest.raises(ValueError):
        P.build_xlocal(2, 0, np.zeros(5))
