"""Honeycomb cluster tables in the layout of pNED's ``set_bond_info``.

The reference hard-codes a few clusters (n = 8..32) as literal ``ipair`` /
``ibond_type`` / ``site_vec`` / ``q_list`` tables
(S_one_half/Hybrid_TPS_params.f90:344-1369).  The workloads this package is
measured on use periodic L1 x L2 clusters that are not among those tables, so
they are generated here with the site/bond convention

    site(x, y, sub) = 2*(x + L1*y) + sub          (0-based; ipair is 1-based)
    z-bond (type 3): A_r  - B_r
    x-bond (type 1): A_r  - B_{r - a1}
    y-bond (type 2): A_r  - B_{r - a2}

Bond types follow the reference's local-matrix slots: type 1 carries the
Kitaev term on S^x S^x (J1x), type 2 on S^y S^y (J1y), type 3 on S^z S^z (J1z)
(S_one_half/Hybrid_TPS_params.f90:1441-1451).

Geometry follows the reference's vectors (params.f90:365-372, 476-488): Bravais
vectors A1 = a1 + a2 = (1, 0), A2 = a1 + a3 = (1/2, sqrt(3)/2), the B
sublattice is displaced by a1 = (1/2, 1/(2 sqrt 3)) from A, and the allowed
momenta of the periodic cluster are q = (m1/L1) b1 + (m2/L2) b2 with
b_i . A_j = 2 pi delta_ij.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

_A1 = np.array([1.0, 0.0])
_A2 = np.array([0.5, math.sqrt(3.0) / 2.0])
_DELTA_B = np.array([0.5, 0.5 / math.sqrt(3.0)])


@dataclass
class Cluster:
    """One periodic honeycomb cluster, in reference table layout."""

    L1: int
    L2: int
    n: int
    ipair: np.ndarray        # int32 [2*nbond], 1-based site numbers (ipair of the reference)
    ibond_type: np.ndarray   # int32 [nbond], 1 = x, 2 = y, 3 = z
    site_vec: np.ndarray     # float64 [n, 2] real-space positions
    q_list: np.ndarray       # float64 [nq, 2] allowed momenta
    q_index: list = field(default_factory=list)  # (m1, m2) per momentum

    @property
    def nbond(self) -> int:
        return int(self.ibond_type.shape[0])

    def site_pairs0(self) -> np.ndarray:
        """Bond sites as 0-based (nbond, 2)."""
        return self.ipair.reshape(-1, 2).astype(np.int64) - 1

    def qr(self, iq: int) -> np.ndarray:
        """q.r_j for momentum iq and every site j (the phase of intalv_zz)."""
        return self.site_vec @ self.q_list[iq]


def honeycomb(L1: int, L2: int, shift: int = 0) -> Cluster:
    """Periodic L1 x L2 honeycomb cluster (n = 2*L1*L2 sites, 3*L1*L2 bonds).

    The torus identifies cell (x, y) with (x + L1, y) and with (x + shift,
    y + L2); shift = 0 is the plain rectangle.  Bonds are listed cell by cell
    (x fastest, then y), and within a cell in the order z, x, y.
    """
    if L1 < 1 or L2 < 1:
        raise ValueError("L1 and L2 must be >= 1")
    n = 2 * L1 * L2

    def site(x: int, y: int, sub: int) -> int:
        k = y // L2
        y -= k * L2
        x -= k * shift
        return 2 * ((x % L1) + L1 * y) + sub

    pairs, types = [], []
    for y in range(L2):
        for x in range(L1):
            a = site(x, y, 0)
            pairs.append((a, site(x, y, 1)))
            types.append(3)
            pairs.append((a, site(x - 1, y, 1)))
            types.append(1)
            pairs.append((a, site(x, y - 1, 1)))
            types.append(2)
    ipair = (np.asarray(pairs, dtype=np.int32) + 1).reshape(-1)
    ibond_type = np.asarray(types, dtype=np.int32)
    site_vec = np.zeros((n, 2))
    for y in range(L2):
        for x in range(L1):
            r = x * _A1 + y * _A2
            site_vec[site(x, y, 0)] = r
            site_vec[site(x, y, 1)] = r + _DELTA_B
    # reciprocal vectors: b_i . A_j = 2 pi delta_ij
    # allowed momenta: q.T1 and q.T2 in 2 pi Z, T1 = L1 A1, T2 = shift A1 + L2 A2
    tmat = np.stack([L1 * _A1, shift * _A1 + L2 * _A2])
    gmat = 2.0 * math.pi * np.linalg.inv(tmat).T   # reciprocal of the torus
    amat = np.stack([_A1, _A2])
    bmat = 2.0 * math.pi * np.linalg.inv(amat).T   # reciprocal of the lattice
    qs, qi = [], []
    seen = set()
    for m2 in range(-2 * (L1 * L2), 2 * (L1 * L2) + 1):
        for m1 in range(-2 * (L1 * L2), 2 * (L1 * L2) + 1):
            qv = m1 * gmat[0] + m2 * gmat[1]
            # fold into the first reciprocal cell
            c = np.linalg.solve(bmat.T, qv)
            c = c - np.floor(c + 1e-9)
            key = (round(c[0] * L1 * L2 * 4), round(c[1] * L1 * L2 * 4))
            if key in seen:
                continue
            seen.add(key)
            qs.append(c[0] * bmat[0] + c[1] * bmat[1])
            qi.append((float(c[0]), float(c[1])))
            if len(qs) == L1 * L2:
                break
        if len(qs) == L1 * L2:
            break
    order = sorted(range(len(qs)), key=lambda i: (round(qi[i][1], 9), round(qi[i][0], 9)))
    qs = [qs[i] for i in order]
    qi = [qi[i] for i in order]
    return Cluster(L1=L1, L2=L2, n=n, ipair=ipair, ibond_type=ibond_type,
                   site_vec=site_vec, q_list=np.asarray(qs), q_index=qi)


def _min_vector2(L1: int, L2: int, shift: int) -> float:
    best = float("inf")
    for m in range(-3, 4):
        for k in range(-3, 4):
            if m == 0 and k == 0:
                continue
            a = m * L1 + k * shift
            b = k * L2
            best = min(best, a * a + a * b + b * b)
    return best


def cluster_for_sites(n: int) -> Cluster:
    """The cluster used for an n-site workload.

    n = 18, 24, 30 are the 3 x 3, 3 x 4 and 3 x 5 rectangles of the measured
    configurations; other sizes use the rectangle or tilted torus whose
    shortest periodic vector is longest (ties: fewer rows).
    """
    fixed = {18: (3, 3, 0), 24: (3, 4, 0), 30: (3, 5, 0)}
    if n in fixed:
        return honeycomb(*fixed[n])
    if n < 2 or n % 2:
        raise ValueError(f"honeycomb clusters need an even number of sites, got {n}")
    cells = n // 2
    best = None
    for L2 in range(1, cells + 1):
        if cells % L2:
            continue
        L1 = cells // L2
        for s in range(L1):
            key = (_min_vector2(L1, L2, s), -L2, -s)
            if best is None or key > best[0]:
                best = (key, (L1, L2, s))
    return honeycomb(*best[1])
