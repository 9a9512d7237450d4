"""Generates tests/golden/golden.npz: frozen H.v products and low eigenvalues of
small pNED models, computed with the independent Kronecker-product
construction of tests/dense.py (numpy / scipy; it shares no indexing code with
the oracle or the library).  The reference ships no golden vectors, so these
fixtures pin the oracle (CPU tests) and the CUDA path (GPU tests) to values
that stay fixed across changes.

    python -m tests.golden.make_golden      (from the repository root)

Cases above 4096 states take their eigenvalues from the iterative eigsh, whose
last bits (about 1e-15 relative) can differ between runs; the committed file
keeps the values of its first generation.

Each case stores the lattice (1-based ipair, bond types), the coupling slots and
field, a seeded input vector v and w = H^T v (the reference's p_mltply_v3
convention, eperbd = 0), and the four lowest eigenvalues of H.  The Sz-sector
cases restrict H to the states of the sector's digit sum, in ascending order.
"""
import math
import os

import numpy as np
import scipy.sparse.linalg as sla

from pned_b200 import couplings as CP
from pned_b200.lattice import honeycomb
from tests import dense

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = {
    # name: (L1, L2, q, tree, couplings, field, store v/w)
    "s12_kh_n8": (2, 2, 2, 0, CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi)), None, True),
    "s12_khg_h111_n12": (3, 2, 2, 0, CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi),
                                                            gamma=0.1), CP.field_111(0.05), True),
    "s1_kh_n6": (3, 1, 3, 1, CP.kitaev_heisenberg(0.2, -1.0), None, True),
    "s1_khg_h111_n8": (2, 2, 3, 1, CP.kitaev_heisenberg(0.2, -1.0, gamma=0.1), CP.field_111(0.05), False),
}
# Heisenberg models conserve Sz (parity_type 0): the Sz = 0 sector, states of digit
# sum n/2 * (q - 1) in ascending order (the reference's mk_list12 order)
SECTOR_CASES = {
    "s12_heis_sz0_n12": (3, 2, 2, 0, CP.kitaev_heisenberg(1.0, 0.0)),
    "s12_heis_sz0_n16": (2, 4, 2, 0, CP.kitaev_heisenberg(1.0, 0.0)),
    "s1_heis_sz0_n8": (2, 2, 3, 1, CP.kitaev_heisenberg(1.0, 0.0)),
}


def main():
    out = {}
    for name, (L1, L2, q, tree, cpl, fld, store_v) in CASES.items():
        cl = honeycomb(L1, L2)
        H = dense.sparse_h(cl.n, q, tree, cl.ipair, cl.ibond_type, cpl, fld)
        D = H.shape[0]
        if D <= 4096:
            e = np.linalg.eigvalsh(H.toarray())[:4]
        else:
            e = np.sort(sla.eigsh(H, k=4, which="SA", tol=1e-14)[0])
        out[f"{name}/q"] = np.array([q, tree, cl.n])
        out[f"{name}/ipair"] = np.asarray(cl.ipair, dtype=np.int32)
        out[f"{name}/btype"] = np.asarray(cl.ibond_type, dtype=np.int32)
        out[f"{name}/couplings"] = np.asarray(cpl, dtype=np.float64)
        out[f"{name}/field"] = np.zeros(3) if fld is None else np.asarray(fld, dtype=np.float64)
        out[f"{name}/has_field"] = np.array([fld is not None])
        out[f"{name}/e"] = e
        if store_v:
            rng = np.random.default_rng(20261203)
            v = rng.standard_normal(D) + 1j * rng.standard_normal(D)
            out[f"{name}/v"] = v
            out[f"{name}/w"] = H.T @ v
    for name, (L1, L2, q, tree, cpl) in SECTOR_CASES.items():
        cl = honeycomb(L1, L2)
        H = dense.sparse_h(cl.n, q, tree, cl.ipair, cl.ibond_type, cpl)
        states = np.arange(q ** cl.n)
        dsum = sum((states // q ** i) % q for i in range(cl.n))
        sel = states[dsum == cl.n // 2 * (q - 1)]
        Hs = H[sel][:, sel]
        D = Hs.shape[0]
        out[f"{name}/q"] = np.array([q, tree, cl.n])
        out[f"{name}/ipair"] = np.asarray(cl.ipair, dtype=np.int32)
        out[f"{name}/btype"] = np.asarray(cl.ibond_type, dtype=np.int32)
        out[f"{name}/couplings"] = np.asarray(cpl, dtype=np.float64)
        out[f"{name}/field"] = np.zeros(3)
        out[f"{name}/has_field"] = np.array([False])
        out[f"{name}/e"] = np.linalg.eigvalsh(Hs.toarray())[:4]
        rng = np.random.default_rng(20261203)
        v = rng.standard_normal(D) + 1j * rng.standard_normal(D)
        out[f"{name}/v"] = v
        out[f"{name}/w"] = Hs.T @ v
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)


if __name__ == "__main__":
    main()
