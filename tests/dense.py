"""Independent dense construction of pNED Hamiltonians for small clusters.

Used only by tests: builds H = sum_bonds sum_ab J_t[a][b] S^a_{s1} S^b_{s2}
(+ field) with numpy Kronecker products from the spin-matrix definitions, so
that the oracle (which restates the reference's loop structure) is checked
against an implementation that shares none of its indexing code.
"""
import math

import numpy as np
import scipy.sparse as sp


def spin_matrices(q, tree_sa):
    if not tree_sa:
        sx = np.array([[0, .5], [.5, 0]], dtype=complex)
        sy = np.array([[0, -.5j], [.5j, 0]], dtype=complex)
        sz = np.array([[.5, 0], [0, -.5]], dtype=complex)
        return [sx, sy, sz]
    s = 0.5 * (q - 1)
    m = np.arange(q) - s
    su = np.zeros((q, q), dtype=complex)
    sd = np.zeros((q, q), dtype=complex)
    for i in range(q - 1):
        su[i, i + 1] = math.sqrt((s - m[i]) * (s + m[i] + 1))
    for i in range(1, q):
        sd[i, i - 1] = math.sqrt((s + m[i]) * (s - m[i] + 1))
    sx = 0.5 * (su + sd)
    sy = -0.5j * (su - sd)
    sz = np.diag(m).astype(complex)
    return [sx, sy, sz]


def site_op(op, site, n, q):
    """Sparse operator acting on `site`; index = sum_j d_j q^j (site n-1 most significant)."""
    out = sp.identity(1, dtype=complex, format="csr")
    for j in range(n - 1, -1, -1):
        out = sp.kron(out, sp.csr_matrix(op) if j == site else sp.identity(q, dtype=complex, format="csr"),
                      format="csr")
    return out


def nn_exchange(cpl, tree_sa):
    """3x3 exchange matrices for bond types 1..3 from the slot vector (J1x, J1y, J1z)."""
    J1, K1, I11, I12, J1p, K1p, J1pp, K1pp, I11p, I12p, I11pp, I12pp = cpl[:12]
    Jz = np.array([[J1, I11, I12], [I11, J1, I12], [I12, I12, K1]])
    Jx = np.array([[K1p, I12pp, I12p], [I12pp, J1pp, I11p], [I12p, I11p, J1p]])
    Jy = np.array([[J1pp, I12pp, I11p], [I12pp, K1p, I12p], [I11p, I12p, J1p]])
    return {1: Jx, 2: Jy, 3: Jz}


def sparse_h(n, q, tree_sa, ipair, btype, cpl, field=None):
    S = spin_matrices(q, tree_sa)
    Jt = nn_exchange(cpl, tree_sa)
    D = q ** n
    H = sp.csr_matrix((D, D), dtype=complex)
    ops = [[site_op(S[a], j, n, q) for a in range(3)] for j in range(n)]
    for b in range(len(btype)):
        i, j = ipair[2 * b] - 1, ipair[2 * b + 1] - 1
        s1, s2 = min(i, j), max(i, j)
        J = Jt[int(btype[b])]
        for a in range(3):
            for c in range(3):
                if J[a][c] != 0:
                    H = H + J[a][c] * (ops[s1][a] @ ops[s2][c])
    if field is not None:
        for j in range(n):
            for a in range(3):
                if field[a] != 0:
                    H = H - field[a] * ops[j][a]
    return H.tocsr()


def dense_h(n, q, tree_sa, ipair, btype, cpl, field=None):
    return sparse_h(n, q, tree_sa, ipair, btype, cpl, field).toarray()
