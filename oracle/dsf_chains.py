"""DSF chains of the oracle for a given start vector, as a separate process, so
that a test can run the oracle's other build (PNED_ORACLE_BUILD=fma) or another
thread count beside the one it has loaded.  Test infrastructure only.

    PNED_ORACLE_BUILD=fma python -m oracle.dsf_chains in.npz out.npz

in.npz holds the model (n, q, tree, ipair, ibond_type, X, skip, parity_type),
the start vector x, the phases qr [R][n], steps and threads; out.npz receives
salpha [R][steps] and sbeta [R][steps + 1].  The chains are intalv_zz +
parallelized_dsflnc1z (S_one_half/Hybrid_TPS_DSF.f90:18-87, 195-261).
"""
import sys

import numpy as np

from oracle import oracle as O


def main(src, dst):
    f = np.load(src)
    O.set_num_threads(int(f["threads"]))
    om = O.Model(int(f["n"]), int(f["q"]), int(f["tree"]), f["ipair"], f["ibond_type"], f["X"], f["skip"],
                 int(f["parity_type"]))
    steps = int(f["steps"])
    sa, sb = [], []
    for qr in f["qr"]:
        vq, cn = om.intalv_zz(qr, f["x"])
        a, b = om.dsf_chain(vq, cn, steps)
        sa.append(a)
        sb.append(b)
    np.savez(dst, salpha=np.array(sa), sbeta=np.array(sb))


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
