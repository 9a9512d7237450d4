"""GPU test of pned_hv_noalloc, the H.v entry point that allocates no device
memory (for hosts that manage all HBM in their own pool, or threads that must
not call cudaMalloc).  Its reduction scratch is a fixed array inside the
library, shared by all calls; two calls in a row must give the same result as
the context-based pned_hv.  This file is collected last on purpose."""
import math

import numpy as np
import pytest

import pned_b200 as P
from pned_b200 import couplings as CP
from pned_b200.lattice import honeycomb

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA GPU", allow_module_level=True)


def _model(L1, L2, field=True):
    cl = honeycomb(L1, L2)
    cpl = CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi), gamma=0.1)
    X, skip, pt = P.build_xlocal(2, 0, cpl, field=CP.field_111(0.05) if field else None)
    return P.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)


@pytest.mark.parametrize("R", [1, 4, 12])
def test_hv_noalloc_matches_pned_hv_on_two_calls(R):
    m = _model(2, 4)
    g = torch.Generator(device="cuda").manual_seed(42 + R)
    n = m.dim * R
    v1 = torch.complex(torch.randn(n, generator=g, device="cuda", dtype=torch.float64),
                       torch.randn(n, generator=g, device="cuda", dtype=torch.float64))
    v0 = 0.3 * torch.complex(torch.randn(n, generator=g, device="cuda", dtype=torch.float64),
                             torch.randn(n, generator=g, device="cuda", dtype=torch.float64))
    eperbd = 0.0625
    ref = v0.clone()
    pr_ref = P.Context(m, R=R).p_mltply_v3(v1, ref, eperbd)
    torch.cuda.synchronize()
    for _ in range(2):
        out = v0.clone()
        pr = P.hv_noalloc(m, R, v1, out, eperbd)
        err = (torch.linalg.vector_norm(out - ref) / torch.linalg.vector_norm(ref)).item()
        assert err <= 1e-12
        assert np.all(np.abs(pr - pr_ref) <= 1e-12 * np.abs(pr_ref))


def test_hv_noalloc_on_a_stream_and_rejects_unsupported_R():
    m = _model(3, 2, field=False)
    n = m.dim
    v1 = torch.ones(n, dtype=torch.complex128, device="cuda")
    v0 = torch.zeros(n, dtype=torch.complex128, device="cuda")
    s = torch.cuda.Stream()
    ref = v0.clone()
    pr_ref = P.Context(m, R=1).p_mltply_v3(v1, ref)
    torch.cuda.synchronize()
    pr = P.hv_noalloc(m, 1, v1, v0, stream=s)
    assert torch.allclose(v0, ref, rtol=0, atol=1e-12 * ref.abs().max().item())
    assert abs(pr[0] - pr_ref[0]) <= 1e-12 * abs(pr_ref[0])
    with pytest.raises(P.PnedError):
        P.hv_noalloc(m, 5, torch.zeros(5 * n, dtype=torch.complex128, device="cuda"),
                     torch.zeros(5 * n, dtype=torch.complex128, device="cuda"))
