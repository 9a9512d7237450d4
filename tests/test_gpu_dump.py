"""Lanczos runs on the GPU stopped and resumed through the reference's
checkpoint files (interval_dump / interval_dump_read, S_one_half/
Hybrid_TPS_output.f90:50-211, as parallelized_lnc1z calls them, S_one_half/
Hybrid_TPS_Lanczos.f90:87-103), in both directions between the GPU and the
CPU oracle.  Bounds: a GPU run resumed on the GPU follows the uninterrupted
run's alpha/beta to 1e-12 (the resumed vectors are rescaled once); across GPU
and oracle, 1e-10 over the 30-step chain."""
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

from tests.test_interval_dump import oracle_loop  # noqa: E402

STEPS, STOP = 30, 9


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


def models():
    cl = honeycomb(2, 4)
    cpl = CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi), gamma=0.1)
    fld = CP.field_111(0.05)
    gm = P.Model.from_couplings(cl, cpl, field=fld)
    X = O.xlocal(2, 0, cpl, field=fld)
    skip, _, pt = O.parity_skip(2, 0, X)
    om = O.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    return cl, gm, om


def start(dim):
    v = O.gaussian(17, dim)
    return v / np.linalg.norm(v)


def test_gpu_run_resumes_on_the_gpu(tmp_path):
    cl, gm, _ = models()
    v = start(gm.dim)
    full = P.Context(gm, R=1).lanczos(v, STEPS)
    ctx = P.Context(gm, R=1)
    ctx.session_begin("lanczos", v, STEPS)
    ctx.session_step(STOP)
    path = str(tmp_path / "vecdump_me00000")
    ctx.lanczos_dump_reference(path)
    ctx.session_end()
    info = P.api.read_interval_dump_info(path)
    assert info["itr_counter"][0] == STOP + 1 and info["n"] == cl.n and info["ibond"] == cl.nbond
    c2 = P.Context(gm, R=1)
    assert c2.lanczos_resume_reference(path, STEPS) == STOP
    c2.session_step(STEPS - STOP)
    r = c2.session_read()
    assert r["steps"] == STEPS
    assert np.array_equal(r["alpha"][:STOP, 0], full["alpha"][:STOP, 0])
    assert rel(r["alpha"][:, 0], full["alpha"][:, 0]) <= 1e-12
    assert rel(r["beta"][:, 0], full["beta"][:, 0]) <= 1e-12


def test_oracle_dump_resumes_on_the_gpu(tmp_path):
    """The state a reference-style run writes at the top of iteration 10 (the
    oracle's loop here) continues on the GPU as the oracle's own run does."""
    cl, gm, om = models()
    v = start(gm.dim)
    al, be, states = oracle_loop(om, v, STEPS)
    i, vs = STOP + 1, P.api.REF_MAX_ITR
    sa, sb = np.zeros(vs), np.zeros(vs)
    sa[:STOP], sb[:STOP] = al[:STOP], be[:STOP]
    path = str(tmp_path / "vecdump_me00000")
    info = P.api.dump_info(cl.n, cl.nbond, (i, vs, 2, vs, 1, 5000, 1, 500, 1, 8, 2, 4096))
    P.api.write_interval_dump(path, info, vs, sa=sa, sb=sb, sc=np.zeros((vs, 9), order="F"), se=np.zeros(vs),
                              vec1=states[i][0], vec2=states[i][1])
    ctx = P.Context(gm, R=1)
    assert ctx.lanczos_resume_reference(path, STEPS) == STOP
    ctx.session_step(STEPS - STOP)
    r = ctx.session_read()
    assert rel(r["alpha"][:, 0], al) <= 1e-10 and rel(r["beta"][:, 0], be) <= 1e-10


def test_gpu_dump_resumes_on_the_oracle(tmp_path):
    """A GPU run's dump, read back as the reference's loop reads it, continues on
    the oracle as the oracle's own uninterrupted run does."""
    cl, gm, om = models()
    v = start(gm.dim)
    al, be, _ = oracle_loop(om, v, STEPS)
    ctx = P.Context(gm, R=1)
    ctx.session_begin("lanczos", v, STEPS)
    ctx.session_step(STOP)
    path = str(tmp_path / "vecdump_me00000")
    ctx.lanczos_dump_reference(path)
    k = P.api.read_interval_dump_info(path)["itr_counter"][0]
    d = P.api.read_interval_dump(path, "lnc1z")
    v0, v1 = d["vec1"].copy(), d["vec2"].copy()
    a, b = d["sa"][k - 2], d["sb"][k - 2]
    got_a, got_b = list(d["sa"][:k - 1]), list(d["sb"][:k - 1])
    for _ in range(k, STEPS + 1):
        a, b = om.lanczos_step(v1, v0, a, b)
        got_a.append(a)
        got_b.append(b)
    assert rel(got_a, al) <= 1e-10 and rel(got_b, be) <= 1e-10
    ene = d["se"][:8]
    assert abs(ene[0] - P.bisec(al[:STOP], be[:STOP], STOP, 1)[0]) <= 1e-10 * abs(ene[0])


def tps_models(cl, L):
    cpl = CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi), gamma=0.1)
    fld = CP.field_111(0.05)
    gm = P.Model.from_couplings(cl, cpl, field=fld, tps_L=L)
    X = O.xlocal(2, 0, cpl, field=fld)
    skip, _, pt = O.parity_skip(2, 0, X)
    X = O.tps_explicit(2, cl.nbond, L, X)
    om = O.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    return gm, om


def test_tps_run_resumes_through_its_dump(tmp_path):
    """An mTPQ vector's run (parallelized_TPSz, S1/2 TPS.f90:325-409) stopped after
    9 steps, written as interval_dump writes it (vec1 = v0, vec2 = v1, vec3 = vg,
    coef with L in its second column) and resumed on a fresh context follows the
    uninterrupted run (alpha, beta, coefficients) to 1e-12 and the oracle's run to
    1e-10."""
    cl = honeycomb(2, 4)
    L = 2.0 * cl.n
    gm, om = tps_models(cl, L)
    v = start(gm.dim)
    full = P.Context(gm, R=1).tps(L, v, STEPS)
    ctx = P.Context(gm, R=1)
    ctx.session_begin("tps", v, STEPS, L=L)
    ctx.session_step(STOP)
    path = str(tmp_path / "vecdump_me00000")
    ctx.tps_dump_reference(path)
    info = P.api.read_interval_dump_info(path)
    assert info["itr_counter"][0] == STOP + 1 and info["dsf_comp"] == "tp"
    d = P.api.read_interval_dump(path, "tpsz")
    w, vk, vg = d["vec1"], d["vec2"], d["vec3"]
    # the loop's state: v1 normalised, v0 = (L - H) v1 with norm beta, vg the vector before v1
    assert abs(np.linalg.norm(vk) - 1.0) <= 1e-13
    assert abs(np.linalg.norm(w) - full["beta"][STOP - 1, 0]) <= 1e-12 * np.linalg.norm(w)
    assert abs(np.linalg.norm(vg) - 1.0) <= 1e-13
    ctx.session_end()
    c2 = P.Context(gm, R=1)
    assert c2.tps_resume_reference(path, STEPS) == STOP
    c2.session_step(STEPS - STOP)
    r = c2.session_read()
    assert rel(r["beta"][:, 0], full["beta"][:, 0]) <= 1e-12
    assert rel(r["alpha"][:, 0], full["alpha"][:, 0]) <= 1e-12
    assert rel(r["coef"][:, 0, :5], full["coef"][:, 0, :5]) <= 1e-12
    ref = om.tps(L, v, STEPS)
    assert rel(r["beta"][:, 0], ref["beta"]) <= 1e-10
    assert rel(r["coef"][:, 0, :5], ref["coef"][:, :5]) <= 1e-10


def test_dsf_chain_resumes_through_its_dump(tmp_path):
    """A DSF chain (parallelized_dsflnc1z, S1/2 DSF.f90:195-261) stopped after 9
    steps and resumed from its interval_dump files (sbeta(1) = cnorm, vec1 = v1,
    vec2 = v0) follows the uninterrupted chain to 1e-12 and the oracle's first 20
    coefficients to 1e-10."""
    cl, gm, om = models()
    x = start(gm.dim)
    qr = np.ascontiguousarray(cl.qr(1)).reshape(1, -1)
    full = P.Context(gm, R=1).dsf(x, qr, STEPS)
    ctx = P.Context(gm, R=1)
    cn = ctx.session_begin_dsf(x, qr, STEPS)
    ctx.session_step(STOP)
    path = str(tmp_path / "vecdump_me00000")
    ctx.dsf_dump_reference(path, cn[0])
    ctx.session_end()
    assert P.api.read_interval_dump_info(path)["itr_counter"][10] == STOP + 1
    c2 = P.Context(gm, R=1)
    k, cnorm = c2.dsf_resume_reference(path, STEPS)
    assert k == STOP and cnorm == cn[0]
    c2.session_step(STEPS - STOP)
    r = c2.session_read()
    assert rel(r["alpha"][:, 0], full["salpha"][:, 0]) <= 1e-12
    assert rel(r["beta"][:, 0], full["sbeta"][1:, 0]) <= 1e-12
    ra, rb = om.dsf_chain(*om.intalv_zz(qr[0], x), STEPS)
    assert rel(r["alpha"][:20, 0], ra[:20]) <= 1e-10 and rel(r["beta"][:19, 0], rb[1:20]) <= 1e-10
