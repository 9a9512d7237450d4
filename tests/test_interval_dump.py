"""The reference's checkpoint files (interval_dump / interval_dump_read /
check_interval_dump, S_one_half/Hybrid_TPS_output.f90:50-211): byte layout of
vecdump_me%05d and vecdump_me%05d.info as gfortran writes them, read-back, and
the Lanczos loop state they carry, round-tripped through the files on the
CPU oracle (parallelized_lnc1z, S_one_half/Hybrid_TPS_Lanczos.f90:80-122)."""
import math
import struct

import numpy as np

import pned_b200 as P
from oracle import oracle as O
from pned_b200 import couplings as CP
from pned_b200.lattice import honeycomb


def rec(payload: bytes) -> bytes:
    return struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload))


def test_interval_dump_layout_and_read_back(tmp_path):
    rng = np.random.default_rng(5)
    vs, ds = 3, 5
    sa, sb, se = rng.standard_normal(vs), rng.standard_normal(vs), rng.standard_normal(7)
    sc = np.asfortranarray(rng.standard_normal((vs, 9)))
    v0 = rng.standard_normal(ds) + 1j * rng.standard_normal(ds)
    v1 = rng.standard_normal(ds) + 1j * rng.standard_normal(ds)
    itr = (4, vs, 2, vs, 1, 5000, 1, 500, 1, 8, 2, 4096)
    info = P.api.dump_info(16, 24, itr, dump_name="vecdump_me00000", position=(1, 0, 1, 0, 0, 0, 0), dsf_comp="ee")
    path = str(tmp_path / "vecdump_me00000")
    P.api.write_interval_dump(path, info, vs, sa=sa, sb=sb, sc=sc, se=se, vec1=v0, vec2=v1)
    want_info = (rec(b"vecdump_me00000".ljust(128, b" ")) + rec(struct.pack("<i", 1)) +
                 rec(struct.pack("<7i", 1, 0, 1, 0, 0, 0, 0)) + rec(struct.pack("<i", 1024)) + rec(b"ee") +
                 rec(struct.pack("<i", 4096)) + rec(struct.pack("<i", 16)) + rec(struct.pack("<i", 24)) +
                 rec(struct.pack("<i", 8)) + rec(struct.pack("<i", 8)) +
                 b"".join(rec(struct.pack("<i", k)) for k in itr))
    assert open(path + ".info", "rb").read() == want_info
    want = (rec(struct.pack("<i", ds)) + rec(struct.pack("<i", vs)) + rec(sa.astype("<f8").tobytes()) +
            rec(sb.astype("<f8").tobytes()) + rec(sc.astype("<f8").tobytes(order="F")) +
            rec(se.astype("<f8").tobytes()) + rec(v0.astype("<c16").tobytes()) + rec(v1.astype("<c16").tobytes()))
    assert open(path, "rb").read() == want
    got = P.api.read_interval_dump_info(path)
    assert got["dump_name"] == "vecdump_me00000" and got["itr_counter"] == itr and got["dsf_comp"] == "ee"
    assert got["position"] == (True, False, True, False, False, False, False) and got["n"] == 16 and got["ibond"] == 24
    d = P.api.read_interval_dump(path, "lnc1z")
    assert d["data_size"] == ds and d["vec_size"] == vs
    assert np.array_equal(d["sa"], sa) and np.array_equal(d["sb"], sb) and np.array_equal(d["se"], se)
    assert np.array_equal(d["sc"], sc.reshape(-1, order="F"))
    assert np.array_equal(d["vec1"], v0) and np.array_equal(d["vec2"], v1)


def test_interval_dump_long_vectors_in_subrecords(tmp_path):
    """Vectors above one subrecord (every N = 27+ dump) round-trip split as gfortran splits them."""
    rng = np.random.default_rng(6)
    v0 = rng.standard_normal(40) + 1j * rng.standard_normal(40)
    v1 = rng.standard_normal(40) + 1j * rng.standard_normal(40)
    info = P.api.dump_info(8, 12, (2, 1, 2, 1, 1, 5000, 1, 500, 1, 8, 2, 4096))
    path = str(tmp_path / "vecdump_me00000")
    try:
        P.api.set_max_subrecord(48)
        P.api.write_interval_dump(path, info, 1, sa=np.ones(1), sb=np.ones(1), vec1=v0, vec2=v1)
    finally:
        P.api.set_max_subrecord()
    raw = open(path, "rb").read()
    assert struct.unpack("<i", raw[24:28])[0] == 8          # sa: one double, one subrecord
    d = P.api.read_interval_dump(path, "dsflnc")
    assert np.array_equal(d["vec1"], v0) and np.array_equal(d["vec2"], v1)


def oracle_loop(om, v, steps):
    """parallelized_lnc1z driven step by step: alpha/beta and the loop state
    (v0, v1) at the top of each iteration i = 2..steps."""
    v1 = v.copy()
    v0 = np.zeros_like(v1)
    pr = om.p_mltply_v3(v1, v0)   # the loop's first product and calc_beta
    d = v0 - pr * v1
    a, b = pr.real, math.sqrt(float(np.vdot(d, d).real))
    al, be, states = [a], [b], {}
    for i in range(2, steps + 1):
        states[i] = (v0.copy(), v1.copy())
        a, b = om.lanczos_step(v1, v0, a, b)
        al.append(a)
        be.append(b)
    return np.array(al), np.array(be), states


def test_lanczos_loop_resumes_from_its_dump_files_on_the_oracle(tmp_path):
    """A run that stops at the top of iteration 7 and resumes from the files it
    wrote continues exactly as the uninterrupted run (the files carry the state
    bit for bit)."""
    cl = honeycomb(2, 2)
    cpl = CP.kitaev_heisenberg(math.cos(0.3 * math.pi), 2 * math.sin(0.3 * math.pi), gamma=0.1)
    X = O.xlocal(2, 0, cpl, field=CP.field_111(0.05))
    skip, _, pt = O.parity_skip(2, 0, X)
    om = O.Model(cl.n, 2, 0, cl.ipair, cl.ibond_type, X, skip, pt)
    v = O.gaussian(3, om.ldim)
    v /= np.linalg.norm(v)
    nth = O.num_threads()
    O.set_num_threads(1)   # one thread: the oracle's reductions then repeat bit for bit
    try:
        al, be, states, rest = resumed(om, v, cl, tmp_path)
    finally:
        O.set_num_threads(nth)
    k = 7
    assert np.array_equal(np.array(rest)[:, 0], al[k - 1:]) and np.array_equal(np.array(rest)[:, 1], be[k - 1:])


def resumed(om, v, cl, tmp_path):
    al, be, states = oracle_loop(om, v, 20)
    i, vs = 7, 1024
    sa, sb = np.zeros(vs), np.zeros(vs)
    sa[:i - 1], sb[:i - 1] = al[:i - 1], be[:i - 1]
    path = str(tmp_path / "vecdump_me00000")
    info = P.api.dump_info(cl.n, cl.nbond, (i, vs, 2, vs, 1, 5000, 1, 500, 1, 8, 2, 4096))
    P.api.write_interval_dump(path, info, vs, sa=sa, sb=sb, sc=np.zeros((vs, 9), order="F"), se=np.zeros(vs),
                              vec1=states[i][0], vec2=states[i][1])
    k = P.api.read_interval_dump_info(path)["itr_counter"][0]
    d = P.api.read_interval_dump(path, "lnc1z")
    v0, v1 = d["vec1"].copy(), d["vec2"].copy()
    a, b = d["sa"][k - 2], d["sb"][k - 2]
    rest = []
    for _ in range(k, 21):
        a, b = om.lanczos_step(v1, v0, a, b)
        rest.append((a, b))
    return al, be, states, rest


def test_tps_dump_layout_reads_back(tmp_path):
    """parallelized_TPSz's dump (S1/2 TPS.f90:368-372) adds vec3 = vg after vec1, vec2."""
    rng = np.random.default_rng(8)
    vs, ds = 4, 6
    vec = [rng.standard_normal(ds) + 1j * rng.standard_normal(ds) for _ in range(3)]
    coef = np.asfortranarray(rng.standard_normal((vs, 5)))
    info = P.api.dump_info(12, 18, (3, vs, 2, vs, 1, 5000, 1, 500, 1, 8, 2, 4096), dsf_comp="tp",
                           position=(0, 0, 0, 0, 0, 0, 1))
    path = str(tmp_path / "vecdump_me00003")
    P.api.write_interval_dump(path, info, vs, sa=np.arange(vs, dtype=float), sb=np.ones(vs), sc=coef,
                              se=np.zeros(9), vec1=vec[0], vec2=vec[1], vec3=vec[2])
    d = P.api.read_interval_dump(path, "tpsz")
    assert np.array_equal(d["sc"].reshape(vs, 5, order="F"), coef) and d["se"].size == 9
    for i in range(3):
        assert np.array_equal(d[f"vec{i + 1}"], vec[i])
    assert P.api.read_interval_dump_info(path)["position"][6]


def test_interval_dump_rejects_mismatched_files(tmp_path):
    """A dump read with another loop's layout, a truncated data file and a missing
    .info file are refused with an error, not misread."""
    import pytest
    rng = np.random.default_rng(9)
    v = [rng.standard_normal(4) + 1j * rng.standard_normal(4) for _ in range(2)]
    info = P.api.dump_info(8, 12, (2, 3, 2, 3, 1, 5000, 1, 500, 1, 8, 2, 4096))
    path = str(tmp_path / "vecdump_me00000")
    P.api.write_interval_dump(path, info, 3, sa=np.ones(3), sb=np.ones(3), vec1=v[0], vec2=v[1])
    with pytest.raises(ValueError):
        P.api.read_interval_dump(path, "lnc1z")          # six arrays expected, four in the file
    raw = open(path, "rb").read()
    open(path, "wb").write(raw[:-20])
    with pytest.raises(P.PnedError):
        P.api.read_interval_dump(path, "dsflnc")
    with pytest.raises(P.PnedError):
        P.api.read_interval_dump_info(str(tmp_path / "missing"))
