"""Host-side API over the C ABI, named after the reference routines it replaces.

Vectors are complex128 with R interleaved columns ([dim][R] flattened).  Every
vector argument may be a numpy array (host memory: copied to and from the
device by the call) or a CUDA torch tensor (device memory: used in place).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import _capi
from ._capi import PTR_DEVICE, PTR_HOST, check, lib
from .couplings import NSLOT

try:  # torch is only plumbing here: device memory for callers that keep vectors on the GPU
    import torch
except Exception:  # pragma: no cover
    torch = None


def _is_dev(x) -> bool:
    return torch is not None and isinstance(x, torch.Tensor) and x.is_cuda


def _ptr(x, writable=False):
    """(pointer, flag) for a numpy array or a CUDA tensor of complex128.

    A CUDA tensor may still be being written by torch's current stream (a
    fill, a copy, a random draw), while the library works on its own stream
    (a context's or a batch's non-blocking stream); the current stream is
    therefore waited for before the pointer is handed over."""
    if _is_dev(x):
        if x.dtype != torch.complex128 or not x.is_contiguous():
            raise TypeError("device vectors must be contiguous complex128 CUDA tensors")
        torch.cuda.current_stream(x.device).synchronize()
        return C.c_void_p(x.data_ptr()), PTR_DEVICE
    if not isinstance(x, np.ndarray) or x.dtype != np.complex128 or not x.flags["C_CONTIGUOUS"]:
        raise TypeError("host vectors must be C-contiguous complex128 numpy arrays")
    if writable and not x.flags["WRITEABLE"]:
        raise TypeError("output vector is read-only")
    return C.c_void_p(x.ctypes.data), PTR_HOST


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _same_flag(*flags):
    if len(set(flags)) != 1:
        raise TypeError("mix of host and device vectors in one call")
    return flags[0]


# --------------------------------------------------------------------------- model input

def build_xlocal(q: int, tree: int, couplings, simple: int = 0, field=None, coord: float = 3.0):
    """set_xlocal_Ham: returns (xlocal (9,Q,Q) [type, col, row], skip (9,Q,Q) uint8, parity_type)."""
    Q = q * q
    cpl = np.ascontiguousarray(couplings, dtype=np.float64)
    if cpl.shape != (NSLOT,):
        raise ValueError(f"couplings must have {NSLOT} slots")
    X = np.zeros((9, Q, Q), dtype=np.complex128)
    skip = np.zeros((9, Q, Q), dtype=np.uint8)
    pt = C.c_int(0)
    fld = None if field is None else np.ascontiguousarray(field, dtype=np.float64)
    check(lib().pned_build_xlocal(q, tree, _dp(cpl), simple, None if fld is None else _dp(fld), coord,
                                  C.c_void_p(X.ctypes.data), skip.ctypes.data_as(C.POINTER(C.c_uint8)),
                                  C.byref(pt)))
    return X, skip, pt.value


def tps_transform(q: int, tree: int, n_bonds: int, xlocal, L=None, c_count: float = 3.0):
    """change_to_TPS_hamiltonian (L=None: the reference's own L) or X <- (L/n_bonds) 1 - X."""
    X = np.ascontiguousarray(xlocal, dtype=np.complex128).copy()
    Lc = C.c_double(0.0 if L is None else float(L))
    check(lib().pned_tps_transform(q, tree, n_bonds, c_count, 0 if L is None else 1, C.c_void_p(X.ctypes.data),
                                   C.byref(Lc)))
    return X, Lc.value


def mk_list12(n: int, q: int, parity_type: int, total_sz: int):
    ldim = C.c_int64(0)
    check(lib().pned_mk_list12(n, q, parity_type, total_sz, C.byref(ldim), None, None, None))
    nA = q ** ((n + 1) // 2)
    nB = q ** (n // 2)
    list1 = np.zeros(ldim.value, dtype=np.int64)
    lo = np.zeros(max(nA, nB), dtype=np.int64)
    hi = np.zeros(max(nA, nB), dtype=np.int64)
    check(lib().pned_mk_list12(n, q, parity_type, total_sz, C.byref(ldim), C.c_void_p(list1.ctypes.data),
                               C.c_void_p(lo.ctypes.data), C.c_void_p(hi.ctypes.data)))
    return list1, lo, hi


def bisec(alpha, beta, ndim: int, ne: int, eps: float = 1e-25):
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    b = np.ascontiguousarray(beta, dtype=np.float64)
    E = np.zeros(max(1, ne))
    check(lib().pned_bisec(_dp(a), _dp(b), ndim, _dp(E), ne, eps))
    return E[:ne]


def vec12(alpha, beta, E, ndim: int, nvec: int):
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    b = np.ascontiguousarray(np.concatenate([np.asarray(beta, dtype=np.float64), np.zeros(2)]))
    e = np.ascontiguousarray(E, dtype=np.float64)
    v = np.zeros((nvec, ndim))
    check(lib().pned_vec12(_dp(a), _dp(b), _dp(e), ndim, nvec, _dp(v)))
    return v


def exec_renbun(i_range: int, s_maxitr: int, split: float, ene: float, epsln: float, salpha, sbeta):
    sa = np.zeros(s_maxitr)
    sb = np.zeros(s_maxitr)
    na, nb = min(len(salpha), s_maxitr), min(len(sbeta), s_maxitr)
    sa[:na] = np.asarray(salpha)[:na]
    sb[:nb] = np.asarray(sbeta)[:nb]
    w = np.zeros(i_range)
    conv = np.zeros(i_range, dtype=np.int32)
    dsf = np.zeros(i_range)
    check(lib().pned_exec_renbun(i_range, s_maxitr, split, ene, epsln, _dp(sa), _dp(sb), _dp(w),
                                 conv.ctypes.data_as(C.POINTER(C.c_int)), _dp(dsf)))
    return w, conv, dsf


def normalize_dsf(i_range: int, split: float, sq_re: float, dsf):
    d = np.ascontiguousarray(dsf, dtype=np.float64).copy()
    check(lib().pned_normalize_dsf(i_range, split, sq_re, _dp(d)))
    return d


# --------------------------------------------------------------------------- mTPQ output chain


def write_salphasbeta(path: str, alpha, beta, coef):
    """dump_alpha_beta_coef: alpha, beta [num_data1], coef [num_data1][num_data2] (written column-major)."""
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    b = np.ascontiguousarray(beta, dtype=np.float64)
    c = np.asfortranarray(np.asarray(coef, dtype=np.float64))
    n1, n2 = c.shape
    if a.shape != (n1,) or b.shape != (n1,):
        raise ValueError("alpha and beta need num_data1 = coef.shape[0] entries")
    cf = np.ascontiguousarray(c.T)   # coef(k, m) with k fastest
    check(lib().pned_write_salphasbeta(os.fsencode(path), n1, n2, _dp(a), _dp(b), _dp(cf)))


def read_salphasbeta(path: str):
    """Returns (alpha, beta, coef [num_data1][num_data2]) of a TPQ coefficient file."""
    n1, n2 = C.c_int(0), C.c_int(0)
    check(lib().pned_read_salphasbeta(os.fsencode(path), C.byref(n1), C.byref(n2), None, None, None, 0))
    a, b = np.zeros(n1.value), np.zeros(n1.value)
    cf = np.zeros(n1.value * n2.value)
    check(lib().pned_read_salphasbeta(os.fsencode(path), C.byref(n1), C.byref(n2), _dp(a), _dp(b), _dp(cf), n1.value))
    return a, b, cf.reshape(n2.value, n1.value).T.copy()


def tpq_thermo(beta, energy, hmix, t_min: float, t_max: float, num_div: int):
    """eval_mpi: canonical T, E(T), C(T), var, d2E/dT2 from mTPQ runs ([n_seeds][num_data1] arrays)."""
    b = np.ascontiguousarray(np.atleast_2d(beta), dtype=np.float64)
    e = np.ascontiguousarray(np.atleast_2d(energy), dtype=np.float64)
    h = np.ascontiguousarray(np.atleast_2d(hmix), dtype=np.float64)
    if not (b.shape == e.shape == h.shape):
        raise ValueError("beta, energy and hmix need the same [n_seeds][num_data1] shape")
    out = np.zeros((num_div + 1, 5))
    check(lib().pned_tpq_thermo(b.shape[1], b.shape[0], _dp(b), _dp(e), _dp(h), float(t_min), float(t_max),
                                int(num_div), _dp(out)))
    return out


def write_vec_data(path: str, e: float, x):
    """readwrite_vec_data (write): the energy and the vector x (complex128, host)."""
    xs = np.ascontiguousarray(x, dtype=np.complex128)
    check(lib().pned_write_vec_data(os.fsencode(path), float(e), C.c_void_p(xs.ctypes.data), xs.size))


def read_vec_data(path: str, ll: int):
    e = C.c_double(0.0)
    x = np.zeros(int(ll), dtype=np.complex128)
    check(lib().pned_read_vec_data(os.fsencode(path), C.byref(e), C.c_void_p(x.ctypes.data), int(ll)))
    return e.value, x


def write_dsf_alpha_beta(path: str, sq: complex, salpha, sbeta):
    a = np.ascontiguousarray(salpha, dtype=np.float64)
    b = np.ascontiguousarray(sbeta, dtype=np.float64)
    if a.shape != b.shape:
        raise ValueError("salpha and sbeta need the same length (s_maxitr)")
    check(lib().pned_write_dsf_alpha_beta(os.fsencode(path), _capi.c128(complex(sq).real, complex(sq).imag),
                                          _dp(a), _dp(b), a.size))


def read_dsf_alpha_beta(path: str, s_maxitr: int):
    sq = _capi.c128(0.0, 0.0)
    a, b = np.zeros(int(s_maxitr)), np.zeros(int(s_maxitr))
    check(lib().pned_read_dsf_alpha_beta(os.fsencode(path), C.byref(sq), _dp(a), _dp(b), int(s_maxitr)))
    return complex(sq.re, sq.im), a, b


def append_dsf_res(path: str, sq_re: float, q, w, dsf, conv):
    q2 = np.ascontiguousarray(q, dtype=np.float64)[:2].copy()
    w_ = np.ascontiguousarray(w, dtype=np.float64)
    d_ = np.ascontiguousarray(dsf, dtype=np.float64)
    c_ = np.ascontiguousarray(conv, dtype=np.int32)
    check(lib().pned_append_dsf_res(os.fsencode(path), float(sq_re), _dp(q2), _dp(w_), _dp(d_),
                                    c_.ctypes.data_as(C.POINTER(C.c_int)), w_.size))


def append_sq(path: str, iq: int, q, norm_re: float):
    """The DSF driver's sq.txt line for momentum iq (q: the two components)."""
    check(lib().pned_append_sq(os.fsencode(path), int(iq), float(q[0]), float(q[1]), float(norm_re)))


def write_dsf_vectors(path: str, indx: int, v1, v2):
    """vec_q... file of a DSF chain (step index, the two Lanczos vectors)."""
    a = np.ascontiguousarray(v1, dtype=np.complex128)
    b = np.ascontiguousarray(v2, dtype=np.complex128)
    if a.shape != b.shape:
        raise ValueError("v1 and v2 need the same length")
    check(lib().pned_write_dsf_vectors(os.fsencode(path), int(indx), C.c_void_p(a.ctypes.data),
                                       C.c_void_p(b.ctypes.data), a.size))


def set_max_subrecord(nbytes: int = 2147483639):
    """Largest subrecord payload of the Fortran record writers (gfortran's
    -fmax-subrecord-length; default 2^31 - 9 bytes)."""
    check(lib().pned_set_max_subrecord(int(nbytes)))


def read_dsf_vectors(path: str, ll: int):
    i = C.c_int(0)
    a = np.zeros(int(ll), dtype=np.complex128)
    b = np.zeros(int(ll), dtype=np.complex128)
    check(lib().pned_read_dsf_vectors(os.fsencode(path), C.byref(i), C.c_void_p(a.ctypes.data),
                                      C.c_void_p(b.ctypes.data), int(ll)))
    return i.value, a, b


# --------------------------------------------------------------------------- interval_dump checkpoints

REF_MAX_ITR = 1024     # max_itr of the reference (S_one_half/Hybrid_TPS_params.f90:39)
REF_S_MAXITR = 4096    # s_maxitr (:42)
REF_NVEC = 8           # nvec (:31)
DUMP_ARRAYS = ("sa", "sb", "sc", "se", "vec0", "vec1", "vec2", "vec3", "vec4")
# what each loop of the reference passes to interval_dump (S1/2 Lanczos.f90:101, 275; TPS.f90:370; DSF.f90:236)
DUMP_LAYOUTS = {"lnc1z": ("sa", "sb", "sc", "se", "vec1", "vec2"),
                "lncv1z": ("sa", "sb", "sc", "se", "vec0", "vec1", "vec2"),
                "tpsz": ("sa", "sb", "sc", "se", "vec1", "vec2", "vec3"),
                "dsflnc": ("sa", "sb", "vec1", "vec2")}


def dump_info(n_sites: int, n_bonds: int, itr_counter, dump_name: str = "vecdump_me00000",
              position=(1, 0, 1, 0, 0, 0, 0), dsf_comp: str = "ee", np_ranks: int = 1, max_itr: int = REF_MAX_ITR,
              s_maxitr: int = REF_S_MAXITR, nvec: int = REF_NVEC, total_sz=None) -> "_capi.DumpInfo":
    """The .info record set of interval_dump (S1/2 output.f90:176-191); total_sz
    defaults to n/2 as the reference sets it (params.f90:149)."""
    info = _capi.DumpInfo()
    info.dump_name = dump_name.encode().ljust(128, b" ")[:128]
    info.np = int(np_ranks)
    for i, p in enumerate(position):
        info.position[i] = 1 if p else 0
    info.max_itr = int(max_itr)
    info.dsf_comp = dsf_comp.encode()[:2].ljust(2, b" ")
    info.s_maxitr, info.n, info.ibond, info.nvec = int(s_maxitr), int(n_sites), int(n_bonds), int(nvec)
    info.total_sz = int(n_sites // 2 if total_sz is None else total_sz)
    for i, k in enumerate(itr_counter):
        info.itr_counter[i] = int(k)
    return info


def info_dict(info: "_capi.DumpInfo") -> dict:
    return {"dump_name": bytes(info.dump_name).decode(errors="replace").rstrip(" \x00"), "np": info.np,
            "position": tuple(bool(x) for x in info.position), "max_itr": info.max_itr,
            "dsf_comp": bytes(info.dsf_comp).decode(errors="replace"), "s_maxitr": info.s_maxitr, "n": info.n,
            "ibond": info.ibond, "nvec": info.nvec, "total_sz": info.total_sz,
            "itr_counter": tuple(info.itr_counter)}


def write_interval_dump(path: str, info: "_capi.DumpInfo", vec_size: int, **arrays):
    """interval_dump's files `path` and `path`.info: arrays by name (DUMP_ARRAYS;
    sa .. se real, sc column-major as given in Fortran order; vec0 .. vec4
    complex, vec1 and vec2 required, all of one length)."""
    d = _capi.DumpData()
    keep = []
    vl = None
    for name in DUMP_ARRAYS:
        x = arrays.get(name)
        if x is None:
            continue
        if name.startswith("vec"):
            a = np.ascontiguousarray(x, dtype=np.complex128)
            if vl is not None and a.size != vl:
                raise ValueError("the dump's vectors need one length")
            vl = a.size
            d.vec[int(name[3])] = a.ctypes.data
        else:
            a = np.asfortranarray(x, dtype=np.float64).reshape(-1, order="F")
            setattr(d, name, _dp(a))
            setattr(d, "n_" + name, a.size)
        keep.append(a)
    if arrays.get("vec1") is None or arrays.get("vec2") is None:
        raise ValueError("interval_dump always writes vec1 and vec2")
    d.data_size, d.vec_size = int(vl), int(vec_size)
    check(lib().pned_write_interval_dump(os.fsencode(path), C.byref(info), C.byref(d)))


def read_interval_dump_info(path: str) -> dict:
    info = _capi.DumpInfo()
    check(lib().pned_read_interval_dump_info(os.fsencode(path), C.byref(info)))
    return info_dict(info)


def read_interval_dump(path: str, layout) -> dict:
    """interval_dump's data file read with the arrays `layout` names (in file order,
    e.g. DUMP_LAYOUTS['lnc1z']), sized from the records themselves."""
    names = DUMP_LAYOUTS[layout] if isinstance(layout, str) else tuple(layout)
    cap = 16
    lens = (C.c_int64 * cap)()
    cnt = C.c_int(0)
    check(lib().pned_interval_dump_records(os.fsencode(path), lens, cap, C.byref(cnt)))
    if cnt.value != 2 + len(names):
        raise ValueError(f"{path}: {cnt.value} records, the layout {names} needs {2 + len(names)}")
    d = _capi.DumpData()
    out = {}
    for name, nb in zip(names, list(lens)[2:cnt.value]):
        if name.startswith("vec"):
            a = np.zeros(nb // 16, dtype=np.complex128)
            d.vec[int(name[3])] = a.ctypes.data
        else:
            a = np.zeros(nb // 8)
            setattr(d, name, _dp(a))
            setattr(d, "n_" + name, a.size)
        out[name] = a
    check(lib().pned_read_interval_dump(os.fsencode(path), C.byref(d)))
    out["data_size"], out["vec_size"] = d.data_size, d.vec_size
    return out


# --------------------------------------------------------------------------- model / context


def hv_noalloc(model, R: int, v1, v0, eperbd: float = 0.0, stream=None):
    """pned_hv_noalloc: v0 += (H - eperbd*ibond)^T v1 on CUDA tensors without
    any device allocation by the library; returns prdct (R complex)."""
    p1, f1 = _ptr(v1)
    p0, f0 = _ptr(v0, writable=True)
    if f1 != PTR_DEVICE or f0 != PTR_DEVICE:
        raise TypeError("hv_noalloc takes CUDA tensors")
    for v in (v1, v0):
        if v.numel() != model.dim * R:
            raise ValueError("vectors must have dim*R elements")
    sp = None if stream is None else C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else stream)
    pr = np.zeros(R, dtype=np.complex128)
    check(lib().pned_hv_noalloc(model._h, int(R), p1, p0, float(eperbd), C.c_void_p(pr.ctypes.data), sp))
    return pr


class ModelInput:
    """Host-side model description (pned_model_desc) with the arrays it points to."""

    def __init__(self, n, q, tree, ipair, bond_type, xlocal, skip, parity_type, total_sz=None):
        if total_sz is None:
            total_sz = n // 2 * (q - 1)
        self.n, self.q, self.tree = int(n), int(q), int(tree)
        self._ipair = np.ascontiguousarray(ipair, dtype=np.int32)
        self._bt = np.ascontiguousarray(bond_type, dtype=np.int32)
        self._x = np.ascontiguousarray(xlocal, dtype=np.complex128)
        self._skip = None if skip is None else np.ascontiguousarray(skip, dtype=np.uint8)
        self.n_bonds = int(self._bt.shape[0])
        self.parity_type = int(parity_type)
        d = _capi.ModelDesc()
        d.n_sites, d.q_spin, d.tree, d.n_bonds = self.n, self.q, self.tree, self.n_bonds
        d.ipair = self._ipair.ctypes.data_as(C.POINTER(C.c_int32))
        d.bond_type = self._bt.ctypes.data_as(C.POINTER(C.c_int32))
        d.xlocal = C.c_void_p(self._x.ctypes.data)
        d.skip = None if self._skip is None else self._skip.ctypes.data_as(C.POINTER(C.c_uint8))
        d.parity_type, d.total_sz = int(parity_type), int(total_sz)
        self.c = d

    @classmethod
    def from_couplings(cls, cluster, couplings, q=2, tree=0, field=None, tps_L=None, simple=0):
        X, skip, pt = build_xlocal(q, tree, couplings, simple=simple, field=field)
        if tps_L is not None:
            X, _ = tps_transform(q, tree, cluster.nbond, X, L=tps_L)
        return cls(cluster.n, q, tree, cluster.ipair, cluster.ibond_type, X, skip, pt)

    @classmethod
    def structure(cls, cluster, tree=0):
        """Generic S = 1/2 structure of a cluster: every local-matrix entry non-zero,
        so every one- and two-site flip of every bond is a term (slot batches)."""
        X = np.ones((9, 4, 4), dtype=np.complex128)
        return cls(cluster.n, 2, tree, cluster.ipair, cluster.ibond_type, X, None, 1)


def tile_plan_export(desc: "ModelInput", row_fixed_bits: int = -1, window_bits: int = -1, max_passes: int = -1,
                     j_bits: int = -1, row_bits: int = 8, objective: int = -1) -> dict:
    """The tile plan (S = 1/2 full basis) with row_bits row bits a tile (8: the
    single-vector plan Model.set_plan builds), computed on the host
    (pned_tile_plan_export): the program's flip terms and, per pass, the tile
    bits, outer order, terms and partner-tile groups."""
    tp = _capi.TilePlan(int(row_fixed_bits), int(window_bits), int(max_passes), int(j_bits), 1, 0, -1, int(objective), -1)
    # all defaults: no plan, the model's own default (as Model.set_plan)
    ptp = None if (row_fixed_bits, window_bits, max_passes, j_bits, objective) == (-1,) * 5 else C.byref(tp)
    n = C.c_int64(0)
    check(lib().pned_tile_plan_export(C.byref(desc.c), int(row_bits), ptp, None, 0, C.byref(n)))
    buf = np.zeros(n.value, dtype=np.int64)
    check(lib().pned_tile_plan_export(C.byref(desc.c), int(row_bits), ptp,
                                      buf.ctypes.data_as(C.POINTER(C.c_int64)), n.value, C.byref(n)))
    it = iter(buf.tolist())
    nx = next(it)
    xterms = [dict(zip(("xmask", "pos4", "tab", "nb"), (next(it) for _ in range(4)))) for _ in range(nx)]
    passes = []
    for _ in range(next(it)):
        tbits, jb, nout, nt, nin, ng = (next(it) for _ in range(6))
        ps = dict(tbits=tbits, jb=jb, nin=nin)
        ps["rowpos"] = [next(it) for _ in range(tbits)]
        ps["jpos"] = [next(it) for _ in range(jb)]
        ps["outer"] = [next(it) for _ in range(nout)]
        ps["terms"] = [dict(zip(("mask", "pos4", "jtab", "tab", "nb", "hasj", "lmask"), (next(it) for _ in range(7))))
                       for _ in range(nt)]
        ps["gstart"] = [next(it) for _ in range(ng + 1)]
        ps["gxor"] = [next(it) for _ in range(ng)]
        passes.append(ps)
    return {"xterms": xterms, "passes": passes}


def qtile_plan_export(desc: "ModelInput", k: int, low: int = 0) -> dict:
    """The mixed-radix tile passes of k sites (q > 2, full basis) that the tiled
    mixed-radix kernel runs, computed on the host (pned_qtile_plan_export)."""
    n = C.c_int64(0)
    check(lib().pned_qtile_plan_export(C.byref(desc.c), int(k), int(low), None, 0, C.byref(n)))
    buf = np.zeros(n.value, dtype=np.int64)
    check(lib().pned_qtile_plan_export(C.byref(desc.c), int(k), int(low), buf.ctypes.data_as(C.POINTER(C.c_int64)),
                                       n.value, C.byref(n)))
    it = iter(buf.tolist())
    q, nsites, nr = next(it), next(it), next(it)
    rterms = [dict(zip(("offset", "s1", "s2", "tab"), (next(it) for _ in range(4)))) for _ in range(nr)]
    nonzero = [next(it) for _ in range(next(it))]
    passes = []
    for _ in range(next(it)):
        kk, nout, nt = (next(it) for _ in range(3))
        ps = {"sites": [next(it) for _ in range(kk)], "outer": [next(it) for _ in range(nout)]}
        ps["terms"] = [dict(zip(("loff", "ls1", "ls2", "tab"), (next(it) for _ in range(4)))) for _ in range(nt)]
        passes.append(ps)
    return {"q": q, "n": nsites, "rterms": rterms, "nonzero": nonzero, "passes": passes}


class Model:
    """A compiled model on the current device (pned_model_create)."""

    def __init__(self, n, q, tree, ipair, bond_type, xlocal, skip, parity_type, total_sz=None):
        self.desc = ModelInput(n, q, tree, ipair, bond_type, xlocal, skip, parity_type, total_sz)
        self.n, self.q, self.tree, self.n_bonds = self.desc.n, self.desc.q, self.desc.tree, self.desc.n_bonds
        d = self.desc.c
        h = C.c_void_p()
        check(lib().pned_model_create(C.byref(d), C.byref(h)))
        self._h = h
        dim, nt, rc_ = C.c_int64(0), C.c_int(0), C.c_int(0)
        check(lib().pned_model_info(h, C.byref(dim), C.byref(nt), C.byref(rc_)))
        self.dim, self.n_terms, self.real = dim.value, nt.value, bool(rc_.value)

    def plan(self, R: int = 1) -> dict:
        """H.v plan for R vectors: tiled-kernel passes, partner tiles, states per tile."""
        p, g, t = C.c_int(0), C.c_int(0), C.c_int(0)
        check(lib().pned_model_plan(self._h, int(R), C.byref(p), C.byref(g), C.byref(t)))
        out = {"tile_passes": p.value, "partner_tiles": g.value, "tile_states": t.value}
        if R == 1:
            md, ns = C.c_int(0), C.c_int(0)
            check(lib().pned_model_tile_staging(self._h, C.byref(md), C.byref(ns)))
            out["staging"], out["ring_stages"] = md.value, ns.value
        return out

    def sector_segments(self, enable: bool | None = None) -> bool:
        """S = 1/2 Sz sector: selects the per-segment one-vector H.v (True) or the
        flat gather (False); None leaves it.  Returns whether the segment kernel runs."""
        act = C.c_int(0)
        check(lib().pned_model_sector_segments(self._h, -1 if enable is None else int(bool(enable)), C.byref(act)))
        return bool(act.value)

    def set_plan(self, R: int = 1, row_fixed_bits: int = -1, window_bits: int = -1, max_passes: int = -1,
                 j_bits: int = -1, l1_carveout: int = 1, stage_partner_tiles: int = 0, blocks_per_sm: int = -1,
                 objective: int = -1, terms_in_flight: int = -1):
        """Re-plans the tiled H.v for R vectors (-1: default); returns the new plan.
        With no plan argument the library's default plan for the size is restored."""
        args = (row_fixed_bits, window_bits, max_passes, j_bits, l1_carveout, stage_partner_tiles, blocks_per_sm,
                objective, terms_in_flight)
        if args == (-1, -1, -1, -1, 1, 0, -1, -1, -1):
            check(lib().pned_model_set_plan(self._h, int(R), None))
            return self.plan(R)
        tp = _capi.TilePlan(*(int(x) for x in args))
        check(lib().pned_model_set_plan(self._h, int(R), C.byref(tp)))
        return self.plan(R)

    @classmethod
    def from_couplings(cls, cluster, couplings, q=2, tree=0, field=None, tps_L=None, simple=0):
        """Model from a cluster table and coupling slots (+ field, + TPS shift L)."""
        X, skip, pt = build_xlocal(q, tree, couplings, simple=simple, field=field)
        if tps_L is not None:
            X, _ = tps_transform(q, tree, cluster.nbond, X, L=tps_L)
        return cls(cluster.n, q, tree, cluster.ipair, cluster.ibond_type, X, skip, pt)

    def close(self):
        if getattr(self, "_h", None):
            lib().pned_model_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class ObservableSpec:
    """O(s) = sum_t c_t T[bit(s, a_t)][bit(s, b_t)] (see pned_observable)."""
    a: np.ndarray
    b: np.ndarray
    c: np.ndarray
    T: np.ndarray


class Context:
    """Device vectors and scratch for R interleaved vectors of one model."""

    def __init__(self, model: Model, R: int = 1, hbm_budget: int = 0, stream=None):
        self.model = model
        self.R = int(R)
        h = C.c_void_p()
        check(lib().pned_ctx_create(model._h, self.R, C.c_size_t(int(hbm_budget)), C.byref(h)))
        self._h = h
        if stream is not None:
            self.set_stream(stream)

    @property
    def n_elem(self):
        return self.model.dim * self.R

    def set_stream(self, stream):
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        check(lib().pned_ctx_set_stream(self._h, C.c_void_p(sp)))

    def synchronize(self):
        check(lib().pned_ctx_synchronize(self._h))

    def bytes(self) -> int:
        b = C.c_size_t(0)
        check(lib().pned_ctx_bytes(self._h, C.byref(b)))
        return b.value

    def close(self):
        if getattr(self, "_h", None):
            lib().pned_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check_len(self, *vs):
        for v in vs:
            n = v.numel() if _is_dev(v) else v.size
            if n != self.n_elem:
                raise ValueError(f"vector has {n} elements, expected dim*R = {self.n_elem}")

    # ----- p_mltply_v3 / calc_vec_inprdct / calc_beta
    def p_mltply_v3(self, v1, v0, eperbd: float = 0.0):
        """v0 += (H - eperbd*ibond)^T v1 (in place); returns prdct (R complex)."""
        self._check_len(v1, v0)
        p1, f1 = _ptr(v1)
        p0, f0 = _ptr(v0, writable=True)
        pr = np.zeros(self.R, dtype=np.complex128)
        check(lib().pned_hv(self._h, p1, p0, float(eperbd), C.c_void_p(pr.ctypes.data), _same_flag(f1, f0)))
        return pr

    def calc_vec_inprdct(self, x1, x2):
        self._check_len(x1, x2)
        p1, f1 = _ptr(x1)
        p2, f2 = _ptr(x2)
        out = np.zeros(self.R, dtype=np.complex128)
        check(lib().pned_inprdct(self._h, p1, p2, C.c_void_p(out.ctypes.data), _same_flag(f1, f2)))
        return out

    def calc_beta(self, alpha, v1, v0):
        self._check_len(v1, v0)
        al = np.ascontiguousarray(np.broadcast_to(np.asarray(alpha, dtype=np.complex128), (self.R,)))
        p1, f1 = _ptr(v1)
        p0, f0 = _ptr(v0)
        out = np.zeros(self.R)
        check(lib().pned_calc_beta(self._h, C.c_void_p(al.ctypes.data), p1, p0, _dp(out), _same_flag(f1, f0)))
        return out

    def fill_gaussian(self, seed: int, out, normalise: bool = True):
        """Seeded complex-Gaussian vectors into a CUDA tensor (dim*R complex128)."""
        self._check_len(out)
        p, f = _ptr(out, writable=True)
        if f != PTR_DEVICE:
            raise TypeError("fill_gaussian writes device memory (a CUDA tensor)")
        check(lib().pned_fill_gaussian(self._h, C.c_uint64(seed), int(normalise), p))
        return out

    # ----- Krylov drivers
    def lanczos(self, v_init, n_steps: int, check_conv: bool = False):
        """parallelized_lnc1z on R chains: alpha/beta [steps][R], Ritz values of chain 0."""
        self._check_len(v_init)
        p, f = _ptr(v_init)
        a = np.zeros(n_steps * self.R)
        b = np.zeros(n_steps * self.R)
        ene = np.zeros(8)
        done = C.c_int(0)
        rc = lib().pned_lanczos_run(self._h, p, n_steps, int(check_conv), _dp(a), _dp(b), _dp(ene),
                                    C.byref(done), f)
        check(rc)
        k = done.value
        return dict(alpha=a[:k * self.R].reshape(k, self.R), beta=b[:k * self.R].reshape(k, self.R), ene=ene, itr=k)

    @staticmethod
    def _obs_array(observables):
        nobs = len(observables)
        keep = []
        arr = (_capi.Observable * max(1, nobs))()
        for o, spec in enumerate(observables):
            a_ = np.ascontiguousarray(spec.a, dtype=np.int32)
            b_ = np.ascontiguousarray(spec.b, dtype=np.int32)
            c_ = np.ascontiguousarray(spec.c, dtype=np.complex128)
            keep += [a_, b_, c_]
            arr[o].n_terms = a_.shape[0]
            arr[o].a = a_.ctypes.data_as(C.POINTER(C.c_int32))
            arr[o].b = b_.ctypes.data_as(C.POINTER(C.c_int32))
            arr[o].c = C.c_void_p(c_.ctypes.data)
            T = np.asarray(spec.T, dtype=np.complex128).reshape(4)
            for i in range(4):
                arr[o].T[i] = _capi.c128(T[i].real, T[i].imag)
        return arr, keep

    def tps(self, L: float, v_init, n_steps: int, observables=()):
        """parallelized_TPSz on R seeds with a model built for L - H."""
        self._check_len(v_init)
        p, f = _ptr(v_init)
        nobs = len(observables)
        arr, keep = self._obs_array(observables)
        ncoef = 5 + 2 * nobs
        al = np.zeros(n_steps * self.R)
        be = np.zeros(n_steps * self.R)
        co = np.zeros(n_steps * self.R * ncoef)
        check(lib().pned_tps_run(self._h, float(L), p, n_steps, nobs, arr, _dp(al), _dp(be), _dp(co), f))
        return dict(alpha=al.reshape(n_steps, self.R), beta=be.reshape(n_steps, self.R),
                    coef=co.reshape(n_steps, self.R, ncoef))

    def dsf(self, x, qr, n_steps: int):
        """intalv_zz + parallelized_dsflnc1z for R momenta (qr: [R][n] phases q.r_j)."""
        qr = np.ascontiguousarray(qr, dtype=np.float64)
        if qr.shape != (self.R, self.model.n):
            raise ValueError("qr must have shape (R, n)")
        n_x = x.numel() if _is_dev(x) else x.size
        if n_x != self.model.dim:
            raise ValueError("x must have dim elements")
        p, f = _ptr(x)
        cn = np.zeros(self.R)
        sa = np.zeros(n_steps * self.R)
        sb = np.zeros((n_steps + 1) * self.R)
        rc = lib().pned_dsf_run(self._h, p, _dp(qr), n_steps, _dp(cn), _dp(sa), _dp(sb), f)
        check(rc)
        return dict(cnorm=cn, salpha=sa.reshape(n_steps, self.R), sbeta=sb.reshape(n_steps + 1, self.R))

    def dsf_xy(self, source: "Model", x, qr, n_steps: int, ipm: int = 1):
        """intalv_xy + parallelized_dsflnc1z: chains of this context's model (the
        target sector) from S^{ipm}_q x, x on `source`'s basis; qr [R][n]."""
        qr = np.ascontiguousarray(qr, dtype=np.float64)
        if qr.shape != (self.R, self.model.n):
            raise ValueError("qr must have shape (R, n)")
        n_x = x.numel() if _is_dev(x) else x.size
        if n_x != source.dim:
            raise ValueError("x must have the source model's dim elements")
        p, f = _ptr(x)
        cn = np.zeros(self.R)
        sa = np.zeros(n_steps * self.R)
        sb = np.zeros((n_steps + 1) * self.R)
        check(lib().pned_dsf_xy_run(self._h, source._h, int(ipm), p, _dp(qr), n_steps, _dp(cn), _dp(sa), _dp(sb), f))
        return dict(cnorm=cn, salpha=sa.reshape(n_steps, self.R), sbeta=sb.reshape(n_steps + 1, self.R))

    def lanczos_vector(self, v_init, alpha, beta, coef, x_out=None):
        """parallelized_lncv1z (R = 1): x = sum_k coef[k] v_k over the replayed chain, normalised."""
        self._check_len(v_init)
        p, f = _ptr(v_init)
        if x_out is None:
            x_out = np.zeros(self.model.dim, dtype=np.complex128) if f == PTR_HOST else \
                torch.zeros(self.model.dim, dtype=torch.complex128, device=v_init.device)
        px, fx = _ptr(x_out, writable=True)
        a = np.ascontiguousarray(alpha, dtype=np.float64)
        b = np.ascontiguousarray(beta, dtype=np.float64)
        c = np.ascontiguousarray(coef, dtype=np.float64)
        n = len(c)
        if len(a) < n or len(b) < n:
            raise ValueError("alpha and beta need at least len(coef) entries")
        check(lib().pned_lanczos_vector(self._h, p, n, _dp(a), _dp(b), _dp(c), px, _same_flag(f, fx)))
        return x_out

    def cg(self, E: float, b_init, inv_max: int = 5000, cg_max: int = 500, x_out=None):
        """parallelized_inv1z + cg1 (R = 1): returns (x, n_inv, n_cg)."""
        self._check_len(b_init)
        p, f = _ptr(b_init)
        if x_out is None:
            x_out = np.zeros(self.model.dim, dtype=np.complex128) if f == PTR_HOST else \
                torch.zeros(self.model.dim, dtype=torch.complex128, device=b_init.device)
        px, fx = _ptr(x_out, writable=True)
        ni, nc = C.c_int(0), C.c_int(0)
        check(lib().pned_cg_run(self._h, float(E), p, inv_max, cg_max, px, C.byref(ni), C.byref(nc),
                                _same_flag(f, fx)))
        return x_out, ni.value, nc.value

    # ----- sessions: the Krylov vectors stay on the device between calls
    def session_begin(self, kind: str, v_init, max_steps: int, L: float = 0.0, observables=()):
        """Starts a 'lanczos' or 'tps' session from v_init ([dim][R])."""
        self._check_len(v_init)
        p, f = _ptr(v_init)
        k = {"lanczos": _capi.SESSION_LANCZOS, "tps": _capi.SESSION_TPS}[kind]
        arr, keep = self._obs_array(observables)
        self._sess = dict(kind=kind, nobs=len(observables), max_steps=max_steps)
        check(lib().pned_session_begin(self._h, k, p, int(max_steps), float(L), len(observables), arr, f))

    def session_begin_dsf(self, x, qr, max_steps: int):
        qr = np.ascontiguousarray(qr, dtype=np.float64)
        p, f = _ptr(x)
        cn = np.zeros(self.R)
        check(lib().pned_session_begin_dsf(self._h, p, _dp(qr), int(max_steps), _dp(cn), f))
        self._sess = dict(kind="dsf", nobs=0, max_steps=max_steps)
        return cn

    def session_step(self, n: int):
        """Enqueues n steps (asynchronous)."""
        check(lib().pned_session_step(self._h, int(n)))

    def session_read(self):
        s = self._sess
        m = s["max_steps"]
        a = np.zeros(m * self.R)
        b = np.zeros(m * self.R)
        nc = 5 + 2 * s["nobs"]
        co = np.zeros(m * self.R * nc) if s["kind"] == "tps" else None
        k, st = C.c_int(0), C.c_int(0)
        check(lib().pned_session_read(self._h, _dp(a), _dp(b), None if co is None else _dp(co), C.byref(k),
                                      C.byref(st)))
        k = k.value
        out = dict(alpha=a[:k * self.R].reshape(k, self.R), beta=b[:k * self.R].reshape(k, self.R), steps=k,
                   breakdown=bool(st.value))
        if co is not None:
            out["coef"] = co[:k * self.R * nc].reshape(k, self.R, nc)
        return out

    def session_profile(self, n: int):
        """Mean (hv_ms, step_ms) over n further steps timed one by one with CUDA events."""
        a, b = C.c_double(0), C.c_double(0)
        check(lib().pned_session_profile(self._h, int(n), C.byref(a), C.byref(b)))
        return a.value, b.value

    def session_vector(self):
        """(device pointer of the current Krylov vector buffer, scales[R])."""
        p = C.c_void_p()
        sc = np.zeros(self.R)
        check(lib().pned_session_vector(self._h, C.byref(p), _dp(sc)))
        return p.value, sc

    def session_save(self, path: str):
        """Checkpoint of the running session (waits for its enqueued steps)."""
        check(lib().pned_session_save(self._h, os.fsencode(path)))

    def session_load(self, path: str, max_steps: int = 0):
        """Resumes a checkpointed session on this context (same basis and R)."""
        check(lib().pned_session_load(self._h, os.fsencode(path), int(max_steps)))
        kind, done, ms, nc = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
        check(lib().pned_session_info(self._h, C.byref(kind), C.byref(done), C.byref(ms), C.byref(nc)))
        names = {_capi.SESSION_LANCZOS: "lanczos", _capi.SESSION_TPS: "tps", _capi.SESSION_DSF: "dsf"}
        self._sess = {"kind": names[kind.value], "max_steps": ms.value, "nobs": max(0, (nc.value - 5) // 2)}

    def session_end(self):
        check(lib().pned_session_end(self._h))
        self._sess = None

    def lanczos_state(self):
        """The running Lanczos session (R = 1) as the reference's loop holds it at the
        top of its next iteration: (v0, v1) = (H v_k - beta v_{k-1}, v_k) on the host."""
        w = np.zeros(self.model.dim, dtype=np.complex128)
        v = np.zeros(self.model.dim, dtype=np.complex128)
        check(lib().pned_session_lanczos_state(self._h, C.c_void_p(w.ctypes.data), C.c_void_p(v.ctypes.data),
                                               PTR_HOST))
        return w, v

    def lanczos_dump_reference(self, path: str, vec_size: int = REF_MAX_ITR, ene_size: int = REF_MAX_ITR, **info_kw):
        """Writes the running Lanczos session (R = 1) as parallelized_lnc1z's
        interval_dump does (S1/2 Lanczos.f90:99-103; files `path`, `path`.info):
        alpha, beta (vec_size each, zero past the steps done), coef (vec_size x
        9, zero: lnc1z keeps none), ene (the 8 lowest Ritz values so far, then
        zeros), vec1 = v0, vec2 = v1, and itr_counter(1) = steps done + 1."""
        r = self.session_read()
        k = r["steps"]
        if k < 1 or k > vec_size:
            raise ValueError("the session needs 1..vec_size steps done")
        a = np.zeros(vec_size)
        b = np.zeros(vec_size)
        a[:k], b[:k] = r["alpha"][:, 0], r["beta"][:, 0]
        ene = np.zeros(ene_size)
        ne = min(k, REF_NVEC)
        ene[:ne] = bisec(a[:k], b[:k], k, ne)
        w, v = self.lanczos_state()
        m = self.model
        itr = (k + 1, vec_size, 2, vec_size, 1, 5000, 1, 500, 1, REF_NVEC, 2, REF_S_MAXITR)
        info = dump_info(m.n, m.n_bonds, itr, **info_kw)
        write_interval_dump(path, info, vec_size, sa=a, sb=b, sc=np.zeros((vec_size, REF_NVEC + 1), order="F"),
                            se=ene, vec1=w, vec2=v)

    def dsf_dump_reference(self, path: str, cnorm: float, vec_size: int = REF_S_MAXITR, iq: int = 1, **info_kw):
        """Writes the running DSF chain session (R = 1) as parallelized_dsflnc1z's
        interval_dump does (S1/2 DSF.f90:234-238): salpha, sbeta (vec_size each;
        sbeta(1) = cnorm, sbeta(i+1) = beta_i), vec1 = v1, vec2 = v0, with
        itr_counter(9) = iq and itr_counter(11) = steps done + 1."""
        r = self.session_read()
        k = r["steps"]
        if k < 1 or k + 1 > vec_size:
            raise ValueError("the session needs 1..vec_size-1 steps done")
        a = np.zeros(vec_size)
        b = np.zeros(vec_size)
        a[:k] = r["alpha"][:, 0]
        b[0] = float(np.real(cnorm))
        b[1:k + 1] = r["beta"][:, 0]
        w, v = self.lanczos_state()
        m = self.model
        itr = (2, REF_MAX_ITR, 2, REF_MAX_ITR, 1, 5000, 1, 500, int(iq), REF_NVEC, k + 1, vec_size)
        info_kw = {"position": (0, 0, 0, 1, 1, 0, 0), "dsf_comp": "zz", **info_kw}
        info = dump_info(m.n, m.n_bonds, itr, s_maxitr=vec_size, **info_kw)
        write_interval_dump(path, info, vec_size, sa=a, sb=b, vec1=v, vec2=w)

    def dsf_resume_reference(self, path: str, max_steps: int):
        """Starts a DSF chain session (R = 1) from parallelized_dsflnc1z's dump files;
        returns (steps done, cnorm)."""
        info = read_interval_dump_info(path)
        k = info["itr_counter"][10] - 1
        d = read_interval_dump(path, "dsflnc")
        if d["data_size"] != self.model.dim or k < 1 or k + 1 > d["sa"].size:
            raise ValueError(f"{path}: not a DSF dump of this basis")
        a = np.ascontiguousarray(d["sa"][:k])
        b = np.ascontiguousarray(d["sb"][1:k + 1])
        check(lib().pned_session_begin_dsf_at(self._h, C.c_void_p(d["vec2"].ctypes.data),
                                              C.c_void_p(d["vec1"].ctypes.data), _dp(a), _dp(b), int(k),
                                              int(max_steps), PTR_HOST))
        self._sess = dict(kind="dsf", nobs=0, max_steps=int(max_steps))
        return k, float(d["sb"][0])

    def tps_dump_reference(self, path: str, vec_size: int | None = None, ene_size: int = REF_MAX_ITR, **info_kw):
        """Writes the running TPS session (R = 1) as parallelized_TPSz's interval_dump
        does (S1/2 TPS.f90:368-372): alpha, beta (vec_size each), coef (vec_size x
        the session's coefficients per step, column-major: the reference's first
        five columns, then two per observable), ene (zeros: TPS keeps none), vec1
        = v0, vec2 = v1, vec3 = vg, and itr_counter(1) = steps done + 1."""
        r = self.session_read()
        k = r["steps"]
        vec_size = int(vec_size or self._sess["max_steps"])
        if k < 1 or k > vec_size:
            raise ValueError("the session needs 1..vec_size steps done")
        a = np.zeros(vec_size)
        b = np.zeros(vec_size)
        a[:k], b[:k] = r["alpha"][:, 0], r["beta"][:, 0]
        nc = r["coef"].shape[-1]
        coef = np.zeros((vec_size, nc), order="F")
        coef[:k] = r["coef"][:, 0, :]
        w = np.zeros(self.model.dim, dtype=np.complex128)
        v = np.zeros_like(w)
        g = np.zeros_like(w)
        check(lib().pned_session_tps_state(self._h, C.c_void_p(w.ctypes.data), C.c_void_p(v.ctypes.data),
                                           C.c_void_p(g.ctypes.data), PTR_HOST))
        m = self.model
        itr = (k + 1, vec_size, 2, vec_size, 1, 5000, 1, 500, 1, REF_NVEC, 2, REF_S_MAXITR)
        info_kw = {"position": (0, 0, 0, 0, 0, 0, 1), "dsf_comp": "tp", **info_kw}
        info = dump_info(m.n, m.n_bonds, itr, **info_kw)
        write_interval_dump(path, info, vec_size, sa=a, sb=b, sc=coef, se=np.zeros(ene_size), vec1=w, vec2=v, vec3=g)

    def tps_resume_reference(self, path: str, max_steps: int):
        """Starts a TPS session (R = 1, this context's model built for L - H) from
        parallelized_TPSz's interval_dump files (S1/2 TPS.f90:359-363), carrying
        alpha, beta and the first five coefficient columns (observable columns are
        not resumed); L is the dump's coef(1, 2).  Returns the steps done."""
        info = read_interval_dump_info(path)
        k = info["itr_counter"][0] - 1
        if info["n"] != self.model.n:
            raise ValueError(f"{path}: dump of {info['n']} sites, the model has {self.model.n}")
        d = read_interval_dump(path, "tpsz")
        vs = d["sa"].size
        if d["data_size"] != self.model.dim or k < 1 or k > vs or d["sc"].size % vs:
            raise ValueError(f"{path}: not a TPS dump of this basis")
        coef = d["sc"].reshape(vs, -1, order="F")
        if coef.shape[1] < 5:
            raise ValueError(f"{path}: fewer than five coefficient columns")
        L = float(coef[0, 1])
        a = np.ascontiguousarray(d["sa"][:k])
        b = np.ascontiguousarray(d["sb"][:k])
        cf = np.ascontiguousarray(coef[:k, :5])
        check(lib().pned_session_begin_tps_at(self._h, L, C.c_void_p(d["vec1"].ctypes.data),
                                              C.c_void_p(d["vec2"].ctypes.data), _dp(a), _dp(b), _dp(cf), int(k),
                                              int(max_steps), PTR_HOST))
        self._sess = dict(kind="tps", nobs=0, max_steps=int(max_steps))
        return k

    def lanczos_resume_reference(self, path: str, max_steps: int):
        """Starts a Lanczos session (R = 1) from parallelized_lnc1z's interval_dump
        files, as interval_dump_read resumes the loop (S1/2 Lanczos.f90:87-93):
        itr_counter(1) - 1 steps done; returns that count."""
        info = read_interval_dump_info(path)
        k = info["itr_counter"][0] - 1
        if info["n"] != self.model.n:
            raise ValueError(f"{path}: dump of {info['n']} sites, the model has {self.model.n}")
        d = read_interval_dump(path, "lnc1z")
        if d["data_size"] != self.model.dim or k < 1 or k > d["sa"].size:
            raise ValueError(f"{path}: not a Lanczos dump of this basis")
        a = np.ascontiguousarray(d["sa"][:k])
        b = np.ascontiguousarray(d["sb"][:k])
        check(lib().pned_session_begin_lanczos_at(self._h, C.c_void_p(d["vec1"].ctypes.data),
                                                  C.c_void_p(d["vec2"].ctypes.data), _dp(a), _dp(b), int(k),
                                                  int(max_steps), PTR_HOST))
        self._sess = dict(kind="lanczos", nobs=0, max_steps=int(max_steps))
        return k


# --------------------------------------------------------------------------- slot batches


def gaussian_column(dim: int, R: int, r: int, seed: int, out, stream=None):
    """Column r of the seeded [dim][R] complex Gaussian start vectors (unnormalised)
    into the CUDA tensor `out` on `stream`; does not wait."""
    p, f = _ptr(out, writable=True)
    if f != PTR_DEVICE or out.numel() != dim:
        raise TypeError("out must be a CUDA tensor of dim elements")
    sp = None if stream is None else C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else stream)
    check(lib().pned_gaussian_column(int(dim), int(R), int(r), C.c_uint64(int(seed) & (2**64 - 1)), p, sp))

SLOT_KINDS = {"free": 0, "lanczos": 1, "tps": 2, "vector": 3}
_SLOT_NAMES = {v: k for k, v in SLOT_KINDS.items()}


class SlotBatch:
    """R slots of independent chains over one S = 1/2 lattice (pned_slots_*).

    Each slot carries its own couplings (a ModelInput on the batch's lattice);
    all slots advance together, one batched H.V per step, and a slot is loaded
    or released between steps while the others keep running."""

    def __init__(self, structure: ModelInput, R: int, max_steps: int, hbm_budget: int = 0, stream=None):
        self.structure = structure
        h = C.c_void_p()
        check(lib().pned_slots_create(C.byref(structure.c), int(R), int(max_steps), C.c_size_t(int(hbm_budget)),
                                      C.byref(h)))
        self._h = h
        dim, r, ms, nb = C.c_int64(0), C.c_int(0), C.c_int(0), C.c_size_t(0)
        check(lib().pned_slots_info(h, C.byref(dim), C.byref(r), C.byref(ms), C.byref(nb)))
        self.dim, self.R, self.max_steps, self.bytes = dim.value, r.value, ms.value, nb.value
        self.n = structure.n
        self._stream = None
        if stream is not None:
            self.set_stream(stream)

    def set_stream(self, stream):
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        check(lib().pned_slots_set_stream(self._h, C.c_void_p(sp)))
        self._stream = stream

    def _vec(self, v):
        p, f = _ptr(v)
        n = v.numel() if _is_dev(v) else v.size
        if n != self.dim:
            raise ValueError(f"vector has {n} elements, expected dim = {self.dim}")
        return p, f

    def load(self, slot: int, kind: str, couplings: ModelInput, v_init, n_steps: int, L: float = 0.0):
        """Starts a Lanczos ('lanczos') or TPS ('tps', shift L) chain in `slot` from v_init (normalised here)."""
        p, f = self._vec(v_init)
        check(lib().pned_slots_load(self._h, int(slot), SLOT_KINDS[kind], C.byref(couplings.c), p, int(n_steps),
                                    float(L), f))

    def load_szq(self, slot: int, couplings: ModelInput, x, qr, n_steps: int):
        """Starts a DSF momentum chain from S^z_q x (phases qr[j] = q.r_j)."""
        p, f = self._vec(x)
        q = np.ascontiguousarray(qr, dtype=np.float64)
        if q.shape != (self.n,):
            raise ValueError("qr must have n entries")
        check(lib().pned_slots_load_szq(self._h, int(slot), C.byref(couplings.c), p, _dp(q), int(n_steps), f))

    def load_vector(self, slot: int, couplings: ModelInput, v_init, alpha, beta, coef, x_dev):
        """Eigenvector pass: replays the chain of v_init with stored alpha/beta and
        accumulates x = sum_k coef[k] v_k into the CUDA tensor x_dev."""
        p, f = self._vec(v_init)
        px, fx = _ptr(x_dev, writable=True)
        if fx != PTR_DEVICE or x_dev.numel() != self.dim:
            raise TypeError("x_dev must be a CUDA tensor of dim elements")
        a = np.ascontiguousarray(alpha, dtype=np.float64)
        b = np.ascontiguousarray(beta, dtype=np.float64)
        c = np.ascontiguousarray(coef, dtype=np.float64)
        n = len(c)
        if len(a) < n or len(b) < n:
            raise ValueError("alpha and beta need at least len(coef) entries")
        check(lib().pned_slots_load_vector(self._h, int(slot), C.byref(couplings.c), p, n, _dp(a), _dp(b), _dp(c),
                                           px, f))

    def release(self, slot: int):
        check(lib().pned_slots_release(self._h, int(slot)))

    def plan(self) -> dict:
        p, g, t = C.c_int(0), C.c_int(0), C.c_int(0)
        check(lib().pned_slots_plan(self._h, C.byref(p), C.byref(g), C.byref(t)))
        return {"tile_passes": p.value, "partner_tiles": g.value, "tile_states": t.value}

    def set_plan(self, row_fixed_bits: int = -1, window_bits: int = -1, max_passes: int = -1,
                 j_bits: int = -1, l1_carveout: int = 1, stage_partner_tiles: int = 0, blocks_per_sm: int = -1,
                 objective: int = -1, terms_in_flight: int = -1) -> dict:
        tp = _capi.TilePlan(int(row_fixed_bits), int(window_bits), int(max_passes), int(j_bits), int(l1_carveout),
                            int(stage_partner_tiles), int(blocks_per_sm), int(objective), int(terms_in_flight))
        check(lib().pned_slots_set_plan(self._h, C.byref(tp)))
        return self.plan()

    def step(self, n: int):
        check(lib().pned_slots_step(self._h, int(n)))

    def query(self) -> bool:
        rc = lib().pned_slots_query(self._h)
        if rc not in (0, 1):
            check(rc)
        return rc == 1

    def synchronize(self):
        check(lib().pned_slots_synchronize(self._h))

    def read(self, slot: int) -> dict:
        kind, steps, status, cn = C.c_int(0), C.c_int(0), C.c_int(0), C.c_double(0.0)
        check(lib().pned_slots_read(self._h, int(slot), C.byref(kind), C.byref(steps), C.byref(status), None, None,
                                    None, None))
        k = steps.value
        a, b, c = np.zeros(max(1, k)), np.zeros(max(1, k)), np.zeros((max(1, k), 5))
        check(lib().pned_slots_read(self._h, int(slot), C.byref(kind), C.byref(steps), C.byref(status), _dp(a),
                                    _dp(b), _dp(c), C.byref(cn)))
        return {"kind": _SLOT_NAMES.get(kind.value, kind.value), "steps": k, "status": status.value,
                "alpha": a[:k], "beta": b[:k], "coef": c[:k], "cnorm": cn.value}

    def close(self):
        if getattr(self, "_h", None):
            lib().pned_slots_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
