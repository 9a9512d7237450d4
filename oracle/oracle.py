"""ctypes wrapper of the CPU oracle (oracle/pned_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, as the checker or the timed CPU baseline.  The
product package ``pned_b200`` never imports it.

Parity unpinned by the reference itself (no Fortran compiler in the image and
no golden vectors shipped with pNED); the restatement is pinned by the dense
and known-answer checks of tests/test_oracle.py.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# PNED_ORACLE_BUILD=fma loads the build with fused multiply-adds (see the Makefile):
# the same algorithm with other rounding, used to measure the spread of long chains
_VARIANT = os.environ.get("PNED_ORACLE_BUILD", "")
_LIB_PATH = os.path.join(_HERE, "_build", "libpned_oracle_fma.so" if _VARIANT == "fma" else "libpned_oracle.so")
_lib = None

c_int_p = C.POINTER(C.c_int)
c_dbl_p = C.POINTER(C.c_double)
c_i64_p = C.POINTER(C.c_int64)
c_u8_p = C.POINTER(C.c_uint8)


class c_cplx(C.Structure):
    """double _Complex by value (same SysV classification as two doubles)."""
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    if force or not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "pned_oracle.c"))):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp = C.c_void_p
        L.oracle_xlocal_matrices.argtypes = [C.c_int, C.c_int, c_dbl_p, C.c_int, vp]
        L.oracle_add_field.argtypes = [C.c_int, C.c_int, c_dbl_p, C.c_double, vp]
        L.oracle_parity_skip.argtypes = [C.c_int, C.c_int, vp, c_u8_p, c_u8_p, c_int_p]
        L.oracle_tps_reference.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, vp]
        L.oracle_tps_reference.restype = C.c_double
        L.oracle_tps_explicit.argtypes = [C.c_int, C.c_int, C.c_double, vp]
        L.oracle_mk_list12.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.POINTER(c_i64_p), C.POINTER(c_i64_p), C.POINTER(c_i64_p), c_i64_p]
        L.oracle_mk_list12.restype = C.c_int64
        L.oracle_free.argtypes = [vp]
        L.oracle_model_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, c_int_p, c_int_p, vp, c_u8_p,
                                          C.c_int, C.c_int, C.c_int]
        L.oracle_model_create.restype = vp
        L.oracle_model_destroy.argtypes = [vp]
        L.oracle_model_ldim.argtypes = [vp]
        L.oracle_model_ldim.restype = C.c_int64
        L.oracle_model_nitem.argtypes = [vp]
        L.oracle_model_item.argtypes = [vp, C.c_int, c_int_p, c_int_p, c_int_p, c_int_p]
        L.oracle_p_mltply_v3.argtypes = [vp, vp, vp, C.c_double, vp]
        L.oracle_p_mltply_v3_slice.argtypes = [vp, vp, vp, C.c_double, C.c_int64, C.c_int64, vp]
        L.oracle_inprdct.argtypes = [C.c_int64, vp, vp]
        L.oracle_inprdct.restype = c_cplx
        L.oracle_calc_beta.argtypes = [C.c_int64, c_cplx, vp, vp]
        L.oracle_calc_beta.restype = C.c_double
        L.oracle_bisec.argtypes = [c_dbl_p, c_dbl_p, C.c_int, c_dbl_p, C.c_int, C.c_double]
        L.oracle_vec12.argtypes = [c_dbl_p, c_dbl_p, c_dbl_p, c_dbl_p, C.c_int, C.c_int]
        L.oracle_lanczos.argtypes = [vp, vp, C.c_int, C.c_int, c_dbl_p, c_dbl_p, c_dbl_p, c_int_p]
        L.oracle_tps.argtypes = [vp, C.c_double, vp, C.c_int, C.c_int, c_int_p, c_int_p, c_int_p, vp, vp,
                                 c_dbl_p, c_dbl_p, c_dbl_p, C.c_int]
        L.oracle_intalv_zz.argtypes = [vp, c_dbl_p, vp, vp, vp]
        L.oracle_intalv_xy.argtypes = [vp, vp, C.c_int, c_dbl_p, vp, vp, vp]
        L.oracle_dsf_chain.argtypes = [vp, vp, c_cplx, C.c_int, c_dbl_p, c_dbl_p]
        L.oracle_exec_renbun.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, c_dbl_p, c_dbl_p,
                                         c_dbl_p, c_int_p, c_dbl_p]
        L.oracle_normalization_dsf.argtypes = [C.c_int, C.c_double, C.c_double, c_dbl_p]
        L.oracle_inverse_iteration.argtypes = [vp, C.c_double, vp, vp, C.c_int, C.c_int, c_int_p, c_int_p]
        L.oracle_lanczos_vector.argtypes = [vp, vp, C.c_int, c_dbl_p, c_dbl_p, c_dbl_p, vp]
        L.oracle_lanczos_step.argtypes = [vp, vp, vp, c_dbl_p, c_dbl_p]
        L.oracle_lanczos_step_slice.argtypes = [vp, vp, vp, C.c_int64, C.c_int64, c_dbl_p, c_dbl_p]
        L.oracle_gaussian.argtypes = [C.c_uint64, C.c_int64, C.c_int, vp]
        L.oracle_num_threads.restype = C.c_int
        L.oracle_set_num_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def _p(a, t=None):
    if t is None:
        return C.c_void_p(a.ctypes.data)
    return a.ctypes.data_as(C.POINTER(t))


def _c128(a):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a


# ----------------------------------------------------------------------------- model building

def xlocal(q: int, tree_sa: int, cpl, simple: int = 0, field=None, coord: float = 3.0) -> np.ndarray:
    """set_xlocal_Ham matrices (+ optional field extension).

    Returns X with shape (9, Q, Q) indexed [type-1, col, row] (Fortran layout).
    """
    Q = q * q
    cpl = np.ascontiguousarray(cpl, dtype=np.float64)
    X = np.zeros((9, Q, Q), dtype=np.complex128)
    rc = lib().oracle_xlocal_matrices(q, tree_sa, _p(cpl, C.c_double), simple, _p(X))
    if rc:
        raise ValueError("oracle_xlocal_matrices failed")
    if field is not None:
        h = np.ascontiguousarray(field, dtype=np.float64)
        lib().oracle_add_field(q, tree_sa, _p(h, C.c_double), coord, _p(X))
    return X


def parity_skip(q: int, tree_sa: int, X: np.ndarray):
    Q = q * q
    X = _c128(X)
    skip = np.zeros((9, Q, Q), dtype=np.uint8)
    pskip = np.zeros((9, Q), dtype=np.uint8)
    pt = C.c_int(0)
    lib().oracle_parity_skip(q, tree_sa, _p(X), _p(skip, C.c_uint8), _p(pskip, C.c_uint8), C.byref(pt))
    return skip, pskip, pt.value


def tps_reference(q: int, tree_sa: int, nbond: int, X: np.ndarray, c_count: float = 3.0):
    X = _c128(X).copy()
    L = lib().oracle_tps_reference(q, tree_sa, nbond, c_count, _p(X))
    return X, L


def tps_explicit(q: int, nbond: int, L: float, X: np.ndarray):
    X = _c128(X).copy()
    lib().oracle_tps_explicit(q, nbond, L, _p(X))
    return X


def mk_list12(n: int, q: int, parity_type: int, tot_sz: int, is_shift: int = 0):
    l1, a, b = c_i64_p(), c_i64_p(), c_i64_p()
    nl3 = C.c_int64(0)
    ldim = lib().oracle_mk_list12(n, q, parity_type, tot_sz, is_shift, C.byref(l1), C.byref(a), C.byref(b),
                                  C.byref(nl3))
    list1 = np.ctypeslib.as_array(l1, shape=(ldim,)).copy()
    l3a = np.ctypeslib.as_array(a, shape=(nl3.value,)).copy()
    l3b = np.ctypeslib.as_array(b, shape=(nl3.value,)).copy()
    for p in (l1, a, b):
        lib().oracle_free(C.cast(p, C.c_void_p))
    return list1, l3a, l3b


def gaussian(seed: int, dim: int, R: int = 1) -> np.ndarray:
    v = np.empty(dim * R, dtype=np.complex128)
    lib().oracle_gaussian(C.c_uint64(seed), dim, R, _p(v))
    return v


def inprdct(x1, x2) -> complex:
    r = lib().oracle_inprdct(x1.shape[0], _p(x1), _p(x2))
    return complex(r.re, r.im)


def bisec(alpha, beta, ndim, ne, eps=1e-25):
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    b = np.ascontiguousarray(beta, dtype=np.float64)
    E = np.zeros(max(ne, 1))
    rc = lib().oracle_bisec(_p(a, C.c_double), _p(b, C.c_double), ndim, _p(E, C.c_double), ne, eps)
    if rc:
        raise ValueError("bisec: bad arguments")
    return E[:ne]


def vec12(alpha, beta, E, ndim, nvec):
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    b = np.ascontiguousarray(beta, dtype=np.float64)
    b = np.concatenate([b, np.zeros(2)])
    e = np.ascontiguousarray(E, dtype=np.float64)
    v = np.zeros((nvec, ndim))
    lib().oracle_vec12(_p(a, C.c_double), _p(b, C.c_double), _p(v, C.c_double), _p(e, C.c_double), ndim, nvec)
    return v


def exec_renbun(i_range, s_maxitr, split, ene, epsln, salpha, sbeta):
    sa = np.zeros(s_maxitr)
    sb = np.zeros(s_maxitr)
    sa[:min(len(salpha), s_maxitr)] = salpha[:s_maxitr]
    sb[:min(len(sbeta), s_maxitr)] = sbeta[:s_maxitr]
    w = np.zeros(i_range)
    conv = np.zeros(i_range, dtype=np.int32)
    dsf = np.zeros(i_range)
    lib().oracle_exec_renbun(i_range, s_maxitr, split, ene, epsln, _p(sa, C.c_double), _p(sb, C.c_double),
                             _p(w, C.c_double), _p(conv, C.c_int), _p(dsf, C.c_double))
    return w, conv, dsf


def normalization_dsf(i_range, split, sq_re, dsf):
    d = np.ascontiguousarray(dsf, dtype=np.float64).copy()
    lib().oracle_normalization_dsf(i_range, split, sq_re, _p(d, C.c_double))
    return d


def set_num_threads(n: int):
    lib().oracle_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().oracle_num_threads())


class Model:
    """Oracle model: the lnp = 1 item schedule and Lin tables of the reference."""

    def __init__(self, n, q, tree_sa, ipair, ibond_type, X, skip, parity_type, tot_sz=None, is_shift=0):
        if tot_sz is None:
            tot_sz = n // 2 * (q - 1)
        self.n, self.q, self.tree_sa = n, q, tree_sa
        self.ipair = np.ascontiguousarray(ipair, dtype=np.int32)
        self.ibond_type = np.ascontiguousarray(ibond_type, dtype=np.int32)
        self.X = _c128(X)
        self.skip = np.ascontiguousarray(skip, dtype=np.uint8)
        self.nbond = int(self.ibond_type.shape[0])
        self._h = lib().oracle_model_create(n, q, tree_sa, self.nbond, _p(self.ipair, C.c_int),
                                            _p(self.ibond_type, C.c_int), _p(self.X), _p(self.skip, C.c_uint8),
                                            parity_type, tot_sz, is_shift)
        self.ldim = int(lib().oracle_model_ldim(self._h))

    def close(self):
        if self._h:
            lib().oracle_model_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def items(self):
        out = []
        a, b, t, e = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        for k in range(lib().oracle_model_nitem(self._h)):
            lib().oracle_model_item(self._h, k, C.byref(a), C.byref(b), C.byref(t), C.byref(e))
            out.append((a.value, b.value, t.value, e.value))
        return out

    def p_mltply_v3(self, v1, v0, eperbd=0.0):
        """v0 += (H - eperbd*ibond)^T v1 in place; returns prdct."""
        assert v1.dtype == np.complex128 and v0.dtype == np.complex128
        pr = np.zeros(1, dtype=np.complex128)
        lib().oracle_p_mltply_v3(self._h, _p(v1), _p(v0), eperbd, _p(pr))
        return complex(pr[0])

    def p_mltply_v3_slice(self, v1, v0_slice, lo, hi, eperbd=0.0):
        pr = np.zeros(1, dtype=np.complex128)
        lib().oracle_p_mltply_v3_slice(self._h, _p(v1), _p(v0_slice), eperbd, lo, hi, _p(pr))
        return complex(pr[0])

    def lanczos_step(self, v1, v0, alpha, beta):
        """One step of the Lanczos loop on (v1, v0) in place: the swap with the
        previous alpha/beta, then p_mltply_v3 and calc_beta; returns (alpha, beta)."""
        a, b = C.c_double(alpha), C.c_double(beta)
        lib().oracle_lanczos_step(self._h, _p(v1), _p(v0), C.byref(a), C.byref(b))
        return a.value, b.value

    def lanczos_step_slice(self, v1, v0_slice, lo, hi, alpha, beta):
        """The same step on the output states [lo, hi) (v0_slice holds them);
        returns the slice's parts (alpha, sqrt of the beta sum)."""
        a, b = C.c_double(alpha), C.c_double(beta)
        lib().oracle_lanczos_step_slice(self._h, _p(v1), _p(v0_slice), lo, hi, C.byref(a), C.byref(b))
        return a.value, b.value

    def lanczos(self, v1, nsteps, check_conv=False):
        v = _c128(v1).copy()
        alpha = np.zeros(nsteps)
        beta = np.zeros(nsteps)
        ene = np.zeros(8)
        itr = C.c_int(0)
        rc = lib().oracle_lanczos(self._h, _p(v), nsteps, int(check_conv), _p(alpha, C.c_double),
                                  _p(beta, C.c_double), _p(ene, C.c_double), C.byref(itr))
        return dict(alpha=alpha[:itr.value], beta=beta[:itr.value], ene=ene, itr=itr.value, rc=rc, v=v)

    def tps(self, L, v1, nsteps, observables=()):
        """observables: list of (terms [(a, b, c complex)], T 2x2 complex)."""
        v = _c128(v1).copy()
        nobs = len(observables)
        off = [0]
        ta, tb, tc, T = [], [], [], []
        for terms, tab in observables:
            for (a, b, c) in terms:
                ta.append(a)
                tb.append(b)
                tc.append(c)
            off.append(len(ta))
            T.append(np.asarray(tab, dtype=np.complex128).reshape(4))
        off = np.asarray(off, dtype=np.int32)
        ta = np.asarray(ta + [0], dtype=np.int32)
        tb = np.asarray(tb + [0], dtype=np.int32)
        tc = np.asarray(tc + [0], dtype=np.complex128)
        T = np.asarray(T if T else [np.zeros(4)], dtype=np.complex128).reshape(-1)
        ncoef = 5 + 2 * nobs
        alpha = np.zeros(nsteps)
        beta = np.zeros(nsteps)
        coef = np.zeros((nsteps, ncoef))
        rc = lib().oracle_tps(self._h, L, _p(v), nsteps, nobs, _p(off, C.c_int), _p(ta, C.c_int), _p(tb, C.c_int),
                              _p(tc), _p(T), _p(alpha, C.c_double), _p(beta, C.c_double), _p(coef, C.c_double),
                              ncoef)
        if rc:
            raise RuntimeError(f"oracle_tps rc={rc}")
        return dict(alpha=alpha, beta=beta, coef=coef, v=v)

    def intalv_zz(self, qr, x):
        qr = np.ascontiguousarray(qr, dtype=np.float64)
        v = np.zeros(self.ldim, dtype=np.complex128)
        cn = np.zeros(1, dtype=np.complex128)
        xs = _c128(x)   # keep the array alive across the call
        lib().oracle_intalv_zz(self._h, _p(qr, C.c_double), _p(xs), _p(v), _p(cn))
        return v, complex(cn[0])

    def intalv_xy(self, source, ipm, qr, x):
        """S^{ipm}_q start vector on this model's basis from x on `source`'s basis."""
        qr = np.ascontiguousarray(qr, dtype=np.float64)
        v = np.zeros(self.ldim, dtype=np.complex128)
        cn = np.zeros(1, dtype=np.complex128)
        xs = _c128(x)   # keep the array alive across the call
        rc = lib().oracle_intalv_xy(self._h, source._h, int(ipm), _p(qr, C.c_double), _p(xs), _p(v), _p(cn))
        if rc:
            raise ValueError(f"oracle_intalv_xy rc={rc}")
        return v, complex(cn[0])

    def dsf_chain(self, v1, cnorm, nsteps):
        v = _c128(v1).copy()
        sa = np.zeros(nsteps)
        sb = np.zeros(nsteps + 1)
        cn = c_cplx(cnorm.real, cnorm.imag)
        rc = lib().oracle_dsf_chain(self._h, _p(v), cn, nsteps, _p(sa, C.c_double), _p(sb, C.c_double))
        if rc:
            raise RuntimeError("oracle_dsf_chain failed")
        return sa, sb

    def lanczos_vector(self, v1, alpha, beta, coef):
        """parallelized_lncv1z: x = sum_k coef[k] v_k over the replayed chain, normalised."""
        x = np.zeros(self.ldim, dtype=np.complex128)
        a = np.ascontiguousarray(alpha, dtype=np.float64)
        b = np.ascontiguousarray(beta, dtype=np.float64)
        c = np.ascontiguousarray(coef, dtype=np.float64)
        v = _c128(v1).copy()   # kept alive across the call
        rc = lib().oracle_lanczos_vector(self._h, _p(v), len(c), _p(a, C.c_double),
                                         _p(b, C.c_double), _p(c, C.c_double), _p(x))
        if rc:
            raise RuntimeError(f"oracle_lanczos_vector rc={rc}")
        return x

    def inverse_iteration(self, E, b, inv_max=5000, cg_max=500):
        x = np.zeros(self.ldim, dtype=np.complex128)
        ni, nc = C.c_int(0), C.c_int(0)
        bw = _c128(b).copy()   # kept alive across the call
        lib().oracle_inverse_iteration(self._h, E, _p(bw), _p(x), inv_max, cg_max, C.byref(ni),
                                       C.byref(nc))
        return x, ni.value, nc.value


# --------------------------------------------------------------------------- mTPQ output chain (numpy)

def tpq_thermo(beta, energy, hmix, t_min, t_max, num_div):
    """eval_mpi restated in numpy/Python loops (S_one_half/Hybrid_TPS_eval_mpi.f90:
    calc_fac :236-281, eval_q :284-313, lsort :315-347, calc_ave :349-363, main
    loop :395-430); arrays [n_seeds][num_data1]; returns [num_div+1][5]:
    T, E(T), dE/dT, variance, d2E/dT2."""
    import math
    beta = np.atleast_2d(np.asarray(beta, dtype=np.float64))
    energy = np.atleast_2d(np.asarray(energy, dtype=np.float64))
    hmix = np.atleast_2d(np.asarray(hmix, dtype=np.float64))
    nseed, nd1 = beta.shape

    def calc_fac(bt, b):
        fac1 = [0.0] * (nd1 + 1)
        fac2 = [0.0] * (nd1 + 1)
        y, maxfac = 0.0, -1e200
        for i in range(1, 2 * (nd1 - 1) + 1):
            m = ((i + 1) >> 1) + 1
            arg = bt / (2 * i) * b[m - 1]
            y += math.log(arg) if arg > 0 else -math.inf
            fac1[m] = y
            maxfac = max(y, maxfac)
        for i in range(1, nd1):
            fac1[i] = math.exp(fac1[i] - maxfac)
            fac2[i] = fac1[i] * bt * b[i] / (2 * i - 1)
        fac1[nd1] = math.exp(fac1[nd1] - maxfac)
        return fac1, fac2

    def eval_q(bt, s):
        fac1, fac2 = calc_fac(bt, beta[s])
        t1 = [fac1[i] * energy[s][i - 1] for i in range(1, nd1)]
        t2 = [fac2[i] * hmix[s][i - 1] for i in range(1, nd1)]
        z = 0.0
        for i in range(1, nd1):
            z = z + fac1[i] + fac2[i]
        x = 0.0
        for v in sorted(t1, reverse=True):
            x += v
        y = 0.0
        for v in sorted(t2, reverse=True):
            y += v
        return (x + y) / z

    lmin, lmax = math.log(t_min), math.log(t_max)
    delta = (lmax - lmin) / num_div
    t_delta = 1e-4 if t_min >= 1e-4 else t_min * 0.9
    out = np.zeros((num_div + 1, 5))
    for i1 in range(num_div + 1):
        t0 = math.exp(lmin + i1 * delta)
        dat = [0.0] * 9
        for i2, bt in enumerate((1.0 / (t0 - t_delta), 1.0 / t0, 1.0 / (t0 + t_delta))):
            tmp = [eval_q(bt, s) for s in range(nseed)]
            ave = 0.0
            var = 0.0
            for v in tmp:
                ave += v
                var += v * v
            ave /= nseed
            var = var / nseed - ave * ave
            dat[3 * i2:3 * i2 + 3] = [bt, ave, var]
        spec = 0.5 * (dat[7] - dat[1]) / t_delta
        d1 = (dat[4] - dat[1]) / t_delta
        d2 = (dat[7] - dat[4]) / t_delta
        out[i1] = [1.0 / dat[3], dat[4], spec, 0.5 * (dat[2] + dat[8]), (d2 - d1) / t_delta]
    return out
