// Krylov drivers of libpned_gpu.so: Lanczos, mTPQ (TPS), DSF chains and CG
// inverse iteration.  Scalars (alpha, beta, scales) stay on the device between
// kernels, so a run of steps needs no host round trip and is replayed as a
// CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "device.cuh"

namespace pned {

// ---------------------------------------------------------------------------
// step epilogues (one block, one thread per vector)
// ---------------------------------------------------------------------------

// Lanczos: alpha = Re(sum0), beta = sqrt(sum1); record; next scales.
__global__ void lanczos_epilogue(const double2 *__restrict__ sa, const double2 *__restrict__ sb, int R,
                                 double *sc, double *pc, double *d_alpha, double *d_beta, int *counter,
                                 int *flag)
{
    __shared__ int k;
    if (threadIdx.x == 0) k = *counter;
    __syncthreads();
    const int r = threadIdx.x;
    if (r < R) {
        const double al = sa[r].x;
        const double be = sqrt(sb[r].x);
        d_alpha[(size_t)k * R + r] = al;
        d_beta[(size_t)k * R + r] = be;
        if (!(be >= 0.5e-30)) atomicOr(flag, 1);
        const double old = sc[r];
        sc[r] = 1.0 / be;
        pc[r] = -be * old;
    }
    __syncthreads();
    if (threadIdx.x == 0) *counter = k + 1;
}

// TPS: alpha1 = Re<v|(L-H)v>, beta = ||(L-H)v||, coef as eval_phys_val.
__global__ void tps_epilogue(const double2 *__restrict__ s, int R, int nobs, const double2 *__restrict__ so, double L,
                             double *sc, double *gsc, double *gscp, double *d_alpha, double *d_beta, double *d_coef,
                             int ncoef, int *counter)
{
    __shared__ int k;
    if (threadIdx.x == 0) k = *counter;
    __syncthreads();
    const int r = threadIdx.x;
    if (r < R) {
        const double a1 = s[0 * R + r].x;
        const double be = sqrt(s[1 * R + r].x);
        const double2 gw = s[2 * R + r], gv = s[3 * R + r];
        d_alpha[(size_t)k * R + r] = L - a1;
        d_beta[(size_t)k * R + r] = be;
        double *cf = d_coef + ((size_t)k * R + r) * ncoef;
        cf[0] = double(2 * (k + 1)) / a1;
        cf[1] = L;
        cf[2] = be;
        cf[3] = L - a1;
        cf[4] = L * gv.x - gw.x;   // Re(L <vg|v1> - <vg|v0>)
        for (int o = 0; o < nobs; ++o) {
            cf[5 + 2 * o] = so[(2 * o) * R + r].x;
            cf[6 + 2 * o] = so[(2 * o + 1) * R + r].x;
        }
        gscp[r] = gsc[r];
        gsc[r] = sc[r];
        sc[r] = 1.0 / be;
    }
    __syncthreads();
    if (threadIdx.x == 0) *counter = k + 1;
}

// Diagonal observables: <v|O v> and <g|O v>, v = sc C, g = gsc G.
__global__ void __launch_bounds__(kThreads) obs_kernel(const double2 *__restrict__ C, const double2 *__restrict__ G,
                                                       const double *__restrict__ sc, const double *__restrict__ gsc,
                                                       int64_t dim, int R, int vpt, int n, int nterm,
                                                       const int *__restrict__ ta, const int *__restrict__ tb,
                                                       const double2 *__restrict__ tc, const double2 *__restrict__ T,
                                                       double2 *partials, const int64_t *__restrict__ list1)
{
    double2 red[2][kMaxVPT];
    for (int k = 0; k < 2; ++k)
        for (int j = 0; j < kMaxVPT; ++j) red[k][j] = make_double2(0.0, 0.0);
    const int Gs = R / vpt, r0 = (threadIdx.x % Gs) * vpt;
    for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < dim * Gs;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int64_t st = it / Gs;
        const int64_t state = list1 ? list1[st] : st;   // sector index -> state
        double2 w = make_double2(0.0, 0.0);
        for (int t = 0; t < nterm; ++t) {
            const int i = ta[t] >= n ? 0 : int((state >> ta[t]) & 1);
            const int k = tb[t] >= n ? 0 : int((state >> tb[t]) & 1);
            w = cfma(tc[t], T[2 * i + k], w);
        }
        const int64_t base = st * R + r0;
#pragma unroll
        for (int j = 0; j < kMaxVPT; ++j) {
            if (j >= vpt) break;
            const double2 v = cscale(sc[r0 + j], C[base + j]);
            const double2 ov = cmul(w, v);
            red[0][j] = cadd(red[0][j], cconjmul(v, ov));
            if (G) red[1][j] = cadd(red[1][j], cconjmul(cscale(gsc[r0 + j], G[base + j]), ov));
        }
    }
    block_reduce_store<2, kMaxVPT>(red, Gs, vpt, R, partials);
}

// S^z_q start vectors: C[s, r] = sum_j (d_j(s) - S) e^{i qr[r, j]} x[s].
__global__ void __launch_bounds__(kThreads) szq_kernel(const double2 *__restrict__ x, const double2 *__restrict__ ph,
                                                       int64_t dim, int R, int vpt, int n, int q, double2 *C,
                                                       double2 *partials, const int64_t *__restrict__ list1)
{
    double2 red[1][kMaxVPT];
    for (int j = 0; j < kMaxVPT; ++j) red[0][j] = make_double2(0.0, 0.0);
    const int Gs = R / vpt, r0 = (threadIdx.x % Gs) * vpt;
    const double S = 0.5 * (q - 1);
    for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < dim * Gs;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int64_t st = it / Gs;
        double2 w[kMaxVPT];
        for (int j = 0; j < kMaxVPT; ++j) w[j] = make_double2(0.0, 0.0);
        int64_t y = list1 ? list1[st] : st;   // sector index -> state
        for (int site = 0; site < n; ++site) {
            int64_t dj;
            if (q == 2) { dj = y & 1; y >>= 1; }
            else { const int64_t z = y / q; dj = y - z * q; y = z; }
            const double f = double(dj) - S;
#pragma unroll
            for (int j = 0; j < kMaxVPT; ++j) {
                if (j >= vpt) break;
                const double2 p = ph[(r0 + j) * n + site];
                w[j].x = fma(f, p.x, w[j].x);
                w[j].y = fma(f, p.y, w[j].y);
            }
        }
        const double2 xs = x[st];
#pragma unroll
        for (int j = 0; j < kMaxVPT; ++j) {
            if (j >= vpt) break;
            const double2 v = cmul(w[j], xs);
            C[st * R + r0 + j] = v;
            red[0][j].x += v.x * v.x + v.y * v.y;
        }
    }
    block_reduce_store<1, kMaxVPT>(red, Gs, vpt, R, partials);
}

// S^{ipm}_q start vectors (intalv_xy) as a gather over the target basis:
// C[st, r] = sum over sites j (ascending) with a valid source digit of
// fac * e^{i qr[r, j]} x[source index of state - ipm q^j].  Target states come
// from t_list1 (null: full basis), source indices from the source Lin tables
// (null: full basis).
__global__ void __launch_bounds__(kThreads) sxy_kernel(const double2 *__restrict__ x, const double2 *__restrict__ ph,
                                                       int64_t dim, int R, int vpt, int n, int q, int ipm,
                                                       const int64_t *__restrict__ t_list1,
                                                       const int64_t *__restrict__ s_lo,
                                                       const int64_t *__restrict__ s_hi, int64_t s_mod, double2 *C,
                                                       double2 *partials)
{
    double2 red[1][kMaxVPT];
    for (int j = 0; j < kMaxVPT; ++j) red[0][j] = make_double2(0.0, 0.0);
    const int Gs = R / vpt, r0 = (threadIdx.x % Gs) * vpt;
    const double ss = 0.5 * (q - 1);
    for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < dim * Gs;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int64_t st = it / Gs;
        const int64_t state = t_list1 ? t_list1[st] : st;
        double2 w[kMaxVPT];
        for (int j = 0; j < kMaxVPT; ++j) w[j] = make_double2(0.0, 0.0);
        int64_t y = state, pw = 1;
        for (int site = 0; site < n; ++site, pw *= q) {
            const int64_t z = y / q;
            const int d = int(y - z * q);
            y = z;
            const int ds = d - ipm;   // the source digit
            if (ds < 0 || ds >= q) continue;
            const double sm = double(ds) - ss;
            const double fac = ipm == 1 ? sqrt((ss - sm) * (ss + sm + 1.0)) : sqrt((ss + sm) * (ss - sm + 1.0));
            const int64_t src = state - int64_t(ipm) * pw;
            const int64_t si = s_lo ? s_lo[src % s_mod] + s_hi[src / s_mod] - 1 : src;
            const double2 xs = x[si];
#pragma unroll
            for (int j = 0; j < kMaxVPT; ++j) {
                if (j >= vpt) break;
                const double2 p = ph[(r0 + j) * n + site];
                const double2 rot = make_double2(p.x * xs.x - p.y * xs.y, p.y * xs.x + p.x * xs.y);
                w[j].x += fac * rot.x;
                w[j].y += fac * rot.y;
            }
        }
#pragma unroll
        for (int j = 0; j < kMaxVPT; ++j) {
            if (j >= vpt) break;
            C[st * R + r0 + j] = w[j];
            red[0][j].x += w[j].x * w[j].x + w[j].y * w[j].y;
        }
    }
    block_reduce_store<1, kMaxVPT>(red, Gs, vpt, R, partials);
}

__global__ void dsf_start_epilogue(const double2 *__restrict__ s, int R, int n, double *sc, double *cnorm)
{
    const int r = threadIdx.x;
    if (r < R) {
        double raw = s[r].x;
        if (raw < 1e-25) raw = 1e-25;
        cnorm[r] = raw / double(n);
        sc[r] = 1.0 / sqrt(raw);
    }
}

// x += a p ; r -= a y    (complex a, one vector)
__global__ void cg_update_xr(double2 *x, double2 *r, const double2 *__restrict__ p, const double2 *__restrict__ y,
                             double2 a, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] = cfma(a, p[i], x[i]);
        const double2 ay = cmul(a, y[i]);
        r[i] = make_double2(r[i].x - ay.x, r[i].y - ay.y);
    }
}

// p = r + b p
__global__ void cg_update_p(double2 *p, const double2 *__restrict__ r, double b, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = make_double2(r[i].x + b * p[i].x, r[i].y + b * p[i].y);
}

__global__ void scale_real_kernel(double2 *v, double f, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = cscale(f, v[i]);
}

// Eigenvector pass: v = sc C; x += c v; Pn = W - a v (Pn may be null: accumulate only).
__global__ void __launch_bounds__(kThreads) lncv_kernel(const double2 *__restrict__ W, const double2 *__restrict__ C,
                                                        double2 *Pn, double2 *x, const double *__restrict__ sc,
                                                        double a, double c, int64_t n)
{
    const double s = *sc;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 v = cscale(s, C[i]);
        const double2 xo = x[i];
        x[i] = make_double2(fma(c, v.x, xo.x), fma(c, v.y, xo.y));
        if (Pn) {
            const double2 w = W[i];
            Pn[i] = make_double2(w.x - a * v.x, w.y - a * v.y);
        }
    }
}

// Resuming a Lanczos chain from the reference's loop state: Rn = W - a V.
__global__ void __launch_bounds__(kThreads) resume_kernel(const double2 *__restrict__ W, const double2 *__restrict__ V,
                                                          double2 *Rn, double a, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 w = W[i], v = V[i];
        Rn[i] = make_double2(w.x - a * v.x, w.y - a * v.y);
    }
}

// sc <- 1/b, pc <- -b sc_old
__global__ void lncv_scal_kernel(double *sc, double *pc, double b)
{
    if (threadIdx.x == 0) {
        const double old = *sc;
        *sc = 1.0 / b;
        *pc = -b * old;
    }
}

// ---------------------------------------------------------------------------
// one step of each kind; buffer roles live in the session
// ---------------------------------------------------------------------------

// Lanczos (b0 = C, b1 = P, b2 = W):
//   W = -beta_{i-1} v_{i-1} + H v_i,  alpha_i = <v_i|H v_i>     (hv kernel)
//   R = W - alpha_i v_i, beta_i = ||W - alpha_i v_i||           (residual kernel)
// written into the old P buffer, which becomes C (v_{i+1} = R / beta_i).
static cudaError_t lanczos_step(pned_ctx *c, Session &S, bool first)
{
    const int R = c->R;
    HvArgs a{};
    a.C = c->buf[S.b0];
    a.P = first ? nullptr : c->buf[S.b1];
    a.W = c->buf[S.b2];
    a.sc = slot(c, kSlotSc);
    a.pc = first ? nullptr : slot(c, kSlotPc);
    a.diag = c->m->d_diag;
    a.shift = 0.0;
    a.table = c->m->d_table;
    a.partials = c->partials;
    a.dim = c->m->dim;
    a.R = R;
    a.K = 1;
    a.err = c->flag;
    ctx_tile_args(c, a);
    double2 *sa = c->sums, *sb = c->sums + kMaxK * kMaxR;
    if (S.ev_hv0) cudaEventRecord(S.ev_hv0, c->stream);
    cudaError_t e = launch_hv(c->m, a, c->nblocks, c->stream);
    if (S.ev_hv1) cudaEventRecord(S.ev_hv1, c->stream);
    if (e == cudaSuccess) e = launch_finish(c->partials, int(hv_partials(c->m, a, c->nblocks)), R, sa, c->stream);
    if (e == cudaSuccess)
        e = launch_residual(c, c->buf[S.b2], c->buf[S.b0], c->buf[S.b1], slot(c, kSlotSc), sa, c->stream);
    if (e == cudaSuccess) e = launch_finish(c->partials, c->nblocks, R, sb, c->stream);
    if (e == cudaSuccess) {
        lanczos_epilogue<<<1, 32 * ((R + 31) / 32), 0, c->stream>>>(sa, sb, R, slot(c, kSlotSc), slot(c, kSlotPc),
                                                                   S.d_alpha, S.d_beta, S.d_counter, S.d_flag);
        e = cudaGetLastError();
    }
    std::swap(S.b0, S.b1);
    return e;
}

// TPS (b0 = C = |k> scaled, b1 = W, b2 = G = |k-1> scaled):
//   W = (L - H)^T v, alpha1 = <v|W>, beta = ||W||, <vg|W>, <vg|v>  (one fused kernel)
// then G <- C, C <- W (scale 1/beta), W <- old G.
static cudaError_t tps_step(pned_ctx *c, Session &S, bool first)
{
    const int R = c->R;
    HvArgs a{};
    a.C = c->buf[S.b0]; a.P = nullptr; a.W = c->buf[S.b1];
    a.sc = slot(c, kSlotSc); a.pc = nullptr;
    a.diag = c->m->d_diag; a.shift = 0.0;
    a.table = c->m->d_table; a.partials = c->partials;
    a.G = first ? nullptr : c->buf[S.b2]; a.gsc = slot(c, kSlotGsc);
    a.dim = c->m->dim; a.R = R; a.K = 4;
    a.err = c->flag;
    ctx_tile_args(c, a);
    if (S.ev_hv0) cudaEventRecord(S.ev_hv0, c->stream);
    cudaError_t e = launch_hv(c->m, a, c->nblocks, c->stream);
    if (S.ev_hv1) cudaEventRecord(S.ev_hv1, c->stream);
    if (e == cudaSuccess)
        e = launch_finish(c->partials, int(hv_partials(c->m, a, c->nblocks)), 4 * R, c->sums, c->stream);
    if (first && e == cudaSuccess) e = cudaMemsetAsync(c->sums + 2 * R, 0, sizeof(double2) * 2 * R, c->stream);
    for (int o = 0; o < S.nobs && e == cudaSuccess; ++o) {
        const DevObs &ob = S.obs[o];
        obs_kernel<<<c->nblocks, kThreads, 0, c->stream>>>(c->buf[S.b0], first ? nullptr : c->buf[S.b2],
                                                          slot(c, kSlotSc), slot(c, kSlotGsc), c->m->dim, R,
                                                          pick_vpt(R), c->m->n, ob.n, ob.a, ob.b, ob.c, ob.T,
                                                          c->partials, c->m->d_list1);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = launch_finish(c->partials, c->nblocks, 2 * R, S.d_osum + 2 * o * R, c->stream);
    }
    if (e == cudaSuccess) {
        tps_epilogue<<<1, 32 * ((R + 31) / 32), 0, c->stream>>>(c->sums, R, S.nobs, S.d_osum, S.L, slot(c, kSlotSc),
                                                               slot(c, kSlotGsc), slot(c, kSlotGscPrev), S.d_alpha,
                                                               S.d_beta, S.d_coef, S.ncoef, S.d_counter);
        e = cudaGetLastError();
    }
    const int og = S.b2;
    S.b2 = S.b0; S.b0 = S.b1; S.b1 = og;
    return e;
}

static cudaError_t one_step(pned_ctx *c, Session &S, bool first)
{
    return S.kind == PNED_SESSION_TPS ? tps_step(c, S, first) : lanczos_step(c, S, first);
}

template <class T> static T *sess_alloc(Session &S, size_t n)
{
    void *q = nullptr;
    if (cudaMalloc(&q, sizeof(T) * std::max<size_t>(1, n)) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    S.allocs.push_back(q);
    return static_cast<T *>(q);
}

void session_release(pned_ctx *c)
{
    Session &S = c->sess;
    if (S.graph) cudaGraphExecDestroy(S.graph);
    for (void *q : S.allocs) cudaFree(q);
    c->sess = Session{};
}

static int session_common_begin(pned_ctx *c, int kind, int max_steps)
{
    if (c->sess.kind) {
        cudaStreamSynchronize(c->stream);
        session_release(c);
    }
    Session &S = c->sess;
    S.kind = kind;
    S.max_steps = max_steps;
    S.period = kind == PNED_SESSION_TPS ? 3 : 2;
    S.b0 = 2; S.b1 = 3; S.b2 = 4;
    int rc = 0;
    for (int k : {2, 3, 4})
        if ((rc = ctx_alloc_buffer(c, k))) { session_release(c); return rc; }
    const int R = c->R;
    S.d_alpha = sess_alloc<double>(S, size_t(max_steps) * R);
    S.d_beta = sess_alloc<double>(S, size_t(max_steps) * R);
    S.d_counter = sess_alloc<int>(S, 2);
    if (!S.d_alpha || !S.d_beta || !S.d_counter) { session_release(c); return fail(PNED_ENOMEM, "session scratch"); }
    S.d_flag = S.d_counter + 1;
    cudaError_t e = cudaMemsetAsync(S.d_counter, 0, 2 * sizeof(int), c->stream);
    if (e != cudaSuccess) { session_release(c); return cuda_fail(e, "session memset"); }
    return PNED_OK;
}

}  // namespace pned

using namespace pned;

extern "C" int pned_session_begin(pned_ctx *c, int kind, const pned_c128 *v_init, int max_steps, double L, int n_obs,
                                  const pned_observable *obs, int flags)
{
    if (!c || !v_init || max_steps < 1 || n_obs < 0 || (n_obs && !obs) || n_obs > 6)
        return fail(PNED_EINVAL, "pned_session_begin: bad arguments");
    if (kind != PNED_SESSION_LANCZOS && kind != PNED_SESSION_TPS)
        return fail(PNED_EINVAL, "pned_session_begin: kind must be LANCZOS or TPS (DSF: pned_session_begin_dsf)");
    if (kind == PNED_SESSION_LANCZOS && n_obs) return fail(PNED_EINVAL, "observables belong to TPS sessions");
    cudaSetDevice(c->m->device);
    int rc = session_common_begin(c, kind, max_steps);
    if (rc) return rc;
    Session &S = c->sess;
    const int R = c->R;
    const size_t bytes = sizeof(double2) * size_t(c->m->dim) * R;
    cudaError_t e = cudaMemcpyAsync(c->buf[S.b0], v_init, bytes,
                                    (flags & PNED_PTR_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                    c->stream);
    if (e != cudaSuccess) { session_release(c); return cuda_fail(e, "pned_session_begin: staging v_init"); }
    if (kind == PNED_SESSION_TPS) {
        S.L = L;
        S.nobs = n_obs;
        S.ncoef = 5 + 2 * n_obs;
        S.d_coef = sess_alloc<double>(S, size_t(max_steps) * R * S.ncoef);
        S.d_osum = sess_alloc<double2>(S, size_t(2 * std::max(1, n_obs)) * R);
        if (!S.d_coef || !S.d_osum) { session_release(c); return fail(PNED_ENOMEM, "session scratch"); }
        for (int o = 0; o < n_obs; ++o) {
            DevObs d;
            d.n = obs[o].n_terms;
            d.a = sess_alloc<int>(S, d.n);
            d.b = sess_alloc<int>(S, d.n);
            d.c = sess_alloc<double2>(S, d.n);
            d.T = sess_alloc<double2>(S, 4);
            if (!d.a || !d.b || !d.c || !d.T) { session_release(c); return fail(PNED_ENOMEM, "observables"); }
            if (d.n) {
                e = cudaMemcpyAsync(d.a, obs[o].a, sizeof(int) * d.n, cudaMemcpyHostToDevice, c->stream);
                if (e == cudaSuccess) e = cudaMemcpyAsync(d.b, obs[o].b, sizeof(int) * d.n, cudaMemcpyHostToDevice, c->stream);
                if (e == cudaSuccess) e = cudaMemcpyAsync(d.c, obs[o].c, sizeof(double2) * d.n, cudaMemcpyHostToDevice, c->stream);
            }
            if (e == cudaSuccess) e = cudaMemcpyAsync(d.T, obs[o].T, sizeof(double2) * 4, cudaMemcpyHostToDevice, c->stream);
            if (e != cudaSuccess) { session_release(c); return cuda_fail(e, "observables"); }
            S.obs.push_back(d);
        }
        // observable uploads read host memory that may go away after this call
        e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) { session_release(c); return cuda_fail(e, "observables"); }
        if ((rc = set_slot(c, kSlotGsc, 0.0))) { session_release(c); return rc; }
    }
    if ((rc = set_slot(c, kSlotSc, 1.0))) { session_release(c); return rc; }
    return PNED_OK;
}

extern "C" int pned_session_begin_dsf(pned_ctx *c, const pned_c128 *x, const double *qr, int max_steps, double *cnorm,
                                      int flags)
{
    if (!c || !x || !qr || max_steps < 1) return fail(PNED_EINVAL, "pned_session_begin_dsf: bad arguments");
    cudaSetDevice(c->m->device);
    int rc = session_common_begin(c, PNED_SESSION_DSF, max_steps);
    if (rc) return rc;
    Session &S = c->sess;
    const int R = c->R, n = c->m->n;
    const size_t dim = size_t(c->m->dim);
    const double2 *dx = reinterpret_cast<const double2 *>(x);
    cudaError_t e = cudaSuccess;
    if (!(flags & PNED_PTR_DEVICE)) {
        double2 *tmp = sess_alloc<double2>(S, dim);
        if (!tmp) { session_release(c); return fail(PNED_ENOMEM, "pned_session_begin_dsf: staging x"); }
        e = cudaMemcpyAsync(tmp, x, sizeof(double2) * dim, cudaMemcpyHostToDevice, c->stream);
        dx = tmp;
    }
    std::vector<double2> ph(size_t(R) * n);
    for (int r = 0; r < R; ++r)
        for (int j = 0; j < n; ++j) ph[size_t(r) * n + j] = make_double2(std::cos(qr[r * n + j]), std::sin(qr[r * n + j]));
    double2 *dph = sess_alloc<double2>(S, ph.size());
    double *dcn = sess_alloc<double>(S, R);
    if (!dph || !dcn) { session_release(c); return fail(PNED_ENOMEM, "pned_session_begin_dsf: scratch"); }
    if (e == cudaSuccess) e = cudaMemcpyAsync(dph, ph.data(), sizeof(double2) * ph.size(), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        szq_kernel<<<c->nblocks, kThreads, 0, c->stream>>>(dx, dph, c->m->dim, R, pick_vpt(R), n, c->m->q,
                                                          c->buf[S.b0], c->partials, c->m->d_list1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = launch_finish(c->partials, c->nblocks, R, c->sums, c->stream);
    if (e == cudaSuccess) {
        dsf_start_epilogue<<<1, 32 * ((R + 31) / 32), 0, c->stream>>>(c->sums, R, n, slot(c, kSlotSc), dcn);
        e = cudaGetLastError();
    }
    std::vector<double> hc(R);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hc.data(), dcn, sizeof(double) * R, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { session_release(c); return cuda_fail(e, "pned_session_begin_dsf: S^z_q"); }
    if (cnorm) std::copy(hc.begin(), hc.end(), cnorm);
    return PNED_OK;
}

extern "C" int pned_session_begin_dsf_xy(pned_ctx *c, const pned_model *source, int ipm, const pned_c128 *x,
                                         const double *qr, int max_steps, double *cnorm, int flags)
{
    if (!c || !source || !x || !qr || max_steps < 1 || (ipm != 1 && ipm != -1))
        return fail(PNED_EINVAL, "pned_session_begin_dsf_xy: bad arguments");
    if (source->n != c->m->n || source->q != c->m->q || source->device != c->m->device)
        return fail(PNED_EINVAL, "pned_session_begin_dsf_xy: source and target models differ in n, q or device");
    // a sector source needs the neighbouring sector as target: every target state
    // minus one ladder step must be a source-sector state for its Lin lookup
    if (source->hp.sector && (!c->m->hp.sector || c->m->hp.total != source->hp.total + ipm))
        return fail(PNED_EINVAL, "pned_session_begin_dsf_xy: for a sector source the context's model must be the "
                                 "sector of digit sum source + ipm");
    cudaSetDevice(c->m->device);
    int rc = session_common_begin(c, PNED_SESSION_DSF, max_steps);
    if (rc) return rc;
    Session &S = c->sess;
    const int R = c->R, n = c->m->n;
    const size_t sdim = size_t(source->dim);
    const double2 *dx = reinterpret_cast<const double2 *>(x);
    cudaError_t e = cudaSuccess;
    if (!(flags & PNED_PTR_DEVICE)) {
        double2 *tmp = sess_alloc<double2>(S, sdim);
        if (!tmp) { session_release(c); return fail(PNED_ENOMEM, "pned_session_begin_dsf_xy: staging x"); }
        e = cudaMemcpyAsync(tmp, x, sizeof(double2) * sdim, cudaMemcpyHostToDevice, c->stream);
        dx = tmp;
    }
    std::vector<double2> ph(size_t(R) * n);
    for (int r = 0; r < R; ++r)
        for (int j = 0; j < n; ++j) ph[size_t(r) * n + j] = make_double2(std::cos(qr[r * n + j]), std::sin(qr[r * n + j]));
    double2 *dph = sess_alloc<double2>(S, ph.size());
    double *dcn = sess_alloc<double>(S, R);
    if (!dph || !dcn) { session_release(c); return fail(PNED_ENOMEM, "pned_session_begin_dsf_xy: scratch"); }
    if (e == cudaSuccess) e = cudaMemcpyAsync(dph, ph.data(), sizeof(double2) * ph.size(), cudaMemcpyHostToDevice, c->stream);
    const bool ssec = source->hp.sector;
    if (e == cudaSuccess) {
        sxy_kernel<<<c->nblocks, kThreads, 0, c->stream>>>(dx, dph, c->m->dim, R, pick_vpt(R), n, c->m->q, ipm,
                                                          c->m->d_list1, ssec ? source->d_lin_lo : nullptr,
                                                          ssec ? source->d_lin_hi : nullptr,
                                                          ssec ? source->lin_mod : 1, c->buf[S.b0], c->partials);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = launch_finish(c->partials, c->nblocks, R, c->sums, c->stream);
    if (e == cudaSuccess) {
        dsf_start_epilogue<<<1, 32 * ((R + 31) / 32), 0, c->stream>>>(c->sums, R, n, slot(c, kSlotSc), dcn);
        e = cudaGetLastError();
    }
    std::vector<double> hc(R);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hc.data(), dcn, sizeof(double) * R, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { session_release(c); return cuda_fail(e, "pned_session_begin_dsf_xy: S^pm_q"); }
    if (cnorm) std::copy(hc.begin(), hc.end(), cnorm);
    return PNED_OK;
}

extern "C" int pned_session_step(pned_ctx *c, int n_steps)
{
    if (!c || n_steps < 0) return fail(PNED_EINVAL, "pned_session_step: bad arguments");
    Session &S = c->sess;
    if (!S.kind) return fail(PNED_EINVAL, "pned_session_step: no session");
    if (S.enqueued + n_steps > S.max_steps)
        return fail(PNED_EINVAL, "pned_session_step: more steps than max_steps of the session");
    cudaSetDevice(c->m->device);
    cudaError_t e = cudaSuccess;
    while (n_steps > 0) {
        if (S.enqueued == 0) {
            e = one_step(c, S, true);
            if (e != cudaSuccess) return cuda_fail(e, "first Krylov step");
            ++S.enqueued; --n_steps;
            continue;
        }
        const bool roles_match = S.graph && S.b0 == S.g0 && S.b1 == S.g1 && S.b2 == S.g2;
        if (roles_match && n_steps >= S.period) {
            e = cudaGraphLaunch(S.graph, c->stream);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
            S.enqueued += S.period; n_steps -= S.period;
            continue;
        }
        if (!S.graph && n_steps >= 2 * S.period) {
            // capture `period` steps: the buffer roles come back to where they started
            cudaGraph_t graph;
            e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
            const int s0 = S.b0, s1 = S.b1, s2 = S.b2;
            cudaError_t ek = cudaSuccess;
            for (int k = 0; k < S.period; ++k) {
                cudaError_t q = one_step(c, S, false);
                if (q != cudaSuccess) ek = q;
            }
            e = cudaStreamEndCapture(c->stream, &graph);
            if (e == cudaSuccess && ek != cudaSuccess) e = ek;
            if (e == cudaSuccess) {
                e = cudaGraphInstantiate(&S.graph, graph, 0);
                cudaGraphDestroy(graph);
            }
            if (e != cudaSuccess) return cuda_fail(e, "capturing the Krylov step graph");
            S.g0 = s0; S.g1 = s1; S.g2 = s2;
            S.b0 = s0; S.b1 = s1; S.b2 = s2;
            continue;
        }
        e = one_step(c, S, false);
        if (e != cudaSuccess) return cuda_fail(e, "Krylov step");
        ++S.enqueued; --n_steps;
    }
    return PNED_OK;
}

extern "C" int pned_session_read(pned_ctx *c, double *alpha, double *beta, double *coef, int *steps_done,
                                 int *status_out)
{
    if (!c) return fail(PNED_EINVAL, "pned_session_read: null context");
    Session &S = c->sess;
    if (!S.kind) return fail(PNED_EINVAL, "pned_session_read: no session");
    cudaSetDevice(c->m->device);
    const int R = c->R, k = S.enqueued;
    cudaError_t e = cudaSuccess;
    if (alpha && k) e = cudaMemcpyAsync(alpha, S.d_alpha, sizeof(double) * size_t(k) * R, cudaMemcpyDeviceToHost, c->stream);
    if (beta && k && e == cudaSuccess)
        e = cudaMemcpyAsync(beta, S.d_beta, sizeof(double) * size_t(k) * R, cudaMemcpyDeviceToHost, c->stream);
    if (coef && k && S.kind == PNED_SESSION_TPS && e == cudaSuccess)
        e = cudaMemcpyAsync(coef, S.d_coef, sizeof(double) * size_t(k) * R * S.ncoef, cudaMemcpyDeviceToHost, c->stream);
    int flag = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, S.d_flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_session_read");
    const int kf = check_kernel_flag(c);
    if (kf) return kf;
    if (steps_done) *steps_done = k;
    if (status_out) *status_out = flag;
    return PNED_OK;
}

extern "C" int pned_session_vector(pned_ctx *c, pned_c128 **dev_ptr, double *scale_out)
{
    if (!c || !dev_ptr) return fail(PNED_EINVAL, "pned_session_vector: bad arguments");
    Session &S = c->sess;
    if (!S.kind) return fail(PNED_EINVAL, "pned_session_vector: no session");
    *dev_ptr = reinterpret_cast<pned_c128 *>(c->buf[S.b0]);
    if (scale_out) {
        double h[kMaxR];
        cudaError_t e = cudaMemcpyAsync(h, slot(c, kSlotSc), sizeof(double) * kMaxR, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return cuda_fail(e, "pned_session_vector");
        for (int r = 0; r < c->R; ++r) scale_out[r] = h[r];
    }
    return PNED_OK;
}

extern "C" int pned_session_profile(pned_ctx *c, int n_steps, double *hv_ms, double *step_ms)
{
    if (!c || n_steps < 1 || !hv_ms || !step_ms) return fail(PNED_EINVAL, "pned_session_profile: bad arguments");
    Session &S = c->sess;
    if (!S.kind || S.enqueued < 1) return fail(PNED_EINVAL, "pned_session_profile: needs a started session");
    if (S.enqueued + n_steps > S.max_steps) return fail(PNED_EINVAL, "pned_session_profile: beyond max_steps");
    cudaSetDevice(c->m->device);
    cudaEvent_t e0, e1, s0, s1;
    cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&s0); cudaEventCreate(&s1);
    double thv = 0, tst = 0;
    cudaError_t e = cudaSuccess;
    S.ev_hv0 = e0; S.ev_hv1 = e1;
    for (int k = 0; k < n_steps && e == cudaSuccess; ++k) {
        cudaEventRecord(s0, c->stream);
        e = one_step(c, S, false);
        cudaEventRecord(s1, c->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(s1);
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, e0, e1);
        cudaEventElapsedTime(&b, s0, s1);
        thv += a; tst += b;
        ++S.enqueued;
    }
    S.ev_hv0 = S.ev_hv1 = nullptr;
    cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(s0); cudaEventDestroy(s1);
    if (e != cudaSuccess) return cuda_fail(e, "pned_session_profile");
    *hv_ms = thv / n_steps;
    *step_ms = tst / n_steps;
    return PNED_OK;
}

extern "C" int pned_session_end(pned_ctx *c)
{
    if (!c) return fail(PNED_EINVAL, "pned_session_end: null context");
    cudaSetDevice(c->m->device);
    cudaStreamSynchronize(c->stream);
    session_release(c);
    return PNED_OK;
}

// ---------------------------------------------------------------------------
// whole-run drivers
// ---------------------------------------------------------------------------
extern "C" int pned_lanczos_run(pned_ctx *c, const pned_c128 *v_init, int n_steps, int check_conv, double *alpha,
                                double *beta, double *ene, int *steps_done, int flags)
{
    if (!c || !v_init || !alpha || !beta || n_steps < 1) return fail(PNED_EINVAL, "pned_lanczos_run: bad arguments");
    if (check_conv && c->R != 1) return fail(PNED_EINVAL, "pned_lanczos_run: check_conv needs R = 1");
    int rc = pned_session_begin(c, PNED_SESSION_LANCZOS, v_init, n_steps, 0.0, 0, nullptr, flags);
    if (rc) return rc;
    const int R = c->R;
    int done = 0;
    if (!check_conv) {
        rc = pned_session_step(c, n_steps);
        done = n_steps;
    } else {
        // the nvec = 8 stop of S1/2 Lanczos.f90:133-155: bisec at i = 32 and every
        // 5th step after it, stop when ene(8) changes by less than 1e-13 relative
        const int nvec2 = 8;
        double ebefor = 0.0;
        std::vector<double> a, b;
        while (done < n_steps && !rc) {
            int next = done < 4 * nvec2 ? std::min(4 * nvec2, n_steps) : std::min((done / 5 + 1) * 5, n_steps);
            if ((rc = pned_session_step(c, next - done))) break;
            done = next;
            if (done < 4 * nvec2 || (done > 4 * nvec2 && done % 5)) continue;
            a.resize(done); b.resize(done);
            if ((rc = pned_session_read(c, a.data(), b.data(), nullptr, nullptr, nullptr))) break;
            double E[8];
            pned_bisec(a.data(), b.data(), done, E, nvec2, 1e-25);
            if (done == 4 * nvec2) { ebefor = E[nvec2 - 1]; continue; }
            if (std::fabs((ebefor - E[nvec2 - 1]) / E[nvec2 - 1]) < 1e-13) break;
            ebefor = E[nvec2 - 1];
        }
    }
    int status = 0, k = 0;
    if (!rc) rc = pned_session_read(c, alpha, beta, nullptr, &k, &status);
    pned_session_end(c);
    if (rc) return rc;
    if (steps_done) *steps_done = k;
    if (ene) {
        std::vector<double> a0(k), b0(k);
        for (int i = 0; i < k; ++i) { a0[i] = alpha[size_t(i) * R]; b0[i] = beta[size_t(i) * R]; }
        for (int i = 0; i < 8; ++i) ene[i] = 0.0;
        pned_bisec(a0.data(), b0.data(), k, ene, std::min(k, 8), 1e-25);
    }
    if (status) return fail(PNED_EBREAKDOWN, "Lanczos beta below 0.5e-30 (tridiagonalisation unsuccessful)");
    return PNED_OK;
}

extern "C" int pned_tps_run(pned_ctx *c, double L, const pned_c128 *v_init, int n_steps, int n_obs,
                            const pned_observable *obs, double *alpha, double *beta, double *coef, int flags)
{
    if (!c || !v_init || !alpha || !beta || !coef || n_steps < 1)
        return fail(PNED_EINVAL, "pned_tps_run: bad arguments");
    int rc = pned_session_begin(c, PNED_SESSION_TPS, v_init, n_steps, L, n_obs, obs, flags);
    if (rc) return rc;
    rc = pned_session_step(c, n_steps);
    if (!rc) rc = pned_session_read(c, alpha, beta, coef, nullptr, nullptr);
    pned_session_end(c);
    return rc;
}

extern "C" int pned_dsf_run(pned_ctx *c, const pned_c128 *x, const double *qr, int n_steps, double *cnorm,
                            double *salpha, double *sbeta, int flags)
{
    if (!c || !x || !qr || !cnorm || !salpha || !sbeta || n_steps < 1)
        return fail(PNED_EINVAL, "pned_dsf_run: bad arguments");
    int rc = pned_session_begin_dsf(c, x, qr, n_steps, cnorm, flags);
    if (rc) return rc;
    const int R = c->R;
    std::vector<double> b(size_t(n_steps) * R);
    rc = pned_session_step(c, n_steps);
    int status = 0;
    if (!rc) rc = pned_session_read(c, salpha, b.data(), nullptr, nullptr, &status);
    pned_session_end(c);
    if (rc) return rc;
    for (int r = 0; r < R; ++r) sbeta[r] = cnorm[r];
    for (size_t i = 0; i < b.size(); ++i) sbeta[R + i] = b[i];
    return PNED_OK;
}

extern "C" int pned_dsf_xy_run(pned_ctx *c, const pned_model *source, int ipm, const pned_c128 *x, const double *qr,
                               int n_steps, double *cnorm, double *salpha, double *sbeta, int flags)
{
    if (!c || !cnorm || !salpha || !sbeta || n_steps < 1) return fail(PNED_EINVAL, "pned_dsf_xy_run: bad arguments");
    int rc = pned_session_begin_dsf_xy(c, source, ipm, x, qr, n_steps, cnorm, flags);
    if (rc) return rc;
    const int R = c->R;
    std::vector<double> b(size_t(n_steps) * R);
    rc = pned_session_step(c, n_steps);
    int status = 0;
    if (!rc) rc = pned_session_read(c, salpha, b.data(), nullptr, nullptr, &status);
    pned_session_end(c);
    if (rc) return rc;
    for (int r = 0; r < R; ++r) sbeta[r] = cnorm[r];
    for (size_t i = 0; i < b.size(); ++i) sbeta[R + i] = b[i];
    return PNED_OK;
}

// parallelized_lncv1z (S1/2 Lanczos.f90:183-329): the chain of v_init is
// replayed with the stored alpha/beta, x = sum_k coef[k] v_k, normalised.
extern "C" int pned_lanczos_vector(pned_ctx *c, const pned_c128 *v_init, int n_steps, const double *alpha,
                                   const double *beta, const double *coef, pned_c128 *x_out, int flags)
{
    if (!c || !v_init || !alpha || !beta || !coef || !x_out || n_steps < 1)
        return fail(PNED_EINVAL, "pned_lanczos_vector: bad arguments");
    if (c->R != 1) return fail(PNED_EINVAL, "pned_lanczos_vector: needs a context with R = 1");
    for (int k = 0; k < n_steps - 1; ++k)
        if (!(beta[k] > 0.0)) return fail(PNED_EINVAL, "pned_lanczos_vector: beta must be positive");
    cudaSetDevice(c->m->device);
    int rc = 0;
    for (int k = 0; k < 4; ++k)
        if ((rc = ctx_alloc_buffer(c, k))) return rc;
    double2 *Cb = c->buf[0], *Pb = c->buf[1], *W = c->buf[2], *x = c->buf[3];
    const int64_t n = c->m->dim;
    const size_t bytes = sizeof(double2) * size_t(n);
    const int nb = c->nblocks;
    cudaError_t e = cudaMemcpyAsync(Cb, v_init, bytes,
                                    (flags & PNED_PTR_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                    c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(x, 0, bytes, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_lanczos_vector: staging");
    if ((rc = set_slot(c, kSlotSc, 1.0)) || (rc = set_slot(c, kSlotPc, 0.0))) return rc;
    for (int k = 0; k < n_steps; ++k) {
        if (k + 1 == n_steps) {
            lncv_kernel<<<nb, kThreads, 0, c->stream>>>(nullptr, Cb, nullptr, x, slot(c, kSlotSc), 0.0, coef[k], n);
            e = cudaGetLastError();
            break;
        }
        HvArgs a{};
        a.C = Cb; a.P = k ? Pb : nullptr; a.W = W;
        a.sc = slot(c, kSlotSc); a.pc = k ? slot(c, kSlotPc) : nullptr;
        a.diag = c->m->d_diag; a.shift = 0.0;
        a.table = c->m->d_table; a.partials = c->partials;
        a.dim = n; a.R = 1; a.K = 1; a.err = c->flag;
        ctx_tile_args(c, a);
        e = launch_hv(c->m, a, nb, c->stream);
        if (e != cudaSuccess) break;
        lncv_kernel<<<nb, kThreads, 0, c->stream>>>(W, Cb, Pb, x, slot(c, kSlotSc), alpha[k], coef[k], n);
        lncv_scal_kernel<<<1, 32, 0, c->stream>>>(slot(c, kSlotSc), slot(c, kSlotPc), beta[k]);
        e = cudaGetLastError();
        if (e != cudaSuccess) break;
        std::swap(Cb, Pb);
    }
    if (e != cudaSuccess) return cuda_fail(e, "pned_lanczos_vector");
    // normalise
    double2 xx;
    e = launch_dot(c, x, x, nullptr, 0, c->sums, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_lanczos_vector: norm");
    if ((rc = sums_to_host(c, 1))) return rc;
    xx = c->h_sums[0];
    scale_real_kernel<<<nb, kThreads, 0, c->stream>>>(x, 1.0 / std::sqrt(xx.x), n);
    e = cudaMemcpyAsync(x_out, x, bytes, (flags & PNED_PTR_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                        c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_lanczos_vector: result");
    return PNED_OK;
}

extern "C" int pned_cg_run(pned_ctx *c, double E, const pned_c128 *b_init, int inv_max, int cg_max, pned_c128 *x_out,
                           int *n_inv, int *n_cg, int flags)
{
    if (!c || !b_init || !x_out || inv_max < 1 || cg_max < 1) return fail(PNED_EINVAL, "pned_cg_run: bad arguments");
    if (c->R != 1) return fail(PNED_EINVAL, "pned_cg_run: needs a context with R = 1");
    cudaSetDevice(c->m->device);
    int rc = 0;
    for (int k = 0; k < 5; ++k)
        if ((rc = ctx_alloc_buffer(c, k))) return rc;
    double2 *x = c->buf[0], *b = c->buf[1], *p = c->buf[2], *r = c->buf[3], *y = c->buf[4];
    const int64_t n = c->m->dim;
    const size_t bytes = sizeof(double2) * size_t(n);
    cudaError_t e = cudaMemcpyAsync(b, b_init, bytes,
                                    (flags & PNED_PTR_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                    c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_cg_run: staging b");
    if ((rc = set_slot(c, kSlotOne, 1.0))) return rc;
    const int nb = c->nblocks;
    auto dot = [&](const double2 *u, const double2 *v, double2 &out) -> int {
        cudaError_t err = launch_dot(c, u, v, nullptr, 0, c->sums, c->stream);
        if (err != cudaSuccess) return cuda_fail(err, "cg dot");
        int q = sums_to_host(c, 1);
        out = c->h_sums[0];
        return q;
    };
    bool cg_loop_saved = false;   // the SAVEd `loop` flag of cg1 (S1/2 cg.f90:118)
    int total_cg = 0, itr_inv = 0;
    for (int it = 1; it <= inv_max; ++it) {
        itr_inv = it;
        // ---- cg1: solve (H - E) x = b
        double2 bc;
        if ((rc = dot(b, b, bc))) return rc;
        e = cudaMemcpyAsync(r, b, bytes, cudaMemcpyDeviceToDevice, c->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(p, b, bytes, cudaMemcpyDeviceToDevice, c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(x, 0, bytes, c->stream);
        if (e != cudaSuccess) return cuda_fail(e, "cg init");
        for (int k = 1; k <= cg_max; ++k) {
            ++total_cg;
            HvArgs a{};
            a.C = p; a.P = nullptr; a.W = y;
            a.sc = slot(c, kSlotOne); a.pc = nullptr;
            a.diag = c->m->d_diag;
            a.shift = (E / double(c->m->nbond)) * double(c->m->nbond);
            a.table = c->m->d_table; a.partials = c->partials;
            a.dim = n; a.R = 1; a.K = 1;
            a.err = c->flag;
            ctx_tile_args(c, a);
            e = launch_hv(c->m, a, nb, c->stream);
            if (e != cudaSuccess) return cuda_fail(e, "cg hv");
            double2 crp, cyp, rc1, rc2;
            if ((rc = dot(p, r, crp)) || (rc = dot(p, y, cyp)) || (rc = dot(r, r, rc1))) return rc;
            const double den = cyp.x * cyp.x + cyp.y * cyp.y;
            const double2 al = make_double2((crp.x * cyp.x + crp.y * cyp.y) / den, (crp.y * cyp.x - crp.x * cyp.y) / den);
            cg_update_xr<<<nb, kThreads, 0, c->stream>>>(x, r, p, y, al, n);
            if ((rc = dot(r, r, rc2))) return rc;
            const double beta = rc2.x / rc1.x;
            cg_update_p<<<nb, kThreads, 0, c->stream>>>(p, r, beta, n);
            e = cudaGetLastError();
            if (e != cudaSuccess) return cuda_fail(e, "cg update");
            if (k % 5 != 0) continue;
            if (std::sqrt(std::hypot(rc2.x, rc2.y)) < 1.0e-9 * std::sqrt(std::hypot(bc.x, bc.y))) cg_loop_saved = true;
            if (cg_loop_saved) break;
        }
        // ---- normalise x, test |<x|b>| = 1
        double2 xx, xb;
        if ((rc = dot(x, x, xx))) return rc;
        scale_real_kernel<<<nb, kThreads, 0, c->stream>>>(x, 1.0 / std::sqrt(xx.x), n);
        if ((rc = dot(x, b, xb))) return rc;
        if (std::fabs(std::hypot(xb.x, xb.y) - 1.0) < 1.0e-12) break;
        e = cudaMemcpyAsync(b, x, bytes, cudaMemcpyDeviceToDevice, c->stream);
        if (e != cudaSuccess) return cuda_fail(e, "cg copy");
    }
    e = cudaMemcpyAsync(x_out, x, bytes, (flags & PNED_PTR_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                        c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_cg_run: result");
    if (n_inv) *n_inv = itr_inv;
    if (n_cg) *n_cg = total_cg;
    return PNED_OK;
}

// ---------------------------------------------------------------------------
// session checkpoint / restart (the role of interval_dump / interval_dump_read,
// S1/2 output.f90:50-211: Krylov arrays and vectors to a file, resumed later)
// ---------------------------------------------------------------------------
namespace pned {
namespace {

constexpr uint32_t kCkptMagic = 0x54504B43u;   // "CKPT"
constexpr int32_t kCkptVersion = 1;

// A section: 8-byte length, payload (vectors exceed the 4-byte Fortran record length).
bool ck_put(FILE *f, const void *p, uint64_t n)
{
    return fwrite(&n, 8, 1, f) == 1 && (n == 0 || fwrite(p, 1, size_t(n), f) == size_t(n));
}

bool ck_get(FILE *f, void *p, uint64_t n)
{
    uint64_t m = 0;
    return fread(&m, 8, 1, f) == 1 && m == n && (n == 0 || fread(p, 1, size_t(n), f) == size_t(n));
}

// Device vector to file (or back) through a bounded host buffer.
bool ck_put_dev(FILE *f, const double2 *d, uint64_t bytes, cudaStream_t st)
{
    if (fwrite(&bytes, 8, 1, f) != 1) return false;
    const uint64_t chunk = uint64_t(1) << 28;
    std::vector<char> h(size_t(std::min(bytes, chunk)));
    for (uint64_t o = 0; o < bytes; o += chunk) {
        const size_t n = size_t(std::min(chunk, bytes - o));
        if (cudaMemcpyAsync(h.data(), reinterpret_cast<const char *>(d) + o, n, cudaMemcpyDeviceToHost, st) !=
                cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess || fwrite(h.data(), 1, n, f) != n)
            return false;
    }
    return true;
}

bool ck_get_dev(FILE *f, double2 *d, uint64_t bytes, cudaStream_t st)
{
    uint64_t m = 0;
    if (fread(&m, 8, 1, f) != 1 || m != bytes) return false;
    const uint64_t chunk = uint64_t(1) << 28;
    std::vector<char> h(size_t(std::min(bytes, chunk)));
    for (uint64_t o = 0; o < bytes; o += chunk) {
        const size_t n = size_t(std::min(chunk, bytes - o));
        if (fread(h.data(), 1, n, f) != n ||
            cudaMemcpyAsync(reinterpret_cast<char *>(d) + o, h.data(), n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return false;
    }
    return true;
}

}  // namespace
}  // namespace pned

extern "C" int pned_session_save(pned_ctx *c, const char *path)
{
    if (!c || !path) return fail(PNED_EINVAL, "pned_session_save: bad arguments");
    Session &S = c->sess;
    if (!S.kind) return fail(PNED_EINVAL, "pned_session_save: no session");
    if (S.nobs) return fail(PNED_ENOTSUP, "pned_session_save: sessions with observables are not checkpointed");
    cudaSetDevice(c->m->device);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_session_save");
    const int R = c->R, k = S.enqueued;
    const size_t nh = size_t(k) * R;
    std::vector<double> scal(size_t(kScalSlots) * kMaxR), a(nh), b(nh), cf(nh * std::max(1, S.ncoef));
    int32_t counters[2] = {0, 0};
    e = cudaMemcpy(scal.data(), c->scal, sizeof(double) * scal.size(), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && nh) e = cudaMemcpy(a.data(), S.d_alpha, sizeof(double) * nh, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && nh) e = cudaMemcpy(b.data(), S.d_beta, sizeof(double) * nh, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && nh && S.d_coef)
        e = cudaMemcpy(cf.data(), S.d_coef, sizeof(double) * nh * S.ncoef, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(counters, S.d_counter, sizeof(int32_t) * 2, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "pned_session_save: reading the session");
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(PNED_EINVAL, std::string("pned_session_save: cannot open ") + path);
    const int64_t dim = c->m->dim;
    int32_t hdr[10] = {int32_t(kCkptMagic), kCkptVersion, S.kind, R, k, S.max_steps, S.ncoef, S.b0, S.b1, S.b2};
    bool ok = ck_put(f, hdr, sizeof(hdr)) && ck_put(f, &dim, 8) && ck_put(f, &S.L, 8) &&
              ck_put(f, counters, sizeof(counters)) && ck_put(f, scal.data(), sizeof(double) * scal.size()) &&
              ck_put(f, a.data(), sizeof(double) * nh) && ck_put(f, b.data(), sizeof(double) * nh) &&
              ck_put(f, cf.data(), sizeof(double) * (S.d_coef ? nh * S.ncoef : 0));
    const uint64_t vb = sizeof(double2) * uint64_t(dim) * R;
    for (int r : {S.b0, S.b1, S.b2})
        if (ok) ok = ck_put_dev(f, c->buf[r], vb, c->stream);
    ok = (std::fclose(f) == 0) && ok;
    return ok ? PNED_OK : fail(PNED_EINVAL, "pned_session_save: write failed");
}

extern "C" int pned_session_load(pned_ctx *c, const char *path, int max_steps)
{
    if (!c || !path) return fail(PNED_EINVAL, "pned_session_load: bad arguments");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(PNED_EINVAL, std::string("pned_session_load: cannot open ") + path);
    int32_t hdr[10];
    int64_t dim = 0;
    double L = 0.0;
    int32_t counters[2];
    bool ok = ck_get(f, hdr, sizeof(hdr)) && hdr[0] == int32_t(kCkptMagic) && hdr[1] == kCkptVersion &&
              ck_get(f, &dim, 8) && ck_get(f, &L, 8) && ck_get(f, counters, sizeof(counters));
    if (!ok) { std::fclose(f); return fail(PNED_EINVAL, "pned_session_load: not a session checkpoint"); }
    const int kind = hdr[2], R = hdr[3], k = hdr[4], ncoef = hdr[6];
    if (R != c->R || dim != c->m->dim) {
        std::fclose(f);
        return fail(PNED_EINVAL, "pned_session_load: checkpoint of another basis size or vector count");
    }
    if (max_steps < k) max_steps = hdr[5];
    cudaSetDevice(c->m->device);
    int rc = session_common_begin(c, kind, std::max(max_steps, k));
    if (rc) { std::fclose(f); return rc; }
    cudaError_t e0 = cudaStreamSynchronize(c->stream);   // the begin's resets land before the restores
    if (e0 != cudaSuccess) { std::fclose(f); session_release(c); return cuda_fail(e0, "pned_session_load"); }
    Session &S = c->sess;
    S.L = L;
    S.ncoef = ncoef;
    S.b0 = hdr[7]; S.b1 = hdr[8]; S.b2 = hdr[9];
    const size_t nh = size_t(k) * R;
    std::vector<double> scal(size_t(kScalSlots) * kMaxR), a(nh), b(nh), cf(kind == PNED_SESSION_TPS ? nh * ncoef : 0);
    if (kind == PNED_SESSION_TPS) {
        S.d_coef = sess_alloc<double>(S, size_t(S.max_steps) * R * ncoef);
        S.d_osum = sess_alloc<double2>(S, size_t(2) * R);
        if (!S.d_coef || !S.d_osum) { std::fclose(f); session_release(c); return fail(PNED_ENOMEM, "session"); }
    }
    ok = ck_get(f, scal.data(), sizeof(double) * scal.size()) && ck_get(f, a.data(), sizeof(double) * nh) &&
         ck_get(f, b.data(), sizeof(double) * nh) && ck_get(f, cf.data(), sizeof(double) * cf.size());
    cudaError_t e = cudaSuccess;
    if (ok) {
        e = cudaMemcpy(c->scal, scal.data(), sizeof(double) * scal.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && nh) e = cudaMemcpy(S.d_alpha, a.data(), sizeof(double) * nh, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && nh) e = cudaMemcpy(S.d_beta, b.data(), sizeof(double) * nh, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !cf.empty())
            e = cudaMemcpy(S.d_coef, cf.data(), sizeof(double) * cf.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(S.d_counter, counters, sizeof(int32_t) * 2, cudaMemcpyHostToDevice);
    }
    const uint64_t vb = sizeof(double2) * uint64_t(dim) * R;
    for (int r : {S.b0, S.b1, S.b2})
        if (ok && e == cudaSuccess) ok = ck_get_dev(f, c->buf[r], vb, c->stream);
    std::fclose(f);
    if (!ok || e != cudaSuccess) {
        session_release(c);
        return e != cudaSuccess ? cuda_fail(e, "pned_session_load") : fail(PNED_EINVAL, "pned_session_load: short file");
    }
    S.enqueued = k;
    return PNED_OK;
}

extern "C" int pned_session_lanczos_state(pned_ctx *c, pned_c128 *w_out, pned_c128 *v_out, int flags)
{
    if (!c || !w_out || !v_out) return fail(PNED_EINVAL, "pned_session_lanczos_state: bad arguments");
    Session &S = c->sess;
    if ((S.kind != PNED_SESSION_LANCZOS && S.kind != PNED_SESSION_DSF) || c->R != 1 || S.enqueued < 1)
        return fail(PNED_EINVAL, "pned_session_lanczos_state: needs a Lanczos or DSF session (R = 1) with steps done");
    cudaSetDevice(c->m->device);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_session_lanczos_state");
    // after step k: b0 = W_k - alpha_k v_k (the next vector times beta_k), b1 = v_k / sc_old,
    // b2 = W_k; sc = 1 / beta_k, pc = -beta_k sc_old
    const int k = S.enqueued;
    double sc = 0.0, pc = 0.0, be = 0.0;
    e = cudaMemcpy(&sc, slot(c, kSlotSc), sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&pc, slot(c, kSlotPc), sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&be, S.d_beta + (k - 1), sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "pned_session_lanczos_state: scalars");
    if (!(be > 0.0)) return fail(PNED_EBREAKDOWN, "pned_session_lanczos_state: beta of the last step is zero");
    const double sc_old = -pc / be;
    const int64_t n = c->m->dim;
    const size_t bytes = sizeof(double2) * size_t(n);
    const bool dev = (flags & PNED_PTR_DEVICE) != 0;
    const cudaMemcpyKind kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    e = cudaMemcpyAsync(w_out, c->buf[S.b2], bytes, kind, c->stream);
    if (e == cudaSuccess && dev) {
        e = cudaMemcpyAsync(v_out, c->buf[S.b1], bytes, kind, c->stream);
        if (e == cudaSuccess) {
            scale_real_kernel<<<c->nblocks, kThreads, 0, c->stream>>>(reinterpret_cast<double2 *>(v_out), sc_old, n);
            e = cudaGetLastError();
        }
    } else if (e == cudaSuccess) {
        // copied out, then scaled on the host (no device memory beyond the session's)
        e = cudaMemcpyAsync(v_out, c->buf[S.b1], bytes, kind, c->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_session_lanczos_state");
    if (!dev) {
        double *p = reinterpret_cast<double *>(v_out);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < 2 * n; ++i) p[i] *= sc_old;
    }
    return PNED_OK;
}

static int begin_chain_at(pned_ctx *c, int kind, const pned_c128 *w, const pned_c128 *v, const double *alpha,
                          const double *beta, int k, int max_steps, int flags)
{
    if (!c || !w || !v || !alpha || !beta || k < 1 || max_steps < k)
        return fail(PNED_EINVAL, "pned_session_begin_lanczos_at: bad arguments");
    if (c->R != 1) return fail(PNED_EINVAL, "pned_session_begin_lanczos_at: needs a context with R = 1");
    if (!(beta[k - 1] > 0.0)) return fail(PNED_EINVAL, "pned_session_begin_lanczos_at: beta[k-1] must be positive");
    cudaSetDevice(c->m->device);
    int rc = session_common_begin(c, kind, max_steps);
    if (rc) return rc;
    Session &S = c->sess;
    const int64_t n = c->m->dim;
    const size_t bytes = sizeof(double2) * size_t(n);
    const cudaMemcpyKind ck = (flags & PNED_PTR_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    // b2 = W, b1 = v (the previous vector, scale 1), b0 = W - alpha v (the next vector times beta)
    cudaError_t e = cudaMemcpyAsync(c->buf[S.b2], w, bytes, ck, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->buf[S.b1], v, bytes, ck, c->stream);
    if (e == cudaSuccess) {
        resume_kernel<<<c->nblocks, kThreads, 0, c->stream>>>(c->buf[S.b2], c->buf[S.b1], c->buf[S.b0], alpha[k - 1], n);
        e = cudaGetLastError();
    }
    const int32_t counters[2] = {k, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(S.d_alpha, alpha, sizeof(double) * k, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(S.d_beta, beta, sizeof(double) * k, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(S.d_counter, counters, sizeof(counters), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);   // host sources may go away after the call
    if (e != cudaSuccess) { session_release(c); return cuda_fail(e, "pned_session_begin_lanczos_at"); }
    if ((rc = set_slot(c, kSlotSc, 1.0 / beta[k - 1])) || (rc = set_slot(c, kSlotPc, -beta[k - 1]))) {
        session_release(c);
        return rc;
    }
    S.enqueued = k;
    return PNED_OK;
}

extern "C" int pned_session_begin_lanczos_at(pned_ctx *c, const pned_c128 *w, const pned_c128 *v, const double *alpha,
                                             const double *beta, int k, int max_steps, int flags)
{
    return begin_chain_at(c, PNED_SESSION_LANCZOS, w, v, alpha, beta, k, max_steps, flags);
}

extern "C" int pned_session_begin_dsf_at(pned_ctx *c, const pned_c128 *w, const pned_c128 *v, const double *alpha,
                                         const double *beta, int k, int max_steps, int flags)
{
    return begin_chain_at(c, PNED_SESSION_DSF, w, v, alpha, beta, k, max_steps, flags);
}

// Copies `src` (scaled by f) into a caller's host or device vector of n states.
static cudaError_t scaled_out(pned_ctx *c, const double2 *src, double f, pned_c128 *out, bool dev, int64_t n)
{
    const size_t bytes = sizeof(double2) * size_t(n);
    cudaError_t e = cudaMemcpyAsync(out, src, bytes, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && dev && f != 1.0) {
        scale_real_kernel<<<c->nblocks, kThreads, 0, c->stream>>>(reinterpret_cast<double2 *>(out), f, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess && !dev && f != 1.0) {
        double *p = reinterpret_cast<double *>(out);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < 2 * n; ++i) p[i] *= f;
    }
    return e;
}

extern "C" int pned_session_tps_state(pned_ctx *c, pned_c128 *w_out, pned_c128 *v_out, pned_c128 *g_out, int flags)
{
    if (!c || !w_out || !v_out || !g_out) return fail(PNED_EINVAL, "pned_session_tps_state: bad arguments");
    Session &S = c->sess;
    if (S.kind != PNED_SESSION_TPS || c->R != 1 || S.enqueued < 1)
        return fail(PNED_EINVAL, "pned_session_tps_state: needs a TPS session (R = 1) with steps done");
    cudaSetDevice(c->m->device);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_session_tps_state");
    // after step k: b0 = (L - H) v_k, b2 = v_k / gsc, b1 = v_{k-1} / gsc_prev (the next step's W)
    double gsc = 0.0, gscp = 0.0;
    e = cudaMemcpy(&gsc, slot(c, kSlotGsc), sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&gscp, slot(c, kSlotGscPrev), sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "pned_session_tps_state: scalars");
    const bool dev = (flags & PNED_PTR_DEVICE) != 0;
    const int64_t n = c->m->dim;
    e = scaled_out(c, c->buf[S.b0], 1.0, w_out, dev, n);
    if (e == cudaSuccess) e = scaled_out(c, c->buf[S.b2], gsc, v_out, dev, n);
    if (e == cudaSuccess) {
        if (S.enqueued >= 2) {
            e = scaled_out(c, c->buf[S.b1], gscp, g_out, dev, n);
        } else {   // no vector before the first
            e = dev ? cudaMemsetAsync(g_out, 0, sizeof(double2) * size_t(n), c->stream) : cudaSuccess;
            if (!dev) std::memset(static_cast<void *>(g_out), 0, sizeof(double2) * size_t(n));
            if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        }
    }
    return e == cudaSuccess ? PNED_OK : cuda_fail(e, "pned_session_tps_state");
}

extern "C" int pned_session_begin_tps_at(pned_ctx *c, double L, const pned_c128 *w, const pned_c128 *v,
                                         const double *alpha, const double *beta, const double *coef, int k,
                                         int max_steps, int flags)
{
    if (!c || !w || !v || !alpha || !beta || !coef || k < 1 || max_steps < k)
        return fail(PNED_EINVAL, "pned_session_begin_tps_at: bad arguments");
    if (c->R != 1) return fail(PNED_EINVAL, "pned_session_begin_tps_at: needs a context with R = 1");
    if (!(beta[k - 1] > 0.0)) return fail(PNED_EINVAL, "pned_session_begin_tps_at: beta[k-1] must be positive");
    cudaSetDevice(c->m->device);
    int rc = session_common_begin(c, PNED_SESSION_TPS, max_steps);
    if (rc) return rc;
    Session &S = c->sess;
    S.L = L;
    S.nobs = 0;
    S.ncoef = 5;
    S.d_coef = sess_alloc<double>(S, size_t(max_steps) * S.ncoef);
    S.d_osum = sess_alloc<double2>(S, 2);
    if (!S.d_coef || !S.d_osum) { session_release(c); return fail(PNED_ENOMEM, "session scratch"); }
    const int64_t n = c->m->dim;
    const size_t bytes = sizeof(double2) * size_t(n);
    const cudaMemcpyKind kind = (flags & PNED_PTR_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    // b0 = C = (L - H) v_k with scale 1/beta_k, b2 = G = v_k with scale 1 (the step rotates them)
    cudaError_t e = cudaMemcpyAsync(c->buf[S.b0], w, bytes, kind, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->buf[S.b2], v, bytes, kind, c->stream);
    const int32_t counters[2] = {k, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(S.d_alpha, alpha, sizeof(double) * k, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(S.d_beta, beta, sizeof(double) * k, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(S.d_coef, coef, sizeof(double) * size_t(k) * S.ncoef, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(S.d_counter, counters, sizeof(counters), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { session_release(c); return cuda_fail(e, "pned_session_begin_tps_at"); }
    if ((rc = set_slot(c, kSlotSc, 1.0 / beta[k - 1])) || (rc = set_slot(c, kSlotGsc, 1.0)) ||
        (rc = set_slot(c, kSlotGscPrev, 1.0))) {
        session_release(c);
        return rc;
    }
    S.enqueued = k;
    return PNED_OK;
}

extern "C" int pned_session_info(const pned_ctx *c, int *kind, int *steps_done, int *max_steps, int *n_coef)
{
    if (!c) return fail(PNED_EINVAL, "pned_session_info: null context");
    const Session &S = c->sess;
    if (kind) *kind = S.kind;
    if (steps_done) *steps_done = S.enqueued;
    if (max_steps) *max_steps = S.max_steps;
    if (n_coef) *n_coef = S.ncoef;
    return PNED_OK;
}
