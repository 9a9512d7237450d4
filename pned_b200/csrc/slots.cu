// Slot batches of libpned_gpu.so: continuous batching of independent Krylov
// chains (Lanczos, TPS, DSF momentum chains, Lanczos eigenvector passes) that
// share one S = 1/2 lattice (n sites, bond list) but each carry their own
// couplings.  The R slots live as the columns of interleaved [dim][R] buffers
// and advance together, one batched H.V per step; a slot is loaded and
// released between steps while the others keep running.
//
// Per step (one CUDA graph per three steps, since buffer roles rotate P -> C -> W):
//   slot_hv_kernel        W = pc P + hsc (H_r - shift) C  with per-slot tables and
//                         diagonal; sums <v|hv>, ||W||^2, <g|W>, <g|v>
//   finish                4R sums
//   slot_residual_kernel  Lanczos slots: W <- W - Re(alpha) v, beta^2 = ||W - alpha v||^2;
//                         eigenvector slots also accumulate x += c_k v
//   finish                R sums
//   slot_epilogue         per-slot alpha/beta/TPS coefficients and next scales
// Lanczos follows S_one_half/Hybrid_TPS_Lanczos.f90:48-163 (alpha from the H.v
// product, beta through the complex alpha, update with the real alpha), TPS
// follows S_one_half/Hybrid_TPS_TPS.f90:325-409 and eval_phys_val :83-111, the
// eigenvector pass follows parallelized_lncv1z :183-329 (stored alpha and beta,
// x = sum_k c_k v_k), the momentum chains intalv_zz and parallelized_dsflnc1z
// (S_one_half/Hybrid_TPS_DSF.f90:18-87, :195-261).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <set>
#include <vector>

#include "device.cuh"

namespace pned {

// per-slot state on the device
struct SlotDev {
    int kind;        // PNED_SLOT_*
    int active;      // 1 while counter < target and no breakdown
    int counter;     // steps done
    int target;      // steps to run
    int status;      // 0 ok, 1 beta breakdown
    int pad;
    double L;        // TPS: L
    double cnorm;    // DSF: ||S^z_q x||^2 / (n ||x||^2)
    double2 *aux;    // eigenvector slots: x accumulated here ([dim])
    const double *vcoef;   // eigenvector slots: c_k, k < target
};

// per-slot step coefficients, [kCf][R]
enum : int { kCfSc = 0, kCfHsc, kCfShift, kCfPc, kCfGsc, kCf };

struct SlotHvArgs {
    const double2 *C;
    const double2 *P;
    double2 *W;
    const double *diag;      // [dim][R]
    const double2 *table;    // [ntab][R]
    const double *cf;        // [kCf][R]
    double2 *partials;       // [nblocks][4][R]
    int64_t dim;
    int R;
};

template <int VPT>
__global__ void __launch_bounds__(kThreads, 2) slot_hv_kernel(const __grid_constant__ XorProgram prog, const SlotHvArgs a)
{
    extern __shared__ double2 s_tab[];
    const int R = a.R, G = R / VPT;
    for (int i = threadIdx.x; i < prog.ntab * R; i += blockDim.x) s_tab[i] = a.table[i];
    __syncthreads();
    const int g = threadIdx.x % G, r0 = g * VPT;
    double sh[VPT];
#pragma unroll
    for (int j = 0; j < VPT; ++j) sh[j] = a.cf[kCfShift * R + r0 + j];
    double2 red[4][VPT];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int j = 0; j < VPT; ++j) red[k][j] = make_double2(0.0, 0.0);
    const int64_t nitems = a.dim * G;
    for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < nitems;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = it / G;
        const uint32_t su = uint32_t(s);
        const int64_t e0 = s * R + r0;
        double2 v[VPT], acc[VPT];
#pragma unroll
        for (int j = 0; j < VPT; ++j) {
            v[j] = a.C[e0 + j];
            acc[j] = cscale(a.diag[e0 + j] - sh[j], v[j]);
        }
        for (int t = 0; t < prog.nterms; ++t) {
            const XorTerm T = prog.t[t];
            uint32_t idx = 0;
#pragma unroll
            for (int k = 0; k < kMaxDeps; ++k)
                if (k < T.nb) idx |= ((su >> ((T.pos4 >> (8 * k)) & 0xffu)) & 1u) << k;
            const double2 *ct = s_tab + (T.tab + idx) * R + r0;
            const double2 *ps = a.C + int64_t(su ^ T.xmask) * R + r0;
#pragma unroll
            for (int j = 0; j < VPT; ++j) acc[j] = cfma(ct[j], __ldg(ps + j), acc[j]);
        }
#pragma unroll
        for (int j = 0; j < VPT; ++j) {
            const double *cf = a.cf + r0 + j;   // per-slot scales, L1-resident
            const double2 hv = cscale(__ldg(cf + kCfHsc * R), acc[j]);
            const double2 p = a.P[e0 + j];
            const double pc = __ldg(cf + kCfPc * R);
            const double2 out = make_double2(fma(pc, p.x, hv.x), fma(pc, p.y, hv.y));
            a.W[e0 + j] = out;
            const double2 vv = cscale(__ldg(cf + kCfSc * R), v[j]);
            const double2 gv = cscale(__ldg(cf + kCfGsc * R), p);
            red[0][j] = cadd(red[0][j], cconjmul(vv, hv));
            red[1][j].x += out.x * out.x + out.y * out.y;
            red[2][j] = cadd(red[2][j], cconjmul(gv, out));
            red[3][j] = cadd(red[3][j], cconjmul(gv, vv));
        }
    }
    block_reduce_store<4, VPT>(red, G, VPT, R, a.partials);
}

struct SlotResArgs {
    double2 *W;
    const double2 *C;
    const double *cf;
    const double2 *sums;     // [4][R] from the H.V pass
    SlotDev *st;
    const double *hist_a;    // [R][max_steps]
    double2 *partials;       // [nblocks][1][R]
    int64_t dim;
    int R, max_steps;
};

// Lanczos residual per slot (see the file comment); other slots are not touched.
template <int VPT>
__global__ void __launch_bounds__(kThreads) slot_residual_kernel(const SlotResArgs a)
{
    __shared__ int s_mode[kMaxR];
    __shared__ double2 s_al[kMaxR];
    __shared__ double s_cx[kMaxR];
    __shared__ double2 *s_aux[kMaxR];
    const int R = a.R, G = R / VPT;
    if (threadIdx.x < R) {
        const int r = threadIdx.x;
        const SlotDev d = a.st[r];
        int mode = 0;
        double2 al = make_double2(0.0, 0.0);
        double cx = 0.0;
        if (d.active && (d.kind == PNED_SLOT_LANCZOS || d.kind == PNED_SLOT_VECTOR)) {
            if (d.kind == PNED_SLOT_LANCZOS) {
                mode = 1;
                al = a.sums[r];
            } else {
                mode = 2;
                al = make_double2(a.hist_a[size_t(r) * a.max_steps + d.counter], 0.0);
                cx = d.vcoef[d.counter];
            }
        }
        s_mode[r] = mode;
        s_al[r] = al;
        s_cx[r] = cx;
        s_aux[r] = mode == 2 ? d.aux : nullptr;
    }
    __syncthreads();
    const int g = threadIdx.x % G, r0 = g * VPT;
    double2 red[1][VPT];
#pragma unroll
    for (int j = 0; j < VPT; ++j) red[0][j] = make_double2(0.0, 0.0);
    const int64_t nitems = a.dim * G;
    for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < nitems;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = it / G;
        const int64_t e0 = s * R + r0;
#pragma unroll
        for (int j = 0; j < VPT; ++j) {
            const int r = r0 + j;
            const int mode = s_mode[r];
            if (!mode) continue;
            const double2 al = s_al[r];
            const double2 w = a.W[e0 + j];
            const double2 v = cscale(a.cf[kCfSc * R + r], a.C[e0 + j]);
            const double2 d = make_double2(w.x - (al.x * v.x - al.y * v.y), w.y - (al.x * v.y + al.y * v.x));
            red[0][j].x += d.x * d.x + d.y * d.y;
            a.W[e0 + j] = make_double2(w.x - al.x * v.x, w.y - al.x * v.y);
            if (mode == 2) {
                double2 *x = s_aux[r] + s;
                const double2 xo = *x;
                *x = make_double2(fma(s_cx[r], v.x, xo.x), fma(s_cx[r], v.y, xo.y));
            }
        }
    }
    block_reduce_store<1, VPT>(red, G, VPT, R, a.partials);
}

__device__ __forceinline__ void slot_idle(double *cf, int R, int r)
{
    for (int f = 0; f < kCf; ++f) cf[f * R + r] = 0.0;
}

// Records the step of every active slot and sets the next step's scales.
__global__ void slot_epilogue(const double2 *__restrict__ s4, const double2 *__restrict__ sb, int R, SlotDev *st,
                              double *cf, double *hist_a, double *hist_b, double *coef, int max_steps)
{
    const int r = threadIdx.x;
    if (r >= R) return;
    SlotDev &d = st[r];
    if (!d.active) { slot_idle(cf, R, r); return; }
    const int k = d.counter;
    const double sc_old = cf[kCfSc * R + r];
    const size_t h = size_t(r) * max_steps + k;
    double be;
    if (d.kind == PNED_SLOT_TPS) {
        const double a1 = s4[0 * R + r].x;
        be = sqrt(s4[1 * R + r].x);
        const double2 gw = s4[2 * R + r], gv = s4[3 * R + r];
        hist_a[h] = d.L - a1;
        hist_b[h] = be;
        double *c = coef + h * 5;
        c[0] = double(2 * (k + 1)) / a1;
        c[1] = d.L;
        c[2] = be;
        c[3] = d.L - a1;
        c[4] = d.L * gv.x - gw.x;
        cf[kCfGsc * R + r] = sc_old;
        cf[kCfSc * R + r] = 1.0 / be;
        cf[kCfHsc * R + r] = -1.0 / be;
        cf[kCfShift * R + r] = d.L;
        cf[kCfPc * R + r] = 0.0;
    } else {
        if (d.kind == PNED_SLOT_LANCZOS) {
            be = sqrt(sb[r].x);
            hist_a[h] = s4[r].x;
            hist_b[h] = be;
        } else {
            be = hist_b[h];
        }
        cf[kCfPc * R + r] = -be * sc_old;
        cf[kCfSc * R + r] = 1.0 / be;
        cf[kCfHsc * R + r] = 1.0 / be;
        cf[kCfShift * R + r] = 0.0;
        cf[kCfGsc * R + r] = 0.0;
    }
    d.counter = k + 1;
    if (!(be >= 0.5e-30)) { d.status = 1; d.active = 0; }
    if (d.counter >= d.target) d.active = 0;
    if (!d.active) slot_idle(cf, R, r);
}

// Writes column r of C (a dense vector, or S^z_q of one), zeroes column r of P
// and W (and the eigenvector target), and sums |column|^2 and |x|^2.
__global__ void __launch_bounds__(kThreads) slot_load_kernel(const double2 *__restrict__ x,
                                                             const double2 *__restrict__ ph, int n, double2 *C,
                                                             double2 *P, double2 *W, double2 *aux, int64_t dim, int R,
                                                             int r, double2 *partials)
{
    double2 red[2][1] = {{make_double2(0.0, 0.0)}, {make_double2(0.0, 0.0)}};
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < dim; s += (int64_t)gridDim.x * blockDim.x) {
        const double2 xs = x[s];
        double2 v = xs;
        if (ph) {
            double2 w = make_double2(0.0, 0.0);
            for (int j = 0; j < n; ++j) {
                const double f = double((s >> j) & 1) - 0.5;
                w.x = fma(f, ph[j].x, w.x);
                w.y = fma(f, ph[j].y, w.y);
            }
            v = cmul(w, xs);
        }
        const int64_t e = s * R + r;
        C[e] = v;
        P[e] = make_double2(0.0, 0.0);
        W[e] = make_double2(0.0, 0.0);
        if (aux) aux[s] = make_double2(0.0, 0.0);
        red[0][0].x += v.x * v.x + v.y * v.y;
        red[1][0].x += xs.x * xs.x + xs.y * xs.y;
    }
    block_reduce_store<2, 1>(red, 1, 1, 1, partials);
}

__global__ void slot_load_epilogue(const double2 *__restrict__ sums, int r, int R, int n, int kind, int target,
                                   double L, int szq, double2 *aux, const double *vcoef, SlotDev *st, double *cf)
{
    if (threadIdx.x != 0) return;
    const double nv = sums[0].x, nx = sums[1].x;
    SlotDev d{};
    d.kind = kind;
    d.target = target;
    d.counter = 0;
    d.status = 0;
    d.L = L;
    d.cnorm = szq ? (nx > 0 ? nv / (double(n) * nx) : 0.0) : 0.0;
    d.aux = aux;
    d.vcoef = vcoef;
    const double sc = nv > 0 ? 1.0 / sqrt(nv) : 0.0;
    d.active = (target > 0 && nv > 0) ? 1 : 0;
    if (!(nv > 0)) d.status = 1;
    st[r] = d;
    cf[kCfSc * R + r] = d.active ? sc : 0.0;
    cf[kCfHsc * R + r] = d.active ? (kind == PNED_SLOT_TPS ? -sc : sc) : 0.0;
    cf[kCfShift * R + r] = (d.active && kind == PNED_SLOT_TPS) ? L : 0.0;
    cf[kCfPc * R + r] = 0.0;
    cf[kCfGsc * R + r] = 0.0;
}

// Per-slot diagonal column: diag[s, r] = sum_b dtab[b][st_b(s)] (real part).
__global__ void slot_diag_kernel(int64_t dim, int nbond, const int *__restrict__ s1, const int *__restrict__ s2,
                                 const double2 *__restrict__ dtab, double *diag, int R, int r)
{
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < dim; s += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int b = 0; b < nbond; ++b) {
            const int stt = int((s >> s1[b]) & 1) | (int((s >> s2[b]) & 1) << 1);
            acc += dtab[b * 4 + stt].x;
        }
        diag[s * R + r] = acc;
    }
}

// Column r of the interleaved [dim][R] Gaussian stream: v[s] = z(s R + r).
__global__ void gaussian_column_kernel(uint64_t key, int64_t dim, int R, int r, double2 *v)
{
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < dim; s += (int64_t)gridDim.x * blockDim.x)
        v[s] = gaussian_at(key, s * R + r);
}

__global__ void slot_release_kernel(SlotDev *st, double *cf, int R, int r)
{
    if (threadIdx.x == 0) {
        st[r].active = 0;
        st[r].kind = PNED_SLOT_FREE;
        st[r].aux = nullptr;
        st[r].vcoef = nullptr;
        slot_idle(cf, R, r);
    }
}

}  // namespace pned

using namespace pned;

struct pned_slots {
    HostProgram hp;
    std::unique_ptr<XorProgram> xprog;
    int device = 0, n = 0, nbond = 0, R = 1, max_steps = 0, ntab = 0, nsm = 148, nblocks = 1;
    int64_t dim = 0;
    size_t bytes = 0, budget = 0;
    cudaStream_t stream = nullptr, own_stream = nullptr;
    double2 *buf[3] = {nullptr, nullptr, nullptr};
    int role[3] = {0, 1, 2};   // P, C, W buffer indices for the next step
    double *diag = nullptr;
    double2 *table = nullptr;
    int *s1 = nullptr, *s2 = nullptr;
    SlotDev *st = nullptr;
    double *cf = nullptr;
    double *hist_a = nullptr, *hist_b = nullptr, *coef = nullptr;
    double *vcoef = nullptr;         // [R][max_steps]
    double2 *partials = nullptr, *sums = nullptr, *scratch = nullptr;   // scratch: [R][n] phases + [R][nbond*4] dtab
    int64_t partials_cap = 0;        // double2 slots at `partials`
    uint32_t *tile_ctr = nullptr;    // R = 1: tile counters of the single-vector kernel's dynamic order
    cudaGraphExec_t graph = nullptr;
    int64_t enqueued = 0;
    // R = 1: the batch's table and diagonal have the layout of a model's, so the
    // tiled single-vector kernel runs the step (tm borrows table and diagonal)
    pned_model tm;
    bool tile = false;
    std::set<std::pair<int, int>> flips;   // (bond, f) pairs of the structure
};

namespace {

template <int VPT>
cudaError_t launch_slot_hv_v(pned_slots *S, const SlotHvArgs &a)
{
    auto kern = slot_hv_kernel<VPT>;
    const size_t smem = sizeof(double2) * size_t(std::max(1, S->ntab)) * S->R;
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void *>(kern), S->device);
    if (e != cudaSuccess) return e;
    kern<<<S->nblocks, kThreads, smem, S->stream>>>(*S->xprog, a);
    return cudaGetLastError();
}

template <int VPT>
cudaError_t launch_slot_res_v(pned_slots *S, const SlotResArgs &a)
{
    slot_residual_kernel<VPT><<<S->nblocks, kThreads, 0, S->stream>>>(a);
    return cudaGetLastError();
}

cudaError_t slot_step(pned_slots *S)
{
    const int R = S->R;
    double2 *P = S->buf[S->role[0]], *C = S->buf[S->role[1]], *W = S->buf[S->role[2]];
    cudaError_t e;
    int nb_hv = S->nblocks;
    if (S->tile) {
        HvArgs a{};
        a.C = C; a.P = P; a.W = W; a.G = P;
        a.sc = S->cf + kCfSc * R; a.pc = S->cf + kCfPc * R; a.gsc = S->cf + kCfGsc * R;
        a.hsc = S->cf + kCfHsc * R; a.shiftv = S->cf + kCfShift * R;
        a.diag = S->diag; a.shift = 0.0; a.table = S->table;
        a.partials = S->partials; a.dim = S->dim; a.R = R; a.K = 4;
        a.slot_tables = R > 1;
        a.tile_counter = S->tile_ctr;
        a.partials_cap = S->partials_cap;
        e = launch_hv(&S->tm, a, S->nblocks, S->stream);
        nb_hv = int(hv_partials(&S->tm, a, S->nblocks));
    } else {
        SlotHvArgs a{};
        a.C = C; a.P = P; a.W = W;
        a.diag = S->diag; a.table = S->table; a.cf = S->cf;
        a.partials = S->partials; a.dim = S->dim; a.R = R;
        switch (pick_vpt(R)) {
        case 4: e = launch_slot_hv_v<4>(S, a); break;
        case 3: e = launch_slot_hv_v<3>(S, a); break;
        case 2: e = launch_slot_hv_v<2>(S, a); break;
        default: e = launch_slot_hv_v<1>(S, a); break;
        }
    }
    double2 *s4 = S->sums, *sb = S->sums + 4 * kMaxR;
    if (e == cudaSuccess) e = launch_finish(S->partials, nb_hv, 4 * R, s4, S->stream);
    SlotResArgs b{};
    b.W = W; b.C = C; b.cf = S->cf; b.sums = s4; b.st = S->st; b.hist_a = S->hist_a;
    b.partials = S->partials; b.dim = S->dim; b.R = R; b.max_steps = S->max_steps;
    if (e == cudaSuccess) {
        switch (pick_vpt(R)) {
        case 4: e = launch_slot_res_v<4>(S, b); break;
        case 3: e = launch_slot_res_v<3>(S, b); break;
        case 2: e = launch_slot_res_v<2>(S, b); break;
        default: e = launch_slot_res_v<1>(S, b); break;
        }
    }
    if (e == cudaSuccess) e = launch_finish(S->partials, S->nblocks, R, sb, S->stream);
    if (e == cudaSuccess) {
        slot_epilogue<<<1, 32 * ((R + 31) / 32), 0, S->stream>>>(s4, sb, R, S->st, S->cf, S->hist_a, S->hist_b,
                                                                 S->coef, S->max_steps);
        e = cudaGetLastError();
    }
    // P <- C, C <- W, W <- P
    const int p = S->role[0];
    S->role[0] = S->role[1];
    S->role[1] = S->role[2];
    S->role[2] = p;
    return e;
}

template <class T> cudaError_t salloc(pned_slots *S, T **p, size_t n)
{
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * std::max<size_t>(1, n));
    if (e == cudaSuccess) S->bytes += sizeof(T) * std::max<size_t>(1, n);
    return e;
}

void slots_free(pned_slots *S)
{
    if (S->graph) cudaGraphExecDestroy(S->graph);
    for (double2 *b : S->buf) cudaFree(b);
    cudaFree(S->diag); cudaFree(S->table); cudaFree(S->s1); cudaFree(S->s2); cudaFree(S->st); cudaFree(S->cf);
    cudaFree(S->hist_a); cudaFree(S->hist_b); cudaFree(S->coef); cudaFree(S->vcoef);
    cudaFree(S->partials); cudaFree(S->sums); cudaFree(S->scratch); cudaFree(S->tile_ctr);
    if (S->own_stream) cudaStreamDestroy(S->own_stream);
}

int check_slot(pned_slots *S, int slot)
{
    if (!S) return fail(PNED_EINVAL, "null slot batch");
    if (slot < 0 || slot >= S->R) return fail(PNED_EINVAL, "slot index out of range");
    return PNED_OK;
}

// Uploads the per-slot coefficient table column and computes the diagonal column.
int load_couplings(pned_slots *S, int slot, const pned_model_desc *d)
{
    std::vector<cd> table, dtab;
    int rc = eval_tables_on_structure(S->hp, d, table, dtab);
    if (rc) return rc;
    // the structure must hold every flip the couplings need
    {
        pned_model_desc dd = *d;
        dd.parity_type = 1;   // slot batches run the full basis
        HostProgram own;
        rc = compile_program(&dd, own);
        if (rc) return rc;
        for (size_t t = 0; t < own.xcontrib.size(); ++t)
            for (const auto &bf : own.xcontrib[t])
                if (!S->flips.count(bf))
                    return fail(PNED_EINVAL, "slot couplings need a spin flip that the batch's structure lacks");
        for (const cd &z : dtab)
            if (z.imag() != 0) return fail(PNED_EINVAL, "slot couplings: the diagonal must be real");
    }
    const int R = S->R;
    // strided column write of the table: [ntab][R]
    std::vector<double2> col(table.size());
    for (size_t i = 0; i < table.size(); ++i) col[i] = make_double2(table[i].real(), table[i].imag());
    cudaError_t e = cudaSuccess;
    if (!col.empty())
        e = cudaMemcpy2DAsync(S->table + slot, sizeof(double2) * R, col.data(), sizeof(double2), sizeof(double2),
                              col.size(), cudaMemcpyHostToDevice, S->stream);
    double2 *dt = S->scratch + size_t(R) * 64 + size_t(slot) * S->nbond * 4;
    std::vector<double2> hd(dtab.size());
    for (size_t i = 0; i < dtab.size(); ++i) hd[i] = make_double2(dtab[i].real(), 0.0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dt, hd.data(), sizeof(double2) * hd.size(), cudaMemcpyHostToDevice, S->stream);
    if (e == cudaSuccess) {
        slot_diag_kernel<<<S->nsm * 8, kThreads, 0, S->stream>>>(S->dim, S->nbond, S->s1, S->s2, dt, S->diag, R, slot);
        e = cudaGetLastError();
    }
    // host staging buffers go away on return
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
    if (e != cudaSuccess) return cuda_fail(e, "loading slot couplings");
    return PNED_OK;
}

int load_vector(pned_slots *S, int slot, int kind, int n_steps, double L, const pned_c128 *v, const double *qr,
                pned_c128 *aux, const double *coef_host, int flags)
{
    const int R = S->R;
    const double2 *dv = reinterpret_cast<const double2 *>(v);
    double2 *tmp = nullptr;
    cudaError_t e = cudaSuccess;
    if (!(flags & PNED_PTR_DEVICE)) {
        e = cudaMallocAsync(reinterpret_cast<void **>(&tmp), sizeof(double2) * size_t(S->dim), S->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(tmp, v, sizeof(double2) * size_t(S->dim), cudaMemcpyHostToDevice, S->stream);
        dv = tmp;
    }
    double2 *ph = nullptr;
    if (qr && e == cudaSuccess) {
        std::vector<double2> hp(S->n);
        for (int j = 0; j < S->n; ++j) hp[j] = make_double2(std::cos(qr[j]), std::sin(qr[j]));
        ph = S->scratch + size_t(slot) * 64;
        e = cudaMemcpyAsync(ph, hp.data(), sizeof(double2) * S->n, cudaMemcpyHostToDevice, S->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
    }
    double *vc = nullptr;
    if (kind == PNED_SLOT_VECTOR && e == cudaSuccess) {
        vc = S->vcoef + size_t(slot) * S->max_steps;
        e = cudaMemcpyAsync(vc, coef_host, sizeof(double) * n_steps, cudaMemcpyHostToDevice, S->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
    }
    double2 *dx = reinterpret_cast<double2 *>(aux);
    if (e == cudaSuccess) {
        slot_load_kernel<<<S->nblocks, kThreads, 0, S->stream>>>(dv, ph, S->n, S->buf[S->role[1]], S->buf[S->role[0]],
                                                                 S->buf[S->role[2]], dx, S->dim, R, slot, S->partials);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = launch_finish(S->partials, S->nblocks, 2, S->sums + 8 * kMaxR, S->stream);
    if (e == cudaSuccess) {
        slot_load_epilogue<<<1, 32, 0, S->stream>>>(S->sums + 8 * kMaxR, slot, R, S->n, kind, n_steps, L, qr ? 1 : 0,
                                                    dx, vc, S->st, S->cf);
        e = cudaGetLastError();
    }
    if (tmp) {
        cudaError_t e2 = cudaFreeAsync(tmp, S->stream);
        if (e == cudaSuccess) e = e2;
    }
    if (e != cudaSuccess) return cuda_fail(e, "loading a slot");
    return PNED_OK;
}

}  // namespace

extern "C" int pned_slots_create(const pned_model_desc *structure, int R, int max_steps, size_t hbm_budget,
                                 pned_slots **out)
{
    if (!structure || !out || pick_vpt(R) == 0 || max_steps < 1)
        return fail(PNED_EINVAL, "pned_slots_create: R must be one of 1, 2, 3, 4, 6, 8, 12, 16 and max_steps >= 1");
    *out = nullptr;
    if (structure->q_spin != 2) return fail(PNED_ENOTSUP, "pned_slots_create: slot batches are S = 1/2");
    std::unique_ptr<pned_slots> S(new pned_slots());
    int rc = compile_program(structure, S->hp);
    if (rc) return rc;
    const HostProgram &hp = S->hp;
    S->n = hp.n; S->nbond = hp.nbond; S->dim = hp.dim; S->R = R; S->max_steps = max_steps;
    S->ntab = int(hp.table.size());
    S->budget = hbm_budget;
    if (S->n > 32) return fail(PNED_ENOTSUP, "pned_slots_create: at most 32 sites");
    const size_t smem = sizeof(double2) * size_t(std::max(1, S->ntab)) * R;
    if (smem > 200 * 1024)
        return fail(PNED_ENOTSUP, "pned_slots_create: per-slot coefficient tables exceed 200 KB of shared memory; "
                                  "use fewer slots");
    for (const auto &c : hp.xcontrib)
        for (const auto &bf : c) S->flips.insert(bf);
    S->xprog.reset(new XorProgram());
    S->xprog->nterms = int(hp.xterms.size());
    S->xprog->ntab = S->ntab;
    std::copy(hp.xterms.begin(), hp.xterms.end(), S->xprog->t);
    // memory: 3 [dim][R] vectors + [dim][R] diagonal
    const size_t vbytes = sizeof(double2) * size_t(S->dim) * R;
    const size_t need = 3 * vbytes + sizeof(double) * size_t(S->dim) * R;
    if (hbm_budget && need > hbm_budget)
        return fail(PNED_EBUDGET, "pned_slots_create: the slot batch needs more than the HBM budget");
    cudaError_t e = cudaSetDevice(current_device());
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    S->device = current_device();
    cudaDeviceGetAttribute(&S->nsm, cudaDevAttrMultiProcessorCount, S->device);
    const int64_t items = S->dim * (R / pick_vpt(R));
    S->nblocks = int(std::max<int64_t>(1, std::min<int64_t>(int64_t(S->nsm) * 8, (items + kThreads - 1) / kThreads)));
    e = cudaStreamCreateWithFlags(&S->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    S->stream = S->own_stream;
    for (int k = 0; k < 3 && e == cudaSuccess; ++k) e = salloc(S.get(), &S->buf[k], size_t(S->dim) * R);
    if (e == cudaSuccess) e = salloc(S.get(), &S->diag, size_t(S->dim) * R);
    if (e != cudaSuccess) {
        cudaGetLastError();
        slots_free(S.get());
        return fail(PNED_ENOMEM, "pned_slots_create: cannot allocate the slot vectors");
    }
    if (e == cudaSuccess) e = salloc(S.get(), &S->table, size_t(std::max(1, S->ntab)) * R);
    if (e == cudaSuccess) e = salloc(S.get(), &S->s1, size_t(S->nbond));
    if (e == cudaSuccess) e = salloc(S.get(), &S->s2, size_t(S->nbond));
    if (e == cudaSuccess) e = salloc(S.get(), &S->st, size_t(R));
    if (e == cudaSuccess) e = salloc(S.get(), &S->cf, size_t(kCf) * R);
    if (e == cudaSuccess) e = salloc(S.get(), &S->hist_a, size_t(R) * max_steps);
    if (e == cudaSuccess) e = salloc(S.get(), &S->hist_b, size_t(R) * max_steps);
    if (e == cudaSuccess) e = salloc(S.get(), &S->coef, size_t(R) * max_steps * 5);
    if (e == cudaSuccess) e = salloc(S.get(), &S->vcoef, size_t(R) * max_steps);
    // per-block sums, and for R = 1 the per-tile sums of the single-vector kernel's
    // dynamic order (any plan of two passes with tiles of >= 2048 states)
    S->partials_cap = int64_t(S->nblocks) * kTileMaxPasses * kMaxK * kMaxR;
    if (R == 1) S->partials_cap = std::max<int64_t>(S->partials_cap, (S->dim / 2048 + 1) * 2 * kMaxK);
    if (e == cudaSuccess) e = salloc(S.get(), &S->partials, size_t(S->partials_cap));
    if (e == cudaSuccess) e = cudaMalloc(&S->tile_ctr, sizeof(uint32_t) * kTileMaxPasses);
    if (e == cudaSuccess) e = salloc(S.get(), &S->sums, size_t(12) * kMaxR);
    if (e == cudaSuccess) e = salloc(S.get(), &S->scratch, size_t(R) * 64 + size_t(R) * S->nbond * 4);
    if (e == cudaSuccess) e = cudaMemcpy(S->s1, hp.dsite1.data(), sizeof(int) * S->nbond, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(S->s2, hp.dsite2.data(), sizeof(int) * S->nbond, cudaMemcpyHostToDevice);
    // zeroed vectors: an idle column multiplies finite values by zero
    for (int k = 0; k < 3 && e == cudaSuccess; ++k) e = cudaMemset(S->buf[k], 0, vbytes);
    if (e == cudaSuccess) e = cudaMemset(S->diag, 0, sizeof(double) * size_t(S->dim) * R);
    if (e == cudaSuccess) e = cudaMemset(S->table, 0, sizeof(double2) * size_t(std::max(1, S->ntab)) * R);
    if (e == cudaSuccess) e = cudaMemset(S->st, 0, sizeof(SlotDev) * R);
    if (e == cudaSuccess) e = cudaMemset(S->cf, 0, sizeof(double) * kCf * R);
    if (e == cudaSuccess) e = cudaMemset(S->hist_a, 0, sizeof(double) * size_t(R) * max_steps);
    if (e == cudaSuccess) e = cudaMemset(S->hist_b, 0, sizeof(double) * size_t(R) * max_steps);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        slots_free(S.get());
        return cuda_fail(e, "pned_slots_create");
    }
    {
        // the batch's table ([ntab][R]) and diagonal ([dim][R]) drive the tiled
        // kernels through a model that borrows them
        pned_model &m = S->tm;
        m.hp = S->hp;
        m.device = S->device; m.n = S->n; m.q = 2; m.nbond = S->nbond; m.dim = S->dim;
        m.real_coef = false; m.real_diag = true;
        m.ntab = S->ntab; m.nterms = S->xprog->nterms; m.nsm = S->nsm;
        m.d_table = S->table; m.d_diag = S->diag;
        if (R == 1) {
            build_tile_programs(&m);
            S->tile = m.use_tile;
        } else {
            S->tile = ensure_rtiles(&m, R, true, nullptr);
        }
    }
    *out = S.release();
    return PNED_OK;
}

extern "C" int pned_slots_destroy(pned_slots *S)
{
    if (!S) return PNED_OK;
    cudaSetDevice(S->device);
    if (S->stream) cudaStreamSynchronize(S->stream);
    slots_free(S);
    delete S;
    return PNED_OK;
}

extern "C" int pned_slots_info(const pned_slots *S, int64_t *dim, int *R, int *max_steps, size_t *bytes)
{
    if (!S) return fail(PNED_EINVAL, "pned_slots_info: null slot batch");
    if (dim) *dim = S->dim;
    if (R) *R = S->R;
    if (max_steps) *max_steps = S->max_steps;
    if (bytes) *bytes = S->bytes;
    return PNED_OK;
}

extern "C" int pned_slots_set_stream(pned_slots *S, void *stream)
{
    if (!S) return fail(PNED_EINVAL, "pned_slots_set_stream: null slot batch");
    cudaStream_t ns = stream ? static_cast<cudaStream_t>(stream) : S->own_stream;
    if (ns != S->stream) {
        cudaStreamSynchronize(S->stream);
        S->stream = ns;
    }
    return PNED_OK;
}

extern "C" int pned_slots_load(pned_slots *S, int slot, int kind, const pned_model_desc *couplings,
                               const pned_c128 *v_init, int n_steps, double L, int flags)
{
    int rc = check_slot(S, slot);
    if (rc) return rc;
    if (kind != PNED_SLOT_LANCZOS && kind != PNED_SLOT_TPS)
        return fail(PNED_EINVAL, "pned_slots_load: kind must be PNED_SLOT_LANCZOS or PNED_SLOT_TPS");
    if (!couplings || !v_init || n_steps < 1 || n_steps > S->max_steps)
        return fail(PNED_EINVAL, "pned_slots_load: bad arguments (n_steps must be in 1..max_steps)");
    cudaSetDevice(S->device);
    if ((rc = load_couplings(S, slot, couplings))) return rc;
    return load_vector(S, slot, kind, n_steps, L, v_init, nullptr, nullptr, nullptr, flags);
}

extern "C" int pned_slots_load_szq(pned_slots *S, int slot, const pned_model_desc *couplings, const pned_c128 *x,
                                   const double *qr, int n_steps, int flags)
{
    int rc = check_slot(S, slot);
    if (rc) return rc;
    if (!couplings || !x || !qr || n_steps < 1 || n_steps > S->max_steps)
        return fail(PNED_EINVAL, "pned_slots_load_szq: bad arguments (n_steps must be in 1..max_steps)");
    cudaSetDevice(S->device);
    if ((rc = load_couplings(S, slot, couplings))) return rc;
    return load_vector(S, slot, PNED_SLOT_LANCZOS, n_steps, 0.0, x, qr, nullptr, nullptr, flags);
}

extern "C" int pned_slots_load_vector(pned_slots *S, int slot, const pned_model_desc *couplings,
                                      const pned_c128 *v_init, int n_steps, const double *alpha, const double *beta,
                                      const double *coef, pned_c128 *x_dev, int flags)
{
    int rc = check_slot(S, slot);
    if (rc) return rc;
    if (!couplings || !v_init || !alpha || !beta || !coef || !x_dev || n_steps < 1 || n_steps > S->max_steps)
        return fail(PNED_EINVAL, "pned_slots_load_vector: bad arguments (n_steps must be in 1..max_steps)");
    cudaSetDevice(S->device);
    if ((rc = load_couplings(S, slot, couplings))) return rc;
    // stored alpha/beta of the first pass drive the recurrence
    const size_t off = size_t(slot) * S->max_steps;
    cudaError_t e = cudaMemcpyAsync(S->hist_a + off, alpha, sizeof(double) * n_steps, cudaMemcpyHostToDevice, S->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(S->hist_b + off, beta, sizeof(double) * n_steps, cudaMemcpyHostToDevice, S->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_slots_load_vector");
    return load_vector(S, slot, PNED_SLOT_VECTOR, n_steps, 0.0, v_init, nullptr, x_dev, coef, flags);
}

extern "C" int pned_slots_release(pned_slots *S, int slot)
{
    int rc = check_slot(S, slot);
    if (rc) return rc;
    cudaSetDevice(S->device);
    slot_release_kernel<<<1, 32, 0, S->stream>>>(S->st, S->cf, S->R, slot);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PNED_OK : cuda_fail(e, "pned_slots_release");
}

extern "C" int pned_slots_step(pned_slots *S, int n_steps)
{
    if (!S || n_steps < 0) return fail(PNED_EINVAL, "pned_slots_step: bad arguments");
    cudaSetDevice(S->device);
    cudaError_t e = cudaSuccess;
    while (n_steps > 0) {
        const bool phase0 = S->role[0] == 0 && S->role[1] == 1 && S->role[2] == 2;
        if (phase0 && n_steps >= 3) {
            if (!S->graph) {
                cudaGraph_t graph;
                e = cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal);
                if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
                cudaError_t ek = cudaSuccess;
                for (int k = 0; k < 3; ++k) {
                    cudaError_t q = slot_step(S);
                    if (q != cudaSuccess) ek = q;
                }
                e = cudaStreamEndCapture(S->stream, &graph);
                if (e == cudaSuccess && ek != cudaSuccess) e = ek;
                if (e == cudaSuccess) {
                    e = cudaGraphInstantiate(&S->graph, graph, 0);
                    cudaGraphDestroy(graph);
                }
                if (e != cudaSuccess) return cuda_fail(e, "capturing the slot step graph");
            }
            e = cudaGraphLaunch(S->graph, S->stream);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
            S->enqueued += 3;
            n_steps -= 3;
            continue;
        }
        e = slot_step(S);
        if (e != cudaSuccess) return cuda_fail(e, "slot step");
        ++S->enqueued;
        --n_steps;
    }
    return PNED_OK;
}

extern "C" int pned_slots_query(pned_slots *S)
{
    if (!S) return fail(PNED_EINVAL, "pned_slots_query: null slot batch");
    cudaError_t e = cudaStreamQuery(S->stream);
    if (e == cudaSuccess) return 1;
    if (e == cudaErrorNotReady) return 0;
    return cuda_fail(e, "pned_slots_query");
}

extern "C" int pned_slots_synchronize(pned_slots *S)
{
    if (!S) return fail(PNED_EINVAL, "pned_slots_synchronize: null slot batch");
    cudaError_t e = cudaStreamSynchronize(S->stream);
    return e == cudaSuccess ? PNED_OK : cuda_fail(e, "pned_slots_synchronize");
}

extern "C" int pned_slots_read(pned_slots *S, int slot, int *kind, int *steps_done, int *status, double *alpha,
                               double *beta, double *coef, double *cnorm)
{
    int rc = check_slot(S, slot);
    if (rc) return rc;
    cudaSetDevice(S->device);
    SlotDev d{};
    cudaError_t e = cudaMemcpyAsync(&d, S->st + slot, sizeof(SlotDev), cudaMemcpyDeviceToHost, S->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_slots_read");
    const size_t off = size_t(slot) * S->max_steps;
    const int k = d.counter;
    if (alpha && k) e = cudaMemcpy(alpha, S->hist_a + off, sizeof(double) * k, cudaMemcpyDeviceToHost);
    if (beta && k && e == cudaSuccess) e = cudaMemcpy(beta, S->hist_b + off, sizeof(double) * k, cudaMemcpyDeviceToHost);
    if (coef && k && e == cudaSuccess)
        e = cudaMemcpy(coef, S->coef + off * 5, sizeof(double) * 5 * k, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "pned_slots_read");
    if (kind) *kind = d.kind;
    if (steps_done) *steps_done = k;
    if (status) *status = d.status;
    if (cnorm) *cnorm = d.cnorm;
    return PNED_OK;
}

extern "C" int pned_gaussian_column(int64_t dim, int R, int r, uint64_t seed, pned_c128 *v_dev, void *stream)
{
    if (dim < 1 || R < 1 || r < 0 || r >= R || !v_dev) return fail(PNED_EINVAL, "pned_gaussian_column: bad arguments");
    cudaSetDevice(current_device());
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, current_device());
    const int64_t nb = std::min<int64_t>(int64_t(nsm) * 8, (dim + kThreads - 1) / kThreads);
    gaussian_column_kernel<<<int(nb), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        splitmix64_host(seed ^ 0x5DEECE66Dull), dim, R, r, reinterpret_cast<double2 *>(v_dev));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PNED_OK : cuda_fail(e, "pned_gaussian_column");
}

extern "C" int pned_slots_set_plan(pned_slots *S, const pned_tile_plan *plan)
{
    if (!S) return fail(PNED_EINVAL, "pned_slots_set_plan: null slot batch");
    if (!S->tile) return PNED_OK;   // the flat kernel runs: nothing to plan
    cudaSetDevice(S->device);
    cudaError_t e = cudaStreamSynchronize(S->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_slots_set_plan");
    if (S->graph) {   // the captured steps hold the old plan
        cudaGraphExecDestroy(S->graph);
        S->graph = nullptr;
    }
    const pned_tile_plan def{-1, -1, -1, -1, -1, -1, -1, -1, -1};
    if (plan) S->tm.carveout = plan->l1_carveout != 0;
    if (S->R == 1) {
        S->tm.plan1 = plan ? *plan : def;
        S->tm.plan1_set = plan != nullptr;
        build_tile_programs(&S->tm);
        S->tile = S->tm.use_tile;
    } else {
        S->tile = ensure_rtiles(&S->tm, S->R, true, plan ? plan : &def);
    }
    return PNED_OK;
}

extern "C" int pned_slots_plan(const pned_slots *S, int *tile_passes, int *partner_tiles, int *tile_states)
{
    if (!S) return fail(PNED_EINVAL, "pned_slots_plan: null slot batch");
    if (!S->tile) {
        if (tile_passes) *tile_passes = 0;
        if (partner_tiles) *partner_tiles = 0;
        if (tile_states) *tile_states = 0;
        return PNED_OK;
    }
    return pned_model_plan(&S->tm, S->R, tile_passes, partner_tiles, tile_states);
}
