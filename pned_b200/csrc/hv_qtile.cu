// Tiled mixed-radix H.V (q > 2, full basis): the kernel, its launchers and
// the tile sets (passes of q^k-state tiles) built per model and R.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "device.cuh"

namespace pned {

// Tiled mixed-radix H.V (q > 2, full basis, R interleaved vectors), one pass
// of a multi-pass program.  A block stages tile t -- the q^k states whose
// outer digits spell t -- in shared memory with cp.async, vector-major
// ([R][nt]: a warp's partner reads fall on distinct banks), then applies the
// pass's terms (bonds with both sites among the k tile sites) there: partner =
// local index + loff, coefficient = the pass's table[tab + pair state].
// G = R / VPT threads share a state, each with VPT consecutive vectors.  The
// epilogue's streams (P or W, the diagonal) of an item are requested before
// its terms run.  The first pass adds the diagonal and pc P; later passes
// accumulate into W; the last forms the K >= 2 sums.
template <int VPT, bool RC, bool RD, int K>
__global__ void __launch_bounds__(kThreads, 2) hv_qtile_kernel(const __grid_constant__ QTileProgram prog, const HvArgs a)
{
    extern __shared__ double2 smem[];
    const int R = a.R, G = R / VPT, nt = prog.nt, q = prog.q;
    double2 *s_v = smem;                                           // [R][nt]
    double2 *s_tab = s_v + size_t(nt) * R;                         // [ntab]
    uint32_t *s_goff = reinterpret_cast<uint32_t *>(s_tab + prog.ntab);   // [nt]
    uint32_t *s_dig = s_goff + nt;                                 // [nt]
    for (int i = threadIdx.x; i < prog.ntab; i += blockDim.x) s_tab[i] = prog.tab[i];
    for (int l = threadIdx.x; l < nt; l += blockDim.x) {
        uint32_t dig = 0, off = 0;
        int x = l;
        for (int i = 0; i < prog.k; ++i) {
            const int d = x % q;
            x /= q;
            dig |= uint32_t(d) << (2 * i);
            off += uint32_t(d) * prog.spow[i];
        }
        s_dig[l] = dig;
        s_goff[l] = off;
    }
    const int g = int(threadIdx.x) % G;
    const int r0 = g * VPT;
    double scr[VPT], pcr[VPT], gsr[VPT];
#pragma unroll
    for (int j = 0; j < VPT; ++j) {
        scr[j] = a.sc[r0 + j];
        pcr[j] = a.pc ? a.pc[r0 + j] : 0.0;
        gsr[j] = a.gsc ? a.gsc[r0 + j] : 0.0;
    }
    double2 red[K][VPT];
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
        for (int j = 0; j < VPT; ++j) red[k][j] = make_double2(0.0, 0.0);
    const int nitems = nt * G;
    __shared__ uint32_t s_base;
    for (int64_t tile = blockIdx.x; tile < prog.ntiles; tile += gridDim.x) {
        __syncthreads();   // the previous tile's shared reads are done (first tile: tables staged)
        if (threadIdx.x == 0) {   // tile -> outer digits -> first state (q^n < 2^32)
            uint32_t b = 0, x = uint32_t(tile);
            for (int i = 0; i < prog.nouter; ++i) {
                const uint32_t y = x / uint32_t(q);
                b += (x - y * uint32_t(q)) * prog.opow[i];
                x = y;
            }
            s_base = b;
        }
        __syncthreads();
        const uint32_t base = s_base;
        for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
            const int l = it / G;
            const double2 *src = a.C + size_t(base + s_goff[l]) * R + r0;
#pragma unroll
            for (int j = 0; j < VPT; ++j) cp_async16(s_v + ((r0 + j) * nt + l), src + j);
        }
        cp_async_commit();
        // the first item's epilogue streams load while the tile lands
        double2 pn[VPT];
        double dn = 0.0;
        double2 dcn = make_double2(0.0, 0.0);
        auto prefetch = [&](int it) {
            if (it >= nitems) return;
            const size_t st = base + s_goff[it / G];
#pragma unroll
            for (int j = 0; j < VPT; ++j) {
                const size_t e = st * R + r0 + j;
                if (!prog.first) pn[j] = __ldcs(a.W + e);
                else if (a.P) pn[j] = __ldcs(a.P + e);
            }
            if (prog.first) {
                if (RD) dn = __ldcs(static_cast<const double *>(a.diag) + st);
                else dcn = __ldcs(static_cast<const double2 *>(a.diag) + st);
            }
        };
        prefetch(threadIdx.x);
        cp_async_wait<0>();
        __syncthreads();
        for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
            const int l = it / G;
            double2 v[VPT], acc[VPT];
#pragma unroll
            for (int j = 0; j < VPT; ++j) {
                v[j] = s_v[(r0 + j) * nt + l];
                acc[j] = make_double2(0.0, 0.0);
            }
            const uint32_t dig = s_dig[l];
            // branch-free: a zero coefficient (target digit out of range, or a
            // zero matrix element) adds zero; its partner index, which may leave
            // the tile, is clamped into it
#pragma unroll 2
            for (int t = 0; t < prog.nterms; ++t) {
                const QTileTerm T = prog.t[t];
                const int pair = int((dig >> (2 * T.ls1)) & 3u) + q * int((dig >> (2 * T.ls2)) & 3u);
                const double2 c = s_tab[T.tab + pair];
                const int pidx = r0 * nt + min(max(l + T.loff, 0), nt - 1);
#pragma unroll
                for (int j = 0; j < VPT; ++j) {
                    const double2 w = s_v[pidx + j * nt];
                    if (RC) {
                        acc[j].x = fma(c.x, w.x, acc[j].x);
                        acc[j].y = fma(c.x, w.y, acc[j].y);
                    } else {
                        acc[j] = cfma(c, w, acc[j]);
                    }
                }
            }
            if (prog.first) {   // the diagonal after the terms: its value arrived meanwhile
#pragma unroll
                for (int j = 0; j < VPT; ++j) {
                    if (RD) {
                        const double dd = dn - a.shift;
                        acc[j].x = fma(dd, v[j].x, acc[j].x);
                        acc[j].y = fma(dd, v[j].y, acc[j].y);
                    } else {
                        double2 dd = dcn;
                        dd.x -= a.shift;
                        acc[j] = cfma(dd, v[j], acc[j]);
                    }
                }
            }
            const size_t st = base + s_goff[l];
#pragma unroll
            for (int j = 0; j < VPT; ++j) {
                const size_t e = st * R + r0 + j;
                const double2 hv = cscale(scr[j], acc[j]);
                double2 out = hv;
                if (!prog.first) {
                    out.x += pn[j].x;
                    out.y += pn[j].y;
                } else if (a.P) {
                    out.x = fma(pcr[j], pn[j].x, out.x);
                    out.y = fma(pcr[j], pn[j].y, out.y);
                }
                __stcs(a.W + e, out);
                const double2 vv = cscale(scr[j], v[j]);
                red[0][j] = cadd(red[0][j], cconjmul(vv, hv));
                if (!prog.last) continue;
                if (K >= 2) red[1][j].x += out.x * out.x + out.y * out.y;
                if (K >= 4 && a.G) {
                    const double2 gv = cscale(gsr[j], a.G[e]);
                    red[2][j] = cadd(red[2][j], cconjmul(gv, out));
                    red[3][j] = cadd(red[3][j], cconjmul(gv, vv));
                }
            }
            prefetch(it + int(blockDim.x));
        }
    }
    // block sums (the pattern of block_reduce_store, in the dynamic buffer)
    for (int off = 16; off >= G; off >>= 1)
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int j = 0; j < VPT; ++j) {
                red[k][j].x += __shfl_xor_sync(0xffffffffu, red[k][j].x, off);
                red[k][j].y += __shfl_xor_sync(0xffffffffu, red[k][j].y, off);
            }
    __syncthreads();   // the tile buffer is free
    double2 *sm = s_v;   // [warps][K][R]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane < G)
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int j = 0; j < VPT; ++j) sm[(size_t(warp) * K + k) * R + lane * VPT + j] = red[k][j];
    __syncthreads();
    const int nw = blockDim.x >> 5;
    for (int idx = threadIdx.x; idx < K * R; idx += blockDim.x) {
        const int k = idx / R, r = idx - k * R;
        double2 sum = make_double2(0.0, 0.0);
        for (int w = 0; w < nw; ++w) sum = cadd(sum, sm[(size_t(w) * K + k) * R + r]);
        a.partials[((size_t)blockIdx.x * K + k) * R + r] = sum;
    }
}

// Tile set of the mixed-radix tiled kernel for R (null: the flat kernel runs).
const pned_model::QTileSet *find_qtiles(const pned_model *m, int R)
{
    std::lock_guard<std::mutex> lock(const_cast<pned_model *>(m)->rtiles_mu);
    auto it = m->qtiles.find(R);
    if (it == m->qtiles.end() || it->second.progs.empty()) return nullptr;
    return &it->second;
}

int qtile_grid(const pned_model *m, const pned_model::QTileSet &qs, int nblocks)
{
    const int per_sm = qs.smem + 1024 <= 113 * 1024 ? 2 : 1;
    return std::max(1, std::min(nblocks, per_sm * m->nsm));
}

template <int VPT, bool RC, bool RD, int K>
static cudaError_t launch_qtile_t(const pned_model *m, const pned_model::QTileSet &qs, const HvArgs &a, int nblocks,
                                  cudaStream_t st)
{
    auto kern = hv_qtile_kernel<VPT, RC, RD, K>;
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void *>(kern), m->device);
    if (e != cudaSuccess) return e;
    const int grid = qtile_grid(m, qs, nblocks);
    HvArgs b = a;
    for (size_t p = 0; p < qs.progs.size(); ++p) {
        b.partials = a.partials + size_t(p) * grid * K * a.R;
        kern<<<grid, kThreads, qs.smem, st>>>(*qs.progs[p], b);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <int VPT, int K>
static cudaError_t launch_qtile_v(const pned_model *m, const pned_model::QTileSet &qs, const HvArgs &a, int nblocks,
                                  cudaStream_t st)
{
    if (m->real_coef && m->real_diag) return launch_qtile_t<VPT, true, true, K>(m, qs, a, nblocks, st);
    if (m->real_diag) return launch_qtile_t<VPT, false, true, K>(m, qs, a, nblocks, st);
    return launch_qtile_t<VPT, false, false, K>(m, qs, a, nblocks, st);
}

template <int K>
static cudaError_t launch_qtile_k(const pned_model *m, const pned_model::QTileSet &qs, const HvArgs &a, int nblocks,
                                  cudaStream_t st)
{
    switch (qs.vpt) {   // 1, 2 or 3 (even R runs two vectors a thread)
    case 3: return launch_qtile_v<3, K>(m, qs, a, nblocks, st);
    case 2: return launch_qtile_v<2, K>(m, qs, a, nblocks, st);
    case 1: return launch_qtile_v<1, K>(m, qs, a, nblocks, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_qtile(const pned_model *m, const pned_model::QTileSet &qs, const HvArgs &a, int nblocks,
                         cudaStream_t st)
{
    if (a.K == 1) return launch_qtile_k<1>(m, qs, a, nblocks, st);
    if (a.K == 4) return launch_qtile_k<4>(m, qs, a, nblocks, st);
    return cudaErrorInvalidValue;
}

// Tiled mixed-radix passes for R vectors (q > 2, full basis, n >= 8): the
// largest tile of q^k states whose [nt][R] values, tables and index arrays
// fit 100 KB of shared memory (two blocks per SM), k <= n - 2.
bool ensure_qtiles(pned_model *m, int R)
{
    const HostProgram &hp = m->hp;
    if (hp.q <= 2 || hp.sector || hp.n < 8 || pick_vpt(R) == 0) return false;
    std::lock_guard<std::mutex> lock(m->rtiles_mu);
    if (m->qtiles.count(R)) return !m->qtiles[R].progs.empty();
    pned_model::QTileSet &qs = m->qtiles[R];
    // the C tile, the pass table, 32-bit offsets and digits
    auto smem_of = [&](int k) {
        int64_t nt = 1;
        for (int i = 0; i < k; ++i) nt *= hp.q;
        return size_t(nt) * (sizeof(double2) * R + 8) + sizeof(double2) * kQTileMaxTab + 64;
    };
    int64_t states = 1;
    for (int i = 0; i < hp.n; ++i) states *= hp.q;
    // digits are packed 2 bits each; state indices and tile offsets are 32-bit
    if (hp.q > 4 || states >= (int64_t(1) << 32)) return false;
    int k = 2;
    while (k + 1 <= std::min(hp.n - 2, kQTileMaxSites) && smem_of(k + 1) <= 110 * 1024) ++k;
    if (smem_of(k) > 110 * 1024) return false;
    std::vector<QTilePass> passes;
    // one vector: 16-byte states; keep site 0 in every tile for 3-state runs
    if (plan_qtiles(hp, k, R == 1 ? 1 : 0, passes) != PNED_OK) return false;
    int64_t pw[64];
    pw[0] = 1;
    for (int i = 1; i <= hp.n; ++i) pw[i] = pw[i - 1] * hp.q;
    for (size_t p = 0; p < passes.size(); ++p) {
        const QTilePass &ps = passes[p];
        if (ps.terms.size() > size_t(kMaxTerms) || ps.outer.size() > 32) { qs.progs.clear(); return false; }
        std::unique_ptr<QTileProgram> T(new QTileProgram());
        T->q = hp.q;
        T->k = int(ps.sites.size());
        T->nt = int(pw[T->k]);
        T->nouter = int(ps.outer.size());
        T->nterms = int(ps.terms.size());
        T->first = p == 0;
        T->last = p + 1 == passes.size();
        T->ntiles = pw[hp.n] / pw[T->k];
        for (int i = 0; i < T->k; ++i) T->spow[i] = uint32_t(pw[ps.sites[i]]);
        for (int i = 0; i < T->nouter; ++i) T->opow[i] = uint32_t(pw[ps.outer[i]]);
        // the pass's own coefficient tables, q^2 entries a term
        const int Q = hp.q * hp.q;
        if (ps.terms.size() * size_t(Q) > size_t(kQTileMaxTab)) { qs.progs.clear(); return false; }
        T->ntab = int(ps.terms.size()) * Q;
        for (size_t t = 0; t < ps.terms.size(); ++t) {
            T->t[t] = ps.terms[t];
            T->t[t].tab = uint16_t(t * Q);
            for (int e = 0; e < Q; ++e) {
                const cd z = hp.table[ps.terms[t].tab + e];
                T->tab[t * Q + e] = make_double2(z.real(), z.imag());
            }
        }
        qs.progs.push_back(std::move(T));
    }
    // two vectors a thread where R is even (the K = 4 sums of four would spill)
    qs.vpt = (R % 2 == 0 && R % 3 != 0) ? 2 : pick_vpt(R);
    qs.smem = smem_of(k);
    return true;
}


}   // namespace pned
