// Device side of libpned_gpu.so: model upload, contexts, H.v kernels,
// deterministic reductions and the C-ABI vector entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "device.cuh"

namespace pned {

// ---------------------------------------------------------------------------
// error helpers
// ---------------------------------------------------------------------------
int cuda_fail(cudaError_t e, const char *what)
{
    return fail(PNED_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// Diagonal d(s) = sum_b X_b[st_b(s), st_b(s)] over all bonds (set-up, once).
template <bool RD>
__global__ void diag_kernel(int64_t dim, int n, int q, int nbond, const int *__restrict__ s1,
                            const int *__restrict__ s2, const double2 *__restrict__ dtab, void *out,
                            const int64_t *__restrict__ list1)
{
    const int Q = q * q;
    for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < dim; l += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = list1 ? list1[l] : l;   // sector index -> state
        double2 acc = make_double2(0.0, 0.0);
        if (q == 2) {
            for (int b = 0; b < nbond; ++b) {
                const int st = int((s >> s1[b]) & 1) | (int((s >> s2[b]) & 1) << 1);
                acc = cadd(acc, dtab[b * Q + st]);
            }
        } else {
            uint64_t digits = pack_digits(s, n, q);
            for (int b = 0; b < nbond; ++b) {
                const int st = digit_at(digits, s1[b]) + q * digit_at(digits, s2[b]);
                acc = cadd(acc, dtab[b * Q + st]);
            }
        }
        if (RD) static_cast<double *>(out)[l] = acc.x;
        else static_cast<double2 *>(out)[l] = acc;
    }
}

// Gathered H.v on the S = 1/2 full basis:
//   W[s,r] = pc_r P[s,r] + sc_r * ( (d(s) - shift) C[s,r] + sum_t c_t(s) C[s ^ m_t, r] )
// with fused per-vector sums: alpha = <v|Hv>, ||W||^2, <G|W>, <G|v> (v = sc C).
template <int VPT, bool RC, bool RD, int K, bool SECTOR>
__global__ void __launch_bounds__(kThreads) hv_xor_kernel(const __grid_constant__ XorProgram prog, const HvArgs a)
{
    extern __shared__ double2 s_tab[];
    for (int i = threadIdx.x; i < prog.ntab; i += blockDim.x) s_tab[i] = a.table[i];
    __syncthreads();
    const int R = a.R, G = R / VPT;
    const int64_t nitems = a.dim * G;
    double2 red[K][VPT];
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
        for (int j = 0; j < VPT; ++j) red[k][j] = make_double2(0.0, 0.0);
    const int g = threadIdx.x % G;
    const int r0 = g * VPT;
    double scr[VPT], pcr[VPT], gsr[VPT];
#pragma unroll
    for (int j = 0; j < VPT; ++j) {
        scr[j] = a.sc[r0 + j];
        pcr[j] = a.pc ? a.pc[r0 + j] : 0.0;
        gsr[j] = a.gsc ? a.gsc[r0 + j] : 0.0;
    }
    for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < nitems;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = G == 1 ? it : it / G;
        const uint32_t su = SECTOR ? uint32_t(a.list1[s]) : uint32_t(s);
        double2 v[VPT], acc[VPT];
        const double2 *cs = a.C + s * R + r0;
#pragma unroll
        for (int j = 0; j < VPT; ++j) v[j] = cs[j];
        if (RD) {
            const double dd = static_cast<const double *>(a.diag)[s] - a.shift;
#pragma unroll
            for (int j = 0; j < VPT; ++j) acc[j] = cscale(dd, v[j]);
        } else {
            double2 dd = static_cast<const double2 *>(a.diag)[s];
            dd.x -= a.shift;
#pragma unroll
            for (int j = 0; j < VPT; ++j) acc[j] = cmul(dd, v[j]);
        }
        int t = 0;
        if (SECTOR && VPT == 1) {
            // sector, one vector a thread: four terms' table and partner reads in flight
            // together, the products added in term order as below
            for (; t + 4 <= prog.nterms; t += 4) {
                double2 c[4], w[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const XorTerm T = prog.t[t + u];
                    uint32_t idx = 0;
#pragma unroll
                    for (int k = 0; k < kMaxDeps; ++k)
                        if (k < T.nb) idx |= ((su >> ((T.pos4 >> (8 * k)) & 0xffu)) & 1u) << k;
                    c[u] = s_tab[T.tab + idx];
                    int64_t pi = lin_index(a, su ^ T.xmask);
                    if (c[u].x == 0.0 && c[u].y == 0.0) pi = s;
                    w[u] = __ldg(a.C + pi * R + r0);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (RC) {
                        acc[0].x = fma(c[u].x, w[u].x, acc[0].x);
                        acc[0].y = fma(c[u].x, w[u].y, acc[0].y);
                    } else {
                        acc[0] = cfma(c[u], w[u], acc[0]);
                    }
                }
            }
        }
        for (; t < prog.nterms; ++t) {
            const XorTerm T = prog.t[t];
            uint32_t idx = 0;
#pragma unroll
            for (int k = 0; k < kMaxDeps; ++k)
                if (k < T.nb) idx |= ((su >> ((T.pos4 >> (8 * k)) & 0xffu)) & 1u) << k;
            const double2 c = s_tab[T.tab + idx];
            // in the sector, zero elements (the reference's skip mask) lead out of it: their
            // partner index is meaningless, so they read the own row and add zero (branch-free;
            // the Lin tables cover every half-state, so the lookup itself stays in bounds)
            int64_t pi = SECTOR ? lin_index(a, su ^ T.xmask) : int64_t(su ^ T.xmask);
            if (SECTOR && c.x == 0.0 && c.y == 0.0) pi = s;
            const double2 *ps = a.C + pi * R + r0;
#pragma unroll
            for (int j = 0; j < VPT; ++j) {
                const double2 w = __ldg(ps + j);
                if (RC) {
                    acc[j].x = fma(c.x, w.x, acc[j].x);
                    acc[j].y = fma(c.x, w.y, acc[j].y);
                } else {
                    acc[j] = cfma(c, w, acc[j]);
                }
            }
        }
        hv_epilogue<K, VPT>(a, s, r0, v, acc, scr, pcr, gsr, red);
    }
    block_reduce_store<K, VPT>(red, G, VPT, R, a.partials);
}

// Tiled single-vector (R = 1) H.v on the S = 1/2 full basis, one pass of a
// multi-pass program (each pass owns a subset of the flip masks).  A block owns
// a tile of 256 * 2^JB states: thread t holds the states of row t (its 8 bits
// placed on the global bits rowpos[], which start with bits 0..2) and j bits
// jexp[j] (j < 2^JB), global index base | jexp[j].  The tile is staged in
// shared memory, so flip masks inside the tile gather from shared memory; the
// others gather through L1/L2 from the partner tile, 2^JB loads per thread in
// flight.  The term decode (coefficient index) is done once per term for the
// thread's 2^JB states.
// Resident blocks per SM the single-vector tile kernel is built for: fewer
// rows per thread, fewer registers, more warps to hide the gather latency.
__host__ __device__ constexpr int tile_blocks_per_sm(int jb) { return jb >= 3 ? 2 : (jb == 2 ? 3 : 4); }

template <int JB, bool RC, bool RD, int K, int BPS = tile_blocks_per_sm(JB)>
__global__ void __launch_bounds__(kThreads, BPS)
    hv_tile_kernel(const __grid_constant__ TileProgram prog, const HvArgs a)
{
    constexpr int SPT = 1 << JB;
    constexpr int CH = SPT < 8 ? SPT : 8;   // rows loaded together (16 rows: two chunks, no spills)
    constexpr int TILE = kThreads * SPT;
    // up to 8 rows a thread the epilogue's rows of P or W are staged too (16 rows:
    // two tiles would not leave room for two blocks per SM)
    constexpr bool PWS = SPT <= 8;
    extern __shared__ double2 smem[];
    double2 *s_v = smem;
    double2 *s_pw = smem + TILE;   // the thread's own rows of P (first pass) or W (later passes)
    double2 *s_tab = smem + (PWS ? 2 : 1) * TILE;
    for (int i = threadIdx.x; i < prog.ntab; i += blockDim.x) s_tab[i] = a.table[i];
    const uint32_t tid = threadIdx.x;
    const int64_t ntiles = int64_t(1) << prog.nouter;
    const double2 *pw_src = PWS ? (prog.first ? a.P : a.W) : nullptr;   // staged rows of the epilogue
    double2 red[K][1];
#pragma unroll
    for (int k = 0; k < K; ++k) red[k][0] = make_double2(0.0, 0.0);
    const double sc = a.sc[0], pc = a.pc ? a.pc[0] : 0.0, gs = a.gsc ? a.gsc[0] : 0.0;
    const double hs = a.hsc ? a.hsc[0] : sc;
    const double shift = a.shift + (a.shiftv ? a.shiftv[0] : 0.0);
    uint32_t rowbase = 0;   // the thread's row on its global bits
#pragma unroll
    for (int k = 0; k < 8; ++k) rowbase |= ((tid >> k) & 1u) << prog.rowpos[k];
    // dynamic order: the block's next tile comes from the pass's counter (taken by
    // thread 0 during the current tile, read after the tile's last barrier)
    __shared__ uint32_t s_next;
    __shared__ double2 s_red[kThreads / 32][K];
    uint32_t *const ctr = a.tile_counter ? a.tile_counter + prog.pass : nullptr;
    int64_t tile = blockIdx.x;
    if (ctr) {
        if (tid == 0) s_next = atomicAdd(ctr, 1u);
        __syncthreads();
        tile = s_next;
    }
    while (tile < ntiles) {
        uint32_t base = rowbase;
        for (int k = 0; k < prog.nouter; ++k) base |= uint32_t((tile >> k) & 1) << prog.outer[k];
        double2 acc[SPT];
#pragma unroll
        for (int j0 = 0; j0 < SPT; j0 += CH) {
            double2 v[CH];
#pragma unroll
            for (int jj = 0; jj < CH; ++jj) v[jj] = __ldg(a.C + (base | prog.jexp[j0 + jj]));
            if (j0 == 0) {
                __syncthreads();   // the previous tile's shared reads are done (first tile: table staged)
                if (ctr && tid == 0) s_next = atomicAdd(ctr, 1u);   // every thread has read s_next
                // the epilogue's rows of P or W are requested now and land in the thread's own
                // slots while the terms run (the thread read its slots of the previous tile
                // before this point)
                if (pw_src) {
#pragma unroll
                    for (int j = 0; j < SPT; ++j)
                        cp_async16(s_pw + tid + kThreads * j, pw_src + (base | prog.jexp[j]));
                    cp_async_commit();
                }
            }
#pragma unroll
            for (int jj = 0; jj < CH; ++jj) s_v[tid + kThreads * (j0 + jj)] = v[jj];
#pragma unroll
            for (int jj = 0; jj < CH; ++jj) {
                const int j = j0 + jj;
                const uint32_t sj = base | prog.jexp[j];
                if (!prog.first) {
                    acc[j] = make_double2(0.0, 0.0);
                } else if (RD) {
                    const double dd = __ldcs(static_cast<const double *>(a.diag) + sj) - shift;
                    acc[j] = cscale(dd, v[jj]);
                } else {
                    double2 dd = __ldcs(static_cast<const double2 *>(a.diag) + sj);
                    dd.x -= shift;
                    acc[j] = cmul(dd, v[jj]);
                }
            }
        }
        __syncthreads();
        // flip masks inside the tile: partners from shared memory
        for (int t = 0; t < prog.nin; ++t) {
            const TileTerm T = prog.t[t];
            uint32_t ib = 0;
#pragma unroll
            for (int d = 0; d < kMaxDeps; ++d)
                if (d < T.nb) ib |= ((base >> ((T.pos4 >> (8 * d)) & 0xffu)) & 1u) << d;
            const double2 *sv = s_v + (tid ^ (T.mask & 0xffu));
            const uint32_t mhi = T.mask >> 8;
            if (!T.hasj) {   // one coefficient for all rows of the thread
                const double2 c = s_tab[T.tab + ib];
#pragma unroll
                for (int j = 0; j < SPT; ++j) {
                    const double2 w = sv[kThreads * (j ^ mhi)];
                    if (RC) { acc[j].x = fma(c.x, w.x, acc[j].x); acc[j].y = fma(c.x, w.y, acc[j].y); }
                    else acc[j] = cfma(c, w, acc[j]);
                }
                continue;
            }
#pragma unroll
            for (int j = 0; j < SPT; ++j) {
                const double2 c = s_tab[T.tab + (ib | ((T.jtab >> (4 * j)) & 15u))];
                const double2 w = sv[kThreads * (j ^ mhi)];
                if (RC) { acc[j].x = fma(c.x, w.x, acc[j].x); acc[j].y = fma(c.x, w.y, acc[j].y); }
                else acc[j] = cfma(c, w, acc[j]);
            }
        }
        // flip masks leaving the tile: partners through L1/L2
        for (int t = prog.nin; t < prog.nterms; ++t) {
            const TileTerm T = prog.t[t];
            // (base | jexp) ^ mask == (base ^ mask) ^ jexp: base has no j bits
            const uint32_t pbx = base ^ T.mask;
            uint32_t ib = 0;
#pragma unroll
            for (int d = 0; d < kMaxDeps; ++d)
                if (d < T.nb) ib |= ((base >> ((T.pos4 >> (8 * d)) & 0xffu)) & 1u) << d;
#pragma unroll
            for (int j0 = 0; j0 < SPT; j0 += CH) {   // CH partner loads in flight
                double2 w0[CH];
#pragma unroll
                for (int jj = 0; jj < CH; ++jj) w0[jj] = __ldg(a.C + (pbx ^ prog.jexp[j0 + jj]));
                if (!T.hasj) {   // one coefficient for all rows of the thread
                    const double2 c = s_tab[T.tab + ib];
#pragma unroll
                    for (int jj = 0; jj < CH; ++jj) {
                        const int j = j0 + jj;
                        if (RC) { acc[j].x = fma(c.x, w0[jj].x, acc[j].x); acc[j].y = fma(c.x, w0[jj].y, acc[j].y); }
                        else acc[j] = cfma(c, w0[jj], acc[j]);
                    }
                    continue;
                }
#pragma unroll
                for (int jj = 0; jj < CH; ++jj) {
                    const int j = j0 + jj;
                    const double2 c = s_tab[T.tab + (ib | uint32_t((T.jtab >> (4 * j)) & 15u))];
                    if (RC) { acc[j].x = fma(c.x, w0[jj].x, acc[j].x); acc[j].y = fma(c.x, w0[jj].y, acc[j].y); }
                    else acc[j] = cfma(c, w0[jj], acc[j]);
                }
            }
        }
        if (pw_src) cp_async_wait<0>();
#pragma unroll
        for (int j = 0; j < SPT; ++j) {
            const int64_t e = base | prog.jexp[j];
            const double2 hv = cscale(hs, acc[j]);
            double2 out = hv;
            if (!prog.first) {
                const double2 w0 = PWS ? s_pw[tid + kThreads * j] : __ldcs(a.W + e);
                out.x += w0.x;
                out.y += w0.y;
            } else if (a.P) {
                const double2 p = PWS ? s_pw[tid + kThreads * j] : __ldcs(a.P + e);
                out.x = fma(pc, p.x, out.x);
                out.y = fma(pc, p.y, out.y);
            }
            __stcs(a.W + e, out);
            const double2 vv = cscale(sc, s_v[tid + kThreads * j]);
            red[0][0] = cadd(red[0][0], cconjmul(vv, hv));
            if (!prog.last) continue;
            if (K >= 2) red[1][0].x += out.x * out.x + out.y * out.y;
            if (K >= 4 && a.G) {
                const double2 gv = cscale(gs, a.G[e]);
                red[2][0] = cadd(red[2][0], cconjmul(gv, out));
                red[3][0] = cadd(red[3][0], cconjmul(gv, vv));
            }
        }
        if (!ctr) {
            tile += gridDim.x;
            continue;
        }
        // the tile's sums (fixed order: lanes, then warps), written at the tile's slot,
        // so that the total does not depend on which block took which tile
        tile_sums_store<K>(red, s_red, a.partials + size_t(tile) * K);
        tile = s_next;
    }
    // static order: the block's sums over its tiles (same reduction order)
    if (!ctr) tile_sums_store<K>(red, s_red, a.partials + size_t(blockIdx.x) * K);
}

// Tiled multi-vector H.V (R > 1 interleaved vectors, S = 1/2 full basis), one
// pass of a multi-pass program.  G = R / VPT threads share a state; a block
// owns a tile of NS * SPT states (NS = 256 / G state rows): thread t serves
// vectors g, g + G, ..., g + (VPT-1) G (g = t mod G) of row l = t / G, whose
// j-th state is base | jexp[j] with the bits of l on the global bits rowpos[]:
// the G threads of a row read its R values as VPT contiguous runs of G
// values, so every load instruction uses whole sectors.  The tile's rows of R
// values are staged in shared memory ([SPT][NS][R]): in-tile flips gather
// there, the others through L1/L2 from the partner tile.  SLOT: per-vector
// coefficient tables ([ntab][R]) and real diagonals ([dim][R]).
template <int VPT, int SPT, bool SLOT, bool RC, bool RD, int K>
__global__ void __launch_bounds__(kThreads, 2) hv_tile_rv_kernel(const __grid_constant__ TileProgram prog, const HvArgs a)
{
    extern __shared__ double2 smem[];
    const int R = a.R, G = R / VPT, NS = kThreads / G;
    const int tbits = prog.tbits;
    const uint32_t tmask = (1u << tbits) - 1u;
    const size_t TS = size_t(SPT) * NS * R;   // elements of a tile
    double2 *s_v = smem;
    double2 *s_pw = smem + TS;   // the thread's own elements of P (first pass) or W (later passes)
    double2 *s_tab = smem + 2 * TS;
    const int tabw = SLOT ? R : 1;
    for (int i = threadIdx.x; i < prog.ntab * tabw; i += blockDim.x) s_tab[i] = a.table[i];
    const int g = threadIdx.x % G, l = threadIdx.x / G;   // vectors g, g + G, ..., g + (VPT-1) G
    const int64_t ntiles = int64_t(1) << prog.nouter;
    const double2 *pw_src = prog.first ? a.P : a.W;   // staged rows of the epilogue (null: none)
    double2 red[K][VPT];
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
        for (int q = 0; q < VPT; ++q) red[k][q] = make_double2(0.0, 0.0);
    uint32_t rowbase = 0;   // the thread's row on its global bits
    for (int k = 0; k < tbits; ++k) rowbase |= ((uint32_t(l) >> k) & 1u) << prog.rowpos[k];
    // dynamic order: blocks take chunks of consecutive tiles (>= 2048 states) from the
    // pass's counter and write the chunk's sums at the chunk's slot; null counter: the
    // static order (tile = block + k * grid) with per-block sums
    __shared__ uint32_t s_next;
    uint32_t *const ctr = a.tile_counter ? a.tile_counter + prog.pass : nullptr;
    const int64_t ctiles = ctr ? int64_t(max(1, a.rv_chunk)) : 1;   // tiles per chunk
    const int64_t nchunks = (ntiles + ctiles - 1) / ctiles;
    int64_t chunk = blockIdx.x;
    if (ctr) {
        if (threadIdx.x == 0) s_next = atomicAdd(ctr, 1u);
        __syncthreads();
        chunk = s_next;
    }
    for (; ctr ? chunk < nchunks : chunk < ntiles;) {
      const int64_t tile_end = ctr ? min(ntiles, (chunk + 1) * ctiles) : chunk + 1;
      for (int64_t tile = ctr ? chunk * ctiles : chunk; tile < tile_end; ++tile) {
        uint32_t base = rowbase;
        for (int k = 0; k < prog.nouter; ++k) base |= uint32_t((tile >> k) & 1) << prog.outer[k];
        double2 acc[SPT][VPT];
        {
            double2 v[SPT][VPT];
#pragma unroll
            for (int j = 0; j < SPT; ++j)
#pragma unroll
                for (int q = 0; q < VPT; ++q) v[j][q] = __ldg(a.C + int64_t(base | prog.jexp[j]) * R + g + q * G);
            __syncthreads();   // the previous tile's shared reads are done (first tile: table staged)
            // the chunk's first tile: every thread has read s_next, so the next chunk is taken now
            if (ctr && threadIdx.x == 0 && tile == chunk * ctiles) s_next = atomicAdd(ctr, 1u);
            // the epilogue's elements of P or W land in the thread's own slots while the terms run
            if (pw_src) {
#pragma unroll
                for (int j = 0; j < SPT; ++j)
#pragma unroll
                    for (int q = 0; q < VPT; ++q)
                        cp_async16(s_pw + (j * NS + l) * R + g + q * G,
                                   pw_src + int64_t(base | prog.jexp[j]) * R + g + q * G);
                cp_async_commit();
            }
#pragma unroll
            for (int j = 0; j < SPT; ++j)
#pragma unroll
                for (int q = 0; q < VPT; ++q) s_v[(j * NS + l) * R + g + q * G] = v[j][q];
#pragma unroll
            for (int j = 0; j < SPT; ++j) {
                const int64_t sj = base | prog.jexp[j];
#pragma unroll
                for (int q = 0; q < VPT; ++q) {
                    const int r = g + q * G;
                    if (!prog.first) {
                        acc[j][q] = make_double2(0.0, 0.0);
                        continue;
                    }
                    const double sh = a.shift + (a.shiftv ? a.shiftv[r] : 0.0);
                    if (SLOT) {
                        acc[j][q] = cscale(__ldcs(static_cast<const double *>(a.diag) + sj * R + r) - sh, v[j][q]);
                    } else if (RD) {
                        acc[j][q] = cscale(__ldcs(static_cast<const double *>(a.diag) + sj) - sh, v[j][q]);
                    } else {
                        double2 dd = __ldcs(static_cast<const double2 *>(a.diag) + sj);
                        dd.x -= sh;
                        acc[j][q] = cmul(dd, v[j][q]);
                    }
                }
            }
        }
        __syncthreads();
        // flip masks inside the tile: partners from shared memory
        for (int t = 0; t < prog.nin; ++t) {
            const TileTerm T = prog.t[t];
            uint32_t ib = 0;
#pragma unroll
            for (int d = 0; d < kMaxDeps; ++d)
                if (d < T.nb) ib |= ((base >> ((T.pos4 >> (8 * d)) & 0xffu)) & 1u) << d;
            const int lp = l ^ int(T.mask & tmask);
            const uint32_t mhi = T.mask >> tbits;
#pragma unroll
            for (int j = 0; j < SPT; ++j) {
                const uint32_t idx = T.hasj ? (ib | ((T.jtab >> (4 * j)) & 15u)) : ib;
                const double2 *ct = s_tab + (T.tab + idx) * tabw + (SLOT ? g : 0);
                const double2 *sv = s_v + ((int(j ^ mhi)) * NS + lp) * R + g;
#pragma unroll
                for (int q = 0; q < VPT; ++q) {
                    const double2 c = ct[SLOT ? q * G : 0];
                    const double2 w = sv[q * G];
                    if (RC && !SLOT) { acc[j][q].x = fma(c.x, w.x, acc[j][q].x); acc[j][q].y = fma(c.x, w.y, acc[j][q].y); }
                    else acc[j][q] = cfma(c, w, acc[j][q]);
                }
            }
        }
        // flip masks leaving the tile: partners through L1/L2
        for (int t = prog.nin; t < prog.nterms; ++t) {
            const TileTerm T = prog.t[t];
            double2 w0[SPT][VPT];
#pragma unroll
            for (int j = 0; j < SPT; ++j)
#pragma unroll
                for (int q = 0; q < VPT; ++q)
                    w0[j][q] = __ldg(a.C + int64_t((base | prog.jexp[j]) ^ T.mask) * R + g + q * G);
            uint32_t ib = 0;
#pragma unroll
            for (int d = 0; d < kMaxDeps; ++d)
                if (d < T.nb) ib |= ((base >> ((T.pos4 >> (8 * d)) & 0xffu)) & 1u) << d;
#pragma unroll
            for (int j = 0; j < SPT; ++j) {
                const uint32_t idx = T.hasj ? (ib | ((T.jtab >> (4 * j)) & 15u)) : ib;
                const double2 *ct = s_tab + (T.tab + idx) * tabw + (SLOT ? g : 0);
#pragma unroll
                for (int q = 0; q < VPT; ++q) {
                    const double2 c = ct[SLOT ? q * G : 0];
                    if (RC && !SLOT) {
                        acc[j][q].x = fma(c.x, w0[j][q].x, acc[j][q].x);
                        acc[j][q].y = fma(c.x, w0[j][q].y, acc[j][q].y);
                    } else {
                        acc[j][q] = cfma(c, w0[j][q], acc[j][q]);
                    }
                }
            }
        }
        if (pw_src) cp_async_wait<0>();
#pragma unroll
        for (int j = 0; j < SPT; ++j) {
#pragma unroll
            for (int q = 0; q < VPT; ++q) {
                const int r = g + q * G;
                const int64_t e = int64_t(base | prog.jexp[j]) * R + r;
                const double sc = a.sc[r];
                const double2 hv = cscale(a.hsc ? a.hsc[r] : sc, acc[j][q]);
                double2 out = hv;
                if (!prog.first) {
                    const double2 w0 = s_pw[(j * NS + l) * R + r];
                    out.x += w0.x;
                    out.y += w0.y;
                } else if (a.P) {
                    const double pc = a.pc[r];
                    const double2 p = s_pw[(j * NS + l) * R + r];
                    out.x = fma(pc, p.x, out.x);
                    out.y = fma(pc, p.y, out.y);
                }
                __stcs(a.W + e, out);
                const double2 vv = cscale(sc, s_v[(j * NS + l) * R + r]);
                red[0][q] = cadd(red[0][q], cconjmul(vv, hv));
                if (!prog.last) continue;
                if (K >= 2) red[1][q].x += out.x * out.x + out.y * out.y;
                if (K >= 4 && a.G) {
                    const double2 gv = cscale(a.gsc[r], a.G[e]);
                    red[2][q] = cadd(red[2][q], cconjmul(gv, out));
                    red[3][q] = cadd(red[3][q], cconjmul(gv, vv));
                }
            }
        }
      }
        if (!ctr) {
            chunk += gridDim.x;
            continue;
        }
        // the chunk's sums at the chunk's slot (fixed order), so that the total does not
        // depend on which block took which chunk; s_next is visible after its barrier
        block_reduce_store<K, VPT, true>(red, G, VPT, R, a.partials, chunk);
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int q = 0; q < VPT; ++q) red[k][q] = make_double2(0.0, 0.0);
        chunk = s_next;
    }
    if (!ctr) block_reduce_store<K, VPT, true>(red, G, VPT, R, a.partials);
}

// Mixed-radix (q > 2) variant: partner = s + offset, coefficient indexed by
// the two bond digits; zero coefficients (target digit out of range) skip the load.
template <int VPT, bool RC, bool RD, int K, bool SECTOR, bool I32>
__global__ void __launch_bounds__(kThreads) hv_radix_kernel(const __grid_constant__ RadixProgram prog, const HvArgs a,
                                                            int q)
{
    extern __shared__ double2 s_tab[];
    for (int i = threadIdx.x; i < prog.ntab; i += blockDim.x) s_tab[i] = a.table[i];
    __syncthreads();
    const int R = a.R, G = R / VPT;
    const int64_t nitems = a.dim * G;
    double2 red[K][VPT];
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
        for (int j = 0; j < VPT; ++j) red[k][j] = make_double2(0.0, 0.0);
    const int g = threadIdx.x % G;
    const int r0 = g * VPT;
    double scr[VPT], pcr[VPT], gsr[VPT];
#pragma unroll
    for (int j = 0; j < VPT; ++j) {
        scr[j] = a.sc[r0 + j];
        pcr[j] = a.pc ? a.pc[r0 + j] : 0.0;
        gsr[j] = a.gsc ? a.gsc[r0 + j] : 0.0;
    }
    for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < nitems;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = G == 1 ? it : it / G;
        double2 v[VPT], acc[VPT];
        const double2 *cs = a.C + s * R + r0;
#pragma unroll
        for (int j = 0; j < VPT; ++j) v[j] = cs[j];
        if (RD) {
            const double dd = static_cast<const double *>(a.diag)[s] - a.shift;
#pragma unroll
            for (int j = 0; j < VPT; ++j) acc[j] = cscale(dd, v[j]);
        } else {
            double2 dd = static_cast<const double2 *>(a.diag)[s];
            dd.x -= a.shift;
#pragma unroll
            for (int j = 0; j < VPT; ++j) acc[j] = cmul(dd, v[j]);
        }
        const int64_t st = SECTOR ? a.list1[s] : s;
        const uint64_t digits = pack_digits(st, prog.n, q);
        // terms come bond by bond: the pair state of a bond is decoded once for its offsets
        for (int t = 0; t < prog.nterms; ++t) {
            const RadixTerm T = prog.t[t];
            const int pair = digit_at(digits, T.s1) + q * digit_at(digits, T.s2);
            const double2 c = s_tab[T.tab + pair];
            if (RC ? c.x == 0.0 : (c.x == 0.0 && c.y == 0.0)) continue;
            const double2 *ps;
            if (SECTOR) ps = a.C + lin_index(a, uint64_t(st + T.offset)) * R + r0;
            else if (I32) ps = a.C + (uint32_t(uint32_t(s) + uint32_t(T.offset)) * uint32_t(R) + uint32_t(r0));
            else ps = a.C + (s + T.offset) * R + r0;
#pragma unroll
            for (int j = 0; j < VPT; ++j) {
                const double2 w = __ldg(ps + j);
                if (RC) {
                    acc[j].x = fma(c.x, w.x, acc[j].x);
                    acc[j].y = fma(c.x, w.y, acc[j].y);
                } else {
                    acc[j] = cfma(c, w, acc[j]);
                }
            }
        }
        hv_epilogue<K, VPT>(a, s, r0, v, acc, scr, pcr, gsr, red);
    }
    block_reduce_store<K, VPT>(red, G, VPT, R, a.partials);
}

// Sums partials[nb][KR] in a fixed order into out[KR] (one block).
// Sums partials[b * stride][kr] over b < nb for each kr into out[kr] (one block,
// fixed order).
__global__ void finish_sum_kernel(const double2 *__restrict__ partials, int nb, int KR, double2 *out, int stride)
{
    __shared__ double2 sm[kThreads];
    for (int kr = 0; kr < KR; ++kr) {
        double2 s = make_double2(0.0, 0.0);
        for (int b = threadIdx.x; b < nb; b += blockDim.x) s = cadd(s, partials[(size_t)b * stride * KR + kr]);
        sm[threadIdx.x] = s;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) sm[threadIdx.x] = cadd(sm[threadIdx.x], sm[threadIdx.x + w]);
            __syncthreads();
        }
        if (threadIdx.x == 0) out[kr] = sm[0];
        __syncthreads();
    }
}

// Dot products: MODE 0: sum conj(x1) x2; MODE 1 (calc_beta): sum |x2 - alpha x1|^2.
template <int MODE>
__global__ void __launch_bounds__(kThreads) dot_kernel(const double2 *__restrict__ x1, const double2 *__restrict__ x2,
                                                       const double2 *__restrict__ alpha, int64_t dim, int R, int vpt,
                                                       double2 *partials)
{
    double2 red[1][kMaxVPT];
    for (int j = 0; j < kMaxVPT; ++j) red[0][j] = make_double2(0.0, 0.0);
    const int G = R / vpt, r0 = (threadIdx.x % G) * vpt;
    for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < dim * G;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int64_t base = (it / G) * R + r0;
#pragma unroll
        for (int j = 0; j < kMaxVPT; ++j) {
            if (j >= vpt) break;
            const double2 a1 = x1[base + j], a2 = x2[base + j];
            if (MODE == 0) {
                red[0][j] = cadd(red[0][j], cconjmul(a1, a2));
            } else {
                const double2 al = alpha[r0 + j];
                const double2 d = make_double2(a2.x - (al.x * a1.x - al.y * a1.y), a2.y - (al.x * a1.y + al.y * a1.x));
                red[0][j].x += d.x * d.x + d.y * d.y;
            }
        }
    }
    block_reduce_store<1, kMaxVPT>(red, G, vpt, R, partials);
}

// Lanczos residual: Rn = W - Re(alpha) v, beta^2 partial = sum |W - alpha v|^2 (v = sc C).
__global__ void __launch_bounds__(kThreads) residual_kernel(const double2 *__restrict__ W, const double2 *__restrict__ C,
                                                            double2 *Rn, const double *__restrict__ sc,
                                                            const double2 *__restrict__ alpha, int64_t dim, int R,
                                                            int vpt, double2 *partials)
{
    double2 red[1][kMaxVPT];
    for (int j = 0; j < kMaxVPT; ++j) red[0][j] = make_double2(0.0, 0.0);
    const int G = R / vpt, r0 = (threadIdx.x % G) * vpt;
    for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < dim * G;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int64_t base = (it / G) * R + r0;
#pragma unroll
        for (int j = 0; j < kMaxVPT; ++j) {
            if (j >= vpt) break;
            const double2 al = alpha[r0 + j];
            const double2 w = W[base + j];
            const double2 v = cscale(sc[r0 + j], C[base + j]);
            const double2 d = make_double2(w.x - (al.x * v.x - al.y * v.y), w.y - (al.x * v.y + al.y * v.x));
            red[0][j].x += d.x * d.x + d.y * d.y;
            Rn[base + j] = make_double2(w.x - al.x * v.x, w.y - al.x * v.y);
        }
    }
    block_reduce_store<1, kMaxVPT>(red, G, vpt, R, partials);
}


__global__ void __launch_bounds__(kThreads) gaussian_kernel(uint64_t key, int64_t dim, double2 *v, int R, int vpt,
                                                            double2 *partials)
{
    double2 red[1][kMaxVPT];
    for (int j = 0; j < kMaxVPT; ++j) red[0][j] = make_double2(0.0, 0.0);
    const int G = R / vpt, r0 = (threadIdx.x % G) * vpt;
    for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < dim * G;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int64_t base = (it / G) * R + r0;
#pragma unroll
        for (int j = 0; j < kMaxVPT; ++j) {
            if (j >= vpt) break;
            const int64_t g = base + j;
            const double2 z = gaussian_at(key, g);
            v[g] = z;
            red[0][j].x += z.x * z.x + z.y * z.y;
        }
    }
    if (partials) block_reduce_store<1, kMaxVPT>(red, G, vpt, R, partials);
}

__global__ void scale_kernel(double2 *v, int64_t n, int R, const double2 *sums, int mode)
{
    // mode 0: v *= 1/sqrt(sums[r].x)
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x) {
        const int r = int(g % R);
        const double f = 1.0 / sqrt(sums[r].x);
        v[g] = cscale(f, v[g]);
    }
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
// Vectors per thread for R interleaved vectors; the R/vpt threads of a state
// form a power-of-two group so that reductions can use xor shuffles.
int pick_vpt(int R)
{
    switch (R) {
    case 1: return 1;
    case 2: return 2;
    case 3: return 3;
    case 4: return 4;
    case 6: return 3;
    case 8: return 4;
    case 12: return 3;
    case 16: return 4;
    default: return 0;
    }
}

// Opts a kernel into more than 48 KB of dynamic shared memory, once per kernel
// and device (static + dynamic above 48 KB fails to launch without it).
cudaError_t allow_dynamic_smem(const void *kern, int device)
{
    static std::mutex mu;
    static std::vector<std::pair<const void *, int>> done;
    std::lock_guard<std::mutex> lock(mu);
    for (auto &d : done)
        if (d.first == kern && d.second == device) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess) done.push_back({kern, device});
    return e;
}

// Shared-memory carveout of a kernel: just what `blocks` resident blocks of
// `smem` dynamic bytes (+ static and reserved bytes) need, so that the rest
// of the SM's 256 KB stays L1, which catches partner rows re-read by the
// terms of one partner tile.
cudaError_t set_carveout(const void *kern, int device, size_t smem, int blocks)
{
    static std::mutex mu;
    static std::vector<std::pair<std::pair<const void *, int>, int>> last;
    const size_t need = size_t(blocks) * (smem + 9 * 1024);
    const int pct = int(std::min<size_t>(100, (need * 100 + 228 * 1024 - 1) / (228 * 1024)));
    std::lock_guard<std::mutex> lock(mu);
    for (auto &l : last)
        if (l.first.first == kern && l.first.second == device) {
            if (l.second == pct) return cudaSuccess;
            l.second = pct;
            return cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
        }
    last.push_back({{kern, device}, pct});
    return cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
}

// Persistent grid of the tiled kernels: all resident blocks, which sweep
// consecutive tiles, so partner tiles on the fast outer bits are found in L2.
int tile_grid(const pned_model *m, int nblocks)
{
    const int per_sm = m->tile_stage == 2 ? 1 : m->tile_bps;
    return std::max(1, std::min(nblocks, per_sm * m->nsm));
}

template <int JB, bool RC, bool RD, int K, int BPS = tile_blocks_per_sm(JB)>
static cudaError_t launch_tile_j(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    auto kern = hv_tile_kernel<JB, RC, RD, K, BPS>;
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void *>(kern), m->device);
    if (e == cudaSuccess && m->carveout)
        e = set_carveout(reinterpret_cast<const void *>(kern), m->device, m->tile_smem, BPS);
    if (e != cudaSuccess) return e;
    const int grid = tile_grid(m, nblocks);
    const bool dyn = tile_dynamic(m, a, nblocks);
    HvArgs b = a;
    if (!dyn) b.tile_counter = nullptr;
    else if ((e = cudaMemsetAsync(a.tile_counter, 0, sizeof(uint32_t) * kTileMaxPasses, st)) != cudaSuccess)
        return e;
    size_t off = 0;
    for (size_t p = 0; p < m->tprogs.size(); ++p) {
        b.partials = a.partials + off;
        off += dyn ? (size_t(1) << m->tprogs[p]->nouter) * K : size_t(grid) * K * a.R;
        kern<<<grid, kThreads, m->tile_smem, st>>>(*m->tprogs[p], b);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <bool RC, bool RD, int K>
static cudaError_t launch_tile_t(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    switch (m->tile_jb) {
    case 1: return launch_tile_j<1, RC, RD, K>(m, a, nblocks, st);
    case 2: return launch_tile_j<2, RC, RD, K>(m, a, nblocks, st);
    case 3:   // 8 rows per thread: two resident blocks (121 registers) or three (85, some spills)
        if (m->tile_bps == 3) return launch_tile_j<3, RC, RD, K, 3>(m, a, nblocks, st);
        return launch_tile_j<3, RC, RD, K>(m, a, nblocks, st);
    case 4: return launch_tile_j<4, RC, RD, K>(m, a, nblocks, st);
    default: return cudaErrorInvalidValue;
    }
}

template <int K>
static cudaError_t launch_tile(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    if (m->real_coef && m->real_diag) return launch_tile_t<true, true, K>(m, a, nblocks, st);
    if (m->real_diag) return launch_tile_t<false, true, K>(m, a, nblocks, st);
    return launch_tile_t<false, false, K>(m, a, nblocks, st);
}

template <int VPT, bool RC, bool RD, int K, bool SECTOR = false>
static cudaError_t launch_hv_t(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    const size_t smem = sizeof(double2) * std::max(1, m->ntab);
    if (m->q == 2) {
        auto kern = hv_xor_kernel<VPT, RC, RD, K, SECTOR>;
        cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void *>(kern), m->device);
        if (e != cudaSuccess) return e;
        kern<<<nblocks, kThreads, smem, st>>>(*m->xprog, a);
    } else if (!SECTOR && uint64_t(m->dim) * uint64_t(a.R) < (uint64_t(1) << 31)) {
        // element indices fit 32 bits (partners stay inside the basis: offsets
        // are only applied where the coefficient, i.e. the target digit, is valid)
        auto kern = hv_radix_kernel<VPT, RC, RD, K, SECTOR, true>;
        cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void *>(kern), m->device);
        if (e != cudaSuccess) return e;
        kern<<<nblocks, kThreads, smem, st>>>(*m->rprog, a, m->q);
    } else {
        auto kern = hv_radix_kernel<VPT, RC, RD, K, SECTOR, false>;
        cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void *>(kern), m->device);
        if (e != cudaSuccess) return e;
        kern<<<nblocks, kThreads, smem, st>>>(*m->rprog, a, m->q);
    }
    return cudaGetLastError();
}

// The call's arguments with the model's sector tables (list1, Lin tables).
static HvArgs sector_args(const pned_model *m, const HvArgs &a)
{
    HvArgs b = a;
    b.list1 = m->d_list1;
    b.lin_lo = m->d_lin_lo;
    b.lin_hi = m->d_lin_hi;
    b.lin_mod = m->lin_mod;
    b.lin_pow2 = 0;
    if ((m->lin_mod & (m->lin_mod - 1)) == 0) {
        int sh = 0;
        while ((int64_t(1) << sh) < m->lin_mod) ++sh;
        b.lin_pow2 = sh + 1;
    }
    return b;
}

template <int VPT, int K>
static cudaError_t launch_hv_v(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    if (m->hp.sector)   // Sz sector: complex coefficients, real diagonal
        return launch_hv_t<VPT, false, true, K, true>(m, sector_args(m, a), nblocks, st);
    if (m->real_coef && m->real_diag) return launch_hv_t<VPT, true, true, K>(m, a, nblocks, st);
    if (m->real_diag) return launch_hv_t<VPT, false, true, K>(m, a, nblocks, st);
    return launch_hv_t<VPT, false, false, K>(m, a, nblocks, st);
}

template <int K>
static cudaError_t launch_hv_k(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    switch (pick_vpt(a.R)) {
    case 4: return launch_hv_v<4, K>(m, a, nblocks, st);
    case 3: return launch_hv_v<3, K>(m, a, nblocks, st);
    case 2: return launch_hv_v<2, K>(m, a, nblocks, st);
    case 1: return launch_hv_v<1, K>(m, a, nblocks, st);
    default: return cudaErrorInvalidValue;
    }
}

static int rtile_grid(const pned_model *m, int nblocks) { return std::max(1, std::min(nblocks, 2 * m->nsm)); }

// Tiles per chunk of one multi-vector pass in the dynamic order: chunks of about
// 2048 states (one partial-sum record each), but at least four chunks per block
// of the grid, so that small bases still spread over the whole device.
int64_t rtile_chunk_tiles(const TileProgram &t, int grid)
{
    const int64_t states = int64_t(1) << (t.tbits + t.jb);   // (256 / G) rows x SPT
    const int64_t ntiles = int64_t(1) << t.nouter;
    return std::max<int64_t>(1, std::min<int64_t>(2048 / states, ntiles / (4 * int64_t(std::max(1, grid)))));
}

int64_t rtile_chunks(const TileProgram &t, int grid)
{
    const int64_t per = rtile_chunk_tiles(t, grid);
    return ((int64_t(1) << t.nouter) + per - 1) / per;
}

// Tile set of the multi-vector kernel for R (null: the flat kernel runs).
static const pned_model::TileSet *find_rtiles(const pned_model *m, int R)
{
    if (R < 2) return nullptr;
    std::lock_guard<std::mutex> lock(const_cast<pned_model *>(m)->rtiles_mu);
    auto it = m->rtiles.find(R);
    if (it == m->rtiles.end() || it->second.progs.empty()) return nullptr;
    return &it->second;
}

template <int VPT, int SPT, bool SLOT, bool RC, bool RD, int K>
static cudaError_t launch_rv_t(const pned_model *m, const pned_model::TileSet &ts, const HvArgs &a, int nblocks,
                               cudaStream_t st)
{
    auto kern = hv_tile_rv_kernel<VPT, SPT, SLOT, RC, RD, K>;
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void *>(kern), m->device);
    if (e == cudaSuccess && m->carveout)
        e = set_carveout(reinterpret_cast<const void *>(kern), m->device, rtile_smem(m, a.R, SLOT), 2);
    if (e != cudaSuccess) return e;
    const int grid = rtile_grid(m, nblocks);
    const size_t smem = rtile_smem(m, a.R, SLOT);
    const bool dyn = tile_dynamic(m, a, nblocks);
    HvArgs b = a;
    if (!dyn) b.tile_counter = nullptr;
    else if ((e = cudaMemsetAsync(a.tile_counter, 0, sizeof(uint32_t) * kTileMaxPasses, st)) != cudaSuccess)
        return e;
    size_t off = 0;
    for (size_t p = 0; p < ts.progs.size(); ++p) {
        b.partials = a.partials + off;
        b.rv_chunk = dyn ? int(rtile_chunk_tiles(*ts.progs[p], grid)) : 1;
        off += (dyn ? size_t(rtile_chunks(*ts.progs[p], grid)) : size_t(grid)) * K * a.R;
        kern<<<grid, kThreads, smem, st>>>(*ts.progs[p], b);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <int VPT, int SPT, int K>
static cudaError_t launch_rv_k(const pned_model *m, const pned_model::TileSet &ts, const HvArgs &a, int nblocks,
                               cudaStream_t st)
{
    if (a.slot_tables) return launch_rv_t<VPT, SPT, true, false, true, K>(m, ts, a, nblocks, st);
    if (m->real_coef && m->real_diag) return launch_rv_t<VPT, SPT, false, true, true, K>(m, ts, a, nblocks, st);
    if (m->real_diag) return launch_rv_t<VPT, SPT, false, false, true, K>(m, ts, a, nblocks, st);
    return launch_rv_t<VPT, SPT, false, false, false, K>(m, ts, a, nblocks, st);
}

template <int K>
static cudaError_t launch_rv(const pned_model *m, const pned_model::TileSet &ts, const HvArgs &a, int nblocks,
                             cudaStream_t st)
{
    if (ts.vpt == 2 && ts.spt == 4) return launch_rv_k<2, 4, K>(m, ts, a, nblocks, st);
    if (ts.vpt == 3 && ts.spt == 2) return launch_rv_k<3, 2, K>(m, ts, a, nblocks, st);
    return cudaErrorInvalidValue;
}

int64_t tile_dynamic_partials(const pned_model *m)
{
    int64_t n = 0;
    for (const auto &t : m->tprogs) n += int64_t(1) << t->nouter;
    return n;
}

int64_t rtile_dynamic_partials(const pned_model *m, int R, int nblocks)
{
    const pned_model::TileSet *ts = find_rtiles(m, R);
    if (!ts) return 0;
    const int grid = rtile_grid(m, nblocks);
    int64_t n = 0;
    for (const auto &t : ts->progs) n += rtile_chunks(*t, grid);
    return n;
}

bool tile_dynamic(const pned_model *m, const HvArgs &a, int nblocks)
{
    if (!a.tile_counter) return false;
    if (a.R == 1) {
        if (m->tprogs.empty() || !m->use_tile || tile_staged(m)) return false;
        return tile_dynamic_partials(m) * a.K <= a.partials_cap;
    }
    if (a.slot_tables || !find_rtiles(m, a.R)) return false;
    return rtile_dynamic_partials(m, a.R, nblocks) * a.K * a.R <= a.partials_cap;
}

int64_t hv_partials(const pned_model *m, const HvArgs &a, int nblocks)
{
    if (tile_dynamic(m, a, nblocks))
        return a.R == 1 ? tile_dynamic_partials(m) : rtile_dynamic_partials(m, a.R, nblocks);
    return hv_partial_blocks(m, a.R, nblocks);
}

int hv_partial_blocks(const pned_model *m, int R, int nblocks)
{
    if (!m->tprogs.empty() && R == 1 && m->use_tile) return int(m->tprogs.size()) * tile_grid(m, nblocks);
    if (const pned_model::TileSet *ts = find_rtiles(m, R)) return int(ts->progs.size()) * rtile_grid(m, nblocks);
    if (const pned_model::QTileSet *qs = find_qtiles(m, R)) return int(qs->progs.size()) * qtile_grid(m, *qs, nblocks);
    if (R == 1 && sector_segments_on(m)) return sector_grid(m, nblocks);
    return nblocks;
}

cudaError_t launch_hv(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    if (!m->tprogs.empty() && a.R == 1 && m->use_tile) {
        if (tile_staged(m)) return launch_tile_staged(m, a, nblocks, st);
        if (m->tile_stage == 3 && tile_tma_usable(m, a)) return launch_tile_tma(m, a, nblocks, st);
        if (a.K == 1) return launch_tile<1>(m, a, nblocks, st);
        if (a.K == 4) return launch_tile<4>(m, a, nblocks, st);
    }
    if (const pned_model::TileSet *ts = find_rtiles(m, a.R)) {
        if (a.K == 1) return launch_rv<1>(m, *ts, a, nblocks, st);
        if (a.K == 4) return launch_rv<4>(m, *ts, a, nblocks, st);
    }
    if (a.slot_tables) return cudaErrorInvalidValue;
    if (const pned_model::QTileSet *qs = find_qtiles(m, a.R)) return launch_qtile(m, *qs, a, nblocks, st);
    if (a.R == 1 && sector_segments_on(m)) return launch_sector(m, sector_args(m, a), nblocks, st);
    switch (a.K) {
    case 1: return launch_hv_k<1>(m, a, nblocks, st);
    case 4: return launch_hv_k<4>(m, a, nblocks, st);
    default: return cudaErrorInvalidValue;
    }
}

// First level of a long finish: block b sums rows [b * chunk, (b + 1) * chunk) of
// partials ([row][KR]) in a fixed order and writes the sum over row b * chunk, the
// first of its own rows, which no other block reads.
__global__ void finish_chunks_kernel(double2 *partials, int nb, int KR, int chunk)
{
    __shared__ double2 sm[kThreads];
    const int64_t lo = int64_t(blockIdx.x) * chunk, hi = min(int64_t(nb), lo + chunk);
    for (int kr = 0; kr < KR; ++kr) {
        double2 s = make_double2(0.0, 0.0);
        for (int64_t b = lo + threadIdx.x; b < hi; b += blockDim.x) s = cadd(s, partials[b * KR + kr]);
        sm[threadIdx.x] = s;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) sm[threadIdx.x] = cadd(sm[threadIdx.x], sm[threadIdx.x + w]);
            __syncthreads();
        }
        if (threadIdx.x == 0) partials[lo * KR + kr] = sm[0];
        __syncthreads();
    }
}

cudaError_t launch_finish(const double2 *partials, int nb, int KR, double2 *out, cudaStream_t st)
{
    // long lists (per-tile sums of the tile kernels) in two levels: one block alone
    // would read them at a single SM's bandwidth
    constexpr int kLevel1Blocks = 512;
    if (nb > 4 * kLevel1Blocks) {
        const int chunk = (nb + kLevel1Blocks - 1) / kLevel1Blocks;
        const int nb2 = (nb + chunk - 1) / chunk;
        finish_chunks_kernel<<<nb2, kThreads, 0, st>>>(const_cast<double2 *>(partials), nb, KR, chunk);
        finish_sum_kernel<<<1, kThreads, 0, st>>>(partials, nb2, KR, out, chunk);
        return cudaGetLastError();
    }
    finish_sum_kernel<<<1, kThreads, 0, st>>>(partials, nb, KR, out, 1);
    return cudaGetLastError();
}

cudaError_t launch_dot(const pned_ctx *c, const double2 *x1, const double2 *x2, const double2 *alpha, int mode,
                       double2 *out, cudaStream_t st)
{
    const int R = c->R;
    const int vpt = pick_vpt(R);
    if (mode == 0) dot_kernel<0><<<c->nblocks, kThreads, 0, st>>>(x1, x2, alpha, c->m->dim, R, vpt, c->partials);
    else dot_kernel<1><<<c->nblocks, kThreads, 0, st>>>(x1, x2, alpha, c->m->dim, R, vpt, c->partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_finish(c->partials, c->nblocks, R, out, st);
}

cudaError_t launch_residual(const pned_ctx *c, const double2 *W, const double2 *C, double2 *Rn, const double *sc,
                            const double2 *alpha, cudaStream_t st)
{
    residual_kernel<<<c->nblocks, kThreads, 0, st>>>(W, C, Rn, sc, alpha, c->m->dim, c->R, pick_vpt(c->R),
                                                     c->partials);
    return cudaGetLastError();
}

cudaError_t launch_gaussian(const pned_ctx *c, uint64_t seed, bool normalise, double2 *v, cudaStream_t st)
{
    uint64_t key = splitmix64_host(seed ^ 0x5DEECE66Dull);
    const int64_t n = c->m->dim * c->R;
    gaussian_kernel<<<c->nblocks, kThreads, 0, st>>>(key, c->m->dim, v, c->R, pick_vpt(c->R),
                                                     normalise ? c->partials : nullptr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !normalise) return e;
    e = launch_finish(c->partials, c->nblocks, c->R, c->sums, st);
    if (e != cudaSuccess) return e;
    scale_kernel<<<c->nblocks, kThreads, 0, st>>>(v, n, c->R, c->sums, 0);
    return cudaGetLastError();
}

}  // namespace pned

// ---------------------------------------------------------------------------
// C ABI: model and context
// ---------------------------------------------------------------------------
using namespace pned;

static thread_local int g_device = 0;

namespace pned {
int current_device() { return g_device; }
}  // namespace pned

extern "C" int pned_set_device(int device)
{
    int cnt = 0;
    cudaError_t e = cudaGetDeviceCount(&cnt);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
    if (device < 0 || device >= cnt) return fail(PNED_EINVAL, "pned_set_device: no such device");
    g_device = device;
    return PNED_OK;
}

namespace pned {

// Device programs of a tile plan (one per pass).
static std::vector<std::unique_ptr<TileProgram>> tile_programs(const HostProgram &h2,
                                                               const std::vector<HostProgram::TilePass> &passes,
                                                               int ntab)
{
    std::vector<std::unique_ptr<TileProgram>> out;
    for (size_t p = 0; p < passes.size(); ++p) {
        const HostProgram::TilePass &ps = passes[p];
        std::unique_ptr<TileProgram> T(new TileProgram());
        T->n = h2.n;
        T->tbits = ps.tbits;
        T->jb = ps.jb;
        T->nin = ps.nin;
        T->nterms = int(ps.tterms.size());
        T->ntab = ntab;
        T->nouter = int(ps.outer.size());
        T->first = p == 0;
        T->last = p + 1 == passes.size();
        T->pass = int(p);
        for (int j = 0; j < (1 << ps.jb); ++j) {
            uint32_t e = 0;
            for (int k = 0; k < ps.jb; ++k) if ((j >> k) & 1) e |= 1u << ps.jpos[k];
            T->jexp[j] = e;
        }
        for (int k = 0; k < T->nouter; ++k) T->outer[k] = uint8_t(ps.outer[k]);
        for (int k = 0; k < 8; ++k) T->rowpos[k] = uint8_t(k < ps.tbits ? ps.rowpos[k] : 0);
        T->ngroups = int(ps.gxor.size());
        for (int g = 0; g <= T->ngroups; ++g) T->gstart[g] = uint16_t(ps.gstart[g]);
        for (int g = 0; g < T->ngroups; ++g) T->gxor[g] = ps.gxor[g];
        std::copy(ps.tterms.begin(), ps.tterms.end(), T->t);
        out.push_back(std::move(T));
    }
    return out;
}

// Tiled single-vector programs (S = 1/2, n >= 12), one launch per pass.
void build_tile_programs(pned_model *m)
{
    m->use_tile = false;
    m->tprogs.clear();
    const HostProgram &hp = m->hp;
    std::vector<HostProgram::TilePass> passes;
    // Without a plan set (pned_model_set_plan with NULL, or never called): from 26
    // sites on, the plan the autotuner picks on B200 at 26-30 sites (tile bits that
    // hold the most flip terms, 7 window bits, two passes, own rows by tensor copies,
    // two out-of-tile terms in flight); below, and for the fields a set plan leaves
    // at -1, the fewest partner tiles with a 10-bit window through the gather kernel.
    const bool big = hp.n >= kTileBigSites && !m->plan1_set;
    const int fixed = m->plan1.row_fixed_bits >= 0 ? m->plan1.row_fixed_bits : (big ? 5 : 8);
    const int window = m->plan1.window_bits >= 0 ? m->plan1.window_bits : (big ? 7 : kTileWindowBits);
    const int mp = m->plan1.max_passes > 0 ? m->plan1.max_passes : (big ? 2 : kTileMaxPasses);
    const int jb = m->plan1.j_bits > 0 ? m->plan1.j_bits : 3;
    const int obj = big ? 1 : (m->plan1.objective > 0 ? m->plan1.objective : 0);
    const int stage = big ? 3 : m->plan1.stage_partner_tiles;
    const int tif = big ? 2 : m->plan1.terms_in_flight;
    if (hp.q == 2 && !hp.sector && hp.n >= 12 && plan_tiles(hp, 8, jb, fixed, window, mp, passes, obj) == PNED_OK) {
        m->tprogs = tile_programs(hp, passes, m->ntab);
        m->tile_jb = jb;
        m->tile_bps = (jb == 3 && m->plan1.blocks_per_sm == 3) ? 3 : tile_blocks_per_sm(jb);
        m->tma_deep = tif == 2;
        m->tile_stage = std::max(0, std::min(3, stage));
        if (m->tile_stage == 3) {
            // own rows, epilogue rows and diagonal by tensor copies: 8 rows a thread, every
            // pass's tile within 5 copy dimensions, two blocks' shared memory per SM
            m->tma_geom.assign(m->tprogs.size(), TmaGeom{});
            bool ok = jb == 3 && tile_tma_encoder() != nullptr;
            for (size_t p = 0; ok && p < m->tprogs.size(); ++p) ok = tile_tma_geometry(*m->tprogs[p], m->tma_geom[p]);
            const size_t smem = tile_tma_smem(m);
            int optin = 0;
            if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerMultiprocessor, m->device) != cudaSuccess)
                optin = 0;
            ok = ok && 2 * (smem + 1024) <= size_t(optin);
            if (!ok) m->tile_stage = 0;
        }
        // own tile, and for up to 8 rows a thread the staged epilogue rows, then the table
        m->tile_smem = sizeof(double2) * ((jb <= 3 ? 2 : 1) * size_t(kThreads) * (1 << jb) + std::max(1, m->ntab));
        m->use_tile = true;
        if (m->tile_stage == 2) {
            // bulk copies: 8 rows per thread, runs of >= 8 consecutive states,
            // and at least two 32 KB stages next to the table
            int optin = 0;
            if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, m->device) != cudaSuccess)
                optin = 0;
            const long room = long(optin) - 1024 - kBulkHead - long(sizeof(double2)) * std::max(1, m->ntab);
            m->bulk_stages = int(std::min<long>(kBulkMaxStages, std::max<long>(0, room) / (kBulkTile * long(sizeof(double2)))));
            bool runs = jb == kBulkJB;
            for (const auto &t : m->tprogs) {
                int f = 0;
                while (f < 8 && t->rowpos[f] == f) ++f;
                runs = runs && f >= kBulkMinRunBits;
            }
            if (!runs || m->bulk_stages < 2) m->tile_stage = 0;
        }
    }
}

// Tile shape of the multi-vector kernel: VPT vectors and SPT state rows per
// thread (VPT * SPT <= 8 accumulators), G = R / VPT threads per state.
static void rtile_shape(int R, int &vpt, int &spt)
{
    switch (R) {
    case 3: case 6: case 12: vpt = 3; spt = 2; break;
    default: vpt = 2; spt = 4; break;   // 2, 4, 8, 16
    }
}

size_t rtile_smem(const pned_model *m, int R, bool slot_tables)
{
    int vpt, spt;
    rtile_shape(R, vpt, spt);
    const int G = R / vpt;
    const size_t tile = size_t(kThreads / G) * spt * R;
    // the tile, the staged epilogue elements (same size), the coefficient tables
    return sizeof(double2) * (2 * tile + size_t(std::max(1, m->ntab)) * (slot_tables ? R : 1));
}

bool ensure_rtiles(pned_model *m, int R, bool slot_tables, const pned_tile_plan *plan)
{
    const HostProgram &hp = m->hp;
    if (hp.q != 2 || hp.sector || hp.n < 12 || R < 2 || pick_vpt(R) == 0) return false;
    if (rtile_smem(m, R, slot_tables) > 200 * 1024) return false;
    std::lock_guard<std::mutex> lock(m->rtiles_mu);
    if (m->rtiles.count(R) && !plan) return !m->rtiles[R].progs.empty();
    pned_model::TileSet &ts = m->rtiles[R];
    ts.progs.clear();
    rtile_shape(R, ts.vpt, ts.spt);
    const int G = R / ts.vpt;
    int tbits = 8;
    while ((1 << tbits) > kThreads / G) --tbits;
    int jb = 0;
    while ((1 << jb) < ts.spt) ++jb;
    // L2 window: about 2^21 vector elements of R
    int lr = 0;
    while ((1 << lr) < R) ++lr;
    int window = std::max(4, 21 - lr - tbits - jb);
    int fixed = tbits;
    int mp = kTileMaxPasses, obj = 0;
    if (plan) {
        if (plan->row_fixed_bits >= 0) fixed = std::min(tbits, plan->row_fixed_bits);
        if (plan->window_bits >= 0) window = plan->window_bits;
        if (plan->max_passes > 0) mp = std::min(kTileMaxPasses, plan->max_passes);
        if (plan->objective > 0) obj = plan->objective;
    }
    std::vector<HostProgram::TilePass> passes;
    if (plan_tiles(hp, tbits, jb, fixed, window, mp, passes, obj) != PNED_OK) return false;
    ts.progs = tile_programs(hp, passes, m->ntab);
    return true;
}


}  // namespace pned

extern "C" int pned_model_create(const pned_model_desc *desc, pned_model **out)
{
    if (!desc || !out) return fail(PNED_EINVAL, "pned_model_create: null argument");
    *out = nullptr;
    // a failure part-way frees what was allocated on the device; one before any
    // allocation (a refused model) makes no CUDA call
    struct Destroy {
        void operator()(pned_model *p) const
        {
            if (p->d_table || p->d_diag || p->d_list1 || p->d_lin_lo || p->d_lin_hi || p->d_seg_start ||
                p->d_seg_hi || p->d_rank_lo)
                pned_model_destroy(p);
            else
                delete p;
        }
    };
    std::unique_ptr<pned_model, Destroy> m(new pned_model());
    int rc = compile_program(desc, m->hp);
    if (rc) return rc;
    cudaError_t e = cudaSetDevice(g_device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    m->device = g_device;
    const HostProgram &hp = m->hp;
    m->n = hp.n; m->q = hp.q; m->dim = hp.dim; m->nbond = hp.nbond;
    m->real_coef = true;
    for (const cd &z : hp.table) if (z.imag() != 0) m->real_coef = false;
    m->real_diag = true;
    for (const cd &z : hp.dtab) if (z.imag() != 0) m->real_diag = false;
    m->ntab = int(hp.table.size());
    // program by value
    if (hp.q == 2) {
        m->xprog.reset(new XorProgram());
        m->xprog->nterms = int(hp.xterms.size());
        m->xprog->ntab = m->ntab;
        std::copy(hp.xterms.begin(), hp.xterms.end(), m->xprog->t);
        m->nterms = m->xprog->nterms;
    } else {
        m->rprog.reset(new RadixProgram());
        m->rprog->nterms = int(hp.rterms.size());
        m->rprog->ntab = m->ntab;
        m->rprog->n = hp.n;
        std::copy(hp.rterms.begin(), hp.rterms.end(), m->rprog->t);
        m->nterms = m->rprog->nterms;
    }
    // tiled single-vector program (S = 1/2, n >= 12), one launch per pass
    {
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, g_device);
        m->nsm = nsm;
    }
    if (hp.sector) {
        if (!m->real_diag)
            return fail(PNED_ENOTSUP, "pned_model_create: the sector basis needs a real diagonal");
        int64_t mod = 1;
        for (int i = 0; i < hp.ihf; ++i) mod *= hp.q;
        m->lin_mod = mod;
        e = cudaMalloc(&m->d_list1, sizeof(int64_t) * hp.list1.size());
        if (e == cudaSuccess) e = cudaMalloc(&m->d_lin_lo, sizeof(int64_t) * hp.lin_lo.size());
        if (e == cudaSuccess) e = cudaMalloc(&m->d_lin_hi, sizeof(int64_t) * hp.lin_hi.size());
        if (e == cudaSuccess)
            e = cudaMemcpy(m->d_list1, hp.list1.data(), sizeof(int64_t) * hp.list1.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(m->d_lin_lo, hp.lin_lo.data(), sizeof(int64_t) * hp.lin_lo.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(m->d_lin_hi, hp.lin_hi.data(), sizeof(int64_t) * hp.lin_hi.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e, "pned_model_create: sector tables");
        e = build_sector_segments(m.get());
        if (e != cudaSuccess) return cuda_fail(e, "pned_model_create: sector segments");
    } else {
        build_tile_programs(m.get());
    }
    // coefficient table
    std::vector<double2> tab(std::max<size_t>(1, hp.table.size()));
    for (size_t i = 0; i < hp.table.size(); ++i) tab[i] = make_double2(hp.table[i].real(), hp.table[i].imag());
    e = cudaMalloc(&m->d_table, sizeof(double2) * tab.size());
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(table)");
    e = cudaMemcpy(m->d_table, tab.data(), sizeof(double2) * tab.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(table)");
    // diagonal
    const size_t dbytes = (m->real_diag ? sizeof(double) : sizeof(double2)) * size_t(m->dim);
    e = cudaMalloc(&m->d_diag, dbytes);
    if (e != cudaSuccess) return fail(PNED_ENOMEM, "pned_model_create: cannot allocate the diagonal");
    int *ds1 = nullptr, *ds2 = nullptr;
    double2 *dt = nullptr;
    const int Q = hp.q * hp.q;
    std::vector<double2> dtab(hp.dtab.size());
    for (size_t i = 0; i < dtab.size(); ++i) dtab[i] = make_double2(hp.dtab[i].real(), hp.dtab[i].imag());
    e = cudaMalloc(&ds1, sizeof(int) * hp.nbond);
    if (e == cudaSuccess) e = cudaMalloc(&ds2, sizeof(int) * hp.nbond);
    if (e == cudaSuccess) e = cudaMalloc(&dt, sizeof(double2) * dtab.size());
    if (e == cudaSuccess) e = cudaMemcpy(ds1, hp.dsite1.data(), sizeof(int) * hp.nbond, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ds2, hp.dsite2.data(), sizeof(int) * hp.nbond, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dt, dtab.data(), sizeof(double2) * dtab.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
        if (m->real_diag)
            diag_kernel<true><<<nsm * 8, kThreads>>>(m->dim, hp.n, hp.q, hp.nbond, ds1, ds2, dt, m->d_diag, m->d_list1);
        else
            diag_kernel<false><<<nsm * 8, kThreads>>>(m->dim, hp.n, hp.q, hp.nbond, ds1, ds2, dt, m->d_diag, m->d_list1);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    cudaFree(ds1); cudaFree(ds2); cudaFree(dt);
    (void)Q;
    if (e != cudaSuccess) return cuda_fail(e, "pned_model_create: diagonal");
    *out = m.release();
    return PNED_OK;
}

extern "C" int pned_model_destroy(pned_model *m)
{
    if (!m) return PNED_OK;
    cudaSetDevice(m->device);
    cudaFree(m->d_table);
    cudaFree(m->d_diag);
    cudaFree(m->d_list1);
    cudaFree(m->d_lin_lo);
    cudaFree(m->d_lin_hi);
    cudaFree(m->d_seg_start);
    cudaFree(m->d_seg_hi);
    cudaFree(m->d_rank_lo);
    delete m;
    return PNED_OK;
}

extern "C" int pned_model_tile_staging(const pned_model *m, int *mode, int *ring_stages)
{
    if (!m) return fail(PNED_EINVAL, "pned_model_tile_staging: null model");
    const int md = m->use_tile ? m->tile_stage : 0;
    if (mode) *mode = md;
    if (ring_stages) *ring_stages = md == 2 ? m->bulk_stages : 0;
    return PNED_OK;
}

extern "C" int pned_model_sector_segments(pned_model *m, int enable, int *active)
{
    if (!m) return fail(PNED_EINVAL, "pned_model_sector_segments: null model");
    if (enable >= 0) m->seg_enabled = enable != 0;
    if (active) *active = sector_segments_on(m) ? 1 : 0;
    return PNED_OK;
}

extern "C" int pned_model_plan(const pned_model *m, int R, int *tile_passes, int *partner_tiles, int *tile_states)
{
    if (!m || R < 1) return fail(PNED_EINVAL, "pned_model_plan: bad arguments");
    int passes = 0, groups = 0, states = 0;
    if (R == 1 && m->use_tile) {
        passes = int(m->tprogs.size());
        for (const auto &t : m->tprogs) groups += t->ngroups;
        states = kThreads * (1 << m->tile_jb);
    } else if (m->q > 2) {
        std::lock_guard<std::mutex> lock(const_cast<pned_model *>(m)->rtiles_mu);
        auto it = m->qtiles.find(R);
        if (it != m->qtiles.end() && !it->second.progs.empty()) {
            passes = int(it->second.progs.size());
            states = it->second.progs[0]->nt;
        }
    } else if (R > 1) {
        std::lock_guard<std::mutex> lock(const_cast<pned_model *>(m)->rtiles_mu);
        auto it = m->rtiles.find(R);
        if (it != m->rtiles.end() && !it->second.progs.empty()) {
            passes = int(it->second.progs.size());
            for (const auto &t : it->second.progs) groups += t->ngroups;
            states = (1 << it->second.progs[0]->tbits) << it->second.progs[0]->jb;
        }
    }
    if (tile_passes) *tile_passes = passes;
    if (partner_tiles) *partner_tiles = groups;
    if (tile_states) *tile_states = states;
    return PNED_OK;
}

extern "C" int pned_model_set_plan(pned_model *m, int R, const pned_tile_plan *plan)
{
    if (!m || pick_vpt(R) == 0) return fail(PNED_EINVAL, "pned_model_set_plan: bad arguments");
    if (plan && (plan->max_passes > kTileMaxPasses || plan->window_bits > 30 || plan->row_fixed_bits > 8 ||
                 plan->j_bits > kTileMaxJB || plan->j_bits == 0 || plan->objective > 1 || plan->terms_in_flight > 2))
        return fail(PNED_EINVAL, "pned_model_set_plan: plan out of range");
    if (R == 1) {
        m->plan1 = plan ? *plan : pned_tile_plan{-1, -1, -1, -1, -1, -1, -1, -1, -1};
        m->plan1_set = plan != nullptr;
        m->carveout = m->plan1.l1_carveout != 0;
        build_tile_programs(m);
        return PNED_OK;
    }
    const pned_tile_plan def{-1, -1, -1, -1, -1, -1, -1, -1, -1};
    if (plan) m->carveout = plan->l1_carveout != 0;
    ensure_rtiles(m, R, false, plan ? plan : &def);
    return PNED_OK;
}

extern "C" int pned_model_info(const pned_model *m, int64_t *dim, int *n_terms, int *real_coef)
{
    if (!m) return fail(PNED_EINVAL, "pned_model_info: null model");
    if (dim) *dim = m->dim;
    if (n_terms) *n_terms = m->nterms;
    if (real_coef) *real_coef = (m->real_coef && m->real_diag) ? 1 : 0;
    return PNED_OK;
}

namespace pned {

int ctx_alloc_buffer(pned_ctx *c, int k)
{
    if (k < 0 || k >= kMaxBuffers) return fail(PNED_EINVAL, "context buffer index out of range");
    if (c->buf[k]) return PNED_OK;
    const size_t bytes = sizeof(double2) * size_t(c->m->dim) * c->R;
    if (c->budget && c->bytes + bytes > c->budget)
        return fail(PNED_EBUDGET, "context HBM budget exceeded by vector buffer " + std::to_string(k));
    cudaError_t e = cudaMalloc(&c->buf[k], bytes);
    if (e != cudaSuccess) {
        c->buf[k] = nullptr;
        cudaGetLastError();
        return fail(PNED_ENOMEM, "cudaMalloc of a vector buffer failed (" + std::to_string(bytes) + " bytes)");
    }
    c->bytes += bytes;
    return PNED_OK;
}

}  // namespace pned

extern "C" int pned_ctx_create(pned_model *m, int R, size_t budget, pned_ctx **out)
{
    if (!m || !out || pick_vpt(R) == 0)
        return fail(PNED_EINVAL, "pned_ctx_create: R must be one of 1, 2, 3, 4, 6, 8, 12, 16");
    *out = nullptr;
    cudaError_t e = cudaSetDevice(m->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    std::unique_ptr<pned_ctx> c(new pned_ctx());
    c->m = m;
    c->R = R;
    c->budget = budget;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
    c->nsm = nsm;
    // fixed grid: the reduction order (and so the result) does not depend on timing
    const int64_t items = m->dim * (R / pick_vpt(R));
    c->nblocks = int(std::min<int64_t>(int64_t(nsm) * 8, (items + kThreads - 1) / kThreads));
    c->nblocks = std::max(1, c->nblocks);
    e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    c->stream = c->own_stream;
    // tiled kernels write one partial sum per block and pass
    if (R > 1) ensure_rtiles(m, R, false, nullptr);
    ensure_qtiles(m, R);
    // room for per-block sums, and for R = 1 for the per-tile sums of the dynamic tile
    // order: the current plan, or any plan of two passes with tiles of >= 2048 states
    size_t pslots = size_t(c->nblocks) * std::max(kTileMaxPasses, kQTileMaxPasses) * kMaxK * kMaxR;
    if (R == 1 && m->use_tile) {
        pslots = std::max<size_t>(pslots, size_t(tile_dynamic_partials(m)) * kMaxK);
        pslots = std::max<size_t>(pslots, size_t(m->dim / 2048) * 2 * kMaxK);
    }
    if (R > 1) {   // per-chunk sums of the multi-vector kernel: the current plan, or two passes
        pslots = std::max<size_t>(pslots, size_t(rtile_dynamic_partials(m, R, c->nblocks)) * kMaxK * R);
        pslots = std::max<size_t>(pslots, size_t(m->dim / 2048 + 1) * 2 * kMaxK * R);
    }
    const size_t pbytes = sizeof(double2) * pslots;
    c->partials_cap = int64_t(pslots);
    e = cudaMalloc(&c->partials, pbytes);
    if (e == cudaSuccess) e = cudaMalloc(&c->tile_ctr, sizeof(uint32_t) * kTileMaxPasses);
    if (e == cudaSuccess) e = cudaMalloc(&c->sums, sizeof(double2) * kMaxK * kMaxR * 4);
    if (e == cudaSuccess) e = cudaMalloc(&c->scal, sizeof(double) * kScalSlots * kMaxR);
    if (e == cudaSuccess) e = cudaMallocHost(&c->h_sums, sizeof(double2) * kMaxK * kMaxR * 4);
    if (e == cudaSuccess) e = cudaMalloc(&c->flag, sizeof(int) * 4);
    if (e == cudaSuccess) e = cudaMemset(c->flag, 0, sizeof(int) * 4);
    if (e != cudaSuccess) {
        pned_ctx_destroy(c.release());
        return cuda_fail(e, "pned_ctx_create: scratch");
    }
    c->bytes = pbytes;
    if (c->budget && c->bytes > c->budget) {
        pned_ctx_destroy(c.release());
        return fail(PNED_EBUDGET, "pned_ctx_create: budget below the context's scratch size");
    }
    *out = c.release();
    return PNED_OK;
}

extern "C" int pned_ctx_destroy(pned_ctx *c)
{
    if (!c) return PNED_OK;
    cudaSetDevice(c->m->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    session_release(c);
    for (int k = 0; k < kMaxBuffers; ++k) cudaFree(c->buf[k]);
    cudaFree(c->partials);
    cudaFree(c->tile_ctr);
    cudaFree(c->sums);
    cudaFree(c->scal);
    cudaFree(c->flag);
    cudaFreeHost(c->h_sums);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return PNED_OK;
}

extern "C" int pned_ctx_set_stream(pned_ctx *c, void *stream)
{
    if (!c) return fail(PNED_EINVAL, "pned_ctx_set_stream: null context");
    c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
    return PNED_OK;
}

extern "C" int pned_ctx_synchronize(pned_ctx *c)
{
    if (!c) return fail(PNED_EINVAL, "pned_ctx_synchronize: null context");
    cudaError_t e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? PNED_OK : cuda_fail(e, "cudaStreamSynchronize");
}

extern "C" int pned_ctx_buffer(pned_ctx *c, int k, pned_c128 **p)
{
    if (!c || !p) return fail(PNED_EINVAL, "pned_ctx_buffer: null argument");
    int rc = ctx_alloc_buffer(c, k);
    if (rc) return rc;
    *p = reinterpret_cast<pned_c128 *>(c->buf[k]);
    return PNED_OK;
}

extern "C" int pned_ctx_bytes(const pned_ctx *c, size_t *bytes)
{
    if (!c || !bytes) return fail(PNED_EINVAL, "pned_ctx_bytes: null argument");
    *bytes = c->bytes + 0;
    return PNED_OK;
}

// ---------------------------------------------------------------------------
// C ABI: vector kernels
// ---------------------------------------------------------------------------
namespace pned {

// Copies [dim][R] host data into buffer k (or returns the device pointer).
int stage_in(pned_ctx *c, const pned_c128 *src, int flags, int k, const double2 **dev)
{
    if (!src) return fail(PNED_EINVAL, "null vector argument");
    if (flags & PNED_PTR_DEVICE) { *dev = reinterpret_cast<const double2 *>(src); return PNED_OK; }
    int rc = ctx_alloc_buffer(c, k);
    if (rc) return rc;
    cudaError_t e = cudaMemcpyAsync(c->buf[k], src, sizeof(double2) * size_t(c->m->dim) * c->R,
                                    cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync H2D");
    *dev = c->buf[k];
    return PNED_OK;
}

int sums_to_host(pned_ctx *c, int KR)
{
    cudaError_t e = cudaMemcpyAsync(c->h_sums, c->sums, sizeof(double2) * KR, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "reading reduction results");
    return check_kernel_flag(c);
}

// PNED_ETIMEOUT (and the flag cleared) if a kernel's bounded wait gave up.
int check_kernel_flag(pned_ctx *c)
{
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, c->flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "reading the kernel error flag");
    if (h) {
        cudaMemsetAsync(c->flag, 0, sizeof(int), c->stream);
        cudaStreamSynchronize(c->stream);
        return fail(PNED_ETIMEOUT, "a kernel's bounded wait for a TMA copy gave up");
    }
    return PNED_OK;
}

// scal slot pointer
double *slot(pned_ctx *c, int s) { return c->scal + s * kMaxR; }

int set_slot(pned_ctx *c, int s, double value)
{
    std::vector<double> h(kMaxR, value);
    cudaError_t e = cudaMemcpyAsync(slot(c, s), h.data(), sizeof(double) * kMaxR, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? PNED_OK : cuda_fail(e, "setting device scalars");
}

}  // namespace pned

extern "C" int pned_hv(pned_ctx *c, const pned_c128 *v1, pned_c128 *v0, double eperbd, pned_c128 *prdct, int flags)
{
    if (!c || !v1 || !v0) return fail(PNED_EINVAL, "pned_hv: null argument");
    cudaSetDevice(c->m->device);
    const double2 *dv1;
    int rc = stage_in(c, v1, flags, 0, &dv1);
    if (rc) return rc;
    const double2 *dv0c;
    rc = stage_in(c, v0, flags, 1, &dv0c);
    if (rc) return rc;
    double2 *dv0 = const_cast<double2 *>(dv0c);
    rc = set_slot(c, kSlotOne, 1.0);
    if (rc) return rc;
    HvArgs a{};
    a.C = dv1; a.P = dv0; a.W = dv0;
    a.sc = slot(c, kSlotOne); a.pc = slot(c, kSlotOne);
    a.diag = c->m->d_diag; a.shift = eperbd * c->m->nbond;
    a.table = c->m->d_table; a.partials = c->partials;
    a.dim = c->m->dim; a.R = c->R; a.K = 1;
    a.err = c->flag;
    ctx_tile_args(c, a);
    cudaError_t e = launch_hv(c->m, a, c->nblocks, c->stream);
    if (e == cudaSuccess)
        e = launch_finish(c->partials, int(hv_partials(c->m, a, c->nblocks)), c->R, c->sums, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_hv launch");
    if (!(flags & PNED_PTR_DEVICE)) {
        e = cudaMemcpyAsync(v0, dv0, sizeof(double2) * size_t(c->m->dim) * c->R, cudaMemcpyDeviceToHost, c->stream);
        if (e != cudaSuccess) return cuda_fail(e, "pned_hv D2H");
    }
    rc = sums_to_host(c, c->R);
    if (rc) return rc;
    if (prdct)
        for (int r = 0; r < c->R; ++r) prdct[r] = pned_c128{c->h_sums[r].x, c->h_sums[r].y};
    return PNED_OK;
}

extern "C" int pned_inprdct(pned_ctx *c, const pned_c128 *x1, const pned_c128 *x2, pned_c128 *out, int flags)
{
    if (!c || !out) return fail(PNED_EINVAL, "pned_inprdct: null argument");
    cudaSetDevice(c->m->device);
    const double2 *a, *b;
    int rc = stage_in(c, x1, flags, 0, &a);
    if (!rc) rc = stage_in(c, x2, flags, 1, &b);
    if (rc) return rc;
    cudaError_t e = launch_dot(c, a, b, nullptr, 0, c->sums, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_inprdct");
    rc = sums_to_host(c, c->R);
    if (rc) return rc;
    for (int r = 0; r < c->R; ++r) out[r] = pned_c128{c->h_sums[r].x, c->h_sums[r].y};
    return PNED_OK;
}

extern "C" int pned_calc_beta(pned_ctx *c, const pned_c128 *alpha, const pned_c128 *v1, const pned_c128 *v0,
                              double *out, int flags)
{
    if (!c || !alpha || !out) return fail(PNED_EINVAL, "pned_calc_beta: null argument");
    cudaSetDevice(c->m->device);
    const double2 *a, *b;
    int rc = stage_in(c, v1, flags, 0, &a);
    if (!rc) rc = stage_in(c, v0, flags, 1, &b);
    if (rc) return rc;
    double2 *dal = c->sums + kMaxK * kMaxR;   // alpha staged after the result slots
    cudaError_t e = cudaMemcpyAsync(dal, alpha, sizeof(double2) * c->R, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = launch_dot(c, a, b, dal, 1, c->sums, c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "pned_calc_beta");
    rc = sums_to_host(c, c->R);
    if (rc) return rc;
    for (int r = 0; r < c->R; ++r) out[r] = c->h_sums[r].x;
    return PNED_OK;
}

extern "C" int pned_fill_gaussian(pned_ctx *c, uint64_t seed, int normalise, pned_c128 *v_dev)
{
    if (!c || !v_dev) return fail(PNED_EINVAL, "pned_fill_gaussian: null argument");
    cudaSetDevice(c->m->device);
    cudaError_t e = launch_gaussian(c, seed, normalise != 0, reinterpret_cast<double2 *>(v_dev), c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? PNED_OK : cuda_fail(e, "pned_fill_gaussian");
}

// ---------------------------------------------------------------------------
// Allocation-free H.v: reduction scratch in a fixed device array
// ---------------------------------------------------------------------------
namespace pned {

// 4096 complex values (64 KB): [0, 16) holds 32 doubles set to 1 (scales),
// [16, 32) the R totals, [32] a kernel error flag, [33, 33 + blocks*R) the
// per-block partial sums.
constexpr int kNoAllocScratch = 4096;
constexpr int kNoAllocHead = 33;
static __device__ __align__(256) double2 g_noalloc_scratch[kNoAllocScratch];

static std::mutex g_noalloc_mu;
static double2 *g_noalloc_addr[64] = {};

// Device address of g_noalloc_scratch on `device` (which must be current),
// resolved once per device.
static int noalloc_address(int device, double2 **out)
{
    if (device < 0 || device >= 64) return fail(PNED_EINVAL, "pned_hv_noalloc: device index above 63");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "pned_hv_noalloc: cudaGetSymbolAddress");
        g_noalloc_addr[device] = static_cast<double2 *>(p);
    }
    *out = g_noalloc_addr[device];
    return PNED_OK;
}

__global__ void noalloc_fill_ones(double *p, int n, int *err)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = 1.0;
    if (threadIdx.x == 0) *err = 0;
}

}  // namespace pned

extern "C" int pned_hv_noalloc(const pned_model *m, int R, const pned_c128 *v1, pned_c128 *v0, double eperbd,
                               pned_c128 *prdct, void *stream)
{
    if (!m || !v1 || !v0) return fail(PNED_EINVAL, "pned_hv_noalloc: null argument");
    if (pick_vpt(R) == 0)
        return fail(PNED_EINVAL, "pned_hv_noalloc: R = " + std::to_string(R) +
                                     " is not one of 1, 2, 3, 4, 6, 8, 12, 16 (the 4096-value scratch limit)");
    cudaError_t e = cudaSetDevice(m->device);
    if (e != cudaSuccess) return cuda_fail(e, "pned_hv_noalloc: cudaSetDevice");
    double2 *scr = nullptr;
    int rc = noalloc_address(m->device, &scr);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
    const int64_t items = m->dim * (R / pick_vpt(R));
    int64_t nb = std::min<int64_t>(int64_t(nsm) * 8, (items + kThreads - 1) / kThreads);
    nb = std::min<int64_t>(nb, (kNoAllocScratch - kNoAllocHead) / R);
    nb = std::max<int64_t>(1, nb);
    while (nb > 1 && int64_t(hv_partial_blocks(m, R, int(nb))) * R > kNoAllocScratch - kNoAllocHead) --nb;
    if (int64_t(hv_partial_blocks(m, R, int(nb))) * R > kNoAllocScratch - kNoAllocHead)
        return fail(PNED_EINVAL, "pned_hv_noalloc: this model's H.v writes " +
                                     std::to_string(hv_partial_blocks(m, R, int(nb))) + " x " + std::to_string(R) +
                                     " partial sums even with one block, more than the " +
                                     std::to_string(kNoAllocScratch - kNoAllocHead) + "-value scratch holds");
    double *ones = reinterpret_cast<double *>(scr);
    double2 *sums = scr + 16;
    double2 *partials = scr + kNoAllocHead;
    int *err = reinterpret_cast<int *>(scr + 32);
    noalloc_fill_ones<<<1, 32, 0, st>>>(ones, 2 * 16, err);
    e = cudaGetLastError();
    HvArgs a{};
    a.C = reinterpret_cast<const double2 *>(v1);
    a.P = reinterpret_cast<double2 *>(v0);
    a.W = reinterpret_cast<double2 *>(v0);
    a.sc = ones;
    a.pc = ones;
    a.diag = m->d_diag;
    a.shift = eperbd * m->nbond;
    a.table = m->d_table;
    a.partials = partials;
    a.dim = m->dim;
    a.R = R;
    a.K = 1;
    a.err = err;
    if (e == cudaSuccess) e = launch_hv(m, a, int(nb), st);
    if (e == cudaSuccess) e = launch_finish(partials, hv_partial_blocks(m, R, int(nb)), R, sums, st);
    if (e == cudaSuccess && prdct) e = cudaMemcpyAsync(prdct, sums, sizeof(double2) * R, cudaMemcpyDeviceToHost, st);
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "pned_hv_noalloc");
    if (herr) return fail(PNED_ETIMEOUT, "pned_hv_noalloc: a bounded wait for a TMA copy gave up");
    return PNED_OK;
}
