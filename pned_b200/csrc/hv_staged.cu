// Staged variants of the single-vector S = 1/2 tile kernel, chosen by the
// plan: partner tiles copied into shared memory with cp.async (stage 1) or
// with cp.async.bulk under mbarriers by a producer warp (stage 2); or the
// gather kernel with the tile's own rows, its epilogue rows and its diagonal
// brought in by tensor copies (stage 3).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <utility>
#include <vector>

#include "device.cuh"

namespace pned {

// Single-vector tiled H.v with staged partner tiles: the same tiles and
// passes as hv_tile_kernel, but each partner tile (the terms of one group) is
// copied into shared memory once with cp.async, two buffers deep (group g + 1
// loads while group g is computed), and all terms of the group gather from
// there.  L2 sends each partner tile once instead of once per term, and the
// copies in flight hold no registers.
template <bool RC, bool RD, int K>
__global__ void __launch_bounds__(kThreads, 2)
    hv_tile_stage_kernel(const __grid_constant__ TileProgram prog, const HvArgs a)
{
    constexpr int SPT = 8;
    constexpr int TILE = kThreads * SPT;
    extern __shared__ double2 smem[];
    double2 *s_v = smem;              // own tile
    double2 *s_p = smem + TILE;       // two partner-tile buffers
    double2 *s_tab = smem + 3 * TILE;
    for (int i = threadIdx.x; i < prog.ntab; i += blockDim.x) s_tab[i] = a.table[i];
    const uint32_t tid = threadIdx.x;
    const int64_t ntiles = int64_t(1) << prog.nouter;
    double2 red[K][1];
#pragma unroll
    for (int k = 0; k < K; ++k) red[k][0] = make_double2(0.0, 0.0);
    const double sc = a.sc[0], pc = a.pc ? a.pc[0] : 0.0, gs = a.gsc ? a.gsc[0] : 0.0;
    const double hs = a.hsc ? a.hsc[0] : sc;
    const double shift = a.shift + (a.shiftv ? a.shiftv[0] : 0.0);
    uint32_t rowbase = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) rowbase |= ((tid >> k) & 1u) << prog.rowpos[k];
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        uint32_t base = rowbase;
        for (int k = 0; k < prog.nouter; ++k) base |= uint32_t((tile >> k) & 1) << prog.outer[k];
        double2 acc[SPT];
        {
            double2 v[SPT];
#pragma unroll
            for (int j = 0; j < SPT; ++j) v[j] = __ldg(a.C + (base | prog.jexp[j]));
            __syncthreads();   // the previous tile's shared reads are done (first tile: table staged)
#pragma unroll
            for (int j = 0; j < SPT; ++j) s_v[tid + kThreads * j] = v[j];
#pragma unroll
            for (int j = 0; j < SPT; ++j) {
                const uint32_t sj = base | prog.jexp[j];
                if (!prog.first) {
                    acc[j] = make_double2(0.0, 0.0);
                } else if (RD) {
                    acc[j] = cscale(__ldcs(static_cast<const double *>(a.diag) + sj) - shift, v[j]);
                } else {
                    double2 dd = __ldcs(static_cast<const double2 *>(a.diag) + sj);
                    dd.x -= shift;
                    acc[j] = cmul(dd, v[j]);
                }
            }
        }
        // the first partner tile loads while the in-tile terms run
        if (prog.ngroups > 0) {
            const uint32_t pb = base ^ prog.gxor[0];
#pragma unroll
            for (int j = 0; j < SPT; ++j) cp_async16(s_p + tid + kThreads * j, a.C + (pb | prog.jexp[j]));
            cp_async_commit();
        }
        __syncthreads();
        for (int t = 0; t < prog.nin; ++t) {
            const TileTerm T = prog.t[t];
            uint32_t ib = 0;
#pragma unroll
            for (int d = 0; d < kMaxDeps; ++d)
                if (d < T.nb) ib |= ((base >> ((T.pos4 >> (8 * d)) & 0xffu)) & 1u) << d;
            const double2 *sv = s_v + (tid ^ (T.mask & 0xffu));
            const uint32_t mhi = T.mask >> 8;
#pragma unroll
            for (int j = 0; j < SPT; ++j) {
                const double2 c = s_tab[T.tab + (T.hasj ? (ib | ((T.jtab >> (4 * j)) & 15u)) : ib)];
                const double2 w = sv[kThreads * (j ^ mhi)];
                if (RC) { acc[j].x = fma(c.x, w.x, acc[j].x); acc[j].y = fma(c.x, w.y, acc[j].y); }
                else acc[j] = cfma(c, w, acc[j]);
            }
        }
        for (int g = 0; g < prog.ngroups; ++g) {
            double2 *buf = s_p + (g & 1) * TILE;
            if (g + 1 < prog.ngroups) {
                // its buffer was released by the barrier that ended group g - 1
                const uint32_t pb = base ^ prog.gxor[g + 1];
                double2 *nb = s_p + ((g + 1) & 1) * TILE;
#pragma unroll
                for (int j = 0; j < SPT; ++j) cp_async16(nb + tid + kThreads * j, a.C + (pb | prog.jexp[j]));
                cp_async_commit();
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();   // group g's tile has landed for every thread
            for (int t = prog.gstart[g]; t < prog.gstart[g + 1]; ++t) {
                const TileTerm T = prog.t[t];
                uint32_t ib = 0;
#pragma unroll
                for (int d = 0; d < kMaxDeps; ++d)
                    if (d < T.nb) ib |= ((base >> ((T.pos4 >> (8 * d)) & 0xffu)) & 1u) << d;
                const double2 *sv = buf + (tid ^ (T.lmask & 0xffu));
                const uint32_t mhi = T.lmask >> 8;
#pragma unroll
                for (int j = 0; j < SPT; ++j) {
                    const double2 c = s_tab[T.tab + (T.hasj ? (ib | ((T.jtab >> (4 * j)) & 15u)) : ib)];
                    const double2 w = sv[kThreads * (j ^ mhi)];
                    if (RC) { acc[j].x = fma(c.x, w.x, acc[j].x); acc[j].y = fma(c.x, w.y, acc[j].y); }
                    else acc[j] = cfma(c, w, acc[j]);
                }
            }
            __syncthreads();   // every thread is done with buf before it is refilled
        }
#pragma unroll
        for (int j = 0; j < SPT; ++j) {
            const int64_t e = base | prog.jexp[j];
            const double2 hv = cscale(hs, acc[j]);
            double2 out = hv;
            if (!prog.first) {
                const double2 w0 = __ldcs(a.W + e);
                out.x += w0.x;
                out.y += w0.y;
            } else if (a.P) {
                const double2 p = __ldcs(a.P + e);
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
    }
    block_reduce_store<K, 1>(red, 1, 1, 1, a.partials);
}

// ---------------------------------------------------------------------------
// Bulk-copy pipeline (TMA engine, mbarriers) for the single-vector tiles
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
// Bounded wait for the phase of parity `parity` to complete: at most
// kBulkSpins polls, each suspended for at most ~1 us; false if it gave up.
constexpr uint32_t kBulkSpins = 1u << 22;
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kBulkSpins; ++i) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(ok)
                     : "r"(bar), "r"(parity), "r"(1000u)
                     : "memory");
        if (ok) return true;
    }
    return false;
}
// The wait of a whole warp in the tile loop (true only if every lane saw the
// phase): as mbar_wait, but it also gives up as soon as another warp of the
// block has raised the block's abort flag, so that one warp that stopped does
// not leave the others waiting out their own limits.
__device__ __forceinline__ bool mbar_wait_or_abort(uint32_t bar, uint32_t parity, volatile int *abort_flag)
{
    for (uint32_t i = 0; i < kBulkSpins; ++i) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(ok)
                     : "r"(bar), "r"(parity), "r"(1000u)
                     : "memory");
        if (ok) return true;
        if (*abort_flag) return false;
    }
    return false;
}
__device__ __forceinline__ bool warp_wait_or_abort(uint32_t bar, uint32_t parity, volatile int *abort_flag)
{
    return __all_sync(0xffffffffu, mbar_wait_or_abort(bar, parity, abort_flag));
}
// One contiguous global -> shared copy by the bulk-copy (TMA) engine, no
// multicast; completion is counted in bytes on the mbarrier.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

constexpr int kBulkConsumerWarps = 16;           // 8: 8 states per thread; 16: 4

// Single-vector tiled H.v with the partner tiles streamed by the bulk-copy
// engine: the same tiles, passes, term order and arithmetic as
// hv_tile_kernel (W is bit-identical; the block sums group the tiles
// differently), with the data movement split off.  Warp CW (producer) walks
// the block's item sequence -- per tile its own tile, then one partner tile
// per group -- and streams each item into a ring of `nst` 32 KB
// shared-memory stages as contiguous runs of 2^f states (the tile's rows keep
// global bits 0..f-1), accounted on the stage's `full` mbarrier.  Warps
// 0..CW-1 (consumers) wait on `full`, gather their terms' partners from the
// stage and release it on `empty` (one arrival per warp); consumer thread c
// serves row c mod 256 and 2048 / (32 CW) of its states.  Up to nst items are
// in flight per SM without holding registers, and no block-wide barrier sits
// in the tile loop.  One block per SM (grid = SM count).  Every wait is
// bounded: on a timeout the block sets *a.err, stops, waits (bounded) for the
// copies it issued and exits.
template <int CW, bool RC, bool RD, int K>
__global__ void __launch_bounds__(32 * (CW + 1), 1)
    hv_tile_bulk_kernel(const __grid_constant__ TileProgram prog, const HvArgs a, int nst)
{
    constexpr int SPT = (1 << kBulkJB) * 8 / CW;   // states per consumer thread
    extern __shared__ __align__(128) unsigned char bulk_smem[];
    uint64_t *full = reinterpret_cast<uint64_t *>(bulk_smem);
    uint64_t *empty = full + kBulkMaxStages;
    volatile int *s_abort = reinterpret_cast<volatile int *>(empty + kBulkMaxStages);
    int *s_count = reinterpret_cast<int *>(bulk_smem) + 2 * 2 * kBulkMaxStages + 1;   // [CW + 1]: consumed, issued
    double2 *ring = reinterpret_cast<double2 *>(bulk_smem + kBulkHead);
    double2 *s_tab = ring + size_t(nst) * kBulkTile;
    __shared__ double2 s_red[CW + 1][kMaxK];

    const uint32_t tid = threadIdx.x;
    const int warp = int(tid >> 5), lane = int(tid & 31);
    for (int i = tid; i < prog.ntab; i += blockDim.x) s_tab[i] = a.table[i];
    if (tid == 0) {
        for (int s = 0; s < nst; ++s) {
            mbar_init(smem_addr(full + s), 1);
            mbar_init(smem_addr(empty + s), CW);
        }
        *s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    __syncthreads();

    const int64_t ntiles = int64_t(1) << prog.nouter;
    const int items = 1 + prog.ngroups;
    double2 red[K];
#pragma unroll
    for (int k = 0; k < K; ++k) red[k] = make_double2(0.0, 0.0);

    if (warp == CW) {
        // ---------------- producer ----------------
        int f = 0;
        while (f < 8 && prog.rowpos[f] == f) ++f;
        const int ncp = kBulkTile >> f;
        const uint32_t bytes = uint32_t(sizeof(double2)) << f;
        uint32_t it = 0;
        bool ok = true;
        for (int64_t tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) {
            uint32_t ob = 0;
            for (int k = 0; k < prog.nouter; ++k) ob |= uint32_t((tile >> k) & 1) << prog.outer[k];
            for (int item = 0; item < items; ++item, ++it) {
                const uint32_t s = it % uint32_t(nst), round = it / uint32_t(nst);
                if (round > 0 && !warp_wait_or_abort(smem_addr(empty + s), (round - 1) & 1u, s_abort)) {
                    ok = false;
                    break;
                }
                if (__any_sync(0xffffffffu, *s_abort != 0)) {
                    ok = false;
                    break;
                }
                const uint32_t src = ob ^ (item == 0 ? 0u : prog.gxor[item - 1]);
                if (lane == 0) mbar_arrive_expect_tx(smem_addr(full + s), uint32_t(kBulkTile * sizeof(double2)));
                __syncwarp();
                const uint32_t dst0 = smem_addr(ring + size_t(s) * kBulkTile);
                for (int c = lane; c < ncp; c += 32) {
                    const uint32_t L = uint32_t(c) << f;
                    uint32_t off = prog.jexp[L >> 8];
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                        if (k >= f) off |= ((L >> k) & 1u) << prog.rowpos[k];
                    bulk_g2s(dst0 + L * uint32_t(sizeof(double2)), a.C + (src | off), bytes, smem_addr(full + s));
                }
            }
        }
        if (!ok) {
            *s_abort = 1;
            if (lane == 0 && a.err) atomicExch(a.err, 1);
        }
        if (lane == 0) s_count[CW] = int(it);
    } else {
        // ---------------- consumers ----------------
        const double sc = a.sc[0], pc = a.pc ? a.pc[0] : 0.0, gs = a.gsc ? a.gsc[0] : 0.0;
        const double hs = a.hsc ? a.hsc[0] : sc;
        const double shift = a.shift + (a.shiftv ? a.shiftv[0] : 0.0);
        const uint32_t row = tid & (kThreads - 1);
        const int j0 = int(tid / kThreads) * SPT;   // first of the thread's states in the row
        uint32_t rowbase = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) rowbase |= ((row >> k) & 1u) << prog.rowpos[k];
        uint32_t it = 0;
        bool ok = true;
        for (int64_t tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) {
            uint32_t base = rowbase;
            for (int k = 0; k < prog.nouter; ++k) base |= uint32_t((tile >> k) & 1) << prog.outer[k];
            // streams of the epilogue and the diagonal, issued before the first wait
            double2 pw[SPT];
            double dr[SPT];
            double2 dc[SPT];
#pragma unroll
            for (int jj = 0; jj < SPT; ++jj) {
                const uint32_t e = base | prog.jexp[j0 + jj];
                if (!prog.first) pw[jj] = __ldcs(a.W + e);
                else if (a.P) pw[jj] = __ldcs(a.P + e);
                if (prog.first) {
                    if (RD) dr[jj] = __ldcs(static_cast<const double *>(a.diag) + e);
                    else dc[jj] = __ldcs(static_cast<const double2 *>(a.diag) + e);
                }
            }
            double2 v[SPT], acc[SPT];
            // own tile: its values, the diagonal and the in-tile terms
            {
                const uint32_t s = it % uint32_t(nst);
                if (!warp_wait_or_abort(smem_addr(full + s), (it / uint32_t(nst)) & 1u, s_abort)) {
                    ok = false;
                    break;
                }
                const double2 *sv0 = ring + size_t(s) * kBulkTile;
#pragma unroll
                for (int jj = 0; jj < SPT; ++jj) {
                    v[jj] = sv0[row + kThreads * (j0 + jj)];
                    if (!prog.first) {
                        acc[jj] = make_double2(0.0, 0.0);
                    } else if (RD) {
                        acc[jj] = cscale(dr[jj] - shift, v[jj]);
                    } else {
                        double2 dd = dc[jj];
                        dd.x -= shift;
                        acc[jj] = cmul(dd, v[jj]);
                    }
                }
                for (int t = 0; t < prog.nin; ++t) {
                    const TileTerm T = prog.t[t];
                    uint32_t ib = 0;
#pragma unroll
                    for (int d = 0; d < kMaxDeps; ++d)
                        if (d < T.nb) ib |= ((base >> ((T.pos4 >> (8 * d)) & 0xffu)) & 1u) << d;
                    const double2 *sv = sv0 + (row ^ (T.mask & 0xffu));
                    const uint32_t mhi = T.mask >> 8;
                    if (!T.hasj) {
                        const double2 c = s_tab[T.tab + ib];
#pragma unroll
                        for (int jj = 0; jj < SPT; ++jj) {
                            const double2 w = sv[kThreads * ((j0 + jj) ^ mhi)];
                            if (RC) { acc[jj].x = fma(c.x, w.x, acc[jj].x); acc[jj].y = fma(c.x, w.y, acc[jj].y); }
                            else acc[jj] = cfma(c, w, acc[jj]);
                        }
                        continue;
                    }
#pragma unroll
                    for (int jj = 0; jj < SPT; ++jj) {
                        const double2 c = s_tab[T.tab + (ib | ((T.jtab >> (4 * (j0 + jj))) & 15u))];
                        const double2 w = sv[kThreads * ((j0 + jj) ^ mhi)];
                        if (RC) { acc[jj].x = fma(c.x, w.x, acc[jj].x); acc[jj].y = fma(c.x, w.y, acc[jj].y); }
                        else acc[jj] = cfma(c, w, acc[jj]);
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_addr(empty + s));
                ++it;
            }
            // partner tiles, one per group, in the program's term order
            for (int g = 0; g < prog.ngroups; ++g, ++it) {
                const uint32_t s = it % uint32_t(nst);
                if (!warp_wait_or_abort(smem_addr(full + s), (it / uint32_t(nst)) & 1u, s_abort)) {
                    ok = false;
                    break;
                }
                const double2 *buf = ring + size_t(s) * kBulkTile;
                for (int t = prog.gstart[g]; t < prog.gstart[g + 1]; ++t) {
                    const TileTerm T = prog.t[t];
                    uint32_t ib = 0;
#pragma unroll
                    for (int d = 0; d < kMaxDeps; ++d)
                        if (d < T.nb) ib |= ((base >> ((T.pos4 >> (8 * d)) & 0xffu)) & 1u) << d;
                    const double2 *sv = buf + (row ^ (T.lmask & 0xffu));
                    const uint32_t mhi = T.lmask >> 8;
                    if (!T.hasj) {
                        const double2 c = s_tab[T.tab + ib];
#pragma unroll
                        for (int jj = 0; jj < SPT; ++jj) {
                            const double2 w = sv[kThreads * ((j0 + jj) ^ mhi)];
                            if (RC) { acc[jj].x = fma(c.x, w.x, acc[jj].x); acc[jj].y = fma(c.x, w.y, acc[jj].y); }
                            else acc[jj] = cfma(c, w, acc[jj]);
                        }
                        continue;
                    }
#pragma unroll
                    for (int jj = 0; jj < SPT; ++jj) {
                        const double2 c = s_tab[T.tab + (ib | ((T.jtab >> (4 * (j0 + jj))) & 15u))];
                        const double2 w = sv[kThreads * ((j0 + jj) ^ mhi)];
                        if (RC) { acc[jj].x = fma(c.x, w.x, acc[jj].x); acc[jj].y = fma(c.x, w.y, acc[jj].y); }
                        else acc[jj] = cfma(c, w, acc[jj]);
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_addr(empty + s));
            }
            if (!ok) break;
#pragma unroll
            for (int jj = 0; jj < SPT; ++jj) {
                const int64_t e = base | prog.jexp[j0 + jj];
                const double2 hv = cscale(hs, acc[jj]);
                double2 out = hv;
                if (!prog.first) {
                    out.x += pw[jj].x;
                    out.y += pw[jj].y;
                } else if (a.P) {
                    out.x = fma(pc, pw[jj].x, out.x);
                    out.y = fma(pc, pw[jj].y, out.y);
                }
                __stcs(a.W + e, out);
                const double2 vv = cscale(sc, v[jj]);
                red[0] = cadd(red[0], cconjmul(vv, hv));
                if (!prog.last) continue;
                if (K >= 2) red[1].x += out.x * out.x + out.y * out.y;
                if (K >= 4 && a.G) {
                    const double2 gv = cscale(gs, a.G[e]);
                    red[2] = cadd(red[2], cconjmul(gv, out));
                    red[3] = cadd(red[3], cconjmul(gv, vv));
                }
            }
        }
        if (!ok) {
            *s_abort = 1;
            if (lane == 0 && a.err) atomicExch(a.err, 1);
        }
        if (lane == 0) s_count[warp] = int(it);
    }
    __syncthreads();
    // after a timeout: wait (bounded) for every copy still in flight before the
    // block's shared memory is released
    if (*s_abort && tid == 0) {
        int lo = s_count[0];
        for (int w = 1; w < CW; ++w) lo = min(lo, s_count[w]);
        for (int i = lo; i < s_count[CW]; ++i)
            mbar_wait(smem_addr(full + (uint32_t(i) % uint32_t(nst))), (uint32_t(i) / uint32_t(nst)) & 1u);
    }
    // deterministic block sum: warps in order (the producer's terms are zero)
#pragma unroll
    for (int k = 0; k < K; ++k)
        for (int off = 16; off >= 1; off >>= 1) {
            red[k].x += __shfl_xor_sync(0xffffffffu, red[k].x, off);
            red[k].y += __shfl_xor_sync(0xffffffffu, red[k].y, off);
        }
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) s_red[warp][k] = red[k];
    __syncthreads();
    if (int(tid) < K) {
        double2 sum = make_double2(0.0, 0.0);
        for (int w = 0; w < CW + 1; ++w) sum = cadd(sum, s_red[w][tid]);
        a.partials[(size_t)blockIdx.x * K + tid] = sum;
    }
}

template <bool RC, bool RD, int K>
static cudaError_t launch_tile_stage(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    auto kern = hv_tile_stage_kernel<RC, RD, K>;
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void *>(kern), m->device);
    const size_t smem = sizeof(double2) * (size_t(3) * kThreads * 8 + std::max(1, m->ntab));
    if (e == cudaSuccess && m->carveout) e = set_carveout(reinterpret_cast<const void *>(kern), m->device, smem, 2);
    if (e != cudaSuccess) return e;
    const int grid = tile_grid(m, nblocks);
    HvArgs b = a;
    for (size_t p = 0; p < m->tprogs.size(); ++p) {
        b.partials = a.partials + size_t(p) * grid * K * a.R;
        kern<<<grid, kThreads, smem, st>>>(*m->tprogs[p], b);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Dynamic shared memory of the bulk-copy kernel: the ring of stages, the
// table and the head (above the 200 KB the other kernels are allowed).
static size_t bulk_smem_bytes(int nst, int ntab)
{
    return size_t(kBulkHead) + sizeof(double2) * (size_t(nst) * kBulkTile + std::max(1, ntab));
}

static cudaError_t bulk_smem_attr(const void *kern, int device, size_t smem)
{
    static std::mutex mu;
    static std::vector<std::pair<std::pair<const void *, int>, size_t>> done;
    std::lock_guard<std::mutex> lock(mu);
    for (auto &d : done)
        if (d.first.first == kern && d.first.second == device && d.second >= smem) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e == cudaSuccess) done.push_back({{kern, device}, smem});
    return e;
}

template <bool RC, bool RD, int K>
static cudaError_t launch_tile_bulk(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    auto kern = hv_tile_bulk_kernel<kBulkConsumerWarps, RC, RD, K>;
    const size_t smem = bulk_smem_bytes(m->bulk_stages, m->ntab);
    cudaError_t e = bulk_smem_attr(reinterpret_cast<const void *>(kern), m->device, smem);
    if (e != cudaSuccess) return e;
    const int grid = tile_grid(m, nblocks);
    HvArgs b = a;
    for (size_t p = 0; p < m->tprogs.size(); ++p) {
        b.partials = a.partials + size_t(p) * grid * K * a.R;
        kern<<<grid, 32 * (kBulkConsumerWarps + 1), smem, st>>>(*m->tprogs[p], b, m->bulk_stages);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <bool RC, bool RD, int K>
static cudaError_t launch_staged_t(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    if (m->tile_stage == 2) return launch_tile_bulk<RC, RD, K>(m, a, nblocks, st);
    return launch_tile_stage<RC, RD, K>(m, a, nblocks, st);
}

template <int K>
static cudaError_t launch_staged_k(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    if (m->real_coef && m->real_diag) return launch_staged_t<true, true, K>(m, a, nblocks, st);
    if (m->real_diag) return launch_staged_t<false, true, K>(m, a, nblocks, st);
    return launch_staged_t<false, false, K>(m, a, nblocks, st);
}

cudaError_t launch_tile_staged(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    if (!tile_staged(m)) return cudaErrorInvalidValue;
    if (a.K == 1) return launch_staged_k<1>(m, a, nblocks, st);
    if (a.K == 4) return launch_staged_k<4>(m, a, nblocks, st);
    return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// Tile kernel with tensor copies of the tile's own rows (stage 3)
// ---------------------------------------------------------------------------
// Every flip term moves a 16-byte value through the SM's load/store data path
// per state, from shared memory or from L1/L2, and that path bounds the gather
// kernel.  Its own-row traffic rides the same path: the tile's rows of C are
// loaded and stored into shared memory, and the epilogue rows of P or W are
// copied in with cp.async and read back.  Here the tensor-copy engine writes
// the tile's rows of C, of P or W and of the diagonal straight into shared
// memory, outside that path; per state and pass that leaves the epilogue's two
// shared reads (three in the first pass) and the store of W beside the terms.
// The copies are issued by one thread when the tile starts and land while the
// block gathers the out-of-tile terms through L1/L2; the in-tile terms follow
// once the own rows have arrived, the diagonal term is added in the epilogue.
// The same tiles, passes and terms as hv_tile_kernel with 8 rows a thread; W
// agrees to rounding (the diagonal term is added last instead of first).

// Tensor maps of one pass: C (own rows), P or W (epilogue rows), diagonal.
struct TmaMaps {
    CUtensorMap c, pw, d;
    TmaGeom g;
    uint32_t bytes_c, bytes_pw, bytes_d;   // bytes of each copy (0: not copied)
};

__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

// One box of a tensor map into shared memory (no multicast), counted in bytes
// on the mbarrier.
__device__ __forceinline__ void tma_box(uint32_t dst, const CUtensorMap *map, const int (&c)[kTmaMaxRank], int rank,
                                        uint32_t bar)
{
    const uint64_t tm = reinterpret_cast<uint64_t>(map);
    switch (rank) {
    case 1:
        asm volatile("cp.async.bulk.tensor.1d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2}], [%3];\n"
                     ::"r"(dst), "l"(tm), "r"(c[0]), "r"(bar) : "memory");
        break;
    case 2:
        asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                     "[%4];\n" ::"r"(dst), "l"(tm), "r"(c[0]), "r"(c[1]), "r"(bar) : "memory");
        break;
    case 3:
        asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
                     "[%5];\n" ::"r"(dst), "l"(tm), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(bar) : "memory");
        break;
    case 4:
        asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
                     "%5}], [%6];\n" ::"r"(dst), "l"(tm), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(bar) : "memory");
        break;
    default:
        asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
                     "%5, %6}], [%7];\n" ::"r"(dst), "l"(tm), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]),
                     "r"(bar) : "memory");
        break;
    }
}

constexpr int kTmaSPT = 8;                          // rows a thread

// acc[j] += c_j w[j] for a term with dependency bits among the j bits: c_j at the
// thread's base ib and its j-th state.  With one such bit the two coefficients are
// read once and chosen per state (two shared reads instead of one per state).
template <int SPT, bool RC>
__device__ __forceinline__ void tma_term_apply_j(const TileTerm &T, uint32_t ib, const double2 *s_tab,
                                                 const double2 (&w)[SPT], double2 (&acc)[SPT])
{
    if (__popc(uint32_t(T.jdep)) == 1) {
        const double2 c0 = s_tab[T.tab + ib], c1 = s_tab[T.tab + (ib | T.jdep)];
#pragma unroll
        for (int j = 0; j < SPT; ++j) {
            const bool on = ((T.jtab >> (4 * j)) & 15u) != 0;
            if (RC) {
                const double cx = on ? c1.x : c0.x;
                acc[j].x = fma(cx, w[j].x, acc[j].x);
                acc[j].y = fma(cx, w[j].y, acc[j].y);
            } else {
                acc[j] = cfma(on ? c1 : c0, w[j], acc[j]);
            }
        }
        return;
    }
#pragma unroll
    for (int j = 0; j < SPT; ++j) {
        const double2 c = s_tab[T.tab + (ib | uint32_t((T.jtab >> (4 * j)) & 15u))];
        if (RC) { acc[j].x = fma(c.x, w[j].x, acc[j].x); acc[j].y = fma(c.x, w[j].y, acc[j].y); }
        else acc[j] = cfma(c, w[j], acc[j]);
    }
}

// acc[j] += c_j w[j] for the thread's states, c_j the term's coefficient at the
// thread's base (and, for terms with dependency bits among the j bits, at its j-th state).
template <int SPT, bool RC>
__device__ __forceinline__ void tma_term_apply(const TileTerm &T, uint32_t base, const double2 *s_tab,
                                               const double2 (&w)[SPT], double2 (&acc)[SPT])
{
    uint32_t ib = 0;
#pragma unroll
    for (int d = 0; d < kMaxDeps; ++d)
        if (d < T.nb) ib |= ((base >> ((T.pos4 >> (8 * d)) & 0xffu)) & 1u) << d;
    if (!T.hasj) {
        const double2 c = s_tab[T.tab + ib];
#pragma unroll
        for (int j = 0; j < SPT; ++j) {
            if (RC) { acc[j].x = fma(c.x, w[j].x, acc[j].x); acc[j].y = fma(c.x, w[j].y, acc[j].y); }
            else acc[j] = cfma(c, w[j], acc[j]);
        }
        return;
    }
    tma_term_apply_j<SPT, RC>(T, ib, s_tab, w, acc);
}
constexpr int kTmaTile = kThreads * kTmaSPT;        // 2048 states

template <bool RC, bool RD, int K, bool DEEP>
__global__ void __launch_bounds__(kThreads, 2)
    hv_tile_tma_kernel(const __grid_constant__ TileProgram prog, const HvArgs a, const __grid_constant__ TmaMaps tm)
{
    constexpr int SPT = kTmaSPT;
    constexpr int TILE = kTmaTile;
    extern __shared__ unsigned char tma_raw[];
    // copies land at 128-byte aligned addresses
    unsigned char *tma_smem = tma_raw + ((128u - (smem_addr(tma_raw) & 127u)) & 127u);
    double2 *s_v = reinterpret_cast<double2 *>(tma_smem);   // own rows of C
    double2 *s_pw = s_v + TILE;                             // rows of P (first pass) or W (later passes)
    double2 *s_dc = s_pw + TILE;                            // diagonal (complex; real: the first half as doubles)
    const double *s_dr = reinterpret_cast<const double *>(s_dc);
    double2 *s_tab = s_dc + (RD ? TILE / 2 : TILE);
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ uint32_t s_next[2];
    __shared__ int s_abort;
    __shared__ double2 s_red[kThreads / 32][K];
    const uint32_t tid = threadIdx.x;
    for (int i = tid; i < prog.ntab; i += blockDim.x) s_tab[i] = a.table[i];
    const uint32_t bar_v = smem_addr(&s_bar[0]), bar_e = smem_addr(&s_bar[1]);
    uint32_t *const ctr = a.tile_counter ? a.tile_counter + prog.pass : nullptr;
    if (tid == 0) {
        mbar_init(bar_v, 1);
        mbar_init(bar_e, 1);
        fence_mbar_init();
        s_abort = 0;
        s_next[0] = ctr ? atomicAdd(ctr, 1u) : 0u;
    }
    const int64_t ntiles = int64_t(1) << prog.nouter;
    const bool pw_on = prog.first ? a.P != nullptr : true;
    const double sc = a.sc[0], pc = a.pc ? a.pc[0] : 0.0, gs = a.gsc ? a.gsc[0] : 0.0;
    const double hs = a.hsc ? a.hsc[0] : sc;
    const double shift = a.shift + (a.shiftv ? a.shiftv[0] : 0.0);
    uint32_t rowbase = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) rowbase |= ((tid >> k) & 1u) << prog.rowpos[k];
    double2 red[K][1];
#pragma unroll
    for (int k = 0; k < K; ++k) red[k][0] = make_double2(0.0, 0.0);
    uint32_t phase = 0;
    int fail = 0;
    bool gave_up = false;
    for (uint32_t it = 0;; ++it) {
        // the previous tile's shared reads are done and s_next[it & 1] is set; a wait
        // that gave up anywhere in the block ends the loop for every thread
        if (__syncthreads_or(fail)) {
            gave_up = true;
            break;
        }
        const int64_t tile = ctr ? int64_t(s_next[it & 1u]) : int64_t(blockIdx.x) + int64_t(it) * gridDim.x;
        if (tile >= ntiles) break;
        uint32_t tbase = 0;
        for (int k = 0; k < prog.nouter; ++k) tbase |= uint32_t((tile >> k) & 1) << prog.outer[k];
        const uint32_t base = rowbase | tbase;
        if (tid == 0) {
            if (ctr) s_next[(it + 1u) & 1u] = atomicAdd(ctr, 1u);
            int c[kTmaMaxRank];
#pragma unroll
            for (int d = 0; d < kTmaMaxRank; ++d)
                c[d] = (d < tm.g.rank && !tm.g.tile[d]) ? int((tbase >> tm.g.lo[d]) & ((1u << tm.g.nbits[d]) - 1u)) : 0;
            fence_proxy_async_smem();   // the previous tile's reads of these buffers come first
            mbar_arrive_expect_tx(bar_v, tm.bytes_c);
            tma_box(smem_addr(s_v), &tm.c, c, tm.g.rank, bar_v);
            mbar_arrive_expect_tx(bar_e, (pw_on ? tm.bytes_pw : 0u) + (prog.first ? tm.bytes_d : 0u));
            if (pw_on) tma_box(smem_addr(s_pw), &tm.pw, c, tm.g.rank, bar_e);
            if (prog.first) tma_box(smem_addr(s_dc), &tm.d, c, tm.g.rank, bar_e);
        }
        double2 acc[SPT];
#pragma unroll
        for (int j = 0; j < SPT; ++j) acc[j] = make_double2(0.0, 0.0);
        // flip masks leaving the tile first: partners through L1/L2 while the own rows
        // arrive, DEEP: the partner rows of two terms in flight at a time
        int t = prog.nin;
        if (DEEP) {
            for (; t + 1 < prog.nterms; t += 2) {
                const TileTerm T0 = prog.t[t], T1 = prog.t[t + 1];
                const uint32_t p0 = base ^ T0.mask, p1 = base ^ T1.mask;
                double2 w0[SPT], w1[SPT];
#pragma unroll
                for (int j = 0; j < SPT; ++j) w0[j] = __ldg(a.C + (p0 ^ prog.jexp[j]));
#pragma unroll
                for (int j = 0; j < SPT; ++j) w1[j] = __ldg(a.C + (p1 ^ prog.jexp[j]));
                tma_term_apply<SPT, RC>(T0, base, s_tab, w0, acc);
                tma_term_apply<SPT, RC>(T1, base, s_tab, w1, acc);
            }
        }
        for (; t < prog.nterms; ++t) {
            const TileTerm T = prog.t[t];
            const uint32_t pbx = base ^ T.mask;
            double2 w0[SPT];
#pragma unroll
            for (int j = 0; j < SPT; ++j) w0[j] = __ldg(a.C + (pbx ^ prog.jexp[j]));
            tma_term_apply<SPT, RC>(T, base, s_tab, w0, acc);
        }
        const bool okv = mbar_wait_or_abort(bar_v, phase, &s_abort);
        // flip masks inside the tile: partners from shared memory
        for (int t = 0; t < prog.nin; ++t) {
            const TileTerm T = prog.t[t];
            uint32_t ib = 0;
#pragma unroll
            for (int d = 0; d < kMaxDeps; ++d)
                if (d < T.nb) ib |= ((base >> ((T.pos4 >> (8 * d)) & 0xffu)) & 1u) << d;
            const double2 *sv = s_v + (tid ^ (T.mask & 0xffu));
            const uint32_t mhi = T.mask >> 8;
            if (!T.hasj) {
                const double2 c = s_tab[T.tab + ib];
#pragma unroll
                for (int j = 0; j < SPT; ++j) {
                    const double2 w = sv[kThreads * (j ^ mhi)];
                    if (RC) { acc[j].x = fma(c.x, w.x, acc[j].x); acc[j].y = fma(c.x, w.y, acc[j].y); }
                    else acc[j] = cfma(c, w, acc[j]);
                }
                continue;
            }
            double2 wi[SPT];
#pragma unroll
            for (int j = 0; j < SPT; ++j) wi[j] = sv[kThreads * (j ^ mhi)];
            tma_term_apply_j<SPT, RC>(T, ib, s_tab, wi, acc);
        }
        const bool oke = mbar_wait_or_abort(bar_e, phase, &s_abort);
        phase ^= 1u;
        if (!(okv && oke)) {
            fail = 1;
            s_abort = 1;
            if (a.err) atomicExch(a.err, 1);
        }
#pragma unroll
        for (int j = 0; j < SPT; ++j) {
            const int sl = int(tid) + kThreads * j;
            const int64_t e = base | prog.jexp[j];
            const double2 v = s_v[sl];
            double2 hsum = acc[j];
            if (prog.first) {
                if (RD) {
                    const double dd = s_dr[sl] - shift;
                    hsum.x = fma(dd, v.x, hsum.x);
                    hsum.y = fma(dd, v.y, hsum.y);
                } else {
                    double2 dd = s_dc[sl];
                    dd.x -= shift;
                    hsum = cfma(dd, v, hsum);
                }
            }
            const double2 hv = cscale(hs, hsum);
            double2 out = hv;
            if (!prog.first) {
                const double2 w0 = s_pw[sl];
                out.x += w0.x;
                out.y += w0.y;
            } else if (a.P) {
                const double2 p = s_pw[sl];
                out.x = fma(pc, p.x, out.x);
                out.y = fma(pc, p.y, out.y);
            }
            if (!fail) __stcs(a.W + e, out);
            const double2 vv = cscale(sc, v);
            red[0][0] = cadd(red[0][0], cconjmul(vv, hv));
            if (!prog.last) continue;
            if (K >= 2) red[1][0].x += out.x * out.x + out.y * out.y;
            if (K >= 4 && a.G) {
                const double2 gv = cscale(gs, a.G[e]);
                red[2][0] = cadd(red[2][0], cconjmul(gv, out));
                red[3][0] = cadd(red[3][0], cconjmul(gv, vv));
            }
        }
        // per-tile sums in a fixed order (dynamic order: independent of which block took the tile)
        if (ctr) tile_sums_store<K>(red, s_red, a.partials + size_t(tile) * K);
    }
    if (!ctr) tile_sums_store<K>(red, s_red, a.partials + size_t(blockIdx.x) * K);
    // after a wait gave up: wait (bounded) for the last tile's copies before the block's
    // shared memory is released
    if (gave_up && tid == 0) {
        mbar_wait(bar_v, phase ^ 1u);
        mbar_wait(bar_e, phase ^ 1u);
    }
}

void *tile_tma_encoder()
{
    static void *fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = f;
    });
    return fn;
}

bool tile_tma_geometry(const TileProgram &p, TmaGeom &g)
{
    g = TmaGeom{};
    if (p.tbits != 8 || p.jb != 3 || p.n > 32) return false;
    uint32_t tmask = 0;
    for (int k = 0; k < 8; ++k) tmask |= 1u << p.rowpos[k];
    tmask |= p.jexp[7];
    // shared memory holds the tile as [j][row]: its bits in ascending order must be
    // the 8 row bits, then the 3 j bits, starting at bit 0
    int bits[32], nb = 0;
    for (int b = 0; b < p.n; ++b)
        if ((tmask >> b) & 1u) bits[nb++] = b;
    if (nb != 11 || bits[0] != 0) return false;
    for (int k = 0; k < 8; ++k)
        if (bits[k] != p.rowpos[k]) return false;
    for (int k = 0; k < 3; ++k)
        if ((1u << bits[8 + k]) != p.jexp[1u << k]) return false;
    for (int b = 0; b < p.n;) {
        const bool in = (tmask >> b) & 1u;
        int e = b;
        while (e < p.n && (((tmask >> e) & 1u) != 0) == in) ++e;
        for (int s = b; s < e;) {
            const int len = std::min(in ? (g.rank == 0 ? 7 : 8) : 31, e - s);
            if (g.rank == kTmaMaxRank) return false;
            g.lo[g.rank] = s;
            g.nbits[g.rank] = len;
            g.tile[g.rank] = in ? 1 : 0;
            ++g.rank;
            s += len;
        }
        b = e;
    }
    return true;
}

size_t tile_tma_smem(const pned_model *m)
{
    const size_t tile = size_t(kTmaTile);
    return 128 + sizeof(double2) * (2 * tile + (m->real_diag ? tile / 2 : tile) + size_t(std::max(1, m->ntab)));
}

bool tile_tma_usable(const pned_model *m, const HvArgs &a)
{
    auto al = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    return a.R == 1 && m->tma_geom.size() == m->tprogs.size() && tile_tma_encoder() && al(a.C) && al(a.W) &&
           al(a.P) && al(a.diag);
}

// Tensor map of one vector (complex: 16-byte states, or real doubles) over the
// pass's copy dimensions, box = the tile.
static bool encode_tile_map(CUtensorMap *map, const TmaGeom &g, const void *base, bool complex)
{
    auto fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(tile_tma_encoder());
    if (!fn || g.rank < 1) return false;
    cuuint64_t dims[kTmaMaxRank], strides[kTmaMaxRank];
    cuuint32_t box[kTmaMaxRank], estr[kTmaMaxRank];
    const cuuint64_t es = complex ? 16 : 8;
    for (int d = 0; d < g.rank; ++d) {
        dims[d] = cuuint64_t(1) << g.nbits[d];
        if (d == 0 && complex) dims[0] *= 2;   // elements are doubles
        box[d] = g.tile[d] ? cuuint32_t(dims[d]) : 1u;
        estr[d] = 1;
        if (d > 0) strides[d - 1] = (cuuint64_t(1) << g.lo[d]) * es;
    }
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, cuuint32_t(g.rank), const_cast<void *>(base), dims, strides, box,
              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <bool RC, bool RD, int K, bool DEEP>
static cudaError_t launch_tile_tma_t(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    auto kern = hv_tile_tma_kernel<RC, RD, K, DEEP>;
    const size_t smem = tile_tma_smem(m);
    cudaError_t e = allow_dynamic_smem(reinterpret_cast<const void *>(kern), m->device);
    if (e == cudaSuccess && m->carveout) e = set_carveout(reinterpret_cast<const void *>(kern), m->device, smem, 2);
    if (e != cudaSuccess) return e;
    const int grid = tile_grid(m, nblocks);
    const bool dyn = tile_dynamic(m, a, nblocks);
    HvArgs b = a;
    if (!dyn) b.tile_counter = nullptr;
    else if ((e = cudaMemsetAsync(a.tile_counter, 0, sizeof(uint32_t) * kTileMaxPasses, st)) != cudaSuccess)
        return e;
    size_t off = 0;
    for (size_t p = 0; p < m->tprogs.size(); ++p) {
        const TileProgram &pg = *m->tprogs[p];
        TmaMaps tm{};
        tm.g = m->tma_geom[p];
        const double2 *pw = pg.first ? a.P : a.W;
        bool ok = encode_tile_map(&tm.c, tm.g, a.C, true);
        if (pw) ok = ok && encode_tile_map(&tm.pw, tm.g, pw, true);
        if (pg.first) ok = ok && encode_tile_map(&tm.d, tm.g, a.diag, !RD);
        if (!ok) return cudaErrorInvalidValue;
        tm.bytes_c = uint32_t(kTmaTile * sizeof(double2));
        tm.bytes_pw = pw ? uint32_t(kTmaTile * sizeof(double2)) : 0u;
        tm.bytes_d = pg.first ? uint32_t(kTmaTile * (RD ? sizeof(double) : sizeof(double2))) : 0u;
        b.partials = a.partials + off;
        off += dyn ? (size_t(1) << pg.nouter) * K : size_t(grid) * K;
        kern<<<grid, kThreads, smem, st>>>(pg, b, tm);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <int K, bool DEEP>
static cudaError_t launch_tile_tma_k(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    if (m->real_coef && m->real_diag) return launch_tile_tma_t<true, true, K, DEEP>(m, a, nblocks, st);
    if (m->real_diag) return launch_tile_tma_t<false, true, K, DEEP>(m, a, nblocks, st);
    return launch_tile_tma_t<false, false, K, DEEP>(m, a, nblocks, st);
}

cudaError_t launch_tile_tma(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    const bool deep = m->tma_deep;
    if (a.K == 1) return deep ? launch_tile_tma_k<1, true>(m, a, nblocks, st) : launch_tile_tma_k<1, false>(m, a, nblocks, st);
    if (a.K == 4) return deep ? launch_tile_tma_k<4, true>(m, a, nblocks, st) : launch_tile_tma_k<4, false>(m, a, nblocks, st);
    return cudaErrorInvalidValue;
}

}   // namespace pned
