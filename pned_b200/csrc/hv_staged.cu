// Staged variants of the single-vector S = 1/2 tile kernel, chosen by the
// plan: partner tiles copied into shared memory with cp.async (stage 1) or
// with cp.async.bulk under mbarriers by a producer warp (stage 2).
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

}   // namespace pned
