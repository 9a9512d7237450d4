// Sz-sector H.v on segments (S = 1/2, one vector).  In mk_list12 order
// (S1/2 parallel.f90:452-578) the sector states that share their high half
// hi = state >> ihf are contiguous: a segment of len(hi) states, the low halves
// of the complementary popcount in ascending order, so the state of rank r has
// index start(hi) + r with start(hi) = lin_hi[hi] and r = lin_lo[lo] - 1.
//   * a term that flips low bits only stays inside the segment: the partner's
//     rank is lin_lo[lo ^ ml] - 1 (one table read instead of two; the segment,
//     at most about 100 KB, is read through L1);
//   * a term that flips high bits only maps the segment onto segment hi ^ mh
//     rank for rank (same popcounts): partner index lin_hi[hi ^ mh] + r, looked
//     up once per block, and a warp's partner reads are one contiguous run;
//   * a term that flips both looks up the partner's rank in its segment.
// These are the flat gather's indices lin_lo[.] + lin_hi[.] - 1, and the terms
// run in program order with the same arithmetic, so W is bit-identical to it.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "device.cuh"

namespace pned {

constexpr int kSegUnroll = 4;   // terms whose loads the segment kernel keeps in flight together

template <bool RC, bool RD, int K>
__global__ void __launch_bounds__(kThreads, 4)
    hv_sector_kernel(const __grid_constant__ XorProgram prog, const HvArgs a, const int64_t *__restrict__ seg_start,
                     const int32_t *__restrict__ seg_hi, const int32_t *__restrict__ rank_lo, int nseg)
{
    extern __shared__ double2 smem[];
    double2 *s_tab = smem;                                                // coefficient table
    int64_t *s_base = reinterpret_cast<int64_t *>(s_tab + prog.ntab);     // per term: lin_hi[hi ^ mh]
    for (int i = threadIdx.x; i < prog.ntab; i += blockDim.x) s_tab[i] = a.table[i];
    const int sh = a.lin_pow2 - 1;
    const uint32_t lomask = (1u << sh) - 1u;
    const double sc = a.sc[0], pc = a.pc ? a.pc[0] : 0.0, gs = a.gsc ? a.gsc[0] : 0.0;
    const double scr[1] = {sc}, pcr[1] = {pc}, gsr[1] = {gs};
    double2 red[K][1];
#pragma unroll
    for (int k = 0; k < K; ++k) red[k][0] = make_double2(0.0, 0.0);
    for (int g = blockIdx.x; g < nseg; g += gridDim.x) {
        const int64_t start = seg_start[g];
        const int len = int(seg_start[g + 1] - start);
        const uint32_t hi = uint32_t(seg_hi[g]);
        __syncthreads();   // the previous segment's shared reads are done (first: table staged)
        for (int t = threadIdx.x; t < prog.nterms; t += blockDim.x) {
            const uint32_t mh = prog.t[t].xmask >> sh;
            s_base[t] = mh ? a.lin_hi[hi ^ mh] : start;
        }
        __syncthreads();
        for (int r = threadIdx.x; r < len; r += blockDim.x) {
            const int64_t s = start + r;
            const uint32_t su = uint32_t(a.list1[s]);
            const uint32_t lo = su & lomask;
            const double2 v[1] = {a.C[s]};
            double2 acc[1];
            if (RD) {
                const double dd = static_cast<const double *>(a.diag)[s] - a.shift;
                acc[0] = cscale(dd, v[0]);
            } else {
                double2 dd = static_cast<const double2 *>(a.diag)[s];
                dd.x -= a.shift;
                acc[0] = cmul(dd, v[0]);
            }
            // four terms at a time: their rank reads, then their partner reads, are in
            // flight together; the products are added in term order as below
            int t = 0;
            for (; t + kSegUnroll <= prog.nterms; t += kSegUnroll) {
                double2 c[kSegUnroll], w[kSegUnroll];
                int64_t pi[kSegUnroll];
#pragma unroll
                for (int u = 0; u < kSegUnroll; ++u) {
                    const XorTerm T = prog.t[t + u];
                    uint32_t idx = 0;
#pragma unroll
                    for (int k = 0; k < kMaxDeps; ++k)
                        if (k < T.nb) idx |= ((su >> ((T.pos4 >> (8 * k)) & 0xffu)) & 1u) << k;
                    c[u] = s_tab[T.tab + idx];
                    const uint32_t ml = T.xmask & lomask;
                    const bool zero = c[u].x == 0.0 && c[u].y == 0.0;
                    const int64_t rk = ml == 0 ? r : __ldg(rank_lo + (lo ^ ml));
                    pi[u] = zero ? s : s_base[t + u] + rk;
                }
#pragma unroll
                for (int u = 0; u < kSegUnroll; ++u) w[u] = __ldg(a.C + pi[u]);
#pragma unroll
                for (int u = 0; u < kSegUnroll; ++u) {
                    if (RC) {
                        acc[0].x = fma(c[u].x, w[u].x, acc[0].x);
                        acc[0].y = fma(c[u].x, w[u].y, acc[0].y);
                    } else {
                        acc[0] = cfma(c[u], w[u], acc[0]);
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
                const uint32_t ml = T.xmask & lomask;
                // zero elements lead out of the sector: they add zero times the own value
                const bool zero = c.x == 0.0 && c.y == 0.0;
                // (the index is chosen before the load: only in-sector partners are read)
                const int64_t rk = ml == 0 ? r : __ldg(rank_lo + (lo ^ ml));       // partner's rank
                const int64_t pi = s_base[t] + rk;                                 // s_base = start if mh == 0
                const double2 w = __ldg(a.C + (zero ? s : pi));
                if (RC) {
                    acc[0].x = fma(c.x, w.x, acc[0].x);
                    acc[0].y = fma(c.x, w.y, acc[0].y);
                } else {
                    acc[0] = cfma(c, w, acc[0]);
                }
            }
            hv_epilogue<K, 1>(a, s, 0, v, acc, scr, pcr, gsr, red);
        }
    }
    block_reduce_store<K, 1>(red, 1, 1, 1, a.partials);
}

// Shared memory of the segment kernel: the table and one partner-segment
// start per term.
static size_t sector_smem(const pned_model *m)
{
    return sizeof(double2) * std::max(1, m->ntab) + sizeof(int64_t) * std::max(1, m->nterms);
}

// Persistent grid: the resident blocks (the occupancy the runtime reports for
// the kernel's shared memory, static reduction buffer included).
int sector_grid(const pned_model *m, int nblocks)
{
    return std::max(1, std::min({nblocks, std::max(1, m->seg_bps) * m->nsm, m->nseg}));
}

// sector models: complex table, real diagonal
template <int K> static const void *sector_kernel() { return reinterpret_cast<const void *>(hv_sector_kernel<false, true, K>); }

template <int K>
static cudaError_t launch_sector_k(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    hv_sector_kernel<false, true, K><<<sector_grid(m, nblocks), kThreads, sector_smem(m), st>>>(
        *m->xprog, a, m->d_seg_start, m->d_seg_hi, m->d_rank_lo, m->nseg);
    return cudaGetLastError();
}

cudaError_t launch_sector(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st)
{
    if (!sector_segments_on(m) || a.R != 1 || a.lin_pow2 <= 0) return cudaErrorInvalidValue;
    if (a.K == 1) return launch_sector_k<1>(m, a, nblocks, st);
    if (a.K == 4) return launch_sector_k<4>(m, a, nblocks, st);
    return cudaErrorInvalidValue;
}

// Segment table of an S = 1/2 sector model: start of every nonempty segment
// (ascending high half) plus the sector dimension, and the high halves.  Used
// when the largest segment has at least 256 states (one per thread).
cudaError_t build_sector_segments(pned_model *m)
{
    const HostProgram &hp = m->hp;
    if (hp.q != 2 || !hp.sector) return cudaSuccess;
    const int sh = hp.ihf;
    std::vector<int64_t> starts;
    std::vector<int32_t> his;
    int64_t prev = -1;
    for (size_t l = 0; l < hp.list1.size(); ++l) {
        const int64_t hi = hp.list1[l] >> sh;
        if (hi != prev) {
            starts.push_back(int64_t(l));
            his.push_back(int32_t(hi));
            prev = hi;
        }
    }
    starts.push_back(int64_t(hp.list1.size()));
    int64_t mx = 0;
    for (size_t g = 0; g + 1 < starts.size(); ++g) mx = std::max(mx, starts[g + 1] - starts[g]);
    m->nseg = int(his.size());
    m->seg_max = int(mx);
    if (mx < kThreads) {
        m->nseg = 0;
        m->seg_max = 0;
        return cudaSuccess;
    }
    // resident blocks per SM (the rest of the SM's memory stays L1)
    const size_t smem = sector_smem(m);
    int bps = 1 << 20;
    for (const void *kern : {sector_kernel<1>(), sector_kernel<4>()}) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        int b = 0;
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, kThreads, smem);
        if (e != cudaSuccess) return e;
        bps = std::min(bps, b);
    }
    if (bps < 1) {   // does not fit: the flat gather runs
        m->nseg = 0;
        m->seg_max = 0;
        return cudaSuccess;
    }
    m->seg_bps = bps;
    // 0-based rank of every low half in its popcount class (lin_lo - 1; 32-bit,
    // half the cache footprint of the 64-bit Lin table)
    const size_t nlo = size_t(1) << sh;
    std::vector<int32_t> rank(nlo);
    for (size_t lo = 0; lo < nlo; ++lo) rank[lo] = int32_t(hp.lin_lo[lo] - 1);
    cudaError_t e = cudaMalloc(&m->d_seg_start, sizeof(int64_t) * starts.size());
    if (e == cudaSuccess) e = cudaMalloc(&m->d_seg_hi, sizeof(int32_t) * his.size());
    if (e == cudaSuccess) e = cudaMalloc(&m->d_rank_lo, sizeof(int32_t) * nlo);
    if (e == cudaSuccess)
        e = cudaMemcpy(m->d_seg_start, starts.data(), sizeof(int64_t) * starts.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->d_seg_hi, his.data(), sizeof(int32_t) * his.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->d_rank_lo, rank.data(), sizeof(int32_t) * nlo, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(m->d_seg_start);
        cudaFree(m->d_seg_hi);
        cudaFree(m->d_rank_lo);
        m->d_seg_start = nullptr;
        m->d_seg_hi = nullptr;
        m->d_rank_lo = nullptr;
        m->nseg = 0;
        m->seg_max = 0;
    }
    return e;
}

}  // namespace pned
