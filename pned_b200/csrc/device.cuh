// Device-side declarations shared by device.cu and krylov.cu.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "kernels.cuh"

struct pned_model {
    pned::HostProgram hp;
    int device = 0;
    int n = 0, q = 2, nbond = 0;
    int64_t dim = 0;
    bool real_coef = true, real_diag = true;
    int ntab = 0, nterms = 0;
    std::unique_ptr<pned::XorProgram> xprog;
    std::unique_ptr<pned::RadixProgram> rprog;
    std::vector<std::unique_ptr<pned::TileProgram>> tprogs;   // tiled single-vector passes (q == 2)
    size_t tile_smem = 0;
    bool use_tile = false;   // single-vector H.v uses the tiled kernel
    // tiled multi-vector passes per R (q == 2): VPT vectors and SPT rows per thread
    struct TileSet {
        std::vector<std::unique_ptr<pned::TileProgram>> progs;
        int vpt = 0, spt = 0;
    };
    std::map<int, TileSet> rtiles;
    std::mutex rtiles_mu;
    // tiled mixed-radix passes per R (q > 2, full basis; guarded by rtiles_mu)
    struct QTileSet {
        std::vector<std::unique_ptr<pned::QTileProgram>> progs;
        int vpt = 0;
        size_t smem = 0;
    };
    std::map<int, QTileSet> qtiles;
    pned_tile_plan plan1{-1, -1, -1, -1, -1, -1, -1};   // single-vector plan parameters (-1: defaults)
    int tile_jb = 3;                        // j bits (rows per thread 2^jb) of the single-vector tiles
    int tile_bps = 2;                       // resident blocks per SM the single-vector tile kernel is built for
    bool carveout = true;                   // size the shared-memory carveout to the tiles (rest L1)
    int tile_stage = 0;                     // single-vector partner tiles: 0 gathered through L1/L2,
                                            // 1 staged in shared memory (cp.async), 2 streamed by bulk copies,
                                            // 3 gathered as 0 with the tile's own rows, epilogue rows and
                                            // diagonal copied in by the tensor-copy engine
    std::vector<pned::TmaGeom> tma_geom;    // stage 3: copy geometry of each pass's tile
    bool tma_deep = false;                  // stage 3: partner rows of two out-of-tile terms in flight
    bool plan1_set = false;                 // plan1 was set by the caller (else the size's default plan)
    int bulk_stages = 0;                    // shared-memory stages of the bulk-copy pipeline
    int nsm = 148;
    double2 *d_table = nullptr;
    void *d_diag = nullptr;
    // Sz sector: index -> state and the Lin tables
    int64_t *d_list1 = nullptr, *d_lin_lo = nullptr, *d_lin_hi = nullptr;
    int64_t lin_mod = 0;
    // S = 1/2 sector segments (states sharing their high half): nseg starts + the
    // dimension, and the high halves; nseg == 0 when the flat gather is used
    int64_t *d_seg_start = nullptr;
    int32_t *d_seg_hi = nullptr;
    int32_t *d_rank_lo = nullptr;   // rank of each low half in its popcount class (lin_lo - 1)
    int nseg = 0, seg_max = 0, seg_bps = 1;   // segments, the largest, resident blocks per SM
    bool seg_enabled = true;   // pned_model_sector_segments switch
};

namespace pned {
constexpr int kMaxBuffers = 6;
// device scalar slots, kMaxR doubles each
enum : int {
    kSlotOne = 0,   // all ones
    kSlotSc,        // scale of the current vector C
    kSlotPc,        // coefficient of the previous vector P in W
    kSlotGsc,       // scale of the vector G (TPS: previous vector)
    kSlotGscPrev,   // TPS: the scale G had before the last step (the W buffer holds that vector then)
    kScalSlots
};

struct DevObs {
    int n = 0;
    int *a = nullptr, *b = nullptr;
    double2 *c = nullptr, *T = nullptr;
};

// State of a Krylov session (see pned_session_begin).
struct Session {
    int kind = 0;              // 0: none; PNED_SESSION_*
    int max_steps = 0;
    int enqueued = 0;          // steps enqueued so far
    double L = 0.0;
    int b0 = 2, b1 = 3, b2 = 4;  // Lanczos: C, P, W;  TPS: C, W, G
    int nobs = 0, ncoef = 0;
    double *d_alpha = nullptr, *d_beta = nullptr, *d_coef = nullptr;
    int *d_counter = nullptr, *d_flag = nullptr;
    double2 *d_osum = nullptr;
    std::vector<DevObs> obs;
    std::vector<void *> allocs;
    cudaGraphExec_t graph = nullptr;
    int g0 = -1, g1 = -1, g2 = -1;  // buffer roles when the graph was captured
    int period = 2;
    cudaEvent_t ev_hv0 = nullptr, ev_hv1 = nullptr;  // set while profiling: events around the H.v kernel
};
}  // namespace pned

struct pned_ctx {
    pned_model *m = nullptr;
    int R = 1;
    size_t budget = 0, bytes = 0;
    int nsm = 148, nblocks = 1;
    cudaStream_t stream = nullptr, own_stream = nullptr;
    double2 *buf[pned::kMaxBuffers] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    double2 *partials = nullptr;   // [nblocks][kMaxK][kMaxR], or per-tile sums of the single-vector tile kernel
    int64_t partials_cap = 0;      // double2 slots at `partials`
    uint32_t *tile_ctr = nullptr;  // [kTileMaxPasses] tile counters of the dynamic tile order
    double2 *sums = nullptr;       // [4][kMaxK*kMaxR]
    double *scal = nullptr;        // [kScalSlots][kMaxR]
    int *flag = nullptr;
    double2 *h_sums = nullptr;     // pinned mirror of sums
    pned::Session sess;
};

namespace pned {

// cp.async (Ampere-style asynchronous global -> shared copies, 16 bytes a thread).
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Bulk-copy staging of the single-vector tile kernel: tiles of 2^kBulkJB
// states a thread, up to kBulkMaxStages ring stages.
constexpr int kBulkJB = 3;
constexpr int kBulkTile = kThreads << kBulkJB;   // 2048 states, 32 KB
constexpr int kBulkMaxStages = 8;
constexpr int kBulkHead = 256;                   // bytes before the ring: mbarriers and bookkeeping
constexpr int kBulkMinRunBits = 3;               // copies of at least 8 states (128 B)

int cuda_fail(cudaError_t e, const char *what);
int ctx_alloc_buffer(pned_ctx *c, int k);
int stage_in(pned_ctx *c, const pned_c128 *src, int flags, int k, const double2 **dev);
int sums_to_host(pned_ctx *c, int KR);
int check_kernel_flag(pned_ctx *c);
double *slot(pned_ctx *c, int s);
int set_slot(pned_ctx *c, int s, double value);
int pick_vpt(int R);
void session_release(pned_ctx *c);

cudaError_t launch_hv(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st);
// Raises a kernel's dynamic shared memory limit to 200 KB (once per kernel and device).
cudaError_t allow_dynamic_smem(const void *kern, int device);
// Device chosen by pned_set_device on this host thread.
int current_device();
// Plans the tiled single-vector passes of m->hp (S = 1/2, n >= 12) and sets m->use_tile.
void build_tile_programs(pned_model *m);
// Plans the tiled multi-vector passes for R vectors (S = 1/2, n >= 12, R > 1),
// once per model and R (again when `plan` is given); returns false when the
// flat kernel is used instead.
bool ensure_rtiles(pned_model *m, int R, bool slot_tables, const pned_tile_plan *plan);
// Shared memory of the tiled multi-vector kernel for R vectors.
size_t rtile_smem(const pned_model *m, int R, bool slot_tables);
bool ensure_qtiles(pned_model *m, int R);
// Tile set of the mixed-radix tiled kernel for R (null: the flat kernel runs).
const pned_model::QTileSet *find_qtiles(const pned_model *m, int R);
// Resident-block grid of the mixed-radix tiled kernel.
int qtile_grid(const pned_model *m, const pned_model::QTileSet &qs, int nblocks);
// All passes of the mixed-radix tiled kernel for a.R vectors and a.K sums.
cudaError_t launch_qtile(const pned_model *m, const pned_model::QTileSet &qs, const HvArgs &a, int nblocks,
                         cudaStream_t st);
// Persistent grid of the single-vector tiled kernels (all resident blocks).
int tile_grid(const pned_model *m, int nblocks);
// Sets a kernel's shared-memory carveout to what `blocks` blocks of `smem` bytes need.
cudaError_t set_carveout(const void *kern, int device, size_t smem, int blocks);
// Segment table of an S = 1/2 sector model (left empty where the flat gather is used).
cudaError_t build_sector_segments(pned_model *m);
inline bool sector_segments_on(const pned_model *m) { return m->nseg > 0 && m->seg_enabled; }
// Resident-block grid of the sector segment kernel.
int sector_grid(const pned_model *m, int nblocks);
// Sector H.v for one vector over segments (a.* Lin fields set).
cudaError_t launch_sector(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st);
// True when the plan runs a staged variant of the single-vector tile kernel.
inline bool tile_staged(const pned_model *m) { return m->tile_stage == 2 || (m->tile_stage == 1 && m->tile_jb == 3); }
// Stage 3 (tile kernel with tensor copies): the driver's tensor-map encoder (null: unavailable),
// a pass's copy geometry, the kernel's dynamic shared memory, whether a call's vectors suit the
// copies (16-byte aligned), and the launch.
void *tile_tma_encoder();
bool tile_tma_geometry(const TileProgram &p, TmaGeom &g);
size_t tile_tma_smem(const pned_model *m);
bool tile_tma_usable(const pned_model *m, const HvArgs &a);
cudaError_t launch_tile_tma(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st);
// All passes of the staged single-vector tile kernel (cp.async or bulk copies).
cudaError_t launch_tile_staged(const pned_model *m, const HvArgs &a, int nblocks, cudaStream_t st);
// Number of partial-sum blocks launch_hv writes for this model, R and grid
// (static tile order).
int hv_partial_blocks(const pned_model *m, int R, int nblocks);
// Tiles of all passes of the single-vector tile plan (the per-tile sums of the dynamic order).
int64_t tile_dynamic_partials(const pned_model *m);
// Tiles per chunk and chunks of one multi-vector pass on a grid, and the chunks of
// all passes for R vectors (the per-chunk sums of the dynamic order; 0: no
// multi-vector plan).
int64_t rtile_chunk_tiles(const TileProgram &t, int grid);
int64_t rtile_chunks(const TileProgram &t, int grid);
int64_t rtile_dynamic_partials(const pned_model *m, int R, int nblocks);
// True when launch_hv runs a tile kernel in dynamic tile order for these
// arguments (tile counters given and room for the per-tile or per-chunk sums).
bool tile_dynamic(const pned_model *m, const HvArgs &a, int nblocks);
// Partial sums launch_hv writes for these arguments (per tile or per block).
int64_t hv_partials(const pned_model *m, const HvArgs &a, int nblocks);
// The context's tile counters and partial-sum capacity into a.
inline void ctx_tile_args(const pned_ctx *c, HvArgs &a)
{
    a.tile_counter = c->tile_ctr;
    a.partials_cap = c->partials_cap;
}
cudaError_t launch_finish(const double2 *partials, int nb, int KR, double2 *out, cudaStream_t st);
cudaError_t launch_dot(const pned_ctx *c, const double2 *x1, const double2 *x2, const double2 *alpha, int mode,
                       double2 *out, cudaStream_t st);
cudaError_t launch_residual(const pned_ctx *c, const double2 *W, const double2 *C, double2 *Rn, const double *sc,
                            const double2 *alpha, cudaStream_t st);
cudaError_t launch_gaussian(const pned_ctx *c, uint64_t seed, bool normalise, double2 *v, cudaStream_t st);

inline uint64_t splitmix64_host(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// 2 bits per base-q digit (q <= 4), digit j at bits 2j..2j+1.
__device__ __forceinline__ uint64_t pack_digits(int64_t s, int n, int q)
{
    uint64_t r = 0;
    uint64_t x = uint64_t(s);
    if (q == 3) {
        for (int j = 0; j < n; ++j) {
            const uint64_t y = x / 3u;
            r |= (x - 3u * y) << (2 * j);
            x = y;
        }
    } else {
        for (int j = 0; j < n; ++j) {
            const uint64_t y = x / uint64_t(q);
            r |= (x - uint64_t(q) * y) << (2 * j);
            x = y;
        }
    }
    return r;
}
__device__ __forceinline__ int digit_at(uint64_t digits, int j) { return int((digits >> (2 * j)) & 3u); }

// Block-level reduction of red[K][VPT] (vector r = g*vpt + j, or g + j*G when
// STRIDED; g = lane % G, G a power of two dividing 32) into
// partials[slot][K][R] (slot < 0: blockIdx.x).
// Block sum of one vector's K sums (lanes, then warps, in a fixed order) into
// dst[0 .. K-1]; the thread's sums are reset.  All threads of the block call it.
template <int K>
__device__ __forceinline__ void tile_sums_store(double2 (&red)[K][1], double2 (*s_red)[K], double2 *dst)
{
    const uint32_t tid = threadIdx.x;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        for (int off = 16; off >= 1; off >>= 1) {
            red[k][0].x += __shfl_xor_sync(0xffffffffu, red[k][0].x, off);
            red[k][0].y += __shfl_xor_sync(0xffffffffu, red[k][0].y, off);
        }
        if ((tid & 31u) == 0) s_red[tid >> 5][k] = red[k][0];
        red[k][0] = make_double2(0.0, 0.0);
    }
    __syncthreads();
    if (tid < uint32_t(K)) {
        double2 sum = make_double2(0.0, 0.0);
        for (int w = 0; w < kThreads / 32; ++w) sum = cadd(sum, s_red[w][tid]);
        dst[tid] = sum;
    }
}

template <int K, int VPT, bool STRIDED = false>
__device__ __forceinline__ void block_reduce_store(double2 (&red)[K][VPT], int G, int vpt, int R, double2 *partials,
                                                   int64_t slot = -1)
{
    const size_t sl = slot < 0 ? size_t(blockIdx.x) : size_t(slot);
    __shared__ double2 sm[kThreads / 32][kMaxK][kMaxR];
    for (int off = 16; off >= G; off >>= 1)
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int j = 0; j < VPT; ++j) {
                red[k][j].x += __shfl_xor_sync(0xffffffffu, red[k][j].x, off);
                red[k][j].y += __shfl_xor_sync(0xffffffffu, red[k][j].y, off);
            }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane < G)
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int j = 0; j < VPT; ++j)
                if (j < vpt) sm[warp][k][STRIDED ? lane + j * G : lane * vpt + j] = red[k][j];
    __syncthreads();
    const int nw = blockDim.x >> 5;
    for (int idx = threadIdx.x; idx < K * R; idx += blockDim.x) {
        const int k = idx / R, r = idx - k * R;
        double2 s = make_double2(0.0, 0.0);
        for (int w = 0; w < nw; ++w) s = cadd(s, sm[w][k][r]);
        partials[(sl * K + k) * R + r] = s;
    }
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// Element g of the seeded complex Gaussian stream (key = splitmix64(seed ^
// 0x5DEECE66D)): Box-Muller on two counter hashes, sqrt(-ln u1) e^{2 pi i u2}.
__device__ __forceinline__ double2 gaussian_at(uint64_t key, int64_t g)
{
    const uint64_t h1 = splitmix64(key ^ uint64_t(2 * g));
    const uint64_t h2 = splitmix64(key ^ uint64_t(2 * g + 1));
    const double u1 = (double(h1 >> 11) + 0.5) * 0x1.0p-53;
    const double u2 = double(h2 >> 11) * 0x1.0p-53;
    const double rad = sqrt(-log(u1));
    const double ang = 2.0 * 3.14159265358979323846 * u2;
    return make_double2(rad * cos(ang), rad * sin(ang));
}

// Common epilogue of the H.v kernels: writes W and accumulates the fused sums.
template <int K, int VPT>
__device__ __forceinline__ void hv_epilogue(const HvArgs &a, int64_t s, int r0, const double2 (&v)[VPT],
                                            const double2 (&acc)[VPT], const double (&scr)[VPT],
                                            const double (&pcr)[VPT], const double (&gsr)[VPT],
                                            double2 (&red)[K][VPT])
{
    const int R = a.R;
#pragma unroll
    for (int j = 0; j < VPT; ++j) {
        const int64_t e = s * R + r0 + j;
        const double2 hv = cscale(scr[j], acc[j]);
        double2 out = hv;
        if (a.P) {
            const double2 p = a.P[e];
            out.x = fma(pcr[j], p.x, out.x);
            out.y = fma(pcr[j], p.y, out.y);
        }
        a.W[e] = out;
        const double2 vv = cscale(scr[j], v[j]);
        red[0][j] = cadd(red[0][j], cconjmul(vv, hv));
        if (K >= 2) red[1][j].x += out.x * out.x + out.y * out.y;
        if (K >= 4) {
            if (a.G) {
                const double2 gv = cscale(gsr[j], a.G[e]);
                red[2][j] = cadd(red[2][j], cconjmul(gv, out));
                red[3][j] = cadd(red[3][j], cconjmul(gv, vv));
            }
        }
    }
}

}  // namespace pned
