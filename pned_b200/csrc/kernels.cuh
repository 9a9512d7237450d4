// Device kernels of libpned_gpu.so (sm_100a).  FP64 complex throughout.
//
// Vectors are interleaved [dim][R]: element (state s, vector r) at s*R + r.
// A thread owns one state and VPT consecutive vectors of it; G = R/VPT
// threads share a state.  All reductions are deterministic: a fixed grid
// writes per-block partial sums in a fixed order and one block finishes them.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pned_internal.h"

namespace pned {

constexpr int kThreads = 256;
constexpr int kMaxR = 16;
constexpr int kMaxK = 4;          // reduction quantities per vector in one pass
constexpr int kMaxVPT = 4;

struct __align__(16) dcplx { double x, y; };

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c)
{   // a*b + c
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ double2 cconjmul(double2 a, double2 b)
{   // conj(a) * b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }

// Term program passed by value as a kernel parameter (constant bank, uniform
// loads).  Coefficient tables live in global memory and are staged into
// shared memory per block.
struct XorProgram {
    int nterms;
    int ntab;
    XorTerm t[kMaxTerms];
};
struct RadixProgram {
    int nterms;
    int ntab;
    int n;
    RadixTerm t[kMaxTerms];
};

// Tiled mixed-radix pass (see QTileTerm): a tile is the q^k states with
// fixed outer digits; tile t's outer digits are t written in base q over
// outer[] (fastest first).
constexpr int kQTileMaxTab = 768;   // coefficient entries of one pass (its terms' tables only)
struct QTileProgram {
    int q, k, nt, nouter, nterms, ntab, first, last;
    int64_t ntiles;
    uint32_t spow[kQTileMaxSites];  // q^site of tile site i (q^n < 2^32)
    uint32_t opow[32];              // q^site of outer site i
    QTileTerm t[kMaxTerms];
    double2 tab[kQTileMaxTab];      // the pass's coefficient tables
};

// Tiled single-vector S = 1/2 program (see TileTerm).
struct TileProgram {
    int n, tbits, jb, nin, nterms, ntab, nouter;
    int first, last;                  // pass flags: first adds diagonal and P, last forms the K >= 2 sums
    int pass;                         // index of the pass (its tile counter under dynamic tile order)
    uint32_t jexp[1 << kTileMaxJB];   // global bits of the thread's j-th state
    uint8_t rowpos[8];                // row bit k -> global bit rowpos[k]
    uint8_t outer[32];                // tile-id bit k -> global bit outer[k]
    int ngroups;                      // out-of-tile groups, one partner tile each
    uint16_t gstart[kTileMaxGroups + 1];
    uint32_t gxor[kTileMaxGroups];
    TileTerm t[kMaxTerms];
};

// Tensor-copy geometry of a single-vector tile (a pass's rows and j bits, in
// ascending global bit order, as the tile is laid out in shared memory): the
// global bits split into up to 5 copy dimensions, each a run of bits, either
// all tile bits (copied whole) or all outer bits (one position, the tile's).
// Dimension 0 starts at bit 0 and holds at most 7 bits (a box row of at most
// 256 doubles of complex data), the other tile runs at most 8.
constexpr int kTmaMaxRank = 5;
struct TmaGeom {
    int rank = 0;
    int lo[kTmaMaxRank] = {};      // lowest global bit of the dimension
    int nbits[kTmaMaxRank] = {};   // its bits
    int tile[kTmaMaxRank] = {};    // 1: tile bits (box spans it), 0: outer bits (box of 1)
};

// Per-call scalars: W = pc_r * P + sc_r * (H - shift) (sc_r * C); all from device memory.
struct HvArgs {
    const double2 *C;       // input vectors (scaled by sc)
    const double2 *P;       // optional added vector (may alias W), scaled by pc
    double2 *W;             // output
    const double *sc;       // [R] scale of C
    const double *pc;       // [R] coefficient of P (nullptr: no P term)
    const void *diag;       // diagonal (double or double2 per state)
    double shift;           // eperbd * n_bonds subtracted from the diagonal
    const double2 *table;   // coefficient table (global)
    double2 *partials;      // [nblocks][K][R]
    const double2 *G;       // optional previous vector (TPS: vg) scaled by gsc
    const double *gsc;      // [R]
    int64_t dim;
    int R;
    int K;                  // 1: alpha; 2: alpha, ||W||^2; 4: + <G|W>, <G|C>
    int *err;               // set to 1 by a kernel whose bounded wait gave up (may be null)
    // tiled single-vector kernel only (slot batches): per-call scale of the H part
    // (null: sc) and an extra diagonal shift (null: none)
    const double *hsc;
    const double *shiftv;
    // tiled multi-vector kernel only: per-vector coefficient tables ([ntab][R])
    // and real diagonals ([dim][R]) instead of shared ones
    int slot_tables;
    // tiled single-vector kernel only: per-pass tile counters, zeroed before the
    // passes; when set, blocks take tiles in order from the counter (all blocks
    // stay on neighbouring tiles, so the L2 window holds) and the sums are
    // written per tile ([tile][K]) instead of per block.  Null: the static
    // order (tile = block + k * grid) with per-block sums.
    uint32_t *tile_counter;
    int64_t partials_cap;   // double2 slots available at `partials` (per-tile sums need sum(tiles) * K)
    int rv_chunk;           // multi-vector kernel, dynamic order: tiles per chunk (set by the launcher)
    // Sz sector (set by launch_hv from the model): index -> state, and the Lin
    // tables, state -> index = lin_lo[state mod lin_mod] + lin_hi[state / lin_mod] - 1
    const int64_t *list1;
    const int64_t *lin_lo;
    const int64_t *lin_hi;
    int64_t lin_mod;
    int lin_pow2;           // log2(lin_mod) + 1 when lin_mod is a power of two (q = 2, 4), else 0
};

// Sector index of a state (the reference's list_lib lookup).
__device__ __forceinline__ int64_t lin_index(const HvArgs &a, uint64_t st)
{
    if (a.lin_pow2 > 0) {   // shift and mask
        const int sh = a.lin_pow2 - 1;
        return a.lin_lo[st & ((uint64_t(1) << sh) - 1)] + a.lin_hi[st >> sh] - 1;
    }
    if ((st >> 32) == 0) {   // 32-bit division (q^n < 2^32)
        const uint32_t s32 = uint32_t(st), m = uint32_t(a.lin_mod), hi = s32 / m;
        return a.lin_lo[s32 - hi * m] + a.lin_hi[hi] - 1;
    }
    return a.lin_lo[st % uint64_t(a.lin_mod)] + a.lin_hi[st / uint64_t(a.lin_mod)] - 1;
}

}  // namespace pned
