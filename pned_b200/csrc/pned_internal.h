// Internal declarations shared by the host and device translation units of
// libpned_gpu.so.  Nothing here is part of the C ABI.
#pragma once

#include <complex>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/pned_gpu.h"

namespace pned {

using cd = std::complex<double>;

// Thread-local error message behind pned_last_error().
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);

// ---------------------------------------------------------------------------
// Compiled term program
// ---------------------------------------------------------------------------
constexpr int kMaxDeps = 4;      // dependency bits per xor term
constexpr int kMaxTerms = 640;   // gather terms per program (kernel parameter space)
constexpr int kMaxTable = 3072;  // coefficient-table entries (48 KB of shared memory)

// One gather term of the S = 1/2 (q = 2) program: partner = s ^ xmask,
// coefficient = table[tab + idx] with idx gathered from the `nb` dependency
// bits (pos packed 8 bits each, bit k of idx = bit pos_k of s).
struct XorTerm {
    uint32_t xmask;
    uint32_t pos4;
    uint16_t tab;
    uint8_t nb;
    uint8_t pad;
};

// One gather term of the mixed-radix (q > 2) program: partner = s + offset,
// coefficient = table[tab + d(s1) + q*d(s2)] (zero where the target digit
// leaves 0..q-1; the load is skipped for zero coefficients).
struct RadixTerm {
    int64_t offset;
    uint8_t s1, s2;
    uint16_t tab;
    uint32_t pad;
};

// Tiled S = 1/2 program (single vector): a tile is 2^(8+JB) states -- global
// bits 0..7 (one per thread of a 256-thread block) times the JB "j-bits" at
// global positions jpos (each thread owns 2^JB states) -- and the remaining
// "outer" bits enumerate tiles, outer[0] varying fastest.
struct TileTerm {
    uint32_t mask;   // in-tile: local xor (bits 0..7 thread part, bits 8.. j part); out-of-tile: global xor
    uint32_t pos4;   // dependency bit positions (global), 8 bits each
    uint64_t jtab;   // coefficient-index bits contributed by j (4 bits per j)
    uint16_t tab;    // coefficient table offset
    uint8_t nb;      // number of dependency bits
    uint8_t hasj;    // 1 if a dependency bit is a j-bit
    uint32_t lmask;  // out-of-tile: local xor of the mask's in-tile part (the offset inside the partner tile)
    uint8_t jdep;    // the coefficient-index bits that j sets (OR of the jtab nibbles)
};
// Tiled mixed-radix (q > 2) pass: the states that agree on all digits but
// those of the k tile sites form a tile of q^k states, staged in shared
// memory; a pass applies the terms of its bonds (both sites in the tile).
constexpr int kQTileMaxSites = 16;
constexpr int kQTileMaxPasses = 16;
struct QTileTerm {
    int32_t loff;    // partner offset inside the tile (local index)
    uint8_t ls1, ls2;   // local digit positions of the bond's sites
    uint16_t tab;    // coefficient table offset (q^2 entries by pair state)
};
constexpr int kTileMaxJB = 4;
constexpr int kTileWindowBits = 10;   // outer bits whose partner tiles stay in L2 during a sweep
constexpr int kTileBigSites = 26;     // from here on the single-vector plan defaults to the tensor-copy kernel
constexpr int kTileMaxPasses = 4;
constexpr int kTileMaxGroups = 64;    // partner tiles per pass

struct QTilePass {
    std::vector<int> sites;              // tile sites, ascending: local digit k is site sites[k]
    std::vector<int> outer;              // the other sites, ascending
    std::vector<QTileTerm> terms;
};

struct HostProgram {
    int n = 0, q = 2;
    int64_t dim = 0;                     // basis size: q^n, or the sector size
    // Sz sector (parity_type == 0): sector index -> state, and the Lin tables
    // (index = lin_lo[state mod q^ihf] + lin_hi[state / q^ihf] - 1)
    bool sector = false;
    int total = 0;                       // digit sum of the sector states (sector only)
    int ihf = 0;
    std::vector<int64_t> list1, lin_lo, lin_hi;
    int nbond = 0;
    bool real = true;                    // every coefficient and diagonal entry real
    std::vector<XorTerm> xterms;         // q == 2
    // per xor term: the (bond index, flip pattern f) contributions summed into its table
    std::vector<std::vector<std::pair<int, int>>> xcontrib;
    std::vector<int> bond_type;          // schedule-order bond types (1..9)
    std::vector<RadixTerm> rterms;       // q > 2
    std::vector<std::pair<int, int>> rdelta;   // per radix term: digit changes (d1, d2) of sites s1, s2
    std::vector<cd> table;               // coefficient tables
    // diagonal: per bond (s1, s2) and q*q diagonal values (pair state st)
    std::vector<int> dsite1, dsite2;
    std::vector<cd> dtab;                // [nbond][Q]
    // tiled program (q == 2): one or more passes, each with its own tile plan
    struct TilePass {
        int tbits = 8;                   // row bits of a tile (state rows of the thread index)
        std::vector<int> rowpos;         // global bit of row bit k (k < tbits)
        int jb = 0;
        int jpos[kTileMaxJB] = {};
        std::vector<int> outer;          // outer bit positions, fastest first
        int nin = 0;                     // in-tile terms first, then out-of-tile terms grouped by partner tile
        std::vector<TileTerm> tterms;
        std::vector<int> gstart;         // out-of-tile group g: terms gstart[g] .. gstart[g+1]-1
        std::vector<uint32_t> gxor;      // partner tile of group g: outer bits flipped by gxor[g]
    };
};

// Splits the flip masks into passes for the tiled kernels (q == 2,
// n >= tbits + jb + 1).  A tile holds the states that agree on all bits but
// its tbits row bits and jb j bits, chosen per pass to minimise the partner
// tiles (objective 0) or to hold the most masks (objective 1); the row bits include the global bits 0..fixed-1, so that a warp's
// loads come in contiguous segments.  Each pass takes the masks whose partner
// tiles lie within `window_bits` outer bits of its own tile order (so they are
// found in L2), the last pass takes what is left.  In-tile terms carry the
// local xor (row bits, then the j bits from bit tbits); out-of-tile terms the
// global one.
// Covers the bonds of a mixed-radix (q > 2, full basis) program with passes
// of k-site tiles, greedily: each pass takes the uncovered bonds inside a
// site set grown from the most connected uncovered bond (plus the `low`
// lowest sites, kept in every tile for contiguous runs of states).
int plan_qtiles(const HostProgram &P, int k, int low, std::vector<QTilePass> &passes);
int plan_tiles(const HostProgram &P, int tbits, int jb, int fixed, int window_bits, int max_passes,
               std::vector<HostProgram::TilePass> &out, int objective = 0);

// Coefficient tables and diagonal tables of `d` evaluated on the term
// structure of S (same lattice and bonds; q == 2): table[i] for the entries of
// S.table, dtab as S.dtab.  Terms that `d` lacks get zeros.
int eval_tables_on_structure(const HostProgram &S, const pned_model_desc *d, std::vector<cd> &table,
                             std::vector<cd> &dtab);

// Builds the program from a model description (bond order, skip mask and
// element order follow make_cpu_list2; see model.cpp).
int compile_program(const pned_model_desc *d, HostProgram &out);

}  // namespace pned
