// tile_order.cuh -- the order in which the persistent TMA hop kernels
// (dslash_tma.cu) take their tiles, and its default blocking per kind of
// launch. Host and device code share it, so the host test of the mapping
// (tests/c/tile_order.cpp) checks the code the kernels run.
//
// A tile is NY rows (y0 .. y0+NY-1) of one (z, t) line of one output parity;
// RHS-tile launches add the first RHS r0 of a group of nr RHS. Tiles are
// numbered y-tile fastest, then z and t inside a block of bz z-lines x bt
// t-slices, then the blocks (z-blocks inner); in front of that the parity
// (full lattice: the two parities of a tile run back to back) or the RHS
// group (RHS tiles: the groups of the same rows run back to back).
#pragma once

#ifdef __CUDACC__
#define PLQCD_TILE_FN __host__ __device__ __forceinline__
#else
#define PLQCD_TILE_FN inline
#endif

namespace plqcd {
namespace dev {

struct TileCoord {
    int p, y0, zt, z, t;
    int r0;  // first RHS of the tile (RHS tiles; 0 otherwise)
};

// Tile `item` of a launch described by g (fields full, out_parity, nr, ngr,
// NY, nty = L1 / NY, bz, bt, L2, t0). MR: RHS tiles.
template <bool MR = false, class G>
PLQCD_TILE_FN TileCoord tile_coord(const G &g, int item) {
    TileCoord c;
    int tile;
    c.r0 = 0;
    if constexpr (MR) {
        c.p = g.out_parity;
        const int grp = item % g.ngr;
        c.r0 = grp * g.nr;
        tile = item / g.ngr;
    } else if (g.full) {
        c.p = item & 1;
        tile = item >> 1;
    } else {
        c.p = g.out_parity;
        tile = item;
    }
    // y-tiles fastest, then z and t inside a (bz x bt) block, then the
    // blocks (z-blocks inner): a block's z and t neighbours are read while
    // they are still in L2
    int k = tile / g.nty;
    c.y0 = (tile - k * g.nty) * g.NY;
    const int zin = k % g.bz;
    k /= g.bz;
    const int tin = k % g.bt;
    k /= g.bt;
    const int nbz = g.L2 / g.bz;
    c.z = (k % nbz) * g.bz + zin;
    c.t = g.t0 + (k / nbz) * g.bt + tin;
    c.zt = c.z + g.L2 * c.t;
    return c;
}

enum TileLaunch { kTileParity = 0, kTileFull = 1, kTileRhs = 2 };

// Default (bz, bt) block for tc t-slices of an L2-line lattice:
// - one parity of one field: all of z x 4 (or 2, 1) t-slices; the t
//   neighbours of a slice are at most a few waves of tiles old (FP64 at
//   32^3x64, 16-row tiles: 829 DRAM read bytes per site against 866 for
//   8 x 8 blocks);
// - full lattice: half of z x all t-slices (FP64 at 32^3x64, 2216: 448.5
//   against 459.2 us per launch for the above, ten interleaved rounds);
// - RHS tiles: a quarter of z x all t-slices (several RHS per tile make a
//   t-slice of whole z lines tens of MB; 32^3x64 / 8 RHS 1630 against 1731
//   us, 16^3x32 / 32 RHS 363 against 385 us).
// Every default block divides its extent.
inline void tile_order_default(int launch, int L2, int tc, int *bz, int *bt) {
    if (launch == kTileFull) {
        *bz = L2 % 2 == 0 ? L2 / 2 : L2;
        *bt = tc;
    } else if (launch == kTileRhs) {
        *bz = L2 % 4 == 0 ? L2 / 4 : L2;
        *bt = tc;
    } else {
        *bz = L2;
        *bt = tc % 4 == 0 ? 4 : (tc % 2 == 0 ? 2 : 1);
    }
}

}  // namespace dev
}  // namespace plqcd
