// Host test of the persistent TMA kernels' tile order (tile_order.cuh, the
// code the kernels run): for every kind of launch, a range of lattice
// shapes, tile heights and (z, t) blocks, the default ones included, the
// items 0 .. nitems-1 must map onto the tiles one to one, every coordinate
// in range. A tile that no item reaches would leave output sites unwritten;
// one reached twice would be computed twice.
#include <cstdio>
#include <vector>

#include "tile_order.cuh"

using plqcd::dev::TileCoord;

struct Launch {
    int full, out_parity, nr, ngr, NY, nty, bz, bt, L2, t0;
};

static int failures = 0, checked = 0;

static void fail(const char *what, int L1, int L2, int tc, int ny, int bz, int bt, int item) {
    if (failures++ < 20)
        std::printf("FAIL %s: L1=%d L2=%d tc=%d NY=%d bz=%d bt=%d item=%d\n", what, L1, L2, tc, ny, bz, bt, item);
}

// one launch: full / parity / RHS tiles (mr), t-slices [t0, t0 + tc) of L3
template <bool MR>
static void check(int L1, int L2, int L3, int t0, int tc, int ny, int bz, int bt, int full, int par, int nr,
                  int ngr) {
    Launch g{full, par, nr, ngr, ny, L1 / ny, bz, bt, L2, t0};
    const long ntiles = (long)g.nty * L2 * tc;
    const int groups = MR ? ngr : (full ? 2 : 1);
    const long nitems = ntiles * groups;
    // seen[(group or parity) * ntiles + ((t - t0) * L2 + z) * nty + y0 / NY]
    std::vector<unsigned char> seen((size_t)nitems, 0);
    for (long item = 0; item < nitems; item++) {
        const TileCoord c = plqcd::dev::tile_coord<MR>(g, (int)item);
        const bool ok = c.y0 >= 0 && c.y0 + ny <= L1 && c.y0 % ny == 0 && c.z >= 0 && c.z < L2 && c.t >= t0 &&
                        c.t < t0 + tc && c.t < L3 && c.zt == c.z + L2 * c.t && c.p >= 0 && c.p <= 1 &&
                        (MR ? (c.r0 % nr == 0 && c.r0 >= 0 && c.r0 < nr * ngr && c.p == par)
                            : (c.r0 == 0 && (full || c.p == par)));
        if (!ok) {
            fail("coordinate out of range", L1, L2, tc, ny, bz, bt, (int)item);
            continue;
        }
        const long grp = MR ? c.r0 / nr : (full ? c.p : 0);
        const long idx = grp * ntiles + ((long)(c.t - t0) * L2 + c.z) * g.nty + c.y0 / ny;
        if (seen[(size_t)idx]++) fail("tile reached twice", L1, L2, tc, ny, bz, bt, (int)item);
    }
    for (size_t i = 0; i < seen.size(); i++)
        if (!seen[i]) {
            fail("tile never reached", L1, L2, tc, ny, bz, bt, (int)i);
            break;
        }
    checked++;
}

static std::vector<int> divisors(int n) {
    std::vector<int> d;
    for (int k = 1; k <= n; k++)
        if (n % k == 0) d.push_back(k);
    return d;
}

int main() {
    const int L1s[] = {4, 6, 8, 16, 24, 32};
    const int L2s[] = {4, 6, 8, 16, 24, 32};
    const int L3s[] = {4, 6, 10, 32, 48, 64};
    for (int L1 : L1s)
        for (int L2 : L2s)
            for (int L3 : L3s)
                for (int ny : divisors(L1)) {
                    if (ny > 16) continue;
                    // the default blocks of each kind of launch
                    for (int launch = 0; launch < 3; launch++) {
                        int bz = 0, bt = 0;
                        plqcd::dev::tile_order_default(launch, L2, L3, &bz, &bt);
                        if (L2 % bz || L3 % bt) {
                            fail("default block does not divide", L1, L2, L3, ny, bz, bt, -1);
                            continue;
                        }
                        if (launch == plqcd::dev::kTileRhs) {
                            for (int ngr : {1, 2, 3, 4}) check<true>(L1, L2, L3, 0, L3, ny, bz, bt, 0, 1, 4, ngr);
                        } else {
                            check<false>(L1, L2, L3, 0, L3, ny, bz, bt, launch == plqcd::dev::kTileFull, 0, 1, 1);
                            check<false>(L1, L2, L3, 0, L3, ny, bz, bt, 0, 1, 1, 1);
                        }
                    }
                    // every block the environment may set, on whole fields
                    // and on a range of t-slices (site-range launches)
                    if (L1 > 8 || L3 > 10) continue;
                    for (int bz : divisors(L2))
                        for (int bt : divisors(L3)) {
                            check<false>(L1, L2, L3, 0, L3, ny, bz, bt, 1, 0, 1, 1);
                            check<true>(L1, L2, L3, 0, L3, ny, bz, bt, 0, 0, 2, 3);
                        }
                    for (int t0 = 1; t0 < L3; t0++)
                        for (int bt : divisors(L3 - t0)) check<false>(L1, L2, L3, t0, L3 - t0, ny, L2, bt, 0, 1, 1, 1);
                }
    std::printf("%d launches checked, %d failures\n", checked, failures);
    return failures ? 1 : 0;
}
