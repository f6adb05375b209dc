// start.cpp -- runtime state, initialisation and geometry of the drop-in API.
//
// Entry points of the reference's include/start.h:30-87 (lib/start.c), kept
// with the same names and meaning for a single process. Where the reference
// prints and calls exit(1) (lib/start.c:118-140, 281-283, 1176-1179,
// 1285-1289), these record an error (plqcd_last_error) and return.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "internal.h"
#include "start.h"

extern "C" {
struct _PLQCD_GLOBAL_PARAMS plqcd_g;
}

namespace plqcd {

static thread_local int g_status = PLQCD_OK;
static thread_local char g_msg[1024] = "";

int set_error(int code, const char *fmt, ...) {
    g_status = code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof g_msg, fmt, ap);
    va_end(ap);
    if (getenv("PLQCD_VERBOSE")) fprintf(stderr, "plqcd: %s\n", g_msg);
    return code;
}

void clear_error() {
    g_status = PLQCD_OK;
    g_msg[0] = 0;
}

// Drop-in path teardown lives in dropin.cu.
void dropin_release();

}  // namespace plqcd

extern "C" const char *plqcd_last_error(void) { return plqcd::g_msg; }
extern "C" int plqcd_last_status(void) { return plqcd::g_status; }
extern "C" void plqcd_clear_error(void) { plqcd::clear_error(); }
extern "C" const char *plqcd_version(void) { return "plqcd-b200 0.1 (sm_100a)"; }

// ---------------------------------------------------------------------------
// geometry helpers (lib/start.c:1169-1343)
// ---------------------------------------------------------------------------

extern "C" int ipr(int n[]) {
    const int *p = plqcd_g.nprocs;
    for (int i = 0; i < 4; i++)
        if (n[i] < 0 || n[i] >= p[i]) {
            plqcd::set_error(PLQCD_ERR_ARG, "ipr: process coordinate %d = %d out of range", i, n[i]);
            return -1;
        }
    return n[0] + p[0] * (n[1] + p[1] * (n[2] + p[2] * n[3]));
}

extern "C" void comp_cpr(int ip, int n[]) {
    const int *p = plqcd_g.nprocs;
    int np = p[0] * p[1] * p[2] * p[3];
    if (ip < 0 || ip >= np) {
        plqcd::set_error(PLQCD_ERR_ARG, "comp_cpr: process id must be 0 <= ip < %d", np);
        return;
    }
    n[0] = ip % p[0];
    n[1] = (ip / p[0]) % p[1];
    n[2] = (ip / p[0] / p[1]) % p[2];
    n[3] = (ip / p[0] / p[1] / p[2]) % p[3];
}

extern "C" void set_npr(void) {
    int n[4];
    for (int mu = 0; mu < 4; mu++) n[mu] = plqcd_g.cpr[mu];
    for (int mu = 0; mu < 4; mu++) {
        int np = plqcd_g.nprocs[mu];
        n[mu] = (plqcd_g.cpr[mu] - 1 + np) % np;
        plqcd_g.npr[2 * mu] = ipr(n);
        n[mu] = (plqcd_g.cpr[mu] + 1) % np;
        plqcd_g.npr[2 * mu + 1] = ipr(n);
        n[mu] = plqcd_g.cpr[mu];
    }
}

extern "C" void lex2cart(int ix, int xcart[]) {
    const int *L = plqcd_g.latdims;
    if (ix < 0 || ix >= plqcd_g.VOLUME) {
        plqcd::set_error(PLQCD_ERR_ARG, "lex2cart: index %d outside 0 <= ix < VOLUME", ix);
        return;
    }
    xcart[0] = ix % L[0];
    xcart[1] = (ix / L[0]) % L[1];
    xcart[2] = (ix / L[0] / L[1]) % L[2];
    xcart[3] = (ix / L[0] / L[1] / L[2]) % L[3];
}

extern "C" int cart2lex(int xcor[]) {
    const int *L = plqcd_g.latdims;
    for (int i = 0; i < 4; i++)
        if (xcor[i] < 0 || xcor[i] >= L[i]) {
            plqcd::set_error(PLQCD_ERR_ARG, "cart2lex: coordinate %d = %d out of bounds", i, xcor[i]);
            return -1;
        }
    return xcor[0] + L[0] * (xcor[1] + L[1] * (xcor[2] + L[2] * xcor[3]));
}

extern "C" void find_site(int xg[], int *pid, int *xeo) {
    int xc[4], pc[4];
    *pid = -1;
    *xeo = -1;
    for (int mu = 0; mu < 4; mu++) {
        if (xg[mu] < 0 || xg[mu] >= plqcd_g.nprocs[mu] * plqcd_g.latdims[mu]) {
            plqcd::set_error(PLQCD_ERR_ARG, "find_site: global coordinate %d out of bounds", mu);
            return;
        }
        pc[mu] = xg[mu] / plqcd_g.latdims[mu];
        xc[mu] = xg[mu] - pc[mu] * plqcd_g.latdims[mu];
    }
    int ilex = cart2lex(xc);
    *xeo = plqcd_g.ipt_eo[ilex];
    *pid = ipr(pc);
}

static void free_tables() {
    if (plqcd_g.iup) {
        free(plqcd_g.iup[0]);
        free(plqcd_g.iup);
    }
    if (plqcd_g.idn) {
        free(plqcd_g.idn[0]);
        free(plqcd_g.idn);
    }
    free(plqcd_g.ipt_eo);
    free(plqcd_g.ipt_lex);
    free(plqcd_g.ipt_eo_yzt);
    free(plqcd_g.ipt_lex_yzt);
    plqcd_g.iup = plqcd_g.idn = nullptr;
    plqcd_g.ipt_eo = plqcd_g.ipt_lex = plqcd_g.ipt_eo_yzt = plqcd_g.ipt_lex_yzt = nullptr;
}

// Tables of lib/start.c:255-560 for one process: even/odd order with the
// parity taken from the sum of global coordinates, periodic neighbours.
// iup/idn are arrays of row pointers into one contiguous block, so
// iup[i][mu] indexing works as in the reference.
static int build_tables() {
    const int *L = plqcd_g.latdims;
    long V = (long)L[0] * L[1] * L[2] * L[3];
    if (V > 0x7fffffffL) return plqcd::set_error(PLQCD_ERR_ARG, "set_geometry: volume exceeds int range");
    free_tables();
    plqcd_g.VOLUME = (int)V;
    plqcd_g.Vsse_split = (int)(V / 2);
    plqcd_g.Vavx_split = (int)(V / 4);
    plqcd_g.Vmic_split = (int)(V / 8);
    for (int mu = 0; mu < 4; mu++) {
        plqcd_g.face[mu] = 0;  // one process: no boundaries (lib/start.c:295-317)
        plqcd_g.nn_bnde[2 * mu] = plqcd_g.nn_bnde[2 * mu + 1] = nullptr;
        plqcd_g.nn_bndo[2 * mu] = plqcd_g.nn_bndo[2 * mu + 1] = nullptr;
    }
    plqcd_g.ipt_eo = (int *)malloc(sizeof(int) * V);
    plqcd_g.ipt_lex = (int *)malloc(sizeof(int) * V);
    plqcd_g.iup = (int **)malloc(sizeof(int *) * V);
    plqcd_g.idn = (int **)malloc(sizeof(int *) * V);
    int *up = (int *)malloc(sizeof(int) * 4 * V);
    int *dn = (int *)malloc(sizeof(int) * 4 * V);
    long Vyzt = (long)L[1] * L[2] * L[3];
    plqcd_g.ipt_eo_yzt = (int *)malloc(sizeof(int) * Vyzt);
    plqcd_g.ipt_lex_yzt = (int *)malloc(sizeof(int) * Vyzt);
    if (!plqcd_g.ipt_eo || !plqcd_g.ipt_lex || !plqcd_g.iup || !plqcd_g.idn || !up || !dn ||
        !plqcd_g.ipt_eo_yzt || !plqcd_g.ipt_lex_yzt) {
        free(up);
        free(dn);
        free_tables();
        return plqcd::set_error(PLQCD_ERR_NOMEM, "set_geometry: insufficient host memory");
    }
    for (long i = 0; i < V; i++) {
        plqcd_g.iup[i] = up + 4 * i;
        plqcd_g.idn[i] = dn + 4 * i;
    }
    long ce = 0, co = V / 2;
    const int *cpr = plqcd_g.cpr;
    for (long ix = 0; ix < V; ix++) {
        int x0 = ix % L[0], x1 = (ix / L[0]) % L[1], x2 = (ix / L[0] / L[1]) % L[2],
            x3 = (int)(ix / L[0] / L[1] / L[2]);
        int gsum = x0 + x1 + x2 + x3 + cpr[0] * L[0] + cpr[1] * L[1] + cpr[2] * L[2] + cpr[3] * L[3];
        long e = (gsum % 2 == 0) ? ce++ : co++;
        plqcd_g.ipt_eo[ix] = (int)e;
        plqcd_g.ipt_lex[e] = (int)ix;
    }
    for (long i = 0; i < V; i++) {
        int ix = plqcd_g.ipt_lex[i];
        int x[4] = {ix % L[0], (ix / L[0]) % L[1], (ix / L[0] / L[1]) % L[2], ix / L[0] / L[1] / L[2]};
        for (int mu = 0; mu < 4; mu++) {
            int y[4] = {x[0], x[1], x[2], x[3]};
            y[mu] = (x[mu] + 1) % L[mu];
            plqcd_g.iup[i][mu] = plqcd_g.ipt_eo[y[0] + L[0] * (y[1] + L[1] * (y[2] + L[2] * y[3]))];
            y[mu] = (x[mu] + L[mu] - 1) % L[mu];
            plqcd_g.idn[i][mu] = plqcd_g.ipt_eo[y[0] + L[0] * (y[1] + L[1] * (y[2] + L[2] * y[3]))];
        }
    }
    // y,z,t block order (lib/start.c:528-560)
    long ye = 0, yo = Vyzt / 2;
    for (int t = 0; t < L[3]; t++)
        for (int z = 0; z < L[2]; z++)
            for (int y = 0; y < L[1]; y++) {
                long il = y + (long)z * L[1] + (long)t * L[1] * L[2];
                long e = ((y + z + t) % 2 == 0) ? ye++ : yo++;
                plqcd_g.ipt_eo_yzt[il] = (int)e;
                plqcd_g.ipt_lex_yzt[e] = (int)il;
            }
    return PLQCD_OK;
}

extern "C" void set_geometry(void) {
    int g[4] = {plqcd_g.LX, plqcd_g.LY, plqcd_g.LZ, plqcd_g.LT};
    for (int i = 0; i < 4; i++) {
        int np = plqcd_g.nprocs[i] > 0 ? plqcd_g.nprocs[i] : 1;
        int l = g[i] / np;
        if (l * np != g[i] || l < 4 || (l % 2) != 0) {
            plqcd::set_error(PLQCD_ERR_ARG,
                             "set_geometry: local extent in direction %d must divide evenly, be >= 4 and even", i);
            return;
        }
        plqcd_g.latdims[i] = l;
    }
    build_tables();
}

// ---------------------------------------------------------------------------
// init / finalize (lib/start.c:19-247)
// ---------------------------------------------------------------------------

extern "C" int init_plqcd(int argc, char *argv[]) {
    plqcd::clear_error();
    if (argc < 2 || !argv || !argv[1])
        return plqcd::set_error(PLQCD_ERR_ARG, "init_plqcd: must pass the input file name as argv[1]");
    if (plqcd_g.init == 1) return 0;  // already initialised (lib/start.c:60-61)

    FILE *fp = fopen(argv[1], "r");
    if (!fp) return plqcd::set_error(PLQCD_ERR_ARG, "init_plqcd: cannot open input file %s", argv[1]);
    int nprocs[4] = {1, 1, 1, 1}, nthread = 1, L[4] = {4, 4, 4, 4}, align = 16;
    char var[128], val[128];
    while (fscanf(fp, "%127s %127s", var, val) == 2) {
        if (!strcmp(var, "NPROC0")) nprocs[0] = atoi(val);
        else if (!strcmp(var, "NPROC1")) nprocs[1] = atoi(val);
        else if (!strcmp(var, "NPROC2")) nprocs[2] = atoi(val);
        else if (!strcmp(var, "NPROC3")) nprocs[3] = atoi(val);
        else if (!strcmp(var, "NTHREAD")) nthread = atoi(val);
        else if (!strcmp(var, "L0")) L[0] = atoi(val);
        else if (!strcmp(var, "L1")) L[1] = atoi(val);
        else if (!strcmp(var, "L2")) L[2] = atoi(val);
        else if (!strcmp(var, "L3")) L[3] = atoi(val);
        else if (!strcmp(var, "ALIGN")) align = atoi(val);
    }
    fclose(fp);

    for (int i = 0; i < 4; i++)
        if (L[i] < 4 || (L[i] % 2) != 0)
            return plqcd::set_error(PLQCD_ERR_ARG,
                                    "init_plqcd: global lattice dimension in each direction must be >= 4 and even");
    for (int i = 0; i < 4; i++)
        if (nprocs[i] < 1 || (nprocs[i] > 1 && (nprocs[i] % 2) != 0))
            return plqcd::set_error(PLQCD_ERR_ARG, "init_plqcd: processes per direction must be 1 or even");
    if (nprocs[0] * nprocs[1] * nprocs[2] * nprocs[3] != 1)
        return plqcd::set_error(PLQCD_ERR_ARG,
                                "init_plqcd: the GPU library runs one process per lattice; NPROC0..3 must be 1");
    if (align < 0 || align > 30) return plqcd::set_error(PLQCD_ERR_ARG, "init_plqcd: ALIGN out of range");

    for (int i = 0; i < 4; i++) plqcd_g.nprocs[i] = nprocs[i];
    plqcd_g.nthread = nthread > 0 ? nthread : 1;
    plqcd_g.LX = L[0];
    plqcd_g.LY = L[1];
    plqcd_g.LZ = L[2];
    plqcd_g.LT = L[3];
    plqcd_g.ALIGN = align;
    for (int i = 0; i < 4; i++) {
        plqcd_g.phip[i] = nullptr;
        plqcd_g.phim[i] = nullptr;
    }
    comp_cpr(0, plqcd_g.cpr);
    set_npr();
    plqcd::clear_error();
    set_geometry();
    if (plqcd_last_status() != PLQCD_OK) return plqcd_last_status();
    plqcd_g.init = 1;
    return 0;
}

extern "C" void finalize_plqcd(void) {
    plqcd::dropin_release();
    free_tables();
    plqcd_g.init = 0;
}

// ---------------------------------------------------------------------------
// print_params (lib/start.c:1351-1428; same text layout)
// ---------------------------------------------------------------------------

extern "C" void print_params(FILE *fp) {
    if (!fp) return;
    fprintf(fp, "grid of processes: nprocs0 %d nprocs1 %d nprocs2 %d nprocs3 %d\n\n", plqcd_g.nprocs[0],
            plqcd_g.nprocs[1], plqcd_g.nprocs[2], plqcd_g.nprocs[3]);
    fprintf(fp, "Number of openmp threads %d\n\n", plqcd_g.nthread);
    fprintf(fp, "Cartesian co-ordinates of my process on the grid of processes: %d %d %d %d\n\n", plqcd_g.cpr[0],
            plqcd_g.cpr[1], plqcd_g.cpr[2], plqcd_g.cpr[3]);
    fprintf(fp,
            "Nearst neighbours of my process (-0 +0 -1 +1 -2 +2 -3 +3): %10d %10d %10d %10d %10d %10d %10d %10d \n\n",
            plqcd_g.npr[0], plqcd_g.npr[1], plqcd_g.npr[2], plqcd_g.npr[3], plqcd_g.npr[4], plqcd_g.npr[5],
            plqcd_g.npr[6], plqcd_g.npr[7]);
    fprintf(fp, "Global lattice size: LX %d LY %d LZ %d LT %d\n\n", plqcd_g.LX, plqcd_g.LY, plqcd_g.LZ, plqcd_g.LT);
    fprintf(fp, "Local lattice size: lx %d ly %d lz %d lt %d, local volume %d\n\n", plqcd_g.latdims[0],
            plqcd_g.latdims[1], plqcd_g.latdims[2], plqcd_g.latdims[3], plqcd_g.VOLUME);
    fprintf(fp, "Sizes of the boundaries: 0-boundary %d 1-boundary %d 2-boundary %d 3-boundary %d\n\n",
            plqcd_g.face[0], plqcd_g.face[1], plqcd_g.face[2], plqcd_g.face[3]);
    fprintf(fp, "printing the lattice sites w.r.t. the local lattice:\n\n");
    fprintf(fp, "%8s %8s %8s %8s %8s %8s %8s %8s %8s %8s %8s %8s %8s %8s\n\n", "x0", "x1", "x2", "x3", "ipt_eo",
            "ipt_lex", "iup[0]", "iup[1]", "iup[2]", "iup[3]", "idn[0]", "idn[1]", "idn[2]", "idn[3]");
    if (plqcd_g.ipt_lex && plqcd_g.iup && plqcd_g.idn) {
        for (int ix = 0; ix < plqcd_g.VOLUME; ix++) {
            int x[4];
            int il = plqcd_g.ipt_lex[ix];
            lex2cart(il, x);
            fprintf(fp, "%8d %8d %8d %8d %8d %8d %8d %8d %8d %8d %8d %8d %8d %8d\n\n", x[0], x[1], x[2], x[3], ix, il,
                    plqcd_g.iup[ix][0], plqcd_g.iup[ix][1], plqcd_g.iup[ix][2], plqcd_g.iup[ix][3],
                    plqcd_g.idn[ix][0], plqcd_g.idn[ix][1], plqcd_g.idn[ix][2], plqcd_g.idn[ix][3]);
        }
    }
    fprintf(fp, "the nn_bnde and nn_bndo arrays\n");
    for (int d = 0; d < 4; d++) {
        // faces are empty for one process: only the headers are printed
        fprintf(fp, "nn_bnde[%d] \n", 2 * d);
        fprintf(fp, "nn_bndo[%d]\n", 2 * d);
        fprintf(fp, "nn_bnde[%d] \n", 2 * d + 1);
        fprintf(fp, "nn_bndo[%d]\n", 2 * d + 1);
    }
    fprintf(fp, "memory alignment in bytes: ALIGN %d\n\n", plqcd_g.ALIGN);
    fprintf(fp, "initialization check parameter: init %d\n\n", plqcd_g.init);
}
