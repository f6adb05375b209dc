/*
 * Setup helper linked into the compiled reference oracle (test
 * infrastructure only). init_plqcd (lib/start.c:19-232) reads an input file
 * and can run once per process; this helper performs the same single-rank
 * steps -- defaults, comp_cpr, set_npr, set_geometry, phip/phim allocation
 * (lib/start.c:76-81, 143-170) -- for given dimensions, so one process can
 * drive several lattice sizes. Tables of an earlier setup are released
 * first.
 */
#include "plqcd.h"

int oracle_ref_setup(int L0, int L1, int L2, int L3, int nthread)
{
    int i;
    if (plqcd_g.init) {
        for (i = 0; i < plqcd_g.VOLUME; i++) { free(plqcd_g.iup[i]); free(plqcd_g.idn[i]); }
        free(plqcd_g.iup); free(plqcd_g.idn);
        free(plqcd_g.ipt_eo); free(plqcd_g.ipt_lex);
        free(plqcd_g.ipt_eo_yzt); free(plqcd_g.ipt_lex_yzt);
        for (i = 0; i < plqcd_g.Vsse_split; i++) { free(plqcd_g.iup_sse_split[i]); free(plqcd_g.idn_sse_split[i]); }
        free(plqcd_g.iup_sse_split); free(plqcd_g.idn_sse_split);
        free(plqcd_g.ipt_eo_sse_split); free(plqcd_g.ipt_lex_sse_split);
        for (i = 0; i < 4; i++) { afree(plqcd_g.phip[i]); afree(plqcd_g.phim[i]); }
    }
    for (i = 0; i < 4; i++) plqcd_g.nprocs[i] = 1;
    plqcd_g.nthread = nthread;
    plqcd_g.LX = L0; plqcd_g.LY = L1; plqcd_g.LZ = L2; plqcd_g.LT = L3;
    plqcd_g.ALIGN = 6;
#ifdef _OPENMP
    omp_set_num_threads(nthread);
#endif
    comp_cpr(0, plqcd_g.cpr);
    set_npr();
    set_geometry();
    for (i = 0; i < 4; i++) {
        plqcd_g.phip[i] = (halfspinor *)amalloc((plqcd_g.VOLUME / 2 + plqcd_g.face[i]) * sizeof(halfspinor), plqcd_g.ALIGN);
        plqcd_g.phim[i] = (halfspinor *)amalloc((plqcd_g.VOLUME / 2 + plqcd_g.face[i]) * sizeof(halfspinor), plqcd_g.ALIGN);
        if (!plqcd_g.phip[i] || !plqcd_g.phim[i]) return -1;
    }
    plqcd_g.init = 1;
    return 0;
}

void oracle_ref_set_threads(int nthread)
{
    plqcd_g.nthread = nthread;
#ifdef _OPENMP
    omp_set_num_threads(nthread);
#endif
}

/* Copy the reference's geometry tables (lib/start.c:406-526) out of plqcd_g:
 * ipt_eo[V], ipt_lex[V], iup[4V], idn[4V] (index 4*i+mu). */
void oracle_ref_tables(int *ipt_eo, int *ipt_lex, int *iup, int *idn)
{
    int i, mu;
    for (i = 0; i < plqcd_g.VOLUME; i++) {
        ipt_eo[i] = plqcd_g.ipt_eo[i];
        ipt_lex[i] = plqcd_g.ipt_lex[i];
        for (mu = 0; mu < 4; mu++) {
            iup[4 * i + mu] = plqcd_g.iup[i][mu];
            idn[4 * i + mu] = plqcd_g.idn[i][mu];
        }
    }
}
