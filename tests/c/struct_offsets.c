/*
 * Prints sizeof and the offset of every member of struct _PLQCD_GLOBAL_PARAMS,
 * one "name value" line each. Compiled once against this library's
 * include/plqcd_global_params.h and once against the reference's
 * include/plqcd_global_params.h (its default build: no AVX_SPLIT, no MIC);
 * tests/test_boundary_c.py compares the two outputs, so an object file
 * built against either header reads plqcd_g at the same offsets.
 */
#include <stddef.h>
#include <stdio.h>
#include "plqcd_global_params.h"

#define OFF(m) printf("%s %zu\n", #m, offsetof(struct _PLQCD_GLOBAL_PARAMS, m))

int main(void) {
    printf("sizeof %zu\n", sizeof(struct _PLQCD_GLOBAL_PARAMS));
    OFF(nprocs);
    OFF(nthread);
    OFF(cpr);
    OFF(npr);
    OFF(LX);
    OFF(LY);
    OFF(LZ);
    OFF(LT);
    OFF(latdims);
    OFF(VOLUME);
    OFF(Vmic_split);
    OFF(Vavx_split);
    OFF(Vsse_split);
    OFF(face);
    OFF(ipt_eo);
    OFF(ipt_lex);
    OFF(nn_bnde);
    OFF(nn_bndo);
    OFF(iup);
    OFF(idn);
    OFF(ipt_eo_yzt);
    OFF(ipt_lex_yzt);
    OFF(ipt_eo_sse_split);
    OFF(ipt_lex_sse_split);
    OFF(iup_sse_split);
    OFF(idn_sse_split);
    OFF(phip);
    OFF(phim);
    OFF(ALIGN);
    OFF(init);
    return 0;
}
