/*
 * A C caller of the drop-in hopping pair, written the way the reference's
 * driver calls it (tests/test_hopping.c:96-115, 296-297): init_plqcd on an
 * input file, amalloc'd API-layout fields, then the eo and oe calls.
 *
 *   hop_caller <input file> <fields in> <spinor out>
 *
 * <fields in> holds qin (VOLUME spinors) followed by u (4*VOLUME su3), as
 * raw doubles in the API layout; <spinor out> receives qout (VOLUME
 * spinors). Exit status 0 when every call succeeded.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "plqcd.h"

int main(int argc, char **argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s input_file fields_in spinor_out\n", argv[0]);
        return 2;
    }
    if (init_plqcd(argc, argv) != 0) {
        fprintf(stderr, "init_plqcd failed: %s\n", plqcd_last_error());
        return 1;
    }
    const size_t V = (size_t)plqcd_g.VOLUME;
    spinor *pin = (spinor *)amalloc(V * sizeof(spinor), plqcd_g.ALIGN);
    spinor *pout = (spinor *)amalloc(V * sizeof(spinor), plqcd_g.ALIGN);
    su3 *ufield = (su3 *)amalloc(4 * V * sizeof(su3), plqcd_g.ALIGN);
    if (!pin || !pout || !ufield) {
        fprintf(stderr, "amalloc failed\n");
        return 1;
    }
    FILE *f = fopen(argv[2], "rb");
    if (!f || fread(pin, sizeof(spinor), V, f) != V || fread(ufield, sizeof(su3), 4 * V, f) != 4 * V) {
        fprintf(stderr, "cannot read %s\n", argv[2]);
        return 1;
    }
    fclose(f);
    memset(pout, 0, V * sizeof(spinor));
    const double t1 = plqcd_hopping_matrix_eo_sse3_assymbly(pin, pout, ufield);
    const double t2 = plqcd_hopping_matrix_oe_sse3_assymbly(pin, pout, ufield);
    if (t1 < 0 || t2 < 0) {
        fprintf(stderr, "hopping call failed: %s\n", plqcd_last_error());
        return 1;
    }
    f = fopen(argv[3], "wb");
    if (!f || fwrite(pout, sizeof(spinor), V, f) != V) {
        fprintf(stderr, "cannot write %s\n", argv[3]);
        return 1;
    }
    fclose(f);
    printf("eo %.6e s, oe %.6e s\n", t1, t2);
    afree(pin);
    afree(pout);
    afree(ufield);
    finalize_plqcd();
    return 0;
}
