/* Packs API-layout arrays the way the reference's test driver does
 * (tests/test_hopping.c:256-275): object k of the packed arrays holds the
 * even/odd sites lanes*k .. lanes*k+lanes-1, built with the copy_*_256/512
 * converters of include/su3_256.h, su3_512.h. Compiled into a small shared
 * object by tests/test_abi.py to pin the Python packing helper. */
#include "su3_256.h"
#include "su3_512.h"

void pack_spinors(int lanes, const spinor *in, void *out, int V)
{
    for (int i = 0; i < V; i += lanes) {
        spinor *p = (spinor *)in + i;
        if (lanes == 2) copy_spinor_to_spinor_256((spinor_256 *)out + i / 2, p, p + 1);
        else copy_spinor_to_spinor_512((spinor_512 *)out + i / 4, p, p + 1, p + 2, p + 3);
    }
}

void pack_links(int lanes, const su3 *u, void *out, int V)
{
    for (int i = 0; i < V; i += lanes)
        for (int j = 0; j < 4; j++) {
            su3 *p = (su3 *)u + 4 * i + j;
            if (lanes == 2) copy_su3_to_su3_256((su3_256 *)out + 4 * i / 2 + j, p, p + 4);
            else copy_su3_to_su3_512((su3_512 *)out + 4 * i / 4 + j, p, p + 4, p + 8, p + 12);
        }
}
