/* Known-answer test of the packed field types (include/su3_256.h,
 * include/su3_512.h): lane k of every packed complex element is that element
 * of the k-th API-layout object, the packed structs have the layout of
 * consecutive lanes, and unpacking inverts packing. Exit status 0 = pass. */
#include <stdio.h>
#include <string.h>

#include "su3_256.h"
#include "su3_512.h"

static double val(int obj, int elem, int part) { return 1000.0 * obj + 2.0 * elem + part + 0.25; }

static void fill(plqcd_complex_t *c, int n, int obj)
{
    double *d = (double *)c;
    for (int e = 0; e < n; e++) {
        d[2 * e] = val(obj, e, 0);
        d[2 * e + 1] = val(obj, e, 1);
    }
}

/* packed element e, lane k, as laid out in memory: lanes are consecutive */
static int check_lanes(const void *packed, int n, int lanes)
{
    const double *d = (const double *)packed;
    for (int e = 0; e < n; e++)
        for (int k = 0; k < lanes; k++)
            for (int part = 0; part < 2; part++)
                if (d[(e * lanes + k) * 2 + part] != val(k, e, part)) return 1;
    return 0;
}

int main(void)
{
    int fail = 0;
    spinor s[4], r[4];
    su3 u[4], w[4];
    halfspinor h[4], g[4];
    for (int k = 0; k < 4; k++) {
        fill(&s[k].s0.c0, 12, k);
        fill(&u[k].c00, 9, k);
        fill(&h[k].s0.c0, 6, k);
    }
    spinor_256 s2;
    su3_256 u2;
    halfspinor_256 h2;
    su3_vector_256 v2;
    copy_spinor_to_spinor_256(&s2, &s[0], &s[1]);
    copy_su3_to_su3_256(&u2, &u[0], &u[1]);
    copy_halfspinor_to_halfspinor_256(&h2, &h[0], &h[1]);
    copy_su3_vector_to_su3_vector_256(&v2, &s[0].s0, &s[1].s0);
    fail |= check_lanes(&s2, 12, 2) << 0;
    fail |= check_lanes(&u2, 9, 2) << 1;
    fail |= check_lanes(&h2, 6, 2) << 2;
    fail |= check_lanes(&v2, 3, 2) << 3;
    memset(r, 0, sizeof r);
    memset(w, 0, sizeof w);
    memset(g, 0, sizeof g);
    copy_spinor_256_to_spinor(&r[0], &r[1], &s2);
    copy_su3_256_to_su3(&w[0], &w[1], &u2);
    copy_halfspinor_256_to_halfspinor(&g[0], &g[1], &h2);
    fail |= (memcmp(r, s, 2 * sizeof(spinor)) != 0) << 4;
    fail |= (memcmp(w, u, 2 * sizeof(su3)) != 0) << 5;
    fail |= (memcmp(g, h, 2 * sizeof(halfspinor)) != 0) << 6;

    spinor_512 s4;
    su3_512 u4;
    halfspinor_512 h4;
    su3_vector_512 v4;
    copy_spinor_to_spinor_512(&s4, &s[0], &s[1], &s[2], &s[3]);
    copy_su3_to_su3_512(&u4, &u[0], &u[1], &u[2], &u[3]);
    copy_halfspinor_to_halfspinor_512(&h4, &h[0], &h[1], &h[2], &h[3]);
    copy_su3_vector_to_su3_vector_512(&v4, &s[0].s0, &s[1].s0, &s[2].s0, &s[3].s0);
    fail |= check_lanes(&s4, 12, 4) << 7;
    fail |= check_lanes(&u4, 9, 4) << 8;
    fail |= check_lanes(&h4, 6, 4) << 9;
    fail |= check_lanes(&v4, 3, 4) << 10;
    memset(r, 0, sizeof r);
    memset(w, 0, sizeof w);
    memset(g, 0, sizeof g);
    copy_spinor_512_to_spinor(&r[0], &r[1], &r[2], &r[3], &s4);
    copy_su3_512_to_su3(&w[0], &w[1], &w[2], &w[3], &u4);
    copy_halfspinor_512_to_halfspinor(&g[0], &g[1], &g[2], &g[3], &h4);
    su3_vector vv[4];
    copy_su3_vector_512_to_su3_vector(&vv[0], &vv[1], &vv[2], &vv[3], &v4);
    fail |= (memcmp(r, s, sizeof r) != 0) << 11;
    fail |= (memcmp(w, u, sizeof w) != 0) << 12;
    fail |= (memcmp(g, h, sizeof g) != 0) << 13;
    for (int k = 0; k < 4; k++) fail |= (memcmp(&vv[k], &s[k].s0, sizeof(su3_vector)) != 0) << 14;
    if (fail) printf("packed types: failure mask 0x%x\n", fail);
    return fail != 0;
}
