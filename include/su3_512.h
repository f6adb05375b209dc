/*
 * su3_512.h -- four-lane packed field types and their converters (plqcd-b200).
 *
 * Same type names, member names, byte layout and converter signatures as the
 * reference's include/su3_512.h:12-216, for legacy callers that pack four
 * API-layout objects into one (tests/test_hopping.c:267-275): every complex
 * element becomes z[0..3] = that element of objects b0..b3. Portable C.
 */
#ifndef _SU3_512_H
#define _SU3_512_H

#include "su3.h"

typedef struct {
    plqcd_complex_t z[4];
} complex4;

typedef struct {
    complex4 c00, c01, c02, c10, c11, c12, c20, c21, c22;
} su3_512;

typedef struct {
    complex4 c00, c01, c02, c10, c11, c12;
} su3_compact_512;

typedef struct {
    complex4 c0, c1, c2;
} su3_vector_512;

typedef struct {
    su3_vector_512 s0, s1, s2, s3;
} spinor_512;

typedef struct {
    su3_vector_512 s0, s1;
} halfspinor_512;

/* the converters walk the members as arrays: no padding between them */
#ifdef __cplusplus
static_assert(sizeof(su3_512) == 9 * sizeof(complex4) && sizeof(spinor_512) == 12 * sizeof(complex4), "packed layout");
#else
_Static_assert(sizeof(su3_512) == 9 * sizeof(complex4) && sizeof(spinor_512) == 12 * sizeof(complex4), "packed layout");
#endif

/* n complex elements of four objects <-> n lane quadruples */
static inline void plqcd_pack4_(complex4 *a, const plqcd_complex_t *b0, const plqcd_complex_t *b1,
                                const plqcd_complex_t *b2, const plqcd_complex_t *b3, int n)
{
    for (int k = 0; k < n; k++) {
        a[k].z[0] = b0[k];
        a[k].z[1] = b1[k];
        a[k].z[2] = b2[k];
        a[k].z[3] = b3[k];
    }
}

static inline void plqcd_unpack4_(plqcd_complex_t *b0, plqcd_complex_t *b1, plqcd_complex_t *b2,
                                  plqcd_complex_t *b3, const complex4 *a, int n)
{
    for (int k = 0; k < n; k++) {
        b0[k] = a[k].z[0];
        b1[k] = a[k].z[1];
        b2[k] = a[k].z[2];
        b3[k] = a[k].z[3];
    }
}

static inline void copy_su3_to_su3_512(su3_512 *a, su3 *b0, su3 *b1, su3 *b2, su3 *b3)
{
    plqcd_pack4_(&a->c00, &b0->c00, &b1->c00, &b2->c00, &b3->c00, 9);
}

static inline void copy_su3_512_to_su3(su3 *b0, su3 *b1, su3 *b2, su3 *b3, su3_512 *a)
{
    plqcd_unpack4_(&b0->c00, &b1->c00, &b2->c00, &b3->c00, &a->c00, 9);
}

static inline void copy_su3_vector_to_su3_vector_512(su3_vector_512 *a, su3_vector *b0, su3_vector *b1,
                                                     su3_vector *b2, su3_vector *b3)
{
    plqcd_pack4_(&a->c0, &b0->c0, &b1->c0, &b2->c0, &b3->c0, 3);
}

static inline void copy_su3_vector_512_to_su3_vector(su3_vector *b0, su3_vector *b1, su3_vector *b2,
                                                     su3_vector *b3, su3_vector_512 *a)
{
    plqcd_unpack4_(&b0->c0, &b1->c0, &b2->c0, &b3->c0, &a->c0, 3);
}

static inline void copy_spinor_to_spinor_512(spinor_512 *a, spinor *b0, spinor *b1, spinor *b2, spinor *b3)
{
    plqcd_pack4_(&a->s0.c0, &b0->s0.c0, &b1->s0.c0, &b2->s0.c0, &b3->s0.c0, 12);
}

static inline void copy_spinor_512_to_spinor(spinor *b0, spinor *b1, spinor *b2, spinor *b3, spinor_512 *a)
{
    plqcd_unpack4_(&b0->s0.c0, &b1->s0.c0, &b2->s0.c0, &b3->s0.c0, &a->s0.c0, 12);
}

static inline void copy_halfspinor_to_halfspinor_512(halfspinor_512 *a, halfspinor *b0, halfspinor *b1,
                                                     halfspinor *b2, halfspinor *b3)
{
    plqcd_pack4_(&a->s0.c0, &b0->s0.c0, &b1->s0.c0, &b2->s0.c0, &b3->s0.c0, 6);
}

static inline void copy_halfspinor_512_to_halfspinor(halfspinor *b0, halfspinor *b1, halfspinor *b2,
                                                     halfspinor *b3, halfspinor_512 *a)
{
    plqcd_unpack4_(&b0->s0.c0, &b1->s0.c0, &b2->s0.c0, &b3->s0.c0, &a->s0.c0, 6);
}

#endif
