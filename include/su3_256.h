/*
 * su3_256.h -- two-lane packed field types and their converters (plqcd-b200).
 *
 * Same type names, member names, byte layout and converter signatures as the
 * reference's include/su3_256.h:14-191, for legacy callers that pack two
 * API-layout objects into one (tests/test_hopping.c:256-264): every complex
 * element becomes a pair {lo = element of the first object, hi = element of
 * the second}. Portable C: no intrinsics header is needed.
 *
 * Difference from the reference: copy_spinor_256_to_spinor and
 * copy_halfspinor_256_to_halfspinor there write every spin of the second
 * object into its s0 (include/su3_256.h:171-177, 187-190); here each spin
 * goes to its own place, so packing and unpacking are exact inverses.
 */
#ifndef _SU3_256_H
#define _SU3_256_H

#include "su3.h"

typedef struct {
    plqcd_complex_t lo, hi;
} complex_pair;

typedef struct {
    complex_pair c00, c01, c02, c10, c11, c12, c20, c21, c22;
} su3_256;

typedef struct {
    complex_pair c00, c01, c02, c10, c11, c12;
} su3_compact_256;

typedef struct {
    complex_pair c0, c1, c2;
} su3_vector_256;

typedef struct {
    su3_vector_256 s0, s1, s2, s3;
} spinor_256;

typedef struct {
    su3_vector_256 s0, s1;
} halfspinor_256;

/* the converters walk the members as arrays: no padding between them */
#ifdef __cplusplus
static_assert(sizeof(su3_256) == 9 * sizeof(complex_pair) && sizeof(spinor_256) == 12 * sizeof(complex_pair), "packed layout");
#else
_Static_assert(sizeof(su3_256) == 9 * sizeof(complex_pair) && sizeof(spinor_256) == 12 * sizeof(complex_pair), "packed layout");
#endif

/* n complex elements of two objects <-> n lane pairs */
static inline void plqcd_pack2_(complex_pair *a, const plqcd_complex_t *b1, const plqcd_complex_t *b2, int n)
{
    for (int k = 0; k < n; k++) {
        a[k].lo = b1[k];
        a[k].hi = b2[k];
    }
}

static inline void plqcd_unpack2_(plqcd_complex_t *b1, plqcd_complex_t *b2, const complex_pair *a, int n)
{
    for (int k = 0; k < n; k++) {
        b1[k] = a[k].lo;
        b2[k] = a[k].hi;
    }
}

static inline void copy_su3_to_su3_256(su3_256 *a, su3 *b1, su3 *b2)
{
    plqcd_pack2_(&a->c00, &b1->c00, &b2->c00, 9);
}

static inline void copy_su3_256_to_su3(su3 *b1, su3 *b2, su3_256 *a)
{
    plqcd_unpack2_(&b1->c00, &b2->c00, &a->c00, 9);
}

static inline void copy_su3_vector_to_su3_vector_256(su3_vector_256 *a, su3_vector *b1, su3_vector *b2)
{
    plqcd_pack2_(&a->c0, &b1->c0, &b2->c0, 3);
}

static inline void copy_su3_vector_256_to_su3_vector(su3_vector *b1, su3_vector *b2, su3_vector_256 *a)
{
    plqcd_unpack2_(&b1->c0, &b2->c0, &a->c0, 3);
}

static inline void copy_spinor_to_spinor_256(spinor_256 *a, spinor *b1, spinor *b2)
{
    plqcd_pack2_(&a->s0.c0, &b1->s0.c0, &b2->s0.c0, 12);
}

static inline void copy_spinor_256_to_spinor(spinor *b1, spinor *b2, spinor_256 *a)
{
    plqcd_unpack2_(&b1->s0.c0, &b2->s0.c0, &a->s0.c0, 12);
}

static inline void copy_halfspinor_to_halfspinor_256(halfspinor_256 *a, halfspinor *b1, halfspinor *b2)
{
    plqcd_pack2_(&a->s0.c0, &b1->s0.c0, &b2->s0.c0, 6);
}

static inline void copy_halfspinor_256_to_halfspinor(halfspinor *b1, halfspinor *b2, halfspinor_256 *a)
{
    plqcd_unpack2_(&b1->s0.c0, &b2->s0.c0, &a->s0.c0, 6);
}

#endif
