/*
 * su3.h -- field types at the PLQCD API boundary (plqcd-b200).
 *
 * Same names and byte layout as the reference's include/su3.h:52-75, which
 * callers fill element by element (tests/test_hopping.c:202-251):
 *   su3        9 complex doubles, row-major c00..c22         (144 bytes)
 *   su3_vector 3 complex doubles c0..c2                       ( 48 bytes)
 *   spinor     4 su3_vector s0..s3 (spin-major, colour inner) (192 bytes)
 *   halfspinor 2 su3_vector s0..s1                            ( 96 bytes)
 * In C the complex type is `_Complex double`; C++ sees a layout-identical
 * {re, im} pair so the library's C++ side can share the header. The
 * reference's SU(3) macro layer (SSE asm, intrinsics) is not part of this
 * boundary.
 */
#ifndef _SU3_H
#define _SU3_H

#ifdef __cplusplus
typedef struct { double re, im; } plqcd_complex_t;
#else
#include <complex.h>
typedef double _Complex plqcd_complex_t;
#endif

typedef struct {
    plqcd_complex_t c00, c01, c02, c10, c11, c12, c20, c21, c22;
} su3;

typedef struct {
    plqcd_complex_t c0, c1, c2;
} su3_vector;

typedef struct {
    su3_vector s0, s1, s2, s3;
} spinor;

typedef struct {
    su3_vector s0, s1;
} halfspinor;

#endif
