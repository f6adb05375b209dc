/*
 * plqcd_global_params.h -- the global parameter struct `plqcd_g`
 * (plqcd-b200).
 *
 * Field names follow the reference's include/plqcd_global_params.h:67-205
 * because callers index them directly (tests/test_hopping.c:33,42,96;
 * tests/test_comms.c). Differences:
 *  - `plqcd_g` is defined once inside the library and declared extern here
 *    (the reference places a tentative definition in the header, which
 *    needs -fcommon to link);
 *  - phip/phim stay NULL: the GPU kernel gathers neighbours directly and
 *    needs no half-spinor buffers;
 *  - the SSE split-layout tables (ipt_eo_sse_split, ipt_lex_sse_split,
 *    iup_sse_split, idn_sse_split) are members, in the reference's place,
 *    so that the struct has the reference's default layout (no AVX_SPLIT,
 *    no MIC: include/plqcd_global_params.h:147-196); they stay NULL. The
 *    AVX and MIC members, which the reference compiles in only under
 *    AVX_SPLIT / MIC, are not declared.
 */
#ifndef PLQCD_GLOBAL_PARAMS_H_
#define PLQCD_GLOBAL_PARAMS_H_

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
/* C callers get what the reference's header gives them
 * (include/plqcd_global_params.h:24-61): <stdbool.h>, <complex.h>, the
 * caller's MPI header when its include path has one (the reference's
 * drivers call MPI_Barrier / MPI_Reduce / MPI_Bcast for their timing,
 * tests/test_hopping.c:293,303-304) and <omp.h> under OpenMP. The library
 * itself uses none of them. */
#ifndef __cplusplus
#include <stdbool.h>
#include <complex.h>
#if defined(__has_include)
#if __has_include("mpi.h")
#include "mpi.h"
#endif
#endif
#endif
#ifdef _OPENMP
#include <omp.h>
#endif
#include "su3.h"
#include "utils.h"

#ifdef __cplusplus
extern "C" {
#endif

struct _PLQCD_GLOBAL_PARAMS {
    int nprocs[4];      /* process grid; this library runs one process (1,1,1,1) */
    int nthread;        /* NTHREAD from the input file (host threads for table setup) */
    int cpr[4];         /* cartesian coordinates of this process */
    int npr[8];         /* neighbour process ids, -mu at 2*mu, +mu at 2*mu+1 */
    int LX, LY, LZ, LT; /* global lattice extents */
    int latdims[4];     /* local extents (= global for one process) */
    int VOLUME;         /* local volume */
    int Vmic_split;     /* VOLUME/8 */
    int Vavx_split;     /* VOLUME/4 */
    int Vsse_split;     /* VOLUME/2 */
    int face[4];        /* boundary sizes; 0 in every direction for one process */
    int *ipt_eo;        /* lexicographic index -> even/odd index (even sites first) */
    int *ipt_lex;       /* even/odd index -> lexicographic index */
    int *nn_bnde[8];    /* boundary neighbour tables; NULL for one process */
    int *nn_bndo[8];
    int **iup;          /* iup[i][mu]: even/odd index of the +mu neighbour (periodic) */
    int **idn;          /* idn[i][mu]: even/odd index of the -mu neighbour (periodic) */
    int *ipt_eo_yzt;    /* even/odd index within the y,z,t block */
    int *ipt_lex_yzt;   /* inverse of ipt_eo_yzt */
    int *ipt_eo_sse_split;  /* SSE split-layout tables: NULL (not built) */
    int *ipt_lex_sse_split;
    int **iup_sse_split;
    int **idn_sse_split;
    halfspinor *phip[4];/* unused by the GPU path (NULL) */
    halfspinor *phim[4];/* unused by the GPU path (NULL) */
    int ALIGN;          /* alignment exponent for amalloc (2^ALIGN bytes) */
    int init;           /* 1 once init_plqcd has succeeded */
};

extern struct _PLQCD_GLOBAL_PARAMS plqcd_g;

#ifdef __cplusplus
}
#endif
#endif
