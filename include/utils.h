/*
 * utils.h -- aligned allocation, timer and tag helpers (plqcd-b200).
 *
 * Same entry points as the reference's include/utils.h:13-45
 * (implementations: lib/utils.c:23-125).
 */
#ifndef _UTILS_H
#define _UTILS_H 1

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* posix_memalign-style aligned block (lib/utils.c:23-33). */
void *alloc(size_t size, size_t alignment);

/* Block of `size` bytes aligned to 2^p bytes, NULL on failure or on
 * size == 0 / p < 0 (lib/utils.c:35-65). When a CUDA device is present the
 * block is page-locked host memory, so host<->device copies of fields kept
 * in it run at full link speed. */
void *amalloc(size_t size, int p);

/* Release a block from amalloc; unknown or already-freed addresses are
 * ignored (lib/utils.c:68-90). */
void afree(void *addr);

/* Message tags (lib/utils.c:94-114). Kept for source compatibility; the
 * single-GPU library exchanges no messages. Returns -1 instead of exiting
 * when the permanent range is exhausted. */
int mpi_permanent_tag(void);
int mpi_tag(void);

/* Wall-clock seconds since t (lib/utils.c:120-125: the unit is seconds). */
double stop_watch(double t);

#ifdef __cplusplus
}
#endif
#endif
