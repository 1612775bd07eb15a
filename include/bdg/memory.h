/*
 * Checked host allocation helpers with the contract of the reference's
 * include/bdg/memory.h:31-98 (64-byte aligned, zero size or exhaustion is
 * fatal, safe_free nulls the caller's pointer).  Test code written against
 * the reference allocates ctx fields with these and hands them to the
 * library, which frees them with safe_free.
 */
#ifndef BDG_MEMORY_H
#define BDG_MEMORY_H

#ifndef LOBPCG_MEMORY_H
#define LOBPCG_MEMORY_H

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static inline void *xmalloc(size_t size) {
  if (size == 0) {
    fprintf(stderr, "xmalloc: refusing a 0-byte allocation\n");
    exit(1);
  }
  const size_t rounded = (size + 63u) & ~(size_t)63u;
  void *p = aligned_alloc(64, rounded);
  if (p == NULL) {
    fprintf(stderr, "xmalloc: %zu bytes not available\n", size);
    exit(1);
  }
  return p;
}

static inline void *xcalloc(size_t num, size_t size) {
  if (num == 0 || size == 0) {
    fprintf(stderr, "xcalloc: refusing a zero-sized allocation\n");
    exit(1);
  }
  if (num > SIZE_MAX / size) {
    fprintf(stderr, "xcalloc: %zu x %zu overflows size_t\n", num, size);
    exit(1);
  }
  void *p = xmalloc(num * size);
  memset(p, 0, num * size);
  return p;
}

static inline void safe_free(void **ptr) {
  if (ptr != NULL && *ptr != NULL) {
    free(*ptr);
    *ptr = NULL;
  }
}

#endif /* LOBPCG_MEMORY_H */
#endif /* BDG_MEMORY_H */
