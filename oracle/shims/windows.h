/* Linux stand-in for <windows.h>, used only when the reference's CPU sources
 * are compiled as a test oracle.  It supplies the handful of MSVC CRT names the
 * reference uses (aligned allocation, __declspec(align), _BitScanForward,
 * fopen_s) with POSIX equivalents. */
#ifndef GF_ORACLE_WINDOWS_SHIM_H
#define GF_ORACLE_WINDOWS_SHIM_H
#include <stdlib.h>
#include <stdio.h>
#include <string.h>
#include <malloc.h>
#include <limits.h>
#include <immintrin.h>

static inline void* gf_shim_aligned_malloc(size_t n, size_t a) {
  void* p = NULL;
  if (a < sizeof(void*)) a = sizeof(void*);
  if (posix_memalign(&p, a, n ? n : a) != 0) return NULL;
  return p;
}
static inline void* gf_shim_aligned_realloc(void* p, size_t n, size_t a) {
  void* q = gf_shim_aligned_malloc(n, a);
  if (q && p) { size_t old = malloc_usable_size(p); memcpy(q, p, old < n ? old : n); free(p); }
  return q;
}
#define _aligned_malloc(n, a) gf_shim_aligned_malloc((n), (a))
#define _aligned_realloc(p, n, a) gf_shim_aligned_realloc((p), (n), (a))
#define _aligned_free(p) free(p)
#define __declspec(x) gf_declspec_##x
#define gf_declspec_align(n) __attribute__((aligned(n)))

static inline unsigned char _BitScanForward(unsigned long* idx, unsigned long mask) {
  if (!mask) return 0;
  *idx = (unsigned long)__builtin_ctzl(mask);
  return 1;
}
static inline int fopen_s(FILE** f, const char* name, const char* mode) {
  *f = fopen(name, mode);
  return *f ? 0 : 1;
}
#endif
