/*
 * ref_cpuonly_harness.c -- links the reference's untouched CPUonly decoder
 * (CPUonly/src/{format,decodeScanCPU,pixelTransformCPU,main}.c, built with
 * main renamed) into oracle/_ref/libref_cpuonly.so and exposes a small C
 * surface for ctypes: decode a file, read its geometry and pixels, and time
 * it on N host threads.  TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.
 *
 * The CPUonly decoder keeps no mutable globals (each JPG is self-contained),
 * so one image per thread is safe.
 *
 * CPUonly cannot decode files with restart markers (CPUonly/src/
 * decodeScanCPU.c:41-43).  For those, once refcpu_use_gputree has loaded
 * oracle/_ref/libref_gputree.so, the harness composes the reference's own
 * parts instead: the GPU tree's serial host decoder (src/decodeScanCPU.cu:
 * 98-152, which handles restart intervals) for the coefficients, then the
 * CPUonly iDCT_row / iDCT_col (called as CPUonly/src/decodeScanCPU.c:101-105
 * calls them) into channel planes laid out as CPUonly's decodeSOF lays them
 * out (CPUonly/src/format.c:121-145), then CPUonly's
 * upsampleAndColourTransform.
 */
#include <dlfcn.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "format.h" /* CPUonly/include/format.h: struct JPG */
#include "pixelTransformCPU.h"

JPG *openJPG(const char *filename); /* CPUonly/src/main.c:10 */

/* the GPU tree's coefficient decoder (ref_gputree_harness.cpp) */
static struct {
  void *(*create)(void);
  void (*destroy)(void *);
  int (*open)(void *, const char *);
  void (*info)(void *, int *);
  void (*coefs)(void *, int, int32_t *);
} g_gt;

int refcpu_use_gputree(const char *so_path) {
  void *h = dlopen(so_path, RTLD_NOW | RTLD_LOCAL);
  if (!h) return 0;
  g_gt.create = (void *(*)(void))dlsym(h, "refgpu_new");
  g_gt.destroy = (void (*)(void *))dlsym(h, "refgpu_del");
  g_gt.open = (int (*)(void *, const char *))dlsym(h, "refgpu_open");
  g_gt.info = (void (*)(void *, int *))dlsym(h, "refgpu_info");
  g_gt.coefs = (void (*)(void *, int, int32_t *))dlsym(h, "refgpu_coefs");
  if (!g_gt.create || !g_gt.destroy || !g_gt.open || !g_gt.info || !g_gt.coefs) {
    g_gt.create = NULL;
    return 0;
  }
  return 1;
}

/* A file CPUonly rejects, decoded by the composition described above;
 * NULL if the GPU tree rejects it too. */
static JPG *restart_decode(const char *path) {
  if (!g_gt.create) return NULL;
  void *r = g_gt.create();
  if (!r) return NULL;
  if (g_gt.open(r, path)) {
    g_gt.destroy(r);
    return NULL;
  }
  int info[18];
  g_gt.info(r, info);
  JPG *j = (JPG *)calloc(1, sizeof(JPG));
  if (!j) {
    g_gt.destroy(r);
    return NULL;
  }
  j->width = (unsigned short)info[0];
  j->height = (unsigned short)info[1];
  j->num_channels = (unsigned char)info[2];
  j->num_blocks_x = (unsigned short)info[3];
  j->num_blocks_y = (unsigned short)info[4];
  int sxm = 1, sym = 1;
  for (int c = 0; c < j->num_channels; c++) {
    if (info[6 + 4 * c] > sxm) sxm = info[6 + 4 * c];
    if (info[7 + 4 * c] > sym) sym = info[7 + 4 * c];
  }
  j->block_size_x = (unsigned short)(sxm << 3);
  j->block_size_y = (unsigned short)(sym << 3);
  int ok = 1;
  for (int c = 0; c < j->num_channels && ok; c++) {
    ColourChannel *ch = &j->channels[c];
    ch->samples_x = info[6 + 4 * c];
    ch->samples_y = info[7 + 4 * c];
    ch->width = (j->width * ch->samples_x + sxm - 1) / sxm;
    ch->height = (j->height * ch->samples_y + sym - 1) / sym;
    ch->stride = j->num_blocks_x * (ch->samples_x << 3);
    ch->pixels = (unsigned char *)malloc((size_t)ch->stride * j->num_blocks_y * (ch->samples_y << 3));
    const int n = info[8 + 4 * c];
    int32_t *coef = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    ok = ch->pixels && coef;
    if (ok) {
      g_gt.coefs(r, c, coef);
      const int per = ch->samples_x * ch->samples_y;
      for (int b = 0; b < n / 64; b++) {
        const int mcu = b / per, loc = b % per;
        const int bx = (mcu % j->num_blocks_x) * ch->samples_x + loc % ch->samples_x;
        const int by = (mcu / j->num_blocks_x) * ch->samples_y + loc / ch->samples_x;
        unsigned char *out = ch->pixels + (size_t)by * 8 * ch->stride + bx * 8;
        int blk[64];
        memcpy(blk, coef + (size_t)b * 64, sizeof(blk));
        for (int k = 0; k < 64; k += 8) iDCT_row(&blk[k]);
        for (int k = 0; k < 8; k++) iDCT_col(&blk[k], &out[k], ch->stride);
      }
    }
    free(coef);
  }
  g_gt.destroy(r);
  if (ok && j->num_channels == 3) {
    j->pixels = (unsigned char *)malloc((size_t)j->width * j->height * 3);
    ok = j->pixels != NULL;
  }
  if (ok) upsampleAndColourTransform(j);
  if (!ok || j->error) {
    delJPG(j);
    return NULL;
  }
  return j;
}

void *refcpu_open(const char *path) { return openJPG(path); }

/* CPUonly, or for a file it rejects the composition above. */
void *refcpu_open_any(const char *path) {
  JPG *j = openJPG(path);
  return j ? j : restart_decode(path);
}

void refcpu_info(void *h, int *info) {
  JPG *j = (JPG *)h;
  info[0] = j->width;
  info[1] = j->height;
  info[2] = j->num_channels;
  info[3] = j->restart_interval;
}

void refcpu_pixels(void *h, uint8_t *out) {
  JPG *j = (JPG *)h;
  size_t n = (size_t)j->width * j->height * j->num_channels;
  memcpy(out, j->num_channels == 1 ? j->channels[0].pixels : j->pixels, n);
}

void refcpu_close(void *h) {
  if (h) delJPG((JPG *)h);
}

typedef struct {
  const char **paths;
  int npaths, first, stride, iters;
  long long pixels;
  int failures;
} BenchArg;

static void *bench_worker(void *p) {
  BenchArg *a = (BenchArg *)p;
  for (int i = 0; i < a->iters; i++) {
    for (int k = a->first; k < a->npaths; k += a->stride) {
      JPG *j = openJPG(a->paths[k]);
      if (!j) j = restart_decode(a->paths[k]);
      if (!j) { a->failures++; continue; }
      a->pixels += (long long)j->width * j->height;
      delJPG(j);
    }
  }
  return NULL;
}

/* Decode every path `iters` times, files split round-robin over `nthreads`
 * threads (a file CPUonly rejects goes through restart_decode when the GPU
 * tree is loaded).  Returns wall seconds; *pixels_out = pixels decoded, *fail_out =
 * decodes that returned an error. */
double refcpu_bench(const char **paths, int npaths, int iters, int nthreads,
                    long long *pixels_out, int *fail_out) {
  if (nthreads < 1) nthreads = 1;
  if (nthreads > npaths) nthreads = npaths;
  pthread_t *th = (pthread_t *)calloc(nthreads, sizeof(pthread_t));
  BenchArg *args = (BenchArg *)calloc(nthreads, sizeof(BenchArg));
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (int t = 0; t < nthreads; t++) {
    args[t] = (BenchArg){paths, npaths, t, nthreads, iters, 0, 0};
    pthread_create(&th[t], NULL, bench_worker, &args[t]);
  }
  long long px = 0;
  int fails = 0;
  for (int t = 0; t < nthreads; t++) {
    pthread_join(th[t], NULL);
    px += args[t].pixels;
    fails += args[t].failures;
  }
  clock_gettime(CLOCK_MONOTONIC, &t1);
  free(th);
  free(args);
  *pixels_out = px;
  *fail_out = fails;
  return (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
}
