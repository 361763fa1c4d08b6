/*
 * ref_cpuonly_harness.c -- links the reference's untouched CPUonly decoder
 * (CPUonly/src/{format,decodeScanCPU,pixelTransformCPU,main}.c, built with
 * main renamed) into oracle/_ref/libref_cpuonly.so and exposes a small C
 * surface for ctypes: decode a file, read its geometry and pixels, and time
 * it on N host threads.  TEST / BASELINE INFRASTRUCTURE ONLY.
 *
 * The CPUonly decoder keeps no mutable globals (each JPG is self-contained),
 * so one image per thread is safe.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "format.h" /* CPUonly/include/format.h: struct JPG */

JPG *openJPG(const char *filename); /* CPUonly/src/main.c:10 */

void *refcpu_open(const char *path) { return openJPG(path); }

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
      if (!j) { a->failures++; continue; }
      a->pixels += (long long)j->width * j->height;
      delJPG(j);
    }
  }
  return NULL;
}

/* Decode every path `iters` times, files split round-robin over `nthreads`
 * threads.  Returns wall seconds; *pixels_out = pixels decoded, *fail_out =
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
