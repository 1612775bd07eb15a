/* bdg_batch.c -- many independent BdG solves on one GPU.
 *
 * No counterpart in the reference, which solves one problem per call.  A
 * sweep of problems (different grids, trap aspects, interaction strengths)
 * leaves a B200 mostly idle when the solves run one after another: a 32^3 or
 * 48^3 problem fills a fraction of the GPU, and every iteration waits on the
 * host for its small dense steps.  bdg_solve_batch keeps `concurrency` solves
 * in flight, each on its own host thread and its own CUDA stream (the
 * problem's device context), so the GPU work of one solve overlaps the host
 * work and small kernels of the others.  Operator applies are replayed as
 * CUDA graphs when `graphs` is set, and the FFT pass family of every
 * context is chosen by the library's autotuner (bdgd_fft_tuning).  After each
 * solve the problem's solver workspace and scratch are released, so device
 * memory holds at most `concurrency` workspaces.
 */
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "bdg/bdg_b200.h"
#include "bdg/bdg_cuda.h"
#include "bdg/bdg_internal.h"
#include "bdg/bdg_learn.h"

void bdg_solver_release(bdg_t *bdg);

typedef struct {
  bdg_t **p;
  int n;
  int next;
  int graphs;
  int *rcs;
  double *secs;
  pthread_mutex_t mu;
} batch_t;

static double wall(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

void bdg_release_device_memory(bdg_t *bdg) {
  if (bdg == NULL) return;
  bdg_solver_release(bdg);
  if (bdg->ctx && bdg->ctx->dev) bdgd_trim(bdg->ctx->dev);
}

static void *batch_worker(void *arg) {
  batch_t *b = (batch_t *)arg;
  for (;;) {
    pthread_mutex_lock(&b->mu);
    const int i = b->next++;
    pthread_mutex_unlock(&b->mu);
    if (i >= b->n) break;
    bdg_t *p = b->p[i];
    const double t0 = wall();
    int rc = 0;
    if (b->graphs) {
      bdgd_ctx *d = bdg_device_context(p);
      if (d) bdgd_set_graphs(d, 1);
    }
    rc = bdg_solve(p);
    if (b->secs) b->secs[i] = wall() - t0;
    if (b->rcs) b->rcs[i] = rc;
    bdg_release_device_memory(p);
  }
  return NULL;
}

int bdg_solve_batch(bdg_t **problems, int n, int concurrency, int graphs, int *rcs_out, double *seconds_out) {
  if (problems == NULL || n < 0) return -1;
  if (n == 0) return 0;
  if (concurrency < 1) concurrency = 1;
  if (concurrency > n) concurrency = n;
  batch_t b;
  memset(&b, 0, sizeof b);
  b.p = problems;
  b.n = n;
  b.graphs = graphs;
  b.rcs = rcs_out ? rcs_out : (int *)calloc((size_t)n, sizeof(int));
  b.secs = seconds_out;
  pthread_mutex_init(&b.mu, NULL);
  pthread_t *th = (pthread_t *)calloc((size_t)concurrency, sizeof(pthread_t));
  int started = 0; /* handles of the threads created, stored contiguously */
  for (int t = 0; t < concurrency; ++t)
    if (pthread_create(&th[started], NULL, batch_worker, &b) == 0) started++;
  if (started == 0) batch_worker(&b); /* no threads available: solve here */
  for (int t = 0; t < started; ++t) pthread_join(th[t], NULL);
  free(th);
  pthread_mutex_destroy(&b.mu);
  int bad = 0;
  for (int i = 0; i < n; ++i)
    if (b.rcs[i]) bad++;
  if (!rcs_out) free(b.rcs);
  return bad ? -2 : 0;
}
