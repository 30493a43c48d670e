/* dist_two_ranks.c -- a C caller of the distributed Jacobi-PCG in one call
 * (celg_dist_pcg_solve), as a CEL application with two ranks would use it.
 *
 * Two POSIX threads play two ranks on one GPU, each with its own handle and
 * stream.  The 7-point Poisson system (diagonal 6, off-diagonals -1, b = 1)
 * on an nx x ny x nz grid is cut into two z-slabs; each rank uploads its rows
 * with the halo columns numbered after the local ones (the plane below,
 * then the plane above, in ascending global order).  The exchange callbacks
 * wait for the rank's stream, meet the other thread at a barrier and go
 * through host memory: the all-reduce adds the two buffers in rank order,
 * the halo copies the boundary planes.  No kernel waits for the other
 * rank's.  Writes the solution (both slabs in order) to a file and prints
 * the iteration count.
 *
 * usage: dist_two_ranks NX NY NZ OUT.bin
 */
#define _POSIX_C_SOURCE 200112L
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime.h>

#include "celgpu.h"

#define NEXCH CELG_DIST_NEXCH

typedef struct {
  pthread_barrier_t bar;
  double xch[2][NEXCH];
  double* halo_lo;  /* rank 0's top plane, read by rank 1 */
  double* halo_hi;  /* rank 1's bottom plane, read by rank 0 */
  int plane;
} Shared;

typedef struct {
  Shared* sh;
  int rank;
  int n, ncols;     /* local rows, local + halo columns */
  int nx, ny, z0, z1, nz;
  double* x;        /* the rank's part of the solution (host) */
  int iters, status;
} Rank;

static int allreduce_cb(void* ctx, double* buf_d, int count, void* stream) {
  Rank* r = (Rank*)ctx;
  Shared* sh = r->sh;
  if (count != NEXCH) return 1;
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return 1;
  if (cudaMemcpy(sh->xch[r->rank], buf_d, sizeof(double) * NEXCH, cudaMemcpyDeviceToHost)) return 1;
  pthread_barrier_wait(&sh->bar);
  double tot[NEXCH];
  for (int k = 0; k < NEXCH; ++k) tot[k] = sh->xch[0][k] + sh->xch[1][k];  /* rank order */
  if (cudaMemcpy(buf_d, tot, sizeof(double) * NEXCH, cudaMemcpyHostToDevice)) return 1;
  pthread_barrier_wait(&sh->bar);
  return 0;
}

static int halo_cb(void* ctx, double* vec_d, void* stream) {
  Rank* r = (Rank*)ctx;
  Shared* sh = r->sh;
  const size_t pb = sizeof(double) * (size_t)sh->plane;
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return 1;
  /* rank 0 sends its top plane, rank 1 its bottom plane */
  if (r->rank == 0) {
    if (cudaMemcpy(sh->halo_lo, vec_d + r->n - sh->plane, pb, cudaMemcpyDeviceToHost)) return 1;
  } else {
    if (cudaMemcpy(sh->halo_hi, vec_d, pb, cudaMemcpyDeviceToHost)) return 1;
  }
  pthread_barrier_wait(&sh->bar);
  const double* src = r->rank == 0 ? sh->halo_hi : sh->halo_lo;
  if (cudaMemcpy(vec_d + r->n, src, pb, cudaMemcpyHostToDevice)) return 1;
  pthread_barrier_wait(&sh->bar);
  return 0;
}

/* rows z0..z1-1 of the grid as local CSR, halo columns after the local ones */
static void build_block(const Rank* r, int** rp_out, int** ci_out, double** v_out, int* nnz_out) {
  const int nx = r->nx, ny = r->ny, nxy = nx * ny;
  const int n = r->n;
  int* rp = malloc(sizeof(int) * (size_t)(n + 1));
  int* ci = malloc(sizeof(int) * (size_t)n * 7);
  double* v = malloc(sizeof(double) * (size_t)n * 7);
  const int has_lo = r->z0 > 0, has_hi = r->z1 < r->nz;
  int k = 0;
  for (int i = 0; i < n; ++i) {
    const int x = i % nx, y = (i / nx) % ny, z = r->z0 + i / nxy;
    rp[i] = k;
    /* stored order: -nxy, -nx, -1, 0, +1, +nx, +nxy (ascending global column) */
    if (z > 0) {
      ci[k] = z - 1 >= r->z0 ? i - nxy : n + (i % nxy);                /* plane below */
      v[k++] = -1.0;
    }
    if (y > 0) { ci[k] = i - nx; v[k++] = -1.0; }
    if (x > 0) { ci[k] = i - 1; v[k++] = -1.0; }
    ci[k] = i; v[k++] = 6.0;
    if (x < nx - 1) { ci[k] = i + 1; v[k++] = -1.0; }
    if (y < ny - 1) { ci[k] = i + nx; v[k++] = -1.0; }
    if (z < r->nz - 1) {
      ci[k] = z + 1 < r->z1 ? i + nxy : n + (has_lo ? nxy : 0) + (i % nxy);  /* plane above */
      v[k++] = -1.0;
    }
  }
  rp[n] = k;
  (void)has_hi;
  *rp_out = rp;
  *ci_out = ci;
  *v_out = v;
  *nnz_out = k;
}

#define CHECK(call)                                                             \
  do {                                                                          \
    int s_ = (call);                                                            \
    if (s_) {                                                                   \
      fprintf(stderr, "rank %d: %s -> %s\n", r->rank, #call, celg_status_string(s_)); \
      r->status = s_;                                                           \
      return NULL;                                                              \
    }                                                                           \
  } while (0)

static void* rank_main(void* arg) {
  Rank* r = (Rank*)arg;
  celg_handle* h = NULL;
  celg_mat* m = NULL;
  celg_dist* d = NULL;
  int *rp, *ci, nnz;
  double* v;
  r->status = 0;
  CHECK(celg_create(&h, 0, NULL));
  build_block(r, &rp, &ci, &v, &nnz);
  CHECK(celg_mat_from_csr_ext(h, r->n, r->ncols, nnz, rp, ci, v, 0, &m));
  CHECK(celg_mat_jacobi(m));
  celg_params p;
  celg_params_default(&p);
  p.x0_mode = CELG_X0_ZERO;
  p.eps_rel = 1e-8;
  p.eps_abs = 0.0;
  p.iter_max = 1000;
  CHECK(celg_dist_create(h, m, &p, NULL, NULL, 0, &d));
  double *b_d = NULL, *x_d = NULL;
  double* ones = malloc(sizeof(double) * (size_t)r->n);
  for (int i = 0; i < r->n; ++i) ones[i] = 1.0;
  if (cudaMalloc((void**)&b_d, sizeof(double) * (size_t)r->n) ||
      cudaMalloc((void**)&x_d, sizeof(double) * (size_t)r->ncols) ||
      cudaMemcpy(b_d, ones, sizeof(double) * (size_t)r->n, cudaMemcpyHostToDevice) ||
      cudaMemset(x_d, 0, sizeof(double) * (size_t)r->ncols)) {
    r->status = CELG_ERR_CUDA;
    return NULL;
  }
  celg_dist_comm comm = {r, allreduce_cb, halo_cb};
  celg_result res;
  memset(&res, 0, sizeof(res));
  const int st = celg_dist_pcg_solve(d, &comm, b_d, x_d, 4, &res);
  if (st) {
    fprintf(stderr, "rank %d: celg_dist_pcg_solve -> %s\n", r->rank, celg_status_string(st));
    r->status = st;
  }
  r->iters = res.iter_done;
  cudaMemcpy(r->x, x_d, sizeof(double) * (size_t)r->n, cudaMemcpyDeviceToHost);
  cudaFree(b_d);
  cudaFree(x_d);
  free(ones);
  free(rp);
  free(ci);
  free(v);
  celg_dist_destroy(d);
  celg_mat_destroy(m);
  celg_destroy(h);
  return NULL;
}

int main(int argc, char** argv) {
  if (argc != 5) {
    fprintf(stderr, "usage: %s NX NY NZ OUT.bin\n", argv[0]);
    return 2;
  }
  const int nx = atoi(argv[1]), ny = atoi(argv[2]), nz = atoi(argv[3]);
  if (nx < 1 || ny < 1 || nz < 2) return 2;
  Shared sh;
  sh.plane = nx * ny;
  sh.halo_lo = malloc(sizeof(double) * (size_t)sh.plane);
  sh.halo_hi = malloc(sizeof(double) * (size_t)sh.plane);
  pthread_barrier_init(&sh.bar, NULL, 2);
  const int zc = nz / 2;  /* the z-slab cut of two ranks */
  Rank ranks[2];
  for (int q = 0; q < 2; ++q) {
    Rank* r = &ranks[q];
    r->sh = &sh;
    r->rank = q;
    r->nx = nx;
    r->ny = ny;
    r->nz = nz;
    r->z0 = q == 0 ? 0 : zc;
    r->z1 = q == 0 ? zc : nz;
    r->n = (r->z1 - r->z0) * sh.plane;
    r->ncols = r->n + sh.plane;  /* one neighbour plane each */
    r->x = malloc(sizeof(double) * (size_t)r->n);
  }
  pthread_t th[2];
  for (int q = 0; q < 2; ++q) pthread_create(&th[q], NULL, rank_main, &ranks[q]);
  for (int q = 0; q < 2; ++q) pthread_join(th[q], NULL);
  if (ranks[0].status || ranks[1].status) return 1;
  if (ranks[0].iters != ranks[1].iters) {
    fprintf(stderr, "ranks disagree on the iteration count\n");
    return 1;
  }
  FILE* f = fopen(argv[4], "wb");
  if (!f) return 1;
  fwrite(ranks[0].x, sizeof(double), (size_t)ranks[0].n, f);
  fwrite(ranks[1].x, sizeof(double), (size_t)ranks[1].n, f);
  fclose(f);
  printf("iterations=%d\n", ranks[0].iters);
  return 0;
}
