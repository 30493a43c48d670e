/*
 * ref_poisson_main.c -- driver for the reference's own C Poisson generator
 * (TEST INFRASTRUCTURE: builds oracle/_ref/ref_poisson from the reference
 * sources in place; see oracle/ref.mk).
 *
 * Calls cel_sparce_matrix_coo_interface (src/base/cel_sparce_matrix_coo_interface.c:22-60)
 * for one sub-domain (dx=dy=dz=1) with the 7-point stencil and the
 * u = x^2+y^2+z^2 Dirichlet problem
 * (src/base/cel_discretisation_poisson_3d.c:100-181, :622-679, :681-734,
 * :789-801) and writes the COO matrix, the right-hand side and the exact
 * nodal solution as raw little-endian binary:
 *   int32 n, int32 nnz, int32 rows[nnz], int32 cols[nnz], f64 vals[nnz],
 *   f64 b[n], f64 u[n]
 * Usage: ref_poisson nx ny nz out.bin
 */
#include <stdio.h>
#include <stdlib.h>

#include "cel_discretisation.h"
#include "cel_domain_3d.h"
#include "cel_sparse_matrix_coo.h"
#include "cel_types.h"
#include "cel_vector.h"

int cel_sparce_matrix_coo_interface(int* rank, cel_discretisation_task* desc_algorithm,
                                    cel_domain_3D* domain_3D,
                                    cel_sparse_matrix_coo* sparse_matrix_coo,
                                    cel_vector* boundary_vector, cel_vector* th_solution_vector,
                                    int* verbose);

int main(int argc, char** argv) {
  if (argc != 5) {
    fprintf(stderr, "usage: %s nx ny nz out.bin\n", argv[0]);
    return 2;
  }
  cel_discretisation_task task;
  task.problem = POISSON_3D;
  task.stencil = STENCIL_7;
  task.boundary_cond = X_2_PLUS_Y_2_PLUS_Z_2;
  cel_domain_3D dom;
  dom.nx = atoi(argv[1]);
  dom.ny = atoi(argv[2]);
  dom.nz = atoi(argv[3]);
  dom.dx = dom.dy = dom.dz = 1;
  cel_sparse_matrix_coo coo;
  cel_vector b, u;
  int rank = 0, verbose = 0;
  int err = cel_sparce_matrix_coo_interface(&rank, &task, &dom, &coo, &b, &u, &verbose);
  if (err) {
    fprintf(stderr, "generator error %d\n", err);
    return 1;
  }
  FILE* f = fopen(argv[4], "wb");
  if (!f) return 1;
  int n = coo.rows_num, nnz = coo.elements_num;
  fwrite(&n, sizeof(int), 1, f);
  fwrite(&nnz, sizeof(int), 1, f);
  fwrite(coo.rows, sizeof(int), (size_t)nnz, f);
  fwrite(coo.cols, sizeof(int), (size_t)nnz, f);
  fwrite(coo.values, sizeof(double), (size_t)nnz, f);
  fwrite(b.values, sizeof(double), (size_t)n, f);
  fwrite(u.values, sizeof(double), (size_t)n, f);
  fclose(f);
  return 0;
}
