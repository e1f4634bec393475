/* Driver written against the C ABI alone (include/gpufem.h), the way a C,
 * Fortran or FFI caller binds the library: assembler in RCM ordering,
 * Jacobian with fused Dirichlet rows / columns, the direct block LU solve,
 * and FP32-factor ILU(2) inside FP64 GMRES with the dataflow sweeps.
 * Usage: c_abi_solve <mesh.bin> <output prefix>   (mesh.bin as for
 * linear_static.cpp). Writes <prefix>.pattern (int32 nn, nnzb, rowPtr,
 * colPtr, perm), <prefix>.K, <prefix>.x_direct, <prefix>.x_gmres and
 * <prefix>.info (float64 direct residual, GMRES residual, GMRES steps). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime.h>

#include "gpufem.h"

#define CHECK(call)                                                                 \
  do {                                                                              \
    gf_status s_ = (call);                                                          \
    if (s_ != GF_OK) {                                                              \
      fprintf(stderr, "%s: %s %s\n", #call, gf_status_string(s_), gf_last_error()); \
      return 5;                                                                     \
    }                                                                               \
  } while (0)

static void wr(const char* prefix, const char* ext, const void* p, size_t bytes) {
  char path[1024];
  snprintf(path, sizeof(path), "%s%s", prefix, ext);
  FILE* f = fopen(path, "wb");
  fwrite(p, 1, bytes, f);
  fclose(f);
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 3;
  int32_t nn, ne, nbc;
  double E, nu;
  if (fread(&nn, 4, 1, f) != 1 || fread(&ne, 4, 1, f) != 1 || fread(&nbc, 4, 1, f) != 1 ||
      fread(&E, 8, 1, f) != 1 || fread(&nu, 8, 1, f) != 1)
    return 4;
  int32_t* conn = malloc(sizeof(int32_t) * 4 * ne);
  int32_t* bcs = malloc(sizeof(int32_t) * (nbc > 0 ? nbc : 1));
  double* xpts = malloc(sizeof(double) * 3 * nn);
  double* thick = malloc(sizeof(double) * ne);
  double* loads = malloc(sizeof(double) * 6 * nn);
  if (fread(conn, 4, 4 * (size_t)ne, f) != 4 * (size_t)ne ||
      fread(xpts, 8, 3 * (size_t)nn, f) != 3 * (size_t)nn ||
      fread(bcs, 4, (size_t)nbc, f) != (size_t)nbc || fread(thick, 8, (size_t)ne, f) != (size_t)ne ||
      fread(loads, 8, 6 * (size_t)nn, f) != 6 * (size_t)nn)
    return 4;
  fclose(f);
  gf_shell_data* data = calloc((size_t)ne, sizeof(gf_shell_data));
  for (int e = 0; e < ne; e++) {
    data[e].E = E;
    data[e].nu = nu;
    data[e].thick = thick[e];
  }
  gf_mesh_desc d;
  memset(&d, 0, sizeof(d));
  d.num_nodes = nn;
  d.num_elements = ne;
  d.conn = conn;
  d.xpts = xpts;
  d.bcs = bcs;
  d.num_bcs = nbc;
  d.data = data;
  d.ordering = GF_ORDER_RCM;
  d.rcm_root = 0;
  gf_assembler* a;
  CHECK(gf_assembler_create(&d, &a));
  gf_bsr* K;
  CHECK(gf_bsr_create(a, &K));
  const size_t n = 6 * (size_t)nn;
  double *d_b, *d_x, *d_x2;
  cudaMalloc((void**)&d_b, n * sizeof(double));
  cudaMalloc((void**)&d_x, n * sizeof(double));
  cudaMalloc((void**)&d_x2, n * sizeof(double));
  cudaMemcpy(d_b, loads, n * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemset(d_x2, 0, n * sizeof(double));
  CHECK(gf_add_jacobian(a, NULL, K, GF_ASSEMBLE_FUSE_BCS, NULL));
  CHECK(gf_apply_bcs_vec(a, d_b, NULL));
  gf_solve_stats sd, sg;
  CHECK(gf_direct_solve(a, K, d_b, d_x, &sd, NULL));
  gf_precond* P;
  CHECK(gf_precond_create_ex(a, 2, GF_PREC_FP32, GF_SWEEP_DATAFLOW, &P));
  CHECK(gf_precond_factor(P, K, NULL));
  gf_solve_opts o;
  gf_solve_opts_default(&o);
  o.side = 1;
  o.rtol = 1e-10;
  o.restart = 200;
  o.max_iters = 4000;
  CHECK(gf_gmres_solve(a, K, P, d_b, d_x2, &o, &sg, NULL));
  const int32_t nnzb = gf_assembler_nnzb(a);
  int32_t* pat = malloc(sizeof(int32_t) * (2 + (size_t)nn + 1 + (size_t)nnzb + (size_t)nn));
  pat[0] = nn;
  pat[1] = nnzb;
  CHECK(gf_assembler_get_pattern(a, pat + 2, pat + 3 + nn, pat + 3 + nn + nnzb, NULL));
  wr(argv[2], ".pattern", pat, sizeof(int32_t) * (2 + (size_t)nn + 1 + nnzb + nn));
  double* hk = malloc(sizeof(double) * 36 * (size_t)nnzb);
  cudaMemcpy(hk, gf_bsr_values(K), sizeof(double) * 36 * (size_t)nnzb, cudaMemcpyDeviceToHost);
  wr(argv[2], ".K", hk, sizeof(double) * 36 * (size_t)nnzb);
  double* hx = malloc(n * sizeof(double));
  cudaMemcpy(hx, d_x, n * sizeof(double), cudaMemcpyDeviceToHost);
  wr(argv[2], ".x_direct", hx, n * sizeof(double));
  cudaMemcpy(hx, d_x2, n * sizeof(double), cudaMemcpyDeviceToHost);
  wr(argv[2], ".x_gmres", hx, n * sizeof(double));
  double info[3] = {sd.rel_residual, sg.rel_residual, (double)sg.iterations};
  wr(argv[2], ".info", info, sizeof(info));
  gf_precond_destroy(P);
  gf_bsr_destroy(K);
  gf_assembler_destroy(a);
  cudaFree(d_b);
  cudaFree(d_x);
  cudaFree(d_x2);
  return 0;
}
