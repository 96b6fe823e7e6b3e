/*
 * cf_oracle.c — CPU oracle for the warp-field Gauss-Newton/PCG solve.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load this library, and only as the
 * checker (or as the timed CPU baseline).  The product path never calls it.
 *
 * It restates CUDAFusion's algorithm for this path:
 *   include/se3_math.cuh            SE(3)/DQ math and warp_point
 *   kernels/solver_kernels.cu       assembly, damping, preconditioner, PCG,
 *                                   sparsity pattern
 *   src/warp_field.cu:250-291       clamped twist update
 * Two instantiations of cf_oracle_impl.h:
 *   *_f32  FP32 in the reference's operand order, sequential accumulation in
 *          correspondence order (one valid order of the reference's atomics);
 *   *_f64  the same schedule in FP64 (the "FP64 oracle").
 * Parity pin: the f32 se3 functions are checked bit for bit against the
 * reference's own host-compiled functions (oracle/_ref, tests/golden).
 *
 * Build: see oracle/Makefile (gcc -O2 -ffp-contract=off -fopenmp).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../include/cudafusion_b200.h"

#define CFO_EXPORT __attribute__((visibility("default")))

/* 0: the reference's ARAP rotation Jacobian sign (kernels/solver_kernels.cu:140-165);
 * 1: the consistent sign.  The product library exposes the same switch. */
static int cfo_arap_consistent = 0;
CFO_EXPORT void cfo_set_arap_consistent(int on) { cfo_arap_consistent = on ? 1 : 0; }

/* ---- FP32 instantiation (reference operand order) ---- */
#define R float
#define F(name) name##_f32
#define SQRT sqrtf
#define SIN sinf
#define COS cosf
#define EXP expf
#define FABS fabsf
#define FMAX fmaxf
#include "cf_oracle_impl.h"
#undef R
#undef F
#undef SQRT
#undef SIN
#undef COS
#undef EXP
#undef FABS
#undef FMAX

/* ---- FP64 instantiation ---- */
#define R double
#define F(name) name##_f64
#define SQRT sqrt
#define SIN sin
#define COS cos
#define EXP exp
#define FABS fabs
#define FMAX fmax
#include "cf_oracle_impl.h"
#undef R
#undef F

static int cmp_int(const void* a, const void* b) {
  int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}

/* kernels/solver_kernels.cu:498-541 — symmetric block pattern: the diagonal
 * plus every directed graph edge in both directions, sorted and unique per
 * row.  Writes row_ptr[N+1]; col_idx when cap is large enough.  Returns nnzb. */
CFO_EXPORT int cfo_build_pattern(const cf_deform_node* nodes, int N, int* row_ptr, int* col_idx, int cap) {
  int* deg = (int*)calloc((size_t)N + 1, sizeof(int));
  for (int i = 0; i < N; i++) {
    deg[i] += 1;
    for (int k = 0; k < nodes[i].num_neighbors && k < CF_K_GRAPH; k++) {
      int nb = nodes[i].neighbors[k];
      if (nb < 0 || nb >= N) continue;
      deg[i]++;
      deg[nb]++;
    }
  }
  int* start = (int*)malloc(sizeof(int) * ((size_t)N + 1));
  start[0] = 0;
  for (int i = 0; i < N; i++) start[i + 1] = start[i] + deg[i];
  int* raw = (int*)malloc(sizeof(int) * ((size_t)start[N] + 1));
  int* fill = (int*)calloc((size_t)N + 1, sizeof(int));
  for (int i = 0; i < N; i++) raw[start[i] + fill[i]++] = i;
  for (int i = 0; i < N; i++)
    for (int k = 0; k < nodes[i].num_neighbors && k < CF_K_GRAPH; k++) {
      int nb = nodes[i].neighbors[k];
      if (nb < 0 || nb >= N) continue;
      raw[start[i] + fill[i]++] = nb;
      raw[start[nb] + fill[nb]++] = i;
    }
  int nnzb = 0;
  for (int i = 0; i < N; i++) {
    int* r = raw + start[i];
    qsort(r, (size_t)deg[i], sizeof(int), cmp_int);
    row_ptr[i] = nnzb;
    for (int k = 0; k < deg[i]; k++) {
      if (k > 0 && r[k] == r[k - 1]) continue;
      if (col_idx && nnzb < cap) col_idx[nnzb] = r[k];
      nnzb++;
    }
  }
  row_ptr[N] = nnzb;
  free(deg); free(start); free(raw); free(fill);
  return nnzb;
}

CFO_EXPORT int cfo_struct_sizes(int* out) {
  out[0] = (int)sizeof(cf_dual_quat);
  out[1] = (int)sizeof(cf_deform_node);
  out[2] = (int)sizeof(cf_correspondence);
  out[3] = (int)sizeof(cf_gn_params);
  return 4;
}
