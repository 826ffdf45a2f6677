// Arguments of the assembly kernels for one system (one collocation row range).
#pragma once

#include "common.cuh"

namespace bem {

struct AsmArgs {
  int n, ne, nbatches;
  int in0, nrows_nodes;  // collocation nodes [in0, in0 + nrows_nodes)
  const int* batches;
  const int* nconec;
  const int* kconec;
  const int* kode;
  const double* bc;
  const int* uknown;
  const double* vp;
  const int* nesim;
  const int* ke;
  const double* x;
  const double* y;
  const double* z;
  const double* tab;
  const double* rec;  // mode A: per-element boundary records (assembly.cu, kRecD doubles each)
  Material mat;
  double* A;  // mode A: (3n, 3n); mode HG: H
  int64_t lda;
  double* FI;  // mode A only
  double* G;   // mode HG only
  int64_t ldg;
  // mode A, last wave split (assembly.cu): tiles >= tail0 run as nparts pieces, each
  // over its share of the element batches; pieces >= 1 add into scratch that
  // tail_merge_*_kernel then adds into A and FI.  nparts <= 1: no split.
  int tail0, nparts, scr_cols;
  const int* slot;  // [(nparts - 1) * n]: scratch column slot of a node in piece p, or -1
  double* scr;      // [piece item][3 * scr_cols][96]: the pieces' A column segments
  double* fd;       // [piece item][32][12]: the pieces' FI and diagonal-block partial sums
};

// Batched H/G assembly of many systems (assembly.cu): d_args[i] describes system i
// (mode HG: H into A with lda, G with ldg).  Regular pairs: one persistent launch over
// the work items `tiles` ((system, 32-node tile), taken in order from `counter`,
// which must be zero).  Singular pairs: one warp per node of every system, the
// systems' node offsets in node_off (nsys + 1 entries).
int launch_batch_hg(cudaStream_t stream, int sm_count, const AsmArgs* d_args, const int2* d_tiles, int ntiles,
                    unsigned* counter, const int* d_node_off, int nsys, int total_nodes, long long* launches);

}  // namespace bem
