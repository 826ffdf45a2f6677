// ghmat8 on the GPU: collocation assembly of A x = FI (assembly_mod.f90:53-223),
// and the separate H/G products used for entrywise parity.
//
// Work split
//   * regular pairs (collocation node not on the element; extin8, :339-384):
//     one CTA owns 32 consecutive collocation nodes (96 rows of A) and walks the
//     whole element list.  Its 8 warps take the 8 elements of one "batch" at a
//     time; the elements of a batch share no node, so the 8 warps write disjoint
//     columns of A and need no atomics, and a __syncthreads between batches orders
//     the read-modify-writes of columns that neighbouring batches share.  Lane L of
//     every warp integrates node (32*blockIdx + L) against the warp's element, so the
//     element's quadrature table is a warp-uniform broadcast and the 3 rows of each
//     lane make every column update one contiguous 768-byte segment.  FI and the
//     rigid-body sums d1 stay in registers and are reduced across warps in a fixed
//     order at the end (deterministic).
//   * singular pairs (node on the element; locin8/triloc8, :386-616): one warp per
//     collocation node, its <= 8 elements in sequence; lane (k, s) integrates the
//     3x3 blocks of element node k over every third point of the sub-triangles, the
//     partial sums meet in shared memory, and d2 = -sum_{k != nodo} h_k is a warp
//     reduction.  Launched after the regular kernel on the same stream.
// The column swap (:125-218) uses a per-(node, component) lookup built on the host
// from the same node->element adjacency the reference scans (uknown / vp).
#include <algorithm>
#include <cstdlib>

#include "asm_args.cuh"
#include "common.cuh"
#include "shape.cuh"

namespace bem {

enum { kModeA = 0, kModeHG = 1 };


// symmetric 3x3 index (jj, ii) -> 0..5 : xx yy zz xy yz zx
__device__ __forceinline__ int sym_idx(int a, int b) {
  if (a == b) return a;
  const int s = a + b;  // 1: xy, 3: yz, 2: zx
  return s == 1 ? 3 : (s == 3 ? 4 : 5);
}

// The boundary record of an element for mode A (the column swap's inputs, staged in
// shared memory with the element's quadrature table so that the element's epilogue
// reads warp-uniform values from shared memory instead of global memory):
//   doubles [k + 9 ld]       bc(k, ld) of the element (its prescribed displacement or
//                            traction value, io_mod layout bc(3k + ld + 27 e))
//   doubles [27 + k + 9 ld]  vp of the element node's dof 3 kc[k] + ld
//   ints    kRecInt + 0      bit ld: kode(ld, e) != 0; bit 3 + k + 9 ld: uknown(dof) != 0
//   ints    kRecInt + 1      the element's node count; + 2..10 its nodes (0-based)
constexpr int kRecD = 60;              // doubles per record (480 B)
constexpr int kRecInt = 2 * 54;        // int offset of the flags
__global__ void elem_record_kernel(AsmArgs P, double* rec) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= P.ne) return;
  double* R = rec + (int64_t)e * kRecD;
  int* I = reinterpret_cast<int*>(R) + kRecInt;
  const int ncone = P.nconec[e];
  unsigned bits = 0;
  for (int ld = 0; ld < 3; ++ld) {
    if (P.kode[3 * e + ld] != 0) bits |= 1u << ld;
    for (int k = 0; k < 9; ++k) {
      double b = 0.0, v = 0.0;
      if (k < ncone) {
        const int64_t dof = 3 * (int64_t)(P.kconec[k + 9 * e] - 1) + ld;
        b = P.bc[3 * k + ld + 27 * e];
        v = P.vp[dof];
        if (P.uknown[dof] != 0) bits |= 1u << (3 + k + 9 * ld);
      }
      R[k + 9 * ld] = b;
      R[27 + k + 9 * ld] = v;
    }
  }
  I[0] = (int)bits;
  I[1] = ncone;
  for (int k = 0; k < 9; ++k) I[2 + k] = (k < ncone) ? P.kconec[k + 9 * e] - 1 : 0;
  I[11] = 0;
}

// fi_acc (3) and d1_acc (9) are this lane's running sums over its elements, kept in
// shared memory so the 9 x NC accumulators below have the register file to themselves.
// T: the element's packed quadrature table, staged in shared memory by the caller.
// Mode A adds column kc[k] (3 DOFs) of the element's block at Ab + dof * ald + row: A
// itself, or a piece's scratch, whose columns are the piece's node slots.
template <int NC, int MODE, typename R>
__device__ __forceinline__ void regular_pair(const AsmArgs& P, int e, const double* T, const double* Rec,
                                             const int* kc, double xi0, double xi1, double xi2, double* Ab,
                                             int64_t ald, int64_t row, double* fi_acc, double* d1) {
  // mode A: the element's boundary record Rec (shared memory)
  const unsigned rbits = (MODE == kModeA) ? (unsigned)reinterpret_cast<const int*>(Rec)[kRecInt] : 0u;
  double fi[3] = {0.0, 0.0, 0.0};
  constexpr int NG = (NC == 9) ? 36 : 16;
  const double c3 = P.mat.c3, c4 = P.mat.c4, c5 = P.mat.c5, c6 = P.mat.c6;

  // ---- G: U* (symmetric, 6 values) x p12 -------------------------------------------
  {
    R g[NC][6];
#pragma unroll
    for (int k = 0; k < NC; ++k)
#pragma unroll
      for (int p = 0; p < 6; ++p) g[k][p] = R(0);
    const R rc3 = (R)c3, rc4 = (R)c4;
#pragma unroll 2
    for (int q = 0; q < NG; ++q) {
      // the coordinate difference is always formed in FP64 (no cancellation in R)
      const R r0 = (R)(T[6 * q + 0] - xi0);
      const R r1 = (R)(T[6 * q + 1] - xi1);
      const R r2 = (R)(T[6 * q + 2] - xi2);
      const R ri = rsqrt(r0 * r0 + r1 * r1 + r2 * r2);
      const R a0 = r0 * ri, a1 = r1 * ri, a2 = r2 * ri;
      const R c3r = rc3 * ri;
      R u[6];
      u[0] = (rc4 + a0 * a0) * c3r;
      u[1] = (rc4 + a1 * a1) * c3r;
      u[2] = (rc4 + a2 * a2) * c3r;
      u[3] = a0 * a1 * c3r;
      u[4] = a1 * a2 * c3r;
      u[5] = a2 * a0 * c3r;
      const double* W = T + kTabGeo + 9 * q;
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        const R w = (R)W[k];
#pragma unroll
        for (int p = 0; p < 6; ++p) g[k][p] = fma(u[p], w, g[k][p]);
      }
    }
    if (MODE == kModeA) {
#pragma unroll
      for (int ld = 0; ld < 3; ++ld) {
        if (((rbits >> ld) & 1u) == 0) {
          // the element's 3 x NC block added into A by reductions at L2 (no load on the
          // SM's critical path); the batches' CTA barrier orders the additions into an
          // entry, so the sums are deterministic
          const double mu = P.mat.mu;
#pragma unroll
          for (int k = 0; k < NC; ++k) {
            double* col = Ab + (3 * (int64_t)kc[k] + ld) * ald + row;
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) atomicAdd(col + jj, -(g[k][sym_idx(jj, ld)] * mu));
          }
        } else {
#pragma unroll
          for (int k = 0; k < NC; ++k) {
            const double b = Rec[k + 9 * ld];
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) fi[jj] = fma(g[k][sym_idx(jj, ld)], b, fi[jj]);
          }
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < NC; ++k)
#pragma unroll
        for (int ii = 0; ii < 3; ++ii) {
          double* col = P.G + (27 * (int64_t)e + 3 * k + ii) * P.ldg + row;
#pragma unroll
          for (int jj = 0; jj < 3; ++jj) col[jj] = g[k][sym_idx(jj, ii)];
        }
    }
  }

  // ---- H: T* (9 values) x p12 ------------------------------------------------------
  {
    R h[NC][9];  // h[k][jj + 3*ii]
#pragma unroll
    for (int k = 0; k < NC; ++k)
#pragma unroll
      for (int p = 0; p < 9; ++p) h[k][p] = R(0);
    const R rc5 = (R)c5, rc6 = (R)c6;
#pragma unroll 1
    for (int q = 0; q < NG; ++q) {
      const R r0 = (R)(T[6 * q + 0] - xi0);
      const R r1 = (R)(T[6 * q + 1] - xi1);
      const R r2 = (R)(T[6 * q + 2] - xi2);
      const R n[3] = {(R)T[6 * q + 3], (R)T[6 * q + 4], (R)T[6 * q + 5]};
      const R ri = rsqrt(r0 * r0 + r1 * r1 + r2 * r2);
      const R a[3] = {r0 * ri, r1 * ri, r2 * ri};
      const R rdn = a[0] * n[0] + a[1] * n[1] + a[2] * n[2];
      const R c5r2 = rc5 * ri * ri;
      // T*(ii, jj) = c5/r^2 (rdn (c6 delta + 3 a_ii a_jj) + c6 (n_jj a_ii - n_ii a_jj)):
      // the symmetric part from the 6 products a_ii a_jj, the antisymmetric part from 3
      const R k1 = R(3) * c5r2 * rdn, k2 = c5r2 * rc6, k3 = k2 * rdn;
      const R s00 = k1 * (a[0] * a[0]) + k3, s11 = k1 * (a[1] * a[1]) + k3, s22 = k1 * (a[2] * a[2]) + k3;
      const R s01 = k1 * (a[0] * a[1]), s12 = k1 * (a[1] * a[2]), s20 = k1 * (a[2] * a[0]);
      const R b01 = k2 * (n[1] * a[0] - n[0] * a[1]);  // antisymmetric (ii, jj) = (0, 1)
      const R b12 = k2 * (n[2] * a[1] - n[1] * a[2]);
      const R b20 = k2 * (n[0] * a[2] - n[2] * a[0]);
      // t[jj + 3 ii]
      const R t[9] = {s00, s01 + b01, s20 - b20, s01 - b01, s11, s12 + b12, s20 + b20, s12 - b12, s22};
      const double* W = T + kTabGeo + 9 * q;
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        const R w = (R)W[k];
#pragma unroll
        for (int p = 0; p < 9; ++p) h[k][p] = fma(t[p], w, h[k][p]);
      }
    }
    // rigid-body partial sums d1(i, j) = -sum_k h(i, 3k + j) (assembly_mod.f90:103-111)
#pragma unroll
    for (int p = 0; p < 9; ++p) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < NC; ++k) s += (double)h[k][p];
      d1[p] -= s;
    }
    if (MODE == kModeA) {
#pragma unroll
      for (int ld = 0; ld < 3; ++ld) {
        if (((rbits >> ld) & 1u) == 0) {
#pragma unroll
          for (int k = 0; k < NC; ++k) {
            const double b = Rec[k + 9 * ld];
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) fi[jj] = fma(-h[k][jj + 3 * ld], b, fi[jj]);
          }
        } else {
          // the same reductions into A for the unknown columns; the prescribed ones go
          // to FI
#pragma unroll
          for (int k = 0; k < NC; ++k) {
            const int64_t dof = 3 * (int64_t)kc[k] + ld;
            if (((rbits >> (3 + k + 9 * ld)) & 1u) == 0) {
              double* col = Ab + dof * ald + row;
#pragma unroll
              for (int jj = 0; jj < 3; ++jj) atomicAdd(col + jj, h[k][jj + 3 * ld]);
            } else {
              const double v = Rec[27 + k + 9 * ld];
#pragma unroll
              for (int jj = 0; jj < 3; ++jj) fi[jj] = fma(-h[k][jj + 3 * ld], v, fi[jj]);
            }
          }
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < NC; ++k)
#pragma unroll
        for (int ii = 0; ii < 3; ++ii)
#pragma unroll
          for (int jj = 0; jj < 3; ++jj)
            atomicAdd(P.A + (3 * (int64_t)kc[k] + ii) * P.lda + row + jj, h[k][jj + 3 * ii]);
    }
  }
  if (MODE == kModeA)
#pragma unroll
    for (int jj = 0; jj < 3; ++jj) fi_acc[jj] += fi[jj];
}

// PREC 0: every regular pair in FP64.  PREC 1: pairs farther than 3.5 element radii
// from the element centroid (the near-field radius of stress_mod.f90:603-604) evaluate
// and accumulate the Kelvin kernels in FP32; nearer pairs stay in FP64.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}

// Dynamic shared memory of the regular tile: two buffers of one quadrature table per
// warp (the batch being integrated and the next one, copied in meanwhile).
constexpr int kTabSmem = 2 * kBatch * (kTabStride + kRecD) * (int)sizeof(double);

// Tile `tile` (32 collocation nodes) against the element batches [b0, b1); piece
// `part` >= 1 of a split tile adds into its scratch instead of A and FI.
template <int MODE, int PREC>
__device__ __forceinline__ void regular_tile(const AsmArgs& P, int tile, int part, int b0, int b1) {
  __shared__ double s_red[kBatch][32][12];
  extern __shared__ __align__(16) double s_tab[];  // [2][kBatch][kTabStride], then [2][kBatch][kRecD]
  double* s_rec = s_tab + 2 * kBatch * kTabStride;
  const int w = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  // each warp copies its own next element's table (16-byte cp.async, 270 per table)
  // while it integrates the current one: the table loads leave the dependent chain
  auto prefetch = [&](int b) {
    if (b < b1) {
      const int e = __ldg(P.batches + kBatch * b + w);
      if (e >= 0) {
        const char* src = reinterpret_cast<const char*>(P.tab + (int64_t)e * kTabStride);
        char* dst = reinterpret_cast<char*>(s_tab + ((b & 1) * kBatch + w) * kTabStride);
        for (int i = lane; i < kTabStride * 8 / 16; i += 32) cp_async16(dst + 16 * i, src + 16 * i);
        if (MODE == kModeA) {  // and its boundary record
          const char* rs = reinterpret_cast<const char*>(P.rec + (int64_t)e * kRecD);
          char* rd = reinterpret_cast<char*>(s_rec + ((b & 1) * kBatch + w) * kRecD);
          if (lane < kRecD * 8 / 16) cp_async16(rd + 16 * lane, rs + 16 * lane);
        }
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  const int local = tile * 32 + lane;  // node offset inside the row range
  const bool active = local < P.nrows_nodes;
  const int in = P.in0 + (active ? local : 0);
  const double xi0 = P.x[in], xi1 = P.y[in], xi2 = P.z[in];
  const int64_t row = 3 * (int64_t)local;
  // where the element blocks go: A's rows of this tile, or the piece's scratch item
  // (96 rows, the piece's node slots as columns)
  const int64_t item = part > 0 ? (int64_t)(tile - P.tail0) * (P.nparts - 1) + (part - 1) : 0;
  double* Ab = part > 0 ? P.scr + item * (3 * (int64_t)P.scr_cols) * 96 : P.A;
  const int64_t ald = part > 0 ? 96 : P.lda;
  const int64_t arow = part > 0 ? 3 * (int64_t)lane : row;
  double* fi = &s_red[w][lane][0];  // running FI sums of this lane
  double* d1 = &s_red[w][lane][3];  // running rigid-body sums d1
#pragma unroll
  for (int p = 0; p < 12; ++p) s_red[w][lane][p] = 0.0;

  prefetch(b0);
  for (int b = b0; b < b1; ++b) {
    const int e = __ldg(P.batches + kBatch * b + w);
    prefetch(b + 1);
    asm volatile("cp.async.wait_group 1;" ::: "memory");  // this batch's table is in
    __syncwarp();
    const double* T = s_tab + ((b & 1) * kBatch + w) * kTabStride;
    const double* R = s_rec + ((b & 1) * kBatch + w) * kRecD;
    if (e >= 0) {
      const int* RI = reinterpret_cast<const int*>(R) + kRecInt;
      const int ncone = (MODE == kModeA) ? RI[1] : __ldg(P.nconec + e);
      int kc[9];
      bool sing = false;
#pragma unroll
      for (int m = 0; m < 9; ++m) {
        kc[m] = (MODE == kModeA) ? RI[2 + m] : ((m < ncone) ? __ldg(P.kconec + m + 9 * e) - 1 : 0);
        sing |= (m < ncone) && (kc[m] == in);
      }
      bool far32 = false;
      if (PREC == 1) {
        double cx = 0.0, cy = 0.0, cz = 0.0;
        for (int m = 0; m < ncone; ++m) {
          cx += P.x[kc[m]];
          cy += P.y[kc[m]];
          cz += P.z[kc[m]];
        }
        cx /= ncone;
        cy /= ncone;
        cz /= ncone;
        double r2 = 0.0;
        for (int m = 0; m < ncone; ++m) {
          const double dx = P.x[kc[m]] - cx, dy = P.y[kc[m]] - cy, dz = P.z[kc[m]] - cz;
          r2 = fmax(r2, dx * dx + dy * dy + dz * dz);
        }
        const double dx = xi0 - cx, dy = xi1 - cy, dz = xi2 - cz;
        far32 = dx * dx + dy * dy + dz * dz > 12.25 * r2;
      }
      if (part > 0)  // a piece's columns are its node slots
#pragma unroll
        for (int m = 0; m < 9; ++m) kc[m] = (m < ncone) ? __ldg(P.slot + (int64_t)(part - 1) * P.n + kc[m]) : 0;
      if (active && !sing) {
        if (ncone == 9) {
          if (far32)
            regular_pair<9, MODE, float>(P, e, T, R, kc, xi0, xi1, xi2, Ab, ald, arow, fi, d1);
          else
            regular_pair<9, MODE, double>(P, e, T, R, kc, xi0, xi1, xi2, Ab, ald, arow, fi, d1);
        } else {
          if (far32)
            regular_pair<6, MODE, float>(P, e, T, R, kc, xi0, xi1, xi2, Ab, ald, arow, fi, d1);
          else
            regular_pair<6, MODE, double>(P, e, T, R, kc, xi0, xi1, xi2, Ab, ald, arow, fi, d1);
        }
      }
    }
    __syncthreads();
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");

  __syncthreads();
  if (w == 0 && active) {
    double F[3] = {0.0, 0.0, 0.0}, D[9];
    for (int p = 0; p < 9; ++p) D[p] = 0.0;
    for (int ww = 0; ww < kBatch; ++ww) {
      for (int p = 0; p < 3; ++p) F[p] += s_red[ww][lane][p];
      for (int p = 0; p < 9; ++p) D[p] += s_red[ww][lane][3 + p];
    }
    if (part > 0) {  // the piece's partial sums, added by tail_merge_fd_kernel
      double* o = P.fd + (item * 32 + lane) * 12;
      for (int p = 0; p < 3; ++p) o[p] = F[p];
      for (int p = 0; p < 9; ++p) o[3 + p] = D[p];
    } else if (MODE == kModeA) {
      // diagonal block from the non-singular elements (assembly_mod.f90:192-218)
      for (int ld = 0; ld < 3; ++ld) {
        const int64_t dof = 3 * (int64_t)in + ld;
        if (P.uknown[dof] == 0) {
          double* col = P.A + dof * P.lda + row;
          for (int r = 0; r < 3; ++r) col[r] += D[r + 3 * ld];
        } else {
          const double v = P.vp[dof];
          for (int r = 0; r < 3; ++r) F[r] -= D[r + 3 * ld] * v;
        }
      }
      for (int r = 0; r < 3; ++r) P.FI[row + r] = F[r];
    } else {
      for (int ld = 0; ld < 3; ++ld) {
        double* col = P.A + (3 * (int64_t)in + ld) * P.lda + row;
        for (int r = 0; r < 3; ++r) col[r] += D[r + 3 * ld];
      }
    }
  }
}

// One CTA per 32-node tile.  With a split last wave (mode A, P.nparts > 1) the CTAs
// from tail0 on are the pieces of the last tiles, nparts per tile, piece p over the
// batches [nbatches p / nparts, nbatches (p + 1) / nparts): the last wave ends after
// about 1 / nparts of a tile's time instead of a whole tile's.
template <int MODE, int PREC>
__global__ void __launch_bounds__(256, 1) ghmat_regular_kernel(AsmArgs P) {
  if (P.nparts > 1 && (int)blockIdx.x >= P.tail0) {
    const int i = blockIdx.x - P.tail0, part = i % P.nparts;
    const int b0 = (int)((int64_t)P.nbatches * part / P.nparts);
    const int b1 = (int)((int64_t)P.nbatches * (part + 1) / P.nparts);
    regular_tile<MODE, PREC>(P, P.tail0 + i / P.nparts, part, b0, b1);
  } else {
    regular_tile<MODE, PREC>(P, blockIdx.x, 0, 0, P.nbatches);
  }
}

// The pieces' A column segments into A: segment (tail tile t, node j, DOF ld) of 96
// rows, one warp each; the pieces' contributions are summed in piece order and added
// once, so the result is deterministic.
__global__ void tail_merge_cols_kernel(AsmArgs P, int ntail) {
  const int lane = threadIdx.x & 31;
  const int64_t nseg = (int64_t)ntail * P.n * 3;
  const int64_t wstride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t sg = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; sg < nseg; sg += wstride) {
    const int ld = (int)(sg % 3);
    const int64_t q = sg / 3;
    const int j = (int)(q % P.n), t = (int)(q / P.n);
    const int tile = P.tail0 + t;
    const int rows = 3 * min(32, P.nrows_nodes - 32 * tile);
    double acc[3] = {0.0, 0.0, 0.0};
    bool any = false;
    for (int p = 1; p < P.nparts; ++p) {
      const int sl = __ldg(P.slot + (int64_t)(p - 1) * P.n + j);
      if (sl >= 0) {
        any = true;
        const int64_t item = (int64_t)t * (P.nparts - 1) + (p - 1);
        const double* src = P.scr + (item * 3 * P.scr_cols + 3 * (int64_t)sl + ld) * 96;
#pragma unroll
        for (int u = 0; u < 3; ++u) acc[u] += src[lane + 32 * u];
      }
    }
    if (any) {
      double* dst = P.A + (3 * (int64_t)j + ld) * P.lda + 96 * (int64_t)tile;
#pragma unroll
      for (int u = 0; u < 3; ++u)
        if (lane + 32 * u < rows) dst[lane + 32 * u] += acc[u];
    }
  }
}

// The pieces' FI and diagonal-block partial sums (assembly_mod.f90:192-218), one
// thread per node of the tail tiles, after tail_merge_cols_kernel.
__global__ void tail_merge_fd_kernel(AsmArgs P, int ntail) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 32 * ntail) return;
  const int t = i >> 5, lane = i & 31;
  const int local = 32 * (P.tail0 + t) + lane;
  if (local >= P.nrows_nodes) return;
  const int in = P.in0 + local;
  const int64_t row = 3 * (int64_t)local;
  double F[3] = {0.0, 0.0, 0.0}, D[9];
  for (int p = 0; p < 9; ++p) D[p] = 0.0;
  for (int p = 1; p < P.nparts; ++p) {
    const double* o = P.fd + (((int64_t)t * (P.nparts - 1) + (p - 1)) * 32 + lane) * 12;
    for (int r = 0; r < 3; ++r) F[r] += o[r];
    for (int r = 0; r < 9; ++r) D[r] += o[3 + r];
  }
  for (int ld = 0; ld < 3; ++ld) {
    const int64_t dof = 3 * (int64_t)in + ld;
    if (P.uknown[dof] == 0) {
      double* col = P.A + dof * P.lda + row;
      for (int r = 0; r < 3; ++r) col[r] += D[r + 3 * ld];
    } else {
      const double v = P.vp[dof];
      for (int r = 0; r < 3; ++r) F[r] -= D[r + 3 * ld] * v;
    }
  }
  for (int r = 0; r < 3; ++r) P.FI[row + r] += F[r];
}

// ---------------------------------------------------------------------------------
// singular elements
// ---------------------------------------------------------------------------------

__constant__ double s_gi[6];
__constant__ double s_ome[6];

// Sub-triangles of locin8 (assembly_mod.f90:399-489) for local node nodo (1-based):
// returns the count and fills vertex parent coordinates (vertex 0 = the node).
__device__ int sub_triangles(int ncone, int nodo, double v1[4][3], double v2[4][3],
                             double area[4]) {
  if (ncone == 9) {
    const double gi1[9] = {-1.0, 0.0, 1.0, 1.0, 1.0, 0.0, -1.0, -1.0, 0.0};
    const double gi2[9] = {-1.0, -1.0, -1.0, 0.0, 1.0, 1.0, 1.0, 0.0, 0.0};
    // gii(p) = gi((p-1) mod 8 + 1) for p = 1..15
    auto G1 = [&](int p) { return gi1[(p - 1) % 8]; };
    auto G2 = [&](int p) { return gi2[(p - 1) % 8]; };
    int cnt = 0;
    if (nodo == 9) {
      for (int k = 1; k <= 4; ++k) {
        const int m = 2 * k - 1;
        v1[cnt][0] = gi1[8];
        v2[cnt][0] = gi2[8];
        v1[cnt][1] = G1(m);
        v2[cnt][1] = G2(m);
        v1[cnt][2] = G1(m + 2);
        v2[cnt][2] = G2(m + 2);
        area[cnt] = 1.0;
        ++cnt;
      }
    } else if (nodo & 1) {
      for (int k = 1; k <= 2; ++k) {
        const int m = 2 * k;
        v1[cnt][0] = gi1[nodo - 1];
        v2[cnt][0] = gi2[nodo - 1];
        v1[cnt][1] = G1(nodo + m);
        v2[cnt][1] = G2(nodo + m);
        v1[cnt][2] = G1(nodo + m + 2);
        v2[cnt][2] = G2(nodo + m + 2);
        area[cnt] = 2.0;
        ++cnt;
      }
    } else {
      for (int k = 1; k <= 3; ++k) {
        const int m = 2 * k - 1;
        double a1[3] = {gi1[nodo - 1], G1(nodo + m), G1(nodo + m + 2)};
        double a2[3] = {gi2[nodo - 1], G2(nodo + m), G2(nodo + m + 2)};
        for (int t = 0; t < 3; ++t) {
          v1[cnt][t] = a1[t];
          v2[cnt][t] = a2[t];
        }
        area[cnt] = 0.5 * (a1[1] * a2[2] + a1[0] * a2[1] + a1[2] * a2[0] - a1[1] * a2[0] -
                           a1[2] * a2[1] - a1[0] * a2[2]);
        ++cnt;
      }
    }
    return cnt;
  }
  const double gi1[6] = {1.0, 0.0, 0.0, 0.5, 0.0, 0.5};
  const double gi2[6] = {0.0, 1.0, 0.0, 0.5, 0.5, 0.0};
  int ta[2], tb[2], cnt;
  double ar;
  switch (nodo) {
    case 1: cnt = 1; ta[0] = 2; tb[0] = 3; ar = 0.5; break;
    case 2: cnt = 1; ta[0] = 3; tb[0] = 1; ar = 0.5; break;
    case 3: cnt = 1; ta[0] = 1; tb[0] = 2; ar = 0.5; break;
    case 4: cnt = 2; ta[0] = 2; tb[0] = 3; ta[1] = 3; tb[1] = 1; ar = 0.25; break;
    case 5: cnt = 2; ta[0] = 3; tb[0] = 1; ta[1] = 1; tb[1] = 2; ar = 0.25; break;
    default: cnt = 2; ta[0] = 1; tb[0] = 2; ta[1] = 2; tb[1] = 3; ar = 0.25; break;
  }
  for (int t = 0; t < cnt; ++t) {
    v1[t][0] = gi1[nodo - 1];
    v2[t][0] = gi2[nodo - 1];
    v1[t][1] = gi1[ta[t] - 1];
    v2[t][1] = gi2[ta[t] - 1];
    v1[t][2] = gi1[tb[t] - 1];
    v2[t][2] = gi2[tb[t] - 1];
    area[t] = ar;
  }
  return cnt;
}

// one warp: collocation node `local` of the row range; s_part is the warp's scratch
template <int MODE>
__device__ __forceinline__ void singular_node(const AsmArgs& P, int local, double (*s_part)[18]) {
  const int lane = threadIdx.x & 31;
  const int in = P.in0 + local;
  const int64_t row = 3 * (int64_t)local;
  const int k = lane % 9;
  const int s = lane / 9;  // 0..2 active, 3 idle (lanes 27..31)
  const double c3 = P.mat.c3, c4 = P.mat.c4, c5 = P.mat.c5, c6 = P.mat.c6;
  const double xi[3] = {P.x[in], P.y[in], P.z[in]};
  double fi[3] = {0.0, 0.0, 0.0};
  double dsum[9];  // diagonal contributions for mode HG
  for (int p = 0; p < 9; ++p) dsum[p] = 0.0;
  const int cnt = min(P.nesim[in], 8);
  for (int je = 0; je < cnt; ++je) {
    const int e = P.ke[je + 8 * in] - 1;
    const int ncone = P.nconec[e];
    int kc[9];
    int nodo = 0;
    double xj1[9], xj2[9], xj3[9];
    for (int m = 0; m < 9; ++m) {
      kc[m] = (m < ncone) ? P.kconec[m + 9 * e] - 1 : 0;
      xj1[m] = (m < ncone) ? P.x[kc[m]] : 0.0;
      xj2[m] = (m < ncone) ? P.y[kc[m]] : 0.0;
      xj3[m] = (m < ncone) ? P.z[kc[m]] : 0.0;
      if (m < ncone && kc[m] == in && nodo == 0) nodo = m + 1;
    }
    double v1[4][3], v2[4][3], area[4];
    const int ntri = sub_triangles(ncone, nodo, v1, v2, area);
    double g[9], h[9];
    for (int p = 0; p < 9; ++p) g[p] = h[p] = 0.0;
    if (s < 3 && k < ncone) {
      const int total = ntri * 36;
      for (int t = s; t < total; t += 3) {
        const int tri = t / 36, q = t % 36, i = q / 6, j = q % 6;
        const double ss1 = 0.5 * (s_gi[i] + 1.0), ss2 = 0.5 * (s_gi[j] + 1.0);
        const double g1 = (1.0 - ss1) * v1[tri][0] + ss1 * (1.0 - ss2) * v1[tri][1] +
                          ss1 * ss2 * v1[tri][2];
        const double g2 = (1.0 - ss1) * v2[tri][0] + ss1 * (1.0 - ss2) * v2[tri][1] +
                          ss1 * ss2 * v2[tri][2];
        double f[9], fd1[9], fd2[9];
        shape_fn<double>(ncone, g1, g2, f, fd1, fd2);
        double xp[3] = {0.0, 0.0, 0.0}, t1[3] = {0.0, 0.0, 0.0}, t2[3] = {0.0, 0.0, 0.0};
        for (int m = 0; m < ncone; ++m) {
          xp[0] += f[m] * xj1[m];
          xp[1] += f[m] * xj2[m];
          xp[2] += f[m] * xj3[m];
          t1[0] += fd1[m] * xj1[m];
          t1[1] += fd1[m] * xj2[m];
          t1[2] += fd1[m] * xj3[m];
          t2[0] += fd2[m] * xj1[m];
          t2[1] += fd2[m] * xj2[m];
          t2[2] += fd2[m] * xj3[m];
        }
        const double cr0 = t1[1] * t2[2] - t1[2] * t2[1];
        const double cr1 = t1[2] * t2[0] - t1[0] * t2[2];
        const double cr2 = t1[0] * t2[1] - t1[1] * t2[0];
        const double J = sqrt(cr0 * cr0 + cr1 * cr1 + cr2 * cr2);
        const double n[3] = {cr0 / J, cr1 / J, cr2 / J};
        const double pk = f[k] * J * (s_gi[i] + 1.0) * area[tri] * 0.25 * s_ome[i] * s_ome[j];
        const double r0 = xp[0] - xi[0], r1 = xp[1] - xi[1], r2 = xp[2] - xi[2];
        const double ri = rsqrt(r0 * r0 + r1 * r1 + r2 * r2);
        const double a[3] = {r0 * ri, r1 * ri, r2 * ri};
        const double rdn = a[0] * n[0] + a[1] * n[1] + a[2] * n[2];
        const double c3r = c3 * ri, c5r2 = c5 * ri * ri;
        for (int ii = 0; ii < 3; ++ii)
          for (int jj = 0; jj < 3; ++jj) {
            const double dl = (ii == jj) ? 1.0 : 0.0;
            const double u = (c4 * dl + a[ii] * a[jj]) * c3r;
            const double tt = c5r2 * (rdn * (c6 * dl + 3.0 * a[ii] * a[jj]) +
                                      c6 * (n[jj] * a[ii] - n[ii] * a[jj]));
            g[jj + 3 * ii] += u * pk;
            h[jj + 3 * ii] += tt * pk;
          }
      }
    }
    // combine the three point subsets of each node k
    if (s < 3)
      for (int p = 0; p < 9; ++p) {
        s_part[lane][p] = g[p];
        s_part[lane][9 + p] = h[p];
      }
    __syncwarp();
    if (s == 0) {
      for (int p = 0; p < 9; ++p) {
        g[p] = s_part[k][p] + s_part[k + 9][p] + s_part[k + 18][p];
        h[p] = s_part[k][9 + p] + s_part[k + 9][9 + p] + s_part[k + 18][9 + p];
      }
    }
    __syncwarp();
    // d2 = -sum_{k != nodo} h_k  (assembly_mod.f90:113-122)
    double d2[9];
    for (int p = 0; p < 9; ++p) {
      double v = (s == 0 && k < ncone && k != nodo - 1) ? h[p] : 0.0;
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      d2[p] = -v;
    }
    if (s == 0 && k < ncone) {
      const int ik = kc[k];
      if (MODE == kModeA) {
        for (int ld = 0; ld < 3; ++ld) {
          const double bcv = P.bc[3 * k + ld + 27 * e];
          const double* hk = (k == nodo - 1) ? d2 : h;  // entry at the node: rigid body
          if (P.kode[3 * e + ld] == 0) {
            double* col = P.A + (3 * (int64_t)ik + ld) * P.lda + row;
            for (int jj = 0; jj < 3; ++jj) col[jj] -= g[jj + 3 * ld] * P.mat.mu;
            for (int jj = 0; jj < 3; ++jj) fi[jj] -= hk[jj + 3 * ld] * bcv;
          } else {
            const int64_t dof = 3 * (int64_t)ik + ld;
            if (P.uknown[dof] == 0) {
              for (int jj = 0; jj < 3; ++jj) fi[jj] += g[jj + 3 * ld] * bcv;
              double* col = P.A + dof * P.lda + row;
              for (int jj = 0; jj < 3; ++jj) col[jj] += hk[jj + 3 * ld];
            } else {
              const double v = P.vp[dof];
              for (int jj = 0; jj < 3; ++jj) fi[jj] += g[jj + 3 * ld] * bcv - hk[jj + 3 * ld] * v;
            }
          }
        }
      } else {
        for (int ii = 0; ii < 3; ++ii) {
          double* gc = P.G + (27 * (int64_t)e + 3 * k + ii) * P.ldg + row;
          for (int jj = 0; jj < 3; ++jj) gc[jj] = g[jj + 3 * ii];
          if (k != nodo - 1) {
            double* hc = P.A + (3 * (int64_t)ik + ii) * P.lda + row;
            for (int jj = 0; jj < 3; ++jj) hc[jj] += h[jj + 3 * ii];
          }
        }
        if (k == 0)
          for (int p = 0; p < 9; ++p) dsum[p] += d2[p];
      }
    }
    __syncwarp();
  }
  if (MODE == kModeA) {
    for (int p = 0; p < 3; ++p) {
      double v = (s == 0) ? fi[p] : 0.0;
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      fi[p] = v;
    }
    if (lane == 0)
      for (int r = 0; r < 3; ++r) P.FI[row + r] += fi[r];
  } else if (lane == 0) {
    for (int ld = 0; ld < 3; ++ld) {
      double* col = P.A + (3 * (int64_t)in + ld) * P.lda + row;
      for (int r = 0; r < 3; ++r) col[r] += dsum[r + 3 * ld];
    }
  }
}

template <int MODE>
__global__ void __launch_bounds__(128) ghmat_singular_kernel(AsmArgs P) {
  __shared__ double s_part[4][27][18];
  const int wib = threadIdx.x >> 5;
  const int local = blockIdx.x * 4 + wib;
  if (local >= P.nrows_nodes) return;  // warp-uniform
  singular_node<MODE>(P, local, s_part[wib]);
}

// Pinned DOFs: row := unit row, rhs := 0.
__global__ void pins_kernel(const int* pins, int npins, int64_t ncol, double* A, int64_t lda,
                            double* FI) {
  const int p = blockIdx.y;
  if (p >= npins) return;
  const int64_t r = pins[p];
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncol;
       c += (int64_t)gridDim.x * blockDim.x)
    A[r + c * lda] = (c == r) ? 1.0 : 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) FI[r] = 0.0;
}

static AsmArgs make_args(bem_ctx* c) {
  AsmArgs P{};
  P.n = c->n;
  P.ne = c->ne;
  P.nbatches = c->nbatches;
  P.in0 = 0;
  P.nrows_nodes = c->n;
  P.batches = c->batches.p;
  P.nconec = c->nconec.p;
  P.kconec = c->kconec.p;
  P.kode = c->kode.p;
  P.bc = c->bc.p;
  P.uknown = c->uknown.p;
  P.vp = c->vp.p;
  P.nesim = c->nesim.p;
  P.ke = c->ke.p;
  P.x = c->x.p;
  P.y = c->y.p;
  P.z = c->z.p;
  P.tab = c->tab.p;
  P.mat = c->mat;
  return P;
}

static int upload_singular_constants(bem_ctx* c) {
  static DeviceOnce once;  // __constant__ tables are per device
  if (!once.pending()) return BEM_OK;
  BEM_CUDA(c, cudaMemcpyToSymbol(s_gi, kGiQuad, sizeof(kGiQuad)));
  BEM_CUDA(c, cudaMemcpyToSymbol(s_ome, kOmeQuad, sizeof(kOmeQuad)));
  once.mark();
  return BEM_OK;
}

// The last wave of the regular kernel: the tiles beyond the last full wave (rem of
// them) run as pieces over shares of the batch list, as many pieces per tile as fill
// the SMs (at most kMaxPieces), so that the kernel ends about (1 - 1 / pieces) of a
// tile's time earlier.  Pieces >= 1 need a scratch item each: 96 rows by the piece's
// node slots (the nodes of its elements), at most kTailScratch bytes in all.  Sets
// P's split fields (nparts = 1: no split) and returns the number of split tiles.
constexpr int kMaxPieces = 8;
constexpr size_t kTailScratch = size_t(4) << 30;

static int plan_tail(bem_ctx* c, AsmArgs& P, int tiles, int& rc) {
  rc = BEM_OK;
  P.nparts = 1;
  P.tail0 = tiles;
  const char* env = std::getenv("BEM_ASM_SPLIT");
  if (env && std::atoi(env) == 0) return 0;
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ghmat_regular_kernel<kModeA, 0>, 256, kTabSmem) !=
          cudaSuccess ||
      occ < 1) {
    cudaGetLastError();
    return 0;
  }
  const int wave = c->sm_count * occ;
  const int rem = tiles % wave;
  if (rem == 0) return 0;
  int pp = std::min(std::min(kMaxPieces, wave / rem), c->nbatches);
  for (; pp >= 2; --pp) {
    if (c->tail_parts != pp) {  // node slots of pieces 1 .. pp-1 (cached per mesh)
      std::vector<int> slot((size_t)(pp - 1) * c->n, -1);
      int cols = 0;
      for (int p = 1; p < pp; ++p) {
        const int b0 = (int)((int64_t)c->nbatches * p / pp), b1 = (int)((int64_t)c->nbatches * (p + 1) / pp);
        int* sl = slot.data() + (size_t)(p - 1) * c->n;
        std::vector<int> nodes;
        for (size_t i = (size_t)b0 * kBatch; i < (size_t)b1 * kBatch; ++i) {
          const int e = c->h_batches[i];
          if (e < 0) continue;
          for (int m = 0; m < c->h_nconec[e]; ++m) nodes.push_back(c->h_kconec[m + 9 * (size_t)e] - 1);
        }
        std::sort(nodes.begin(), nodes.end());
        nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
        for (size_t k = 0; k < nodes.size(); ++k) sl[nodes[k]] = (int)k;
        cols = std::max(cols, (int)nodes.size());
      }
      const size_t bytes = (size_t)rem * (pp - 1) * ((size_t)3 * cols * 96 + 32 * 12) * sizeof(double);
      if (bytes > kTailScratch) continue;
      c->tail_parts = 0;
      if (c->tail_slot.alloc(slot.size()) != cudaSuccess) {
        cudaGetLastError();
        return 0;
      }
      if (cudaMemcpy(c->tail_slot.p, slot.data(), slot.size() * sizeof(int), cudaMemcpyHostToDevice) !=
          cudaSuccess) {
        rc = bem_fail(c, BEM_ERR_CUDA, "uploading the assembly's piece slots");
        return 0;
      }
      c->tail_parts = pp;
      c->tail_cols = cols;
    }
    const size_t nscr = (size_t)rem * (pp - 1) * 3 * c->tail_cols * 96, nfd = (size_t)rem * (pp - 1) * 32 * 12;
    if ((c->tail_scr.count < nscr && c->tail_scr.alloc(nscr) != cudaSuccess) ||
        (c->tail_fd.count < nfd && c->tail_fd.alloc(nfd) != cudaSuccess)) {
      cudaGetLastError();  // no room: no split
      c->tail_scr.release();
      c->tail_fd.release();
      return 0;
    }
    if (cudaMemsetAsync(c->tail_scr.p, 0, nscr * sizeof(double), c->stream) != cudaSuccess) {
      rc = bem_fail(c, BEM_ERR_CUDA, "clearing the assembly's piece scratch");
      return 0;
    }
    P.nparts = pp;
    P.tail0 = tiles - rem;
    P.scr_cols = c->tail_cols;
    P.slot = c->tail_slot.p;
    P.scr = c->tail_scr.p;
    P.fd = c->tail_fd.p;
    return rem;
  }
  return 0;
}

int launch_ghmat8(bem_ctx* c, int precision) {
  if (!c->have_geometry || !c->have_bc || !c->have_material)
    return bem_fail(c, BEM_ERR_STATE, "ghmat8 needs mesh, material, bc and geometry");
  if (precision != BEM_ASM_FP64 && precision != BEM_ASM_FP32_FAR)
    return bem_fail(c, BEM_ERR_ARG, "unknown assembly precision");
  int rc = upload_singular_constants(c);
  if (rc) return rc;
  const int64_t N = 3 * (int64_t)c->n;
  const int64_t lda = (N + 31) / 32 * 32;
  if (c->A.count != (size_t)(lda * N)) {
    c->A.release();
    cudaError_t e = c->A.alloc((size_t)(lda * N));
    if (e != cudaSuccess) return bem_fail(c, BEM_ERR_OOM, "allocating the system matrix");
  }
  c->lda = lda;
  BEM_CUDA(c, c->FI.alloc(N));
  BEM_CUDA(c, cudaMemsetAsync(c->A.p, 0, c->A.bytes(), c->stream));
  AsmArgs P = make_args(c);
  P.A = c->A.p;
  P.lda = lda;
  P.FI = c->FI.p;
  BEM_CUDA(c, c->erec.alloc((size_t)c->ne * kRecD));
  elem_record_kernel<<<(c->ne + 127) / 128, 128, 0, c->stream>>>(P, c->erec.p);
  BEM_LAUNCH_CHECK(c);
  P.rec = c->erec.p;
  const int tiles = (c->n + 31) / 32;
  static DeviceOnce attr;  // the tables' double buffer is above the 48 KB default
  if (attr.pending()) {
    BEM_CUDA(c, cudaFuncSetAttribute(ghmat_regular_kernel<kModeA, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kTabSmem));
    BEM_CUDA(c, cudaFuncSetAttribute(ghmat_regular_kernel<kModeA, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kTabSmem));
    attr.mark();
  }
  const int ntail = plan_tail(c, P, tiles, rc);
  if (rc) return rc;
  const int grid = P.nparts > 1 ? P.tail0 + ntail * P.nparts : tiles;
  if (precision == BEM_ASM_FP32_FAR)
    ghmat_regular_kernel<kModeA, 1><<<grid, 256, kTabSmem, c->stream>>>(P);
  else
    ghmat_regular_kernel<kModeA, 0><<<grid, 256, kTabSmem, c->stream>>>(P);
  BEM_LAUNCH_CHECK(c);
  if (P.nparts > 1) {
    const int64_t segs = (int64_t)ntail * c->n * 3;
    const int blocks = (int)std::min<int64_t>((segs + 7) / 8, 8 * (int64_t)c->sm_count);
    tail_merge_cols_kernel<<<blocks, 256, 0, c->stream>>>(P, ntail);
    BEM_LAUNCH_CHECK(c);
    tail_merge_fd_kernel<<<(32 * ntail + 127) / 128, 128, 0, c->stream>>>(P, ntail);
    BEM_LAUNCH_CHECK(c);
  }
  ghmat_singular_kernel<kModeA><<<(c->n + 3) / 4, 128, 0, c->stream>>>(P);
  BEM_LAUNCH_CHECK(c);
  if (c->npins > 0) {
    dim3 grid(64, c->npins);
    pins_kernel<<<grid, 256, 0, c->stream>>>(c->pins.p, c->npins, N, c->A.p, lda, c->FI.p);
    BEM_LAUNCH_CHECK(c);
  }
  c->have_system = true;
  c->mesh_system = true;
  c->nsys = N;
  c->have_solution = false;
  c->factored_fp64 = false;
  return BEM_OK;
}

int launch_hg(bem_ctx* c, int in0, int in1, double* dH, int64_t ldh, double* dG, int64_t ldg) {
  if (!c->have_geometry || !c->have_material)
    return bem_fail(c, BEM_ERR_STATE, "get_hg needs mesh, material and geometry");
  int rc = upload_singular_constants(c);
  if (rc) return rc;
  AsmArgs P = make_args(c);
  P.in0 = in0;
  P.nrows_nodes = in1 - in0;
  P.A = dH;
  P.lda = ldh;
  P.G = dG;
  P.ldg = ldg;
  const int tiles = (P.nrows_nodes + 31) / 32;
  static DeviceOnce attr;
  if (attr.pending()) {
    BEM_CUDA(c, cudaFuncSetAttribute(ghmat_regular_kernel<kModeHG, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kTabSmem));
    attr.mark();
  }
  ghmat_regular_kernel<kModeHG, 0><<<tiles, 256, kTabSmem, c->stream>>>(P);
  BEM_LAUNCH_CHECK(c);
  ghmat_singular_kernel<kModeHG><<<(P.nrows_nodes + 3) / 4, 128, 0, c->stream>>>(P);
  BEM_LAUNCH_CHECK(c);
  return BEM_OK;
}


// ---------------------------------------------------------------------------------
// batched H/G assembly of many systems
// ---------------------------------------------------------------------------------

// Persistent: every CTA takes (system, tile) items from a global counter until the
// list is exhausted; the host orders the items by cost (largest systems first), so the
// uneven systems of a batch balance over the SMs.  An item is the body of
// ghmat_regular_kernel for that system's tile, with the system's arguments staged in
// shared memory.
__global__ void __launch_bounds__(256, 1)
    batch_regular_kernel(const AsmArgs* __restrict__ args, const int2* __restrict__ tiles, int ntiles,
                         unsigned* counter) {
  __shared__ AsmArgs sP;
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int it = s_item;
    if (it >= ntiles) return;
    const int2 w = tiles[it];
    if (threadIdx.x == 0) sP = args[w.x];
    __syncthreads();
    regular_tile<kModeHG, 0>(sP, w.y, 0, 0, sP.nbatches);
    __syncthreads();
  }
}

// one warp per node of any system: the system by binary search of the node offsets
__global__ void __launch_bounds__(128)
    batch_singular_kernel(const AsmArgs* __restrict__ args, const int* __restrict__ node_off, int nsys,
                          int total_nodes) {
  __shared__ double s_part[4][27][18];
  __shared__ AsmArgs sP[4];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gnode = blockIdx.x * 4 + wib;
  if (gnode >= total_nodes) return;  // warp-uniform
  int lo = 0, hi = nsys - 1;         // largest i with node_off[i] <= gnode
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(node_off + mid) <= gnode) lo = mid;
    else hi = mid - 1;
  }
  if (lane == 0) sP[wib] = args[lo];
  __syncwarp();
  singular_node<kModeHG>(sP[wib], gnode - __ldg(node_off + lo), s_part[wib]);
}

int launch_batch_hg(cudaStream_t stream, int sm_count, const AsmArgs* d_args, const int2* d_tiles, int ntiles,
                    unsigned* counter, const int* d_node_off, int nsys, int total_nodes, long long* launches) {
  static DeviceOnce constants;
  if (constants.pending()) {
    if (cudaMemcpyToSymbol(s_gi, kGiQuad, sizeof(kGiQuad)) != cudaSuccess ||
        cudaMemcpyToSymbol(s_ome, kOmeQuad, sizeof(kOmeQuad)) != cudaSuccess)
      return BEM_ERR_CUDA;
    constants.mark();
  }
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned), stream) != cudaSuccess) return BEM_ERR_CUDA;
  static DeviceOnce attr;  // the tables' double buffer is above the 48 KB default
  if (attr.pending()) {
    if (cudaFuncSetAttribute(batch_regular_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTabSmem) !=
        cudaSuccess)
      return BEM_ERR_CUDA;
    attr.mark();
  }
  batch_regular_kernel<<<std::max(1, std::min(ntiles, sm_count)), 256, kTabSmem, stream>>>(d_args, d_tiles,
                                                                                            ntiles, counter);
  if (cudaGetLastError() != cudaSuccess) return BEM_ERR_CUDA;
  batch_singular_kernel<<<(total_nodes + 3) / 4, 128, 0, stream>>>(d_args, d_node_off, nsys, total_nodes);
  if (cudaGetLastError() != cudaSuccess) return BEM_ERR_CUDA;
  if (launches) *launches += 2;
  return BEM_OK;
}

}  // namespace bem
