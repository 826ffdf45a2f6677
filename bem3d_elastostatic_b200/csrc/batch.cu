// Many small systems in few launches: each system is a boundary mesh of its own
// (size, material, supports) with nrhs load cases (sets of prescribed values).
//
//   geometry    one etaxja launch over the elements of every system
//   assembly    H (rigid-body diagonal included) and G of every system in two
//               launches (assembly.cu: a persistent work queue over (system, 32-node
//               tile) items for the regular pairs, one warp per node for the singular
//               ones)
//   combine     per system: FI of every load case, FI_r = G[:, t known] t_r -
//               H[:, u known] u_r, then A in place of H by the column swap of
//               assembly_mod.f90:125-218 (A(:, dof) = H(:, dof) unless u is known there,
//               minus mu G for every element that prescribes u at that node), then
//               the pinned rows
//   solve       a persistent kernel factors one system per CTA (LAPACK dgetrf: row
//               pivoting of A, 32-wide panels, SMEM-staged 64 x 64 trailing tiles), in
//               FP32 (refined) or FP64 (plain); the substitution for all load cases
//               and the FP64 residual / backward error of each system follow, one CTA
//               per system, for a fixed number of refinement sweeps in which converged
//               systems skip their work.  The whole solve is captured once in a CUDA
//               graph and replayed.
//
// The column swap is formed from H and G, so a node's prescribed displacement must be
// the same in every element that prescribes it (the single-system path takes each
// element's own value); bem_batch_add rejects meshes that break this.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "asm_args.cuh"
#include "common.cuh"

namespace bem {
namespace {

constexpr int kLuNB = 32;              // panel width of the per-system LU
constexpr int kTM = 128, kTN = 64;     // trailing-update tile (kTM x kTN)
constexpr int kMaxRhs = 8;             // load cases per system
constexpr int kSolveThreads = 512;
constexpr size_t kSolveSmem = 200 * 1024;  // substitution workspace per CTA

struct SysDev {
  int n, ne, N, nrhs;
  int64_t lda;   // of H / A and of the factor copy
  int64_t ldg;   // of G
  int64_t a_off, g_off, f_off;  // A (FP64), G (FP64), factor (T) in their arenas
  int64_t v_off;                // FI, X, R: N x nrhs each (ld N) in the vector arena
  int64_t piv_off;
  int64_t cs_off, ncs;          // column-swap list: (dof, G column) pairs
  int64_t fl_off, nfl;          // FI terms: (matrix, column) and nrhs coefficients each
  int64_t pin_off, npins;
  int64_t uk_off;               // u known per dof
  double mu;
};

// ---------------------------------------------------------------------------------
// combine
// ---------------------------------------------------------------------------------

// FI_r = sum_terms coef[t][r] * M_t(:, col_t), M = G (kind 0) or H (kind 1)
__global__ void batch_fi_kernel(const SysDev* __restrict__ sys, const double* __restrict__ H,
                                const double* __restrict__ G, const int2* __restrict__ terms,
                                const double* __restrict__ coef, double* __restrict__ FI) {
  const SysDev S = sys[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.N) return;
  double acc[kMaxRhs];
  for (int r = 0; r < kMaxRhs; ++r) acc[r] = 0.0;
  const double* Hs = H + S.a_off;
  const double* Gs = G + S.g_off;
  for (int64_t t = 0; t < S.nfl; ++t) {
    const int2 tm = terms[S.fl_off + t];
    const double m = tm.x == 0 ? Gs[i + tm.y * S.ldg] : Hs[i + tm.y * S.lda];
    const double* cf = coef + (S.fl_off + t) * kMaxRhs;
    for (int r = 0; r < S.nrhs; ++r) acc[r] = fma(m, cf[r], acc[r]);
  }
  double* F = FI + S.v_off;
  for (int r = 0; r < S.nrhs; ++r) F[i + (int64_t)r * S.N] = acc[r];
}

// A(:, dof) = (u known at dof ? 0 : H(:, dof)) - mu * sum of the dof's G columns, in
// place of H; one CTA per (system, dof).  ukcsr holds per system the N u-known flags
// and the N + 1 offsets of the dof's entries in the (dof, G column) list cs.
__global__ void batch_a_kernel(const SysDev* __restrict__ sys, double* __restrict__ HA,
                               const double* __restrict__ G, const int2* __restrict__ cs,
                               const int* __restrict__ ukcsr) {
  const SysDev S = sys[blockIdx.y];
  const int d = blockIdx.x;
  if (d >= S.N) return;
  double* col = HA + S.a_off + (int64_t)d * S.lda;
  const double* Gs = G + S.g_off;
  const int* uk = ukcsr + S.uk_off;
  const int beg = uk[S.N + d], end = uk[S.N + d + 1];
  const bool known = uk[d] != 0;
  for (int i = threadIdx.x; i < S.N; i += blockDim.x) {
    double a = known ? 0.0 : col[i];
    for (int q = beg; q < end; ++q) a -= S.mu * Gs[i + (int64_t)cs[S.cs_off + q].y * S.ldg];
    col[i] = a;
  }
}

__global__ void batch_pins_kernel(const SysDev* __restrict__ sys, const int* __restrict__ pins,
                                  double* __restrict__ A, double* __restrict__ FI) {
  const SysDev S = sys[blockIdx.y];
  if (blockIdx.x >= S.npins) return;
  const int p = pins[S.pin_off + blockIdx.x];
  double* As = A + S.a_off;
  for (int c = threadIdx.x; c < S.N; c += blockDim.x) As[p + (int64_t)c * S.lda] = (c == p) ? 1.0 : 0.0;
  if (threadIdx.x < S.nrhs) FI[S.v_off + p + (int64_t)threadIdx.x * S.N] = 0.0;
}

// ---------------------------------------------------------------------------------
// per-system LU (one CTA), substitution and residual
// ---------------------------------------------------------------------------------

template <typename T>
__global__ void batch_copy_kernel(const SysDev* __restrict__ sys, const double* __restrict__ A,
                                  T* __restrict__ F) {
  const SysDev S = sys[blockIdx.y];
  const int64_t total = (int64_t)S.N * S.lda;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x)
    F[S.f_off + k] = (T)A[S.a_off + k];
}

__device__ __forceinline__ void take_max(double& bv, int& bi, double v, int i) {
  if (v > bv || (v == bv && i < bi)) {
    bv = v;
    bi = i;
  }
}

// dynamic shared memory of the LU kernel: the L21 (kLuNB x kTM) and U12 (kLuNB x kTN) tiles
template <typename T>
constexpr size_t lu_smem() { return (size_t)kLuNB * (kTM + kTN) * sizeof(T); }

template <typename T, int NT>
__device__ void cta_getrf(T* A, int64_t lda, int N, int* ipiv, int* info, T* s_a, T* s_b) {
  __shared__ double s_v[NT / 32];
  __shared__ int s_i[NT / 32];
  __shared__ int s_piv[kLuNB];
  __shared__ int s_rows[2 * kLuNB], s_src[2 * kLuNB], s_nrows;
  __shared__ T s_row[kLuNB];
  __shared__ T s_L[kLuNB][kLuNB + 1];
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  if (tid == 0) *info = 0;
  for (int j0 = 0; j0 < N; j0 += kLuNB) {
    const int jb = min(kLuNB, N - j0);
    // ---- panel: columns j0 .. j0+jb-1 ------------------------------------------------
    for (int j = j0; j < j0 + jb; ++j) {
      double bv = -1.0;
      int bi = INT_MAX;
      for (int i = j + tid; i < N; i += NT) take_max(bv, bi, fabs((double)A[i + (int64_t)j * lda]), i);
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        take_max(bv, bi, ov, oi);
      }
      if (lane == 0) {
        s_v[wp] = bv;
        s_i[wp] = bi;
      }
      __syncthreads();
      if (tid == 0) {
        for (int w = 1; w < NT / 32; ++w) take_max(bv, bi, s_v[w], s_i[w]);
        s_piv[j - j0] = bi;
        ipiv[j] = bi;
        if (bv == 0.0 && *info == 0) *info = j + 1;
      }
      __syncthreads();
      const int p = s_piv[j - j0];
      if (p != j && tid < jb) {
        T* a = A + j + (int64_t)(j0 + tid) * lda;
        T* b = A + p + (int64_t)(j0 + tid) * lda;
        const T t = *a;
        *a = *b;
        *b = t;
      }
      __syncthreads();
      const T piv = A[j + (int64_t)j * lda];
      if (tid < jb) s_row[tid] = A[j + (int64_t)(j0 + tid) * lda];
      __syncthreads();
      if (piv != T(0)) {
        for (int i = j + 1 + tid; i < N; i += NT) {
          T* ri = A + i;
          const T l = ri[(int64_t)j * lda] / piv;
          ri[(int64_t)j * lda] = l;
          for (int c = j + 1 - j0; c < jb; ++c) ri[(int64_t)(j0 + c) * lda] -= l * s_row[c];
        }
      }
      __syncthreads();
    }
    // ---- the panel's interchanges on the other columns, as one gather per column ---
    if (tid == 0) {
      int nr = 0;
      for (int q = 0; q < jb; ++q) {  // rows touched: j0+q and their pivots
        const int cand[2] = {j0 + q, s_piv[q]};
        for (int u = 0; u < 2; ++u) {
          int f = -1;
          for (int m = 0; m < nr; ++m)
            if (s_rows[m] == cand[u]) f = m;
          if (f < 0) {
            s_rows[nr] = cand[u];
            s_src[nr] = cand[u];
            ++nr;
          }
        }
      }
      for (int q = 0; q < jb; ++q) {  // apply the swaps to the labels in order
        int a = -1, b = -1;
        for (int m = 0; m < nr; ++m) {
          if (s_rows[m] == j0 + q) a = m;
          if (s_rows[m] == s_piv[q]) b = m;
        }
        const int t = s_src[a];
        s_src[a] = s_src[b];
        s_src[b] = t;
      }
      s_nrows = nr;
    }
    __syncthreads();
    {
      const int nr = s_nrows;
      for (int c = wp; c < N; c += NT / 32) {
        if (c >= j0 && c < j0 + jb) continue;
        T* col = A + (int64_t)c * lda;
        T v0 = T(0), v1 = T(0);
        if (lane < nr) v0 = col[s_src[lane]];
        if (lane + 32 < nr) v1 = col[s_src[lane + 32]];
        __syncwarp();
        if (lane < nr) col[s_rows[lane]] = v0;
        if (lane + 32 < nr) col[s_rows[lane + 32]] = v1;
      }
    }
    __syncthreads();
    const int t0 = j0 + jb;
    if (t0 >= N) break;
    // ---- U12 = L11^{-1} A12 (unit lower), one column per thread -------------------
    for (int idx = tid; idx < jb * jb; idx += NT) {
      const int r = idx % jb, c = idx / jb;
      s_L[r][c] = A[j0 + r + (int64_t)(j0 + c) * lda];
    }
    __syncthreads();
    for (int c = t0 + tid; c < N; c += NT) {
      T* col = A + j0 + (int64_t)c * lda;
      T x[kLuNB];
#pragma unroll
      for (int q = 0; q < kLuNB; ++q) {
        if (q < jb) {
          T v = col[q];
#pragma unroll
          for (int t = 0; t < q; ++t) v -= s_L[q][t] * x[t];
          x[q] = v;
        }
      }
#pragma unroll
      for (int q = 0; q < kLuNB; ++q)
        if (q < jb) col[q] = x[q];
    }
    __syncthreads();
    // ---- A22 -= L21 U12, tiles of kTM x kTN: the tile of C is loaded with the operand
    //      tiles, so a tile costs one memory round trip before its FMAs ---------------
    const int m = N - t0;
    const int tm = (m + kTM - 1) / kTM, tn = (m + kTN - 1) / kTN;
    constexpr int CPT = kTM * kTN / NT;  // columns per thread
    const int r = tid % kTM, cg = tid / kTM;
    for (int tt = 0; tt < tm * tn; ++tt) {
      const int ti = tt % tm, tj = tt / tm;
      const int rb = t0 + ti * kTM, cb = t0 + tj * kTN;
      for (int idx = tid; idx < kLuNB * kTM; idx += NT) {
        const int rr = idx % kTM, k = idx / kTM;  // L21(rb + rr, j0 + k)
        s_a[k * kTM + rr] = (k < jb && rb + rr < N) ? A[rb + rr + (int64_t)(j0 + k) * lda] : T(0);
      }
      for (int idx = tid; idx < kLuNB * kTN; idx += NT) {
        const int kk = idx % kLuNB, cc = idx / kLuNB;  // U12(j0 + kk, cb + cc)
        s_b[kk * kTN + cc] = (kk < jb && cb + cc < N) ? A[j0 + kk + (int64_t)(cb + cc) * lda] : T(0);
      }
      T acc[CPT];
      const bool row_ok = rb + r < N;
#pragma unroll
      for (int q = 0; q < CPT; ++q) {
        const int cc = cb + cg * CPT + q;
        acc[q] = (row_ok && cc < N) ? A[rb + r + (int64_t)cc * lda] : T(0);
      }
      __syncthreads();
#pragma unroll 4
      for (int k = 0; k < kLuNB; ++k) {
        const T l = s_a[k * kTM + r];
#pragma unroll
        for (int q = 0; q < CPT; ++q) acc[q] = fma(-l, s_b[k * kTN + cg * CPT + q], acc[q]);
      }
      if (row_ok) {
#pragma unroll
        for (int q = 0; q < CPT; ++q) {
          const int cc = cb + cg * CPT + q;
          if (cc < N) A[rb + r + (int64_t)cc * lda] = acc[q];
        }
      }
      __syncthreads();
    }
  }
}

template <typename T, int NT>
__global__ void __launch_bounds__(NT) batch_lu_kernel(const SysDev* __restrict__ sys, const int* __restrict__ order,
                                                      int nsys, T* F, int* piv, int* info, unsigned* counter) {
  extern __shared__ __align__(16) unsigned char lu_dyn[];
  T* s_a = reinterpret_cast<T*>(lu_dyn);
  T* s_b = s_a + kLuNB * kTM;
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= nsys) return;
    const int s = order[it];
    const SysDev S = sys[s];
    cta_getrf<T, NT>(F + S.f_off, S.lda, S.N, piv + S.piv_off, info + s, s_a, s_b);
    __syncthreads();
  }
}

// X (+)= U^{-1} L^{-1} P^T R for the system's load cases, in shared memory chunks of
// nc columns (B is [N][nc]); converged systems are skipped
template <typename T>
__global__ void __launch_bounds__(kSolveThreads)
    batch_solve_kernel(const SysDev* __restrict__ sys, const int* __restrict__ order, int nsys,
                       const T* __restrict__ F, const int* __restrict__ piv, const double* __restrict__ R,
                       double* __restrict__ X, const int* __restrict__ conv, const int* __restrict__ info,
                       int accumulate, unsigned* counter) {
  extern __shared__ double sB[];
  __shared__ int s_item;
  __shared__ double s_x[kLuNB][kMaxRhs];
  __shared__ double s_d[kLuNB][kLuNB + 1];
  const int tid = threadIdx.x, lane = tid & 31;
  for (;;) {
    if (tid == 0) s_item = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= nsys) return;
    const int s = order[it];
    if (conv[s] || info[s]) continue;  // converged, or a zero pivot
    const SysDev S = sys[s];
    const int N = S.N;
    const T* A = F + S.f_off;
    const int* pv = piv + S.piv_off;
    const int nc_max = max(1, min(S.nrhs, (int)(kSolveSmem / (sizeof(double) * (size_t)N))));
    for (int r0 = 0; r0 < S.nrhs; r0 += nc_max) {
      const int nc = min(nc_max, S.nrhs - r0);
      for (int i = tid; i < N; i += kSolveThreads)
        _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nc) sB[i * nc + r] = R[S.v_off + i + (int64_t)(r0 + r) * N];
      __syncthreads();
      if (tid < nc)
        for (int j = 0; j < N; ++j) {
          const int p = pv[j];
          if (p != j) {
            const double t = sB[j * nc + tid];
            sB[j * nc + tid] = sB[p * nc + tid];
            sB[p * nc + tid] = t;
          }
        }
      __syncthreads();
      // forward, unit lower, blocks of 32
      for (int j0 = 0; j0 < N; j0 += kLuNB) {
        const int jb = min(kLuNB, N - j0);
        for (int idx = tid; idx < kLuNB * kLuNB; idx += kSolveThreads) {  // the diagonal block
          const int rr = idx % kLuNB, cc = idx / kLuNB;
          s_d[rr][cc] = (rr < jb && cc < jb) ? (double)A[j0 + rr + (int64_t)(j0 + cc) * S.lda] : 0.0;
        }
        __syncthreads();
        if (tid < 32) {
          double b[kMaxRhs];
          _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nc) b[r] = (lane < jb) ? sB[(j0 + lane) * nc + r] : 0.0;
          for (int t = 0; t < jb; ++t) {
            const double l = (lane > t && lane < jb) ? s_d[lane][t] : 0.0;
            _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nc) {
              const double xt = __shfl_sync(0xffffffffu, b[r], t);
              b[r] = fma(-l, xt, b[r]);
            }
          }
          _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nc)
            if (lane < jb) {
              sB[(j0 + lane) * nc + r] = b[r];
              s_x[lane][r] = b[r];
            }
        }
        __syncthreads();
        for (int i = j0 + jb + tid; i < N; i += kSolveThreads) {
          double acc[kMaxRhs];
          _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nc) acc[r] = sB[i * nc + r];
          for (int q0 = 0; q0 < jb; q0 += 8) {  // eight loads in flight, then their FMAs
            T lv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) lv[u] = (q0 + u < jb) ? A[i + (int64_t)(j0 + q0 + u) * S.lda] : T(0);
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              const double l = (double)lv[u];
              _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nc) acc[r] = fma(-l, s_x[q0 + u < jb ? q0 + u : 0][r], acc[r]);
            }
          }
          _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nc) sB[i * nc + r] = acc[r];
        }
        __syncthreads();
      }
      // backward, non-unit upper, blocks of 32 from the last
      for (int j0 = ((N - 1) / kLuNB) * kLuNB; j0 >= 0; j0 -= kLuNB) {
        const int jb = min(kLuNB, N - j0);
        for (int idx = tid; idx < kLuNB * kLuNB; idx += kSolveThreads) {
          const int rr = idx % kLuNB, cc = idx / kLuNB;
          s_d[rr][cc] = (rr < jb && cc < jb) ? (double)A[j0 + rr + (int64_t)(j0 + cc) * S.lda] : 0.0;
        }
        __syncthreads();
        if (tid < 32) {
          double b[kMaxRhs];
          _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nc) b[r] = (lane < jb) ? sB[(j0 + lane) * nc + r] : 0.0;
          for (int t = jb - 1; t >= 0; --t) {
            const double d = s_d[t][t];
            const double u = (lane < t) ? s_d[lane][t] : 0.0;
            _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nc) {
              const double xt = __shfl_sync(0xffffffffu, b[r], t) / d;
              if (lane == t) b[r] = xt;
              else b[r] = fma(-u, xt, b[r]);
            }
          }
          _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nc)
            if (lane < jb) {
              sB[(j0 + lane) * nc + r] = b[r];
              s_x[lane][r] = b[r];
            }
        }
        __syncthreads();
        for (int i = tid; i < j0; i += kSolveThreads) {
          double acc[kMaxRhs];
          _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nc) acc[r] = sB[i * nc + r];
          for (int q0 = 0; q0 < jb; q0 += 8) {  // eight loads in flight, then their FMAs
            T uv[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) uv[k] = (q0 + k < jb) ? A[i + (int64_t)(j0 + q0 + k) * S.lda] : T(0);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
              const double u = (double)uv[k];
              _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nc) acc[r] = fma(-u, s_x[q0 + k < jb ? q0 + k : 0][r], acc[r]);
            }
          }
          _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nc) sB[i * nc + r] = acc[r];
        }
        __syncthreads();
      }
      for (int i = tid; i < N; i += kSolveThreads)
        _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nc) {
          double* xo = X + S.v_off + i + (int64_t)(r0 + r) * N;
          *xo = accumulate ? *xo + sB[i * nc + r] : sB[i * nc + r];
        }
      __syncthreads();
    }
  }
}

// R = B - A X (FP64) and the backward error max_r ||R_r|| / (||A|| ||X_r|| + ||B_r||)
// (infinity norms); conv[s] = 1 once it is <= tol, 2 once a sweep gains less than 10 %
__global__ void __launch_bounds__(kSolveThreads)
    batch_residual_kernel(const SysDev* __restrict__ sys, const int* __restrict__ order, int nsys,
                          const double* __restrict__ A, const double* __restrict__ B, const double* __restrict__ X,
                          double* __restrict__ R, double* __restrict__ berr, int* __restrict__ conv,
                          const int* __restrict__ info, double tol, int first, unsigned* counter) {
  extern __shared__ double sX[];
  __shared__ int s_item;
  __shared__ double s_red[kSolveThreads / 32][3 * kMaxRhs + 1];
  const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  for (;;) {
    if (tid == 0) s_item = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= nsys) return;
    const int s = order[it];
    if (conv[s] || info[s]) continue;
    const SysDev S = sys[s];
    const int N = S.N, nrhs = S.nrhs;
    const double* As = A + S.a_off;
    // X staged in chunks of columns; the row loop keeps all nrhs partial sums
    double rmax[kMaxRhs], xmax[kMaxRhs], bmax[kMaxRhs], amax = 0.0;
    for (int r = 0; r < kMaxRhs; ++r) rmax[r] = xmax[r] = bmax[r] = 0.0;
    const int rows_per = (N + kSolveThreads - 1) / kSolveThreads;
    for (int rb = 0; rb < rows_per; ++rb) {
      const int i = tid + rb * kSolveThreads;
      double acc[kMaxRhs], asum = 0.0;
      _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nrhs) acc[r] = (i < N) ? B[S.v_off + i + (int64_t)r * N] : 0.0;
      const int ncol = max(1, (int)(kSolveSmem / (sizeof(double) * (size_t)nrhs)));
      for (int c0 = 0; c0 < N; c0 += ncol) {
        const int cn = min(ncol, N - c0);
        __syncthreads();
        for (int k = tid; k < cn * nrhs; k += kSolveThreads) {
          const int c = k % cn, r = k / cn;
          sX[c * nrhs + r] = X[S.v_off + c0 + c + (int64_t)r * N];
        }
        __syncthreads();
        if (i < N) {
          // eight columns per step: eight independent loads in flight per thread (one
          // CTA per system streams its whole A, so memory-level parallelism sets the time)
          int c = 0;
          for (; c + 8 <= cn; c += 8) {
            double a[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) a[u] = As[i + (int64_t)(c0 + c + u) * S.lda];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              asum += fabs(a[u]);
              _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nrhs) acc[r] = fma(-a[u], sX[(c + u) * nrhs + r], acc[r]);
            }
          }
          for (; c < cn; ++c) {
            const double a = As[i + (int64_t)(c0 + c) * S.lda];
            asum += fabs(a);
            _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nrhs) acc[r] = fma(-a, sX[c * nrhs + r], acc[r]);
          }
        }
      }
      if (i < N) {
        amax = fmax(amax, asum);
        _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nrhs) {
          R[S.v_off + i + (int64_t)r * N] = acc[r];
          rmax[r] = fmax(rmax[r], fabs(acc[r]));
          xmax[r] = fmax(xmax[r], fabs(X[S.v_off + i + (int64_t)r * N]));
          bmax[r] = fmax(bmax[r], fabs(B[S.v_off + i + (int64_t)r * N]));
        }
      }
    }
    for (int off = 16; off > 0; off >>= 1) {
      amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, off));
      _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nrhs) {
        rmax[r] = fmax(rmax[r], __shfl_xor_sync(0xffffffffu, rmax[r], off));
        xmax[r] = fmax(xmax[r], __shfl_xor_sync(0xffffffffu, xmax[r], off));
        bmax[r] = fmax(bmax[r], __shfl_xor_sync(0xffffffffu, bmax[r], off));
      }
    }
    if (lane == 0) {
      _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nrhs) {
        s_red[wp][r] = rmax[r];
        s_red[wp][kMaxRhs + r] = xmax[r];
        s_red[wp][2 * kMaxRhs + r] = bmax[r];
      }
      s_red[wp][3 * kMaxRhs] = amax;
    }
    __syncthreads();
    if (tid == 0) {
      double an = 0.0, be = 0.0;
      for (int w = 0; w < kSolveThreads / 32; ++w) an = fmax(an, s_red[w][3 * kMaxRhs]);
      _Pragma("unroll") for (int r = 0; r < kMaxRhs; ++r) if (r < nrhs) {
        double rn = 0.0, xn = 0.0, bn = 0.0;
        for (int w = 0; w < kSolveThreads / 32; ++w) {
          rn = fmax(rn, s_red[w][r]);
          xn = fmax(xn, s_red[w][kMaxRhs + r]);
          bn = fmax(bn, s_red[w][2 * kMaxRhs + r]);
        }
        const double den = an * xn + bn;
        be = fmax(be, den > 0.0 ? rn / den : 0.0);
      }
      const double prev = berr[s];
      berr[s] = be;
      if (!first) {
        if (be <= tol) conv[s] = 1;
        else if (be > 0.9 * prev) conv[s] = 2;
      }
    }
    __syncthreads();
  }
}

__global__ void zero_kernel(double* p, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = 0.0;
}

}  // namespace
}  // namespace bem

// =====================================================================================
// host side
// =====================================================================================

struct bem_batch {
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  std::string err;
  long long launches = 0;
  int nrhs = 0;
  struct Sys {
    int n, ne, npins;
    double mu, nu;
    std::vector<double> x, y, z, bc;
    std::vector<int> nconec, kconec, kode, pins;
  };
  std::vector<Sys> sys;
  std::vector<bem::SysDev> hdev;
  std::vector<int> order;  // systems by decreasing order
  bool assembled = false, factored = false;
  int factored_precision = -1;
  // device storage
  bem::DBuf<double> x, y, z, ref, tab, H, G, vec, berr, A64f;
  bem::DBuf<float> A32;
  bem::DBuf<int> nconec, kconec_loc, kconec_glob, nesim, ke, batches, node_off, piv, info, conv, uk_csr, ord;
  bem::DBuf<int2> tiles, cs, terms;
  bem::DBuf<double> coef;
  bem::DBuf<int> pins;
  bem::DBuf<bem::AsmArgs> args;
  bem::DBuf<bem::SysDev> dsys;
  bem::DBuf<unsigned> counters;
  int ntiles = 0, total_nodes = 0, total_elems = 0;
  // solve graph
  cudaGraphExec_t graph = nullptr;
  int graph_key[3] = {-1, -1, -1};
  double graph_tol = -1.0;
  int lu_threads = 0;  // autotuned per batch: 256 or 512
  float lu_ms[2] = {0.f, 0.f};
  ~bem_batch() {
    if (graph) cudaGraphExecDestroy(graph);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

int bfail(bem_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  return code;
}
#define BB_CUDA(b, call)                                                                      \
  do {                                                                                        \
    cudaError_t _e = (call);                                                                  \
    if (_e != cudaSuccess) return bfail((b), BEM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

template <typename T>
int up(bem_batch* b, bem::DBuf<T>& d, const std::vector<T>& h) {
  BB_CUDA(b, d.alloc(std::max<size_t>(1, h.size())));
  if (!h.empty()) BB_CUDA(b, cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, b->stream));
  return BEM_OK;
}

}  // namespace

extern "C" {

int bem_batch_create(bem_batch** out, int device) {
  if (!out) return BEM_ERR_ARG;
  *out = nullptr;
  bem_batch* b = new bem_batch();
  b->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) {
    delete b;
    return BEM_ERR_CUDA;
  }
  *out = b;
  return BEM_OK;
}

int bem_batch_destroy(bem_batch* b) {
  if (!b) return BEM_OK;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  delete b;
  return BEM_OK;
}

const char* bem_batch_last_error(const bem_batch* b) { return b ? b->err.c_str() : "null batch"; }

int bem_batch_add(bem_batch* b, int n, int ne, const double* x, const double* y, const double* z, const int* nconec,
                  const int* kconec, double mu, double nu, const int* kode, int nrhs, const double* bc, int npins,
                  const int* pins) {
  if (!b || n <= 0 || ne <= 0 || !x || !y || !z || !nconec || !kconec || !kode || !bc || nrhs < 1 ||
      nrhs > bem::kMaxRhs || npins < 0 || (npins > 0 && !pins) || !(mu > 0.0))
    return bfail(b, BEM_ERR_ARG, "batch_add: bad arguments");
  if (b->nrhs == 0) b->nrhs = nrhs;
  if (nrhs != b->nrhs) return bfail(b, BEM_ERR_ARG, "batch_add: every system needs the same number of load cases");
  bem_batch::Sys s;
  s.n = n;
  s.ne = ne;
  s.mu = mu;
  s.nu = nu;
  s.npins = npins;
  s.x.assign(x, x + n);
  s.y.assign(y, y + n);
  s.z.assign(z, z + n);
  s.nconec.assign(nconec, nconec + ne);
  s.kconec.assign(kconec, kconec + 9 * (size_t)ne);
  s.kode.assign(kode, kode + 3 * (size_t)ne);
  s.bc.assign(bc, bc + 27 * (size_t)ne * nrhs);
  s.pins.assign(pins, pins + npins);
  std::vector<int> cnt(n, 0);
  for (int e = 0; e < ne; ++e) {
    if (nconec[e] != 9 && nconec[e] != 6) return bfail(b, BEM_ERR_MESH, "batch_add: nconec must be 6 or 9");
    for (int m = 0; m < 9; ++m) {
      if (m >= nconec[e]) {
        s.kconec[m + 9 * (size_t)e] = 1;
        continue;
      }
      const int k = kconec[m + 9 * (size_t)e];
      if (k < 1 || k > n) return bfail(b, BEM_ERR_MESH, "batch_add: kconec references a node out of range");
      if (++cnt[k - 1] > 8) return bfail(b, BEM_ERR_MESH, "batch_add: a node lies in more than 8 elements");
    }
    for (int ld = 0; ld < 3; ++ld)
      if (kode[3 * e + ld] != 0 && kode[3 * e + ld] != 1) return bfail(b, BEM_ERR_ARG, "batch_add: kode must be 0 or 1");
  }
  // a node's prescribed displacement must agree over the elements that prescribe it
  for (int r = 0; r < nrhs; ++r) {
    std::vector<double> val(3 * (size_t)n, 0.0);
    std::vector<char> set(3 * (size_t)n, 0);
    const double* bcr = bc + 27 * (size_t)ne * r;
    for (int e = 0; e < ne; ++e)
      for (int ld = 0; ld < 3; ++ld)
        if (kode[3 * e + ld] == 0)
          for (int m = 0; m < nconec[e]; ++m) {
            const size_t d = 3 * (size_t)(kconec[m + 9 * (size_t)e] - 1) + ld;
            const double v = bcr[3 * m + ld + 27 * (size_t)e];
            if (set[d] && val[d] != v)
              return bfail(b, BEM_ERR_MESH, "batch_add: elements prescribe different displacements at one node");
            set[d] = 1;
            val[d] = v;
          }
  }
  for (int i = 0; i < npins; ++i)
    if (pins[i] < 0 || pins[i] >= 3 * n) return bfail(b, BEM_ERR_ARG, "batch_add: pin out of range");
  b->sys.push_back(std::move(s));
  b->assembled = b->factored = false;
  return (int)b->sys.size() - 1;
}

int bem_batch_assemble(bem_batch* b) {
  if (!b || b->sys.empty()) return bfail(b, BEM_ERR_STATE, "batch_assemble: no systems");
  BB_CUDA(b, cudaSetDevice(b->device));
  const int ns = (int)b->sys.size(), nrhs = b->nrhs;
  // host packing
  std::vector<double> hx, hy, hz;
  std::vector<int> hnc, hkl, hkg, hnesim, hke, hbatch, hnode_off(ns + 1, 0), hpins;
  std::vector<int2> htiles, hcs, hterms;
  std::vector<double> hcoef;
  std::vector<int> huk;  // per system: N u-known flags, then N + 1 row pointers of the cs list
  std::vector<bem::SysDev> hs(ns);
  int64_t a_off = 0, g_off = 0, v_off = 0, piv_off = 0, elem_off = 0, batch_off = 0;
  std::vector<int64_t> elem_offs(ns), batch_offs(ns), node_offs(ns);
  std::vector<int> nbatches(ns);
  for (int si = 0; si < ns; ++si) {
    const auto& S = b->sys[si];
    const int n = S.n, ne = S.ne, N = 3 * n;
    bem::SysDev& D = hs[si];
    D.n = n;
    D.ne = ne;
    D.N = N;
    D.nrhs = nrhs;
    D.lda = ((int64_t)N + 31) / 32 * 32;
    D.ldg = D.lda;
    D.a_off = a_off;
    a_off += D.lda * N;
    D.g_off = g_off;
    g_off += D.ldg * 27 * (int64_t)ne;
    D.f_off = D.a_off;
    D.v_off = v_off;
    v_off += (int64_t)N * nrhs;
    D.piv_off = piv_off;
    piv_off += N;
    D.mu = S.mu;
    node_offs[si] = hx.size();
    hnode_off[si] = (int)hx.size();
    hx.insert(hx.end(), S.x.begin(), S.x.end());
    hy.insert(hy.end(), S.y.begin(), S.y.end());
    hz.insert(hz.end(), S.z.begin(), S.z.end());
    elem_offs[si] = elem_off;
    elem_off += ne;
    hnc.insert(hnc.end(), S.nconec.begin(), S.nconec.end());
    for (size_t k = 0; k < S.kconec.size(); ++k) {
      hkl.push_back(S.kconec[k]);
      hkg.push_back(S.kconec[k] + (int)node_offs[si]);
    }
    // adjacency (io_mod.f90:125-135)
    std::vector<int> nes(n, 0), kel(8 * (size_t)n, 0);
    for (int e = 0; e < ne; ++e)
      for (int m = 0; m < S.nconec[e]; ++m) {
        const int in = S.kconec[m + 9 * (size_t)e] - 1;
        kel[nes[in]++ + 8 * (size_t)in] = e + 1;
      }
    hnesim.insert(hnesim.end(), nes.begin(), nes.end());
    hke.insert(hke.end(), kel.begin(), kel.end());
    // conflict-free element batches of the regular kernel (elements sharing no node)
    {
      std::vector<int> sched;
      std::vector<char> used(ne, 0);
      int left = ne, start = 0;
      while (left > 0) {
        std::vector<int> batch;
        std::vector<int> touched;
        for (int e = start; e < ne && (int)batch.size() < bem::kBatch; ++e) {
          if (used[e]) continue;
          bool clash = false;
          for (int m = 0; m < S.nconec[e] && !clash; ++m)
            for (int t : touched)
              if (t == S.kconec[m + 9 * (size_t)e]) clash = true;
          if (clash) continue;
          batch.push_back(e);
          used[e] = 1;
          --left;
          for (int m = 0; m < S.nconec[e]; ++m) touched.push_back(S.kconec[m + 9 * (size_t)e]);
        }
        while (start < ne && used[start]) ++start;
        for (int w = 0; w < bem::kBatch; ++w) sched.push_back(w < (int)batch.size() ? batch[w] : -1);
      }
      nbatches[si] = (int)sched.size() / bem::kBatch;
      batch_offs[si] = batch_off;
      batch_off += sched.size();
      hbatch.insert(hbatch.end(), sched.begin(), sched.end());
    }
    for (int t = 0; t < (n + 31) / 32; ++t) htiles.push_back(make_int2(si, t));
    // column swap: per dof, G columns of the elements prescribing u there; u-known flags
    std::vector<std::vector<int>> lists(N);
    std::vector<int> uk(N, 0);
    std::vector<double> vp(3 * (size_t)n * nrhs, 0.0);
    for (int in = 0; in < n; ++in)  // first element in ke order prescribing u (as build_lookup)
      for (int ld = 0; ld < 3; ++ld)
        for (int i = 0; i < nes[in] && i < 8 && !uk[3 * in + ld]; ++i) {
          const int e = kel[i + 8 * (size_t)in] - 1;
          if (S.kode[3 * e + ld] == 0)
            for (int m = 0; m < S.nconec[e]; ++m)
              if (S.kconec[m + 9 * (size_t)e] - 1 == in) {
                uk[3 * in + ld] = 1;
                for (int r = 0; r < nrhs; ++r)
                  vp[3 * in + ld + 3 * (size_t)n * r] = S.bc[3 * m + ld + 27 * (size_t)e + 27 * (size_t)ne * r];
                break;
              }
        }
    D.fl_off = (int64_t)hterms.size();
    for (int e = 0; e < ne; ++e)
      for (int k = 0; k < S.nconec[e]; ++k)
        for (int ld = 0; ld < 3; ++ld) {
          const int dof = 3 * (S.kconec[k + 9 * (size_t)e] - 1) + ld;
          const int gcol = 27 * e + 3 * k + ld;
          if (S.kode[3 * e + ld] == 0) {
            lists[dof].push_back(gcol);
          } else {  // traction known: FI += G(:, gcol) t
            bool any = false;
            double cf[bem::kMaxRhs] = {0};
            for (int r = 0; r < nrhs; ++r) {
              cf[r] = S.bc[3 * k + ld + 27 * (size_t)e + 27 * (size_t)ne * r];
              any |= cf[r] != 0.0;
            }
            if (any) {
              hterms.push_back(make_int2(0, gcol));
              hcoef.insert(hcoef.end(), cf, cf + bem::kMaxRhs);
            }
          }
        }
    for (int d = 0; d < N; ++d)  // u known: FI -= H(:, dof) u
      if (uk[d]) {
        bool any = false;
        double cf[bem::kMaxRhs] = {0};
        for (int r = 0; r < nrhs; ++r) {
          cf[r] = -vp[d + 3 * (size_t)n * r];
          any |= cf[r] != 0.0;
        }
        if (any) {
          hterms.push_back(make_int2(1, d));
          hcoef.insert(hcoef.end(), cf, cf + bem::kMaxRhs);
        }
      }
    D.nfl = (int64_t)hterms.size() - D.fl_off;
    D.cs_off = (int64_t)hcs.size();
    D.uk_off = (int64_t)huk.size();
    huk.insert(huk.end(), uk.begin(), uk.end());
    int acc = 0;
    for (int d = 0; d < N; ++d) {
      huk.push_back(acc);
      for (int gcol : lists[d]) hcs.push_back(make_int2(d, gcol));
      acc += (int)lists[d].size();
    }
    huk.push_back(acc);
    D.ncs = acc;
    D.pin_off = (int64_t)hpins.size();
    D.npins = S.npins;
    hpins.insert(hpins.end(), S.pins.begin(), S.pins.end());
  }
  hnode_off[ns] = (int)hx.size();
  b->total_nodes = (int)hx.size();
  b->total_elems = (int)elem_off;
  // the regular work items, largest systems first
  std::vector<int> ordsys(ns);
  for (int i = 0; i < ns; ++i) ordsys[i] = i;
  std::stable_sort(ordsys.begin(), ordsys.end(), [&](int a, int c) {
    return (int64_t)b->sys[a].n * b->sys[a].ne > (int64_t)b->sys[c].n * b->sys[c].ne;
  });
  std::vector<int2> sorted_tiles;
  for (int si : ordsys)
    for (int t = 0; t < (b->sys[si].n + 31) / 32; ++t) sorted_tiles.push_back(make_int2(si, t));
  b->ntiles = (int)sorted_tiles.size();
  b->order = ordsys;
  std::stable_sort(b->order.begin(), b->order.end(), [&](int a, int c) { return b->sys[a].n > b->sys[c].n; });
  // device
  int rc;
  if ((rc = up(b, b->x, hx)) || (rc = up(b, b->y, hy)) || (rc = up(b, b->z, hz)) || (rc = up(b, b->nconec, hnc)) ||
      (rc = up(b, b->kconec_loc, hkl)) || (rc = up(b, b->kconec_glob, hkg)) || (rc = up(b, b->nesim, hnesim)) ||
      (rc = up(b, b->ke, hke)) || (rc = up(b, b->batches, hbatch)) || (rc = up(b, b->node_off, hnode_off)) ||
      (rc = up(b, b->tiles, sorted_tiles)) || (rc = up(b, b->cs, hcs)) || (rc = up(b, b->terms, hterms)) ||
      (rc = up(b, b->coef, hcoef)) || (rc = up(b, b->uk_csr, huk)) || (rc = up(b, b->pins, hpins)) ||
      (rc = up(b, b->ord, b->order)))
    return rc;
  const size_t ng = (size_t)bem::kGp * elem_off;
  BB_CUDA(b, b->ref.alloc(16 * ng));
  BB_CUDA(b, b->tab.alloc((size_t)bem::kTabStride * elem_off));
  BB_CUDA(b, b->H.alloc((size_t)std::max<int64_t>(1, a_off)));
  BB_CUDA(b, b->G.alloc((size_t)std::max<int64_t>(1, g_off)));
  BB_CUDA(b, b->vec.alloc((size_t)3 * std::max<int64_t>(1, v_off)));  // FI, X, R
  BB_CUDA(b, b->piv.alloc((size_t)std::max<int64_t>(1, piv_off)));
  BB_CUDA(b, b->info.alloc(ns));
  BB_CUDA(b, b->conv.alloc(ns));
  BB_CUDA(b, b->berr.alloc(ns));
  BB_CUDA(b, b->counters.alloc(64));
  // per-system assembly arguments (mode HG)
  std::vector<bem::AsmArgs> hargs(ns);
  for (int si = 0; si < ns; ++si) {
    const auto& S = b->sys[si];
    bem::AsmArgs& P = hargs[si];
    P = bem::AsmArgs{};
    P.n = S.n;
    P.ne = S.ne;
    P.nbatches = nbatches[si];
    P.in0 = 0;
    P.nrows_nodes = S.n;
    P.batches = b->batches.p + batch_offs[si];
    P.nconec = b->nconec.p + elem_offs[si];
    P.kconec = b->kconec_loc.p + 9 * elem_offs[si];
    P.nesim = b->nesim.p + node_offs[si];
    P.ke = b->ke.p + 8 * node_offs[si];
    P.x = b->x.p + node_offs[si];
    P.y = b->y.p + node_offs[si];
    P.z = b->z.p + node_offs[si];
    P.tab = b->tab.p + (size_t)bem::kTabStride * elem_offs[si];
    P.mat = bem::make_material(S.mu, S.nu);
    P.A = b->H.p + hs[si].a_off;
    P.lda = hs[si].lda;
    P.G = b->G.p + hs[si].g_off;
    P.ldg = hs[si].ldg;
  }
  if ((rc = up(b, b->args, hargs)) || (rc = up(b, b->dsys, hs))) return rc;
  b->hdev = hs;
  // geometry of every element, then H and G of every system
  if (bem::launch_geometry_arrays(b->stream, (int)elem_off, b->x.p, b->y.p, b->z.p, b->nconec.p, b->kconec_glob.p,
                                  b->ref.p, b->tab.p))
    return bfail(b, BEM_ERR_CUDA, "batch geometry launch failed");
  ++b->launches;
  BB_CUDA(b, cudaMemsetAsync(b->H.p, 0, b->H.bytes(), b->stream));
  if (bem::launch_batch_hg(b->stream, b->sm_count, b->args.p, b->tiles.p, b->ntiles, b->counters.p, b->node_off.p,
                           ns, b->total_nodes, &b->launches))
    return bfail(b, BEM_ERR_CUDA, "batch assembly launch failed");
  // FI of every load case, then A in place of H, then the pinned rows
  int maxN = 0, maxp = 1;
  for (auto& D : hs) {
    maxN = std::max(maxN, D.N);
    maxp = std::max<int>(maxp, (int)D.npins);
  }
  bem::batch_fi_kernel<<<dim3((maxN + 127) / 128, ns), 128, 0, b->stream>>>(b->dsys.p, b->H.p, b->G.p, b->terms.p,
                                                                             b->coef.p, b->vec.p);
  bem::batch_a_kernel<<<dim3(maxN, ns), 128, 0, b->stream>>>(b->dsys.p, b->H.p, b->G.p, b->cs.p, b->uk_csr.p);
  bem::batch_pins_kernel<<<dim3(maxp, ns), 256, 0, b->stream>>>(b->dsys.p, b->pins.p, b->H.p, b->vec.p);
  BB_CUDA(b, cudaGetLastError());
  b->launches += 3;
  BB_CUDA(b, cudaStreamSynchronize(b->stream));
  b->assembled = true;
  b->factored = false;
  return BEM_OK;
}

}  // extern "C"

// bem_batch_info: include/bem3d_b200.h

namespace {

template <typename T, int NT>
int launch_lu(bem_batch* b, T* F) {
  static bem::DeviceOnce attr;
  if (attr.pending()) {
    if (cudaFuncSetAttribute(bem::batch_lu_kernel<T, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)bem::lu_smem<T>()) != cudaSuccess)
      return BEM_ERR_CUDA;
    attr.mark();
  }
  bem::batch_lu_kernel<T, NT><<<std::min((int)b->sys.size(), b->sm_count), NT, bem::lu_smem<T>(), b->stream>>>(
      b->dsys.p, b->ord.p, (int)b->sys.size(), F, b->piv.p, b->info.p, b->counters.p + 0);
  return cudaGetLastError() == cudaSuccess ? BEM_OK : BEM_ERR_CUDA;
}

template <typename T>
int enqueue_solve(bem_batch* b, int precision, double tol, int sweeps, T* F) {
  const int ns = (int)b->sys.size();
  const int64_t nv = b->vec.count / 3;
  double *FI = b->vec.p, *X = b->vec.p + nv, *R = b->vec.p + 2 * nv;
  const int grid = std::min(ns, b->sm_count);
  BB_CUDA(b, cudaMemsetAsync(b->counters.p, 0, b->counters.bytes(), b->stream));
  BB_CUDA(b, cudaMemsetAsync(b->conv.p, 0, b->conv.bytes(), b->stream));
  bem::batch_copy_kernel<T><<<dim3(64, ns), 256, 0, b->stream>>>(b->dsys.p, b->H.p, F);
  BB_CUDA(b, cudaGetLastError());
  int rc = (b->lu_threads == 256) ? launch_lu<T, 256>(b, F) : launch_lu<T, 512>(b, F);
  if (rc) return bfail(b, rc, "batch LU launch failed");
  unsigned* cnt = b->counters.p + 1;
  if (precision == BEM_PREC_FP64) {
    bem::batch_solve_kernel<T><<<grid, bem::kSolveThreads, bem::kSolveSmem, b->stream>>>(
        b->dsys.p, b->ord.p, ns, F, b->piv.p, FI, X, b->conv.p, b->info.p, 0, cnt++);
    bem::batch_residual_kernel<<<grid, bem::kSolveThreads, bem::kSolveSmem, b->stream>>>(
        b->dsys.p, b->ord.p, ns, b->H.p, FI, X, R, b->berr.p, b->conv.p, b->info.p, tol, 1, cnt++);
  } else {
    bem::zero_kernel<<<256, 256, 0, b->stream>>>(X, nv);
    bem::batch_residual_kernel<<<grid, bem::kSolveThreads, bem::kSolveSmem, b->stream>>>(
        b->dsys.p, b->ord.p, ns, b->H.p, FI, X, R, b->berr.p, b->conv.p, b->info.p, tol, 1, cnt++);
    for (int it = 0; it < sweeps; ++it) {
      bem::batch_solve_kernel<T><<<grid, bem::kSolveThreads, bem::kSolveSmem, b->stream>>>(
          b->dsys.p, b->ord.p, ns, F, b->piv.p, R, X, b->conv.p, b->info.p, 1, cnt++);
      bem::batch_residual_kernel<<<grid, bem::kSolveThreads, bem::kSolveSmem, b->stream>>>(
          b->dsys.p, b->ord.p, ns, b->H.p, FI, X, R, b->berr.p, b->conv.p, b->info.p, tol, 0, cnt++);
    }
  }
  BB_CUDA(b, cudaGetLastError());
  return BEM_OK;
}

template <typename T>
int set_smem() {
  static bem::DeviceOnce done;
  if (!done.pending()) return BEM_OK;
  if (cudaFuncSetAttribute(bem::batch_solve_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)bem::kSolveSmem) != cudaSuccess ||
      cudaFuncSetAttribute(bem::batch_residual_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)bem::kSolveSmem) != cudaSuccess)
    return BEM_ERR_CUDA;
  done.mark();
  return BEM_OK;
}

// the LU's CTA size: both candidates timed on this batch, the faster kept
template <typename T>
int autotune_lu(bem_batch* b, T* F) {
  if (b->lu_threads) return BEM_OK;
  const int ns = (int)b->sys.size();
  cudaEvent_t e[3];
  for (auto& x : e) BB_CUDA(b, cudaEventCreate(&x));
  BB_CUDA(b, cudaMemsetAsync(b->counters.p, 0, sizeof(unsigned), b->stream));
  bem::batch_copy_kernel<T><<<dim3(64, ns), 256, 0, b->stream>>>(b->dsys.p, b->H.p, F);
  BB_CUDA(b, cudaEventRecord(e[0], b->stream));
  if (launch_lu<T, 256>(b, F)) return bfail(b, BEM_ERR_CUDA, "batch LU launch failed");
  BB_CUDA(b, cudaEventRecord(e[1], b->stream));
  BB_CUDA(b, cudaMemsetAsync(b->counters.p, 0, sizeof(unsigned), b->stream));
  bem::batch_copy_kernel<T><<<dim3(64, ns), 256, 0, b->stream>>>(b->dsys.p, b->H.p, F);
  BB_CUDA(b, cudaEventRecord(e[2], b->stream));
  if (launch_lu<T, 512>(b, F)) return bfail(b, BEM_ERR_CUDA, "batch LU launch failed");
  cudaEvent_t e3;
  BB_CUDA(b, cudaEventCreate(&e3));
  BB_CUDA(b, cudaEventRecord(e3, b->stream));
  BB_CUDA(b, cudaEventSynchronize(e3));
  cudaEventElapsedTime(&b->lu_ms[0], e[0], e[1]);
  cudaEventElapsedTime(&b->lu_ms[1], e[2], e3);
  for (auto& x : e) cudaEventDestroy(x);
  cudaEventDestroy(e3);
  b->lu_threads = (b->lu_ms[0] <= b->lu_ms[1]) ? 256 : 512;
  b->launches += 4;
  return BEM_OK;
}

}  // namespace

extern "C" {

int bem_batch_solve(bem_batch* b, int precision, double tol, int max_iter, bem_batch_info* info) {
  if (!b || !b->assembled) return bfail(b, BEM_ERR_STATE, "batch_solve before batch_assemble");
  if (precision != BEM_PREC_FP64 && precision != BEM_PREC_FP32_IR)
    return bfail(b, BEM_ERR_ARG, "batch_solve: precision must be BEM_PREC_FP64 or BEM_PREC_FP32_IR");
  if (max_iter < 1 || max_iter > 30) return bfail(b, BEM_ERR_ARG, "batch_solve: max_iter must be in 1..30");
  for (const auto& D : b->hdev)
    if ((size_t)D.N * sizeof(double) > bem::kSolveSmem)
      return bfail(b, BEM_ERR_TOO_LARGE, "batch_solve: a system of order above 25,600");
  BB_CUDA(b, cudaSetDevice(b->device));
  int rc;
  const int ns = (int)b->sys.size();
  const int sweeps = precision == BEM_PREC_FP64 ? 0 : max_iter;
  if (precision == BEM_PREC_FP64) {
    if ((rc = set_smem<double>())) return bfail(b, rc, "batch_solve: shared memory attribute");
    if (b->A64f.count < b->H.count) BB_CUDA(b, b->A64f.alloc(b->H.count));
    if ((rc = autotune_lu<double>(b, b->A64f.p))) return rc;
  } else {
    if ((rc = set_smem<float>())) return bfail(b, rc, "batch_solve: shared memory attribute");
    if (b->A32.count < b->H.count) BB_CUDA(b, b->A32.alloc(b->H.count));
    if ((rc = autotune_lu<float>(b, b->A32.p))) return rc;
  }
  // the solve as one CUDA graph, captured once per (precision, sweeps, tol)
  if (!b->graph || b->graph_key[0] != precision || b->graph_key[1] != sweeps || b->graph_tol != tol) {
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    BB_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    rc = (precision == BEM_PREC_FP64) ? enqueue_solve<double>(b, precision, tol, sweeps, b->A64f.p)
                                      : enqueue_solve<float>(b, precision, tol, sweeps, b->A32.p);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ce != cudaSuccess) return bfail(b, BEM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    ce = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return bfail(b, BEM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
    b->graph_key[0] = precision;
    b->graph_key[1] = sweeps;
    b->graph_tol = tol;
  }
  cudaEvent_t e0, e1;
  BB_CUDA(b, cudaEventCreate(&e0));
  BB_CUDA(b, cudaEventCreate(&e1));
  BB_CUDA(b, cudaEventRecord(e0, b->stream));
  BB_CUDA(b, cudaGraphLaunch(b->graph, b->stream));
  BB_CUDA(b, cudaEventRecord(e1, b->stream));
  BB_CUDA(b, cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->launches += 5 + 2 * sweeps;
  std::vector<int> hconv(ns), hinfo(ns);
  std::vector<double> hbe(ns);
  BB_CUDA(b, cudaMemcpy(hconv.data(), b->conv.p, ns * sizeof(int), cudaMemcpyDeviceToHost));
  BB_CUDA(b, cudaMemcpy(hinfo.data(), b->info.p, ns * sizeof(int), cudaMemcpyDeviceToHost));
  BB_CUDA(b, cudaMemcpy(hbe.data(), b->berr.p, ns * sizeof(double), cudaMemcpyDeviceToHost));
  bem_batch_info st{};
  st.systems = ns;
  st.sweeps = sweeps;
  for (int s = 0; s < ns; ++s) {
    if (hinfo[s]) ++st.singular;
    else {
      st.max_backward_error = std::max(st.max_backward_error, hbe[s]);
      if (hconv[s] == 1 || hbe[s] <= tol) ++st.converged;
    }
  }
  st.solve_seconds = ms * 1e-3;
  st.lu_threads = b->lu_threads;
  st.lu_ms_256 = b->lu_ms[0];
  st.lu_ms_512 = b->lu_ms[1];
  if (info) *info = st;
  b->factored = true;
  b->factored_precision = precision;
  return st.singular ? BEM_ERR_NOCONV : BEM_OK;
}

int bem_batch_get_solution(bem_batch* b, int i, double* x) {
  if (!b || !b->factored || i < 0 || i >= (int)b->sys.size() || !x)
    return bfail(b, BEM_ERR_ARG, "batch_get_solution: bad arguments or no solve");
  const auto& D = b->hdev[i];
  const int64_t nv = b->vec.count / 3;
  BB_CUDA(b, cudaMemcpy(x, b->vec.p + nv + D.v_off, (size_t)D.N * D.nrhs * sizeof(double), cudaMemcpyDeviceToHost));
  return BEM_OK;
}

int bem_batch_get_system(bem_batch* b, int i, double* A, double* FI) {
  if (!b || !b->assembled || i < 0 || i >= (int)b->sys.size())
    return bfail(b, BEM_ERR_ARG, "batch_get_system: bad arguments or no assembly");
  const auto& D = b->hdev[i];
  if (A)
    BB_CUDA(b, cudaMemcpy2D(A, (size_t)D.N * sizeof(double), b->H.p + D.a_off, (size_t)D.lda * sizeof(double),
                            (size_t)D.N * sizeof(double), D.N, cudaMemcpyDeviceToHost));
  if (FI)
    BB_CUDA(b, cudaMemcpy(FI, b->vec.p + D.v_off, (size_t)D.N * D.nrhs * sizeof(double), cudaMemcpyDeviceToHost));
  return BEM_OK;
}

long long bem_batch_launches(const bem_batch* b) { return b ? b->launches : -1; }

}  // extern "C"
