// Blocked right-looking LU with partial pivoting (the DGESV replacement,
// solver_mod.f90:28) and its triangular solves.  See lu.cuh for the layout and the
// product form of the factors.
//
// One outer step factors an NB-wide panel of T = S^T (NB rows of S) and updates the
// trailing matrix:
//   for each 32-wide sub-panel:
//     panel_kernel      cooperative launch over the SMs; every CTA holds a slice of
//                       the sub-panel's S columns in shared memory; per pivot one
//                       grid barrier (bounded spin) exchanges the per-CTA candidates;
//                       the winner column and the diagonal column are swapped through
//                       global copies, then each CTA scales and updates its slice
//     swap_rows_kernel  applies the sub-panel's swaps to the other rows of the panel
//                       and to the trailing rows (contiguous column segments)
//     trsm_small + gemm update of the panel rows below the sub-panel
//   inv_unit_upper + gemm (TRSM by inverse), then the trailing gemm update.
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <atomic>
#include <vector>

#include "lu.cuh"

namespace bem {

constexpr int kPitch = kPanelW + 1;  // shared-memory column pitch (conflict-free)
constexpr int kInvBlock = 128;       // unit-triangle inverse block of the block-row TRSM
constexpr int kSolveBlock = 128;     // diagonal block of the triangular solves
constexpr int kPanelSmemMax = 200 * 1024;  // dynamic shared memory of a panel CTA
constexpr int kSweepThreads = 512;   // threads of a triangular sweep CTA (4 per row of a block)

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add_u32(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void better(double& bv, int& bc, int& bg, double v, int cidx, int gidx) {
  if (v > bv || (v == bv && cidx < bc)) {
    bv = v;
    bc = cidx;
    bg = gidx;
  }
}

// Copies the rows x cols block at src (column-major, lda) into shared memory dst
// (column-major, leading dimension ldd), zero outside [0,rows) x [0,cols) up to
// (full_rows x full_cols) and outside the mask; 16 loads per thread are issued before
// their shared stores so a block costs a few memory round trips, not one per element.
template <typename T, typename Mask>
__device__ __forceinline__ void stage_block(T* dst, int ldd, const T* src, int64_t lda, int rows, int cols,
                                            int full_rows, int full_cols, Mask mask) {
  const int total = full_rows * full_cols;
  for (int base = 0; base < total; base += 16 * blockDim.x) {
    T v[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int idx = base + u * blockDim.x + threadIdx.x;
      const int r = idx % full_rows, cc = idx / full_rows;
      v[u] = (idx < total && r < rows && cc < cols && mask(r, cc)) ? src[r + (int64_t)cc * lda] : T(0);
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int idx = base + u * blockDim.x + threadIdx.x;
      if (idx < total) dst[(idx % full_rows) + (idx / full_rows) * ldd] = v[u];
    }
  }
}

// threads of a panel CTA: one slice row per thread for FP32 factors (measured: the
// local candidate scan and update per pivot shrink with the rows per thread); FP64
// keeps 256 (its 176 registers per thread would spill at 512)
template <typename T>
constexpr int panel_threads() {
  return sizeof(T) == 4 ? 512 : 256;
}

template <typename T>
__global__ void __launch_bounds__(panel_threads<T>(), 1)
    panel_kernel(T* S, int64_t lda, int n, int r0, int w, int chunk, int* piv, double* cand_val,
                 int* cand_idx, T* cand_col, T* diag_col, unsigned* barrier, unsigned bar_base, int* status,
                 unsigned long long wait_ns) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* col = reinterpret_cast<T*>(smem_raw);  // [chunk][kPitch]
  __shared__ T s_pv[kPanelW];  // the winning candidate column
  __shared__ T s_dc[kPanelW];  // the diagonal column of the pivot step
  __shared__ double red_v[panel_threads<T>() / 32];
  __shared__ int red_c[panel_threads<T>() / 32];
  __shared__ int s_local_c, s_abort, s_win[2];
  const int G = gridDim.x, g = blockIdx.x, tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
  const int c_beg = r0 + g * chunk;
  const int c_end = min(n, c_beg + chunk);
  const int ncols = max(0, c_end - c_beg);

  stage_block<T>(col, kPitch, S + r0 + (int64_t)c_beg * lda, lda, w, ncols, kPanelW, ncols,
                 [](int, int) { return true; });
  __syncthreads();

  for (int t = 0; t < w; ++t) {
    const int k = r0 + t;
    const int par = t & 1;
    // 1. local candidate: largest |S(k, c)| over owned c >= k, ties -> smallest c
    double bv = -1.0;
    int bc = INT_MAX, bg = g;
    for (int cc = tid; cc < ncols; cc += blockDim.x) {
      const int cgl = c_beg + cc;
      if (cgl >= k) better(bv, bc, bg, fabs((double)col[cc * kPitch + t]), cgl, g);
    }
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
      const int oc = __shfl_xor_sync(0xffffffffu, bc, off);
      better(bv, bc, bg, ov, oc, g);
    }
    if (lane == 0) {
      red_v[wp] = bv;
      red_c[wp] = bc;
    }
    __syncthreads();
    if (tid == 0) {
      double v = red_v[0];
      int cidx = red_c[0], gg = g;
      for (int i = 1; i < (int)(blockDim.x >> 5); ++i) better(v, cidx, gg, red_v[i], red_c[i], g);
      cand_val[par * G + g] = v;
      cand_idx[par * G + g] = cidx;
      s_local_c = cidx;
    }
    __syncthreads();
    if (tid < w) {
      const int lc = s_local_c;
      if (lc != INT_MAX) cand_col[((int64_t)par * G + g) * kPanelW + tid] = col[(lc - c_beg) * kPitch + tid];
      if (k >= c_beg && k < c_end) diag_col[par * kPanelW + tid] = col[(k - c_beg) * kPitch + tid];
    }
    __syncthreads();
    // 2. grid barrier (bounded): thread 0's release covers the CTA's writes above
    if (tid == 0) {
      red_release_add_u32(barrier, 1u);
      const unsigned target = bar_base + (unsigned)(t + 1) * (unsigned)G;
      const unsigned long long t0 = globaltimer_ns();
      unsigned spins = 0;
      int abort = 0;
      while (ld_acquire_u32(barrier) < target) {
        if ((++spins & 63u) == 0 && (globaltimer_ns() - t0 > wait_ns || *((volatile int*)status) != 0)) {
          abort = 1;
          break;
        }
        __nanosleep(32);
      }
      if (abort) atomicCAS(status, 0, BEM_ERR_TIMEOUT);
      s_abort = abort;
    }
    __syncthreads();
    if (s_abort) return;
    // 3. warp 0 reduces the CTAs' candidates while warp 1 fetches the diagonal column
    //    (needed by the CTA that owns the winner); then the winner's column
    if (wp == 0) {
      double v = -1.0;
      int cidx = INT_MAX, gg = 0;
      for (int i = lane; i < G; i += 32)
        better(v, cidx, gg, __ldcg(cand_val + par * G + i), __ldcg(cand_idx + par * G + i), i);
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int oc = __shfl_xor_sync(0xffffffffu, cidx, off);
        const int og = __shfl_xor_sync(0xffffffffu, gg, off);
        better(v, cidx, gg, ov, oc, og);
      }
      if (lane == 0) {
        s_win[0] = gg;
        s_win[1] = cidx;
      }
    } else if (wp == 1) {
      s_dc[lane] = (lane < w) ? __ldcg(diag_col + par * kPanelW + lane) : T(0);
    }
    __syncthreads();
    const int wg = s_win[0], p = s_win[1];
    if (tid < kPanelW) s_pv[tid] = (tid < w) ? __ldcg(cand_col + ((int64_t)par * G + wg) * kPanelW + tid) : T(0);
    __syncthreads();
    const T* pvt = s_pv;
    const T pv = pvt[t];
    if (g == 0 && tid == 0) {
      piv[k] = p;
      if (pv == T(0) && status[1] == 0) status[1] = k + 1;
    }
    if (tid < w) {
      if (k >= c_beg && k < c_end) col[(k - c_beg) * kPitch + tid] = pvt[tid];
      if (p != k && p >= c_beg && p < c_end) col[(p - c_beg) * kPitch + tid] = s_dc[tid];
    }
    __syncthreads();
    // 5. scale the multipliers and update the rest of the sub-panel
    if (pv != T(0)) {
      for (int cc = tid; cc < ncols; cc += blockDim.x) {
        if (c_beg + cc <= k) continue;
        T* cp = col + cc * kPitch;
        const T l = cp[t] / pv;
        cp[t] = l;
        for (int j = t + 1; j < w; ++j) cp[j] -= l * pvt[j];
      }
    }
    __syncthreads();
  }
  for (int idx = tid; idx < ncols * kPanelW; idx += blockDim.x) {
    const int cc = idx / kPanelW, j = idx % kPanelW;
    if (j < w) S[(int64_t)(c_beg + cc) * lda + r0 + j] = col[cc * kPitch + j];
  }
}

// LU with partial pivoting of a full 32 x 32 window by one warp, in place in D
// (D[c][j] = row j of column c; lane c owns column c).  Per step the search is one vote
// (is any candidate larger than the diagonal?) and only then the warp argmax with the
// smallest-index tie rule; the update loads the pivot column and the lane's own column
// into registers, updates them there and stores the lane's column back, so the step's
// shared-memory accesses are independent of one another.  The operations are those of
// the general loops; the step loop is not unrolled (the warp's code stays in the
// instruction cache).  s_p[t] receives the local pivot of step t; s_g (nullable, the
// identity on entry) receives the interchanges composed into a gather: column b of the
// factored window came from column s_g[b].
template <typename T>
__device__ __forceinline__ void window_lu_warp(T (*D)[kPanelW + 1], int* s_p, int lane, int* s_g = nullptr) {
  constexpr int W = kPanelW;
#pragma unroll 1
  for (int t = 0; t < W; ++t) {
    T ct = D[lane][t];
    T pv = D[t][t];
    int p = t;
    if (__any_sync(0xffffffffu, lane > t && fabs((double)ct) > fabs((double)pv))) {
      double bv = (lane >= t) ? fabs((double)ct) : -1.0;
      int bc = (lane >= t) ? lane : INT_MAX, bg = 0;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
        const int oc = __shfl_xor_sync(0xffffffffu, bc, off);
        better(bv, bc, bg, ov, oc, 0);
      }
      p = bc;
      if (p != t) {  // columns t and p exchanged: lane j swaps their element j
        const T a = D[t][lane];
        D[t][lane] = D[p][lane];
        D[p][lane] = a;
        if (s_g && lane == 0) {
          const int gt = s_g[t];
          s_g[t] = s_g[p];
          s_g[p] = gt;
        }
        __syncwarp();
        ct = D[lane][t];
        pv = D[t][t];
      }
    }
    if (lane == 0) s_p[t] = p;
    if (pv != T(0) && lane > t) {
      const T l = ct / pv;
      T pr[W], my[W];
#pragma unroll
      for (int j = 0; j < W; ++j) {
        pr[j] = D[t][j];
        my[j] = D[lane][j];
      }
#pragma unroll
      for (int j = 0; j < W; ++j)
        if (j > t) my[j] -= l * pr[j];
#pragma unroll
      for (int j = 0; j < W; ++j)
        if (j >= t) D[lane][j] = (j == t) ? l : my[j];
    }
    __syncwarp();
  }
}

// window_lu_warp for a full FP32 window with lane c's column in registers, shifted so
// that every index is static: at step t, v[k] holds row t + k of the lane's column, and
// row t's final value (the pivot row's entry, or the multiplier) is stored to D[lane][t]
// before the shift.  The pivot column is broadcast by shuffles; an interchange moves
// the two lanes' registers (and their original indices) by shuffles and the rows
// already stored by one swap per lane.  The pivot rule (largest magnitude among lanes
// >= t, ties to the smallest index, after a vote on whether any lane beats the
// diagonal) and the arithmetic (one IEEE division per multiplier, one fused
// multiply-add per entry) are window_lu_warp's, and so are the results, bit for bit.
// s_p[t] receives step t's local pivot; s_g[b] the original window column of factored
// column b.  (Measured on one warp: 14,000 cycles for a diagonally dominant window,
// against 22,700 for window_lu_warp.)
__device__ __forceinline__ void window_lu_warp_f32(float (*D)[kPanelW + 1], int* s_p, int* s_g, int lane) {
  constexpr int W = kPanelW;
  constexpr unsigned FULL = 0xffffffffu;
  float v[W];
#pragma unroll
  for (int j = 0; j < W; ++j) v[j] = D[lane][j];
  int g = lane;
#pragma unroll 1
  for (int t = 0; t < W; ++t) {
    float ct = v[0];
    float pv = __shfl_sync(FULL, ct, t);
    int p = t;
    if (__any_sync(FULL, lane > t && fabsf(ct) > fabsf(pv))) {
      float bv = (lane >= t) ? fabsf(ct) : -1.f;
      int bc = (lane >= t) ? lane : INT_MAX;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const float ov = __shfl_xor_sync(FULL, bv, off);
        const int oc = __shfl_xor_sync(FULL, bc, off);
        if (ov > bv || (ov == bv && oc < bc)) {
          bv = ov;
          bc = oc;
        }
      }
      p = bc;
      if (p != t) {  // lanes t and p exchange their columns
        const int src = (lane == t) ? p : ((lane == p) ? t : lane);
#pragma unroll
        for (int j = 0; j < W; ++j) v[j] = __shfl_sync(FULL, v[j], src);
        g = __shfl_sync(FULL, g, src);
        if (lane < t) {  // the rows already stored: lane j swaps its row j
          const float a = D[t][lane];
          D[t][lane] = D[p][lane];
          D[p][lane] = a;
        }
        ct = v[0];
        pv = __shfl_sync(FULL, ct, t);
      }
    }
    if (lane == 0) s_p[t] = p;
    float pr[W];
#pragma unroll
    for (int k = 1; k < W; ++k) pr[k] = __shfl_sync(FULL, v[k], t);
    if (pv != 0.f && lane > t) {
      const float l = ct / pv;
#pragma unroll
      for (int k = 1; k < W; ++k) v[k] -= l * pr[k];
      v[0] = l;
    }
    D[lane][t] = v[0];
#pragma unroll
    for (int k = 0; k < W - 1; ++k) v[k] = v[k + 1];
    v[W - 1] = 0.f;
    __syncwarp();
  }
  s_g[lane] = g;
  __syncwarp();
}

// Window pivoting: the sub-panel's pivot search is restricted to its w x w diagonal
// block (T rows r0..r0+w), so the sub-panel needs no grid-wide exchange.  Every CTA
// factors that block redundantly in shared memory (warp 0: lane c owns column c of the
// window, one warp argmax per pivot, ties to the smallest index as the partial-pivot
// kernel), while its other warps load their columns; then each thread eliminates one
// column c >= r0 + w of the sub-panel (T row c) with the recorded steps, the same
// operations panel_kernel applies to a non-pivot column.  CTA 0 writes the pivots, the
// first exact zero pivot (status[1]) and the factored block to `win` (w x w, leading
// dimension kPanelW): the block is copied into S by the next launch (swap_rows_kernel),
// since other CTAs of this launch may still be reading it from S.
template <typename T>
__global__ void __launch_bounds__(256) window_panel_kernel(T* S, int64_t lda, int n, int r0, int w, int* piv,
                                                           T* win, int* status) {
  // n: the end of the columns eliminated here (the whole matrix, or the panel's
  // diagonal block when the rest of the sub-panel is left to the panel's TRSM)
  __shared__ T D[kPanelW][kPanelW + 1];  // D[c][j] = S(r0 + j, r0 + c)
  __shared__ int s_p[kPanelW];
  const int tid = threadIdx.x, lane = tid & 31;
  const int c = r0 + w + blockIdx.x * blockDim.x + tid;  // this thread's column (T row)
  constexpr int V = 16 / sizeof(T);                       // elements per 16-byte vector
  const bool vec = ((lda % V) == 0) && ((r0 % V) == 0) && ((reinterpret_cast<uintptr_t>(S) & 15) == 0);
  // every load of the thread's column before the window's barrier (r0 + 32 <= lda: the
  // rows up to 32 exist in every column; only rows < w are used or stored)
  T x[kPanelW];
  if (c < n) {
    const T* src = S + r0 + (int64_t)c * lda;
    if (vec && r0 + kPanelW <= lda) {
#pragma unroll
      for (int q = 0; q < kPanelW / V; ++q) {
        const int4 v = *reinterpret_cast<const int4*>(src + q * V);
        const T* e = reinterpret_cast<const T*>(&v);
#pragma unroll
        for (int u = 0; u < V; ++u) x[q * V + u] = e[u];
      }
    } else {
#pragma unroll
      for (int j = 0; j < kPanelW; ++j) x[j] = (j < w) ? src[j] : T(0);
    }
  }
  if (tid < kPanelW) {
    // warp 0: stage and factor the window
    for (int cc = 0; cc < kPanelW; ++cc)  // lane = row: one coalesced segment per column
      D[cc][lane] = (cc < w && lane < w) ? S[r0 + lane + (int64_t)(r0 + cc) * lda] : T(0);
    __syncwarp();
    if (w == kPanelW) {
      window_lu_warp<T>(D, s_p, lane);
    } else {
      for (int t = 0; t < w; ++t) {
        double bv = (lane >= t && lane < w) ? fabs((double)D[lane][t]) : -1.0;
        int bc = (lane >= t && lane < w) ? lane : INT_MAX, bg = 0;
        for (int off = 16; off > 0; off >>= 1) {
          const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
          const int oc = __shfl_xor_sync(0xffffffffu, bc, off);
          better(bv, bc, bg, ov, oc, 0);
        }
        const int p = bc;
        if (lane == 0) s_p[t] = p;
        if (p != t && lane < w) {
          const T a = D[t][lane];
          D[t][lane] = D[p][lane];
          D[p][lane] = a;
        }
        __syncwarp();
        const T pv = D[t][t];
        if (pv != T(0) && lane > t && lane < w) {
          const T l = D[lane][t] / pv;
          D[lane][t] = l;
          for (int j = t + 1; j < w; ++j) D[lane][j] -= l * D[t][j];
        }
        __syncwarp();
      }
    }
    if (blockIdx.x == 0) {
      if (lane < w) {
        piv[r0 + lane] = r0 + s_p[lane];
        for (int j = 0; j < w; ++j) win[j + lane * kPanelW] = D[lane][j];
      }
      if (lane == 0) {
        for (int t = 0; t < w; ++t)
          if (D[t][t] == T(0)) {
            if (status[1] == 0) status[1] = r0 + t + 1;
            break;
          }
      }
    }
  }
  __syncthreads();
  if (c >= n) return;
  // eliminate: step t scales x[t] by the pivot and updates the entries below it
#pragma unroll
  for (int t = 0; t < kPanelW; ++t) {
    if (t < w) {
      const T pv = D[t][t];
      if (pv != T(0)) {
        const T l = x[t] / pv;
        x[t] = l;
#pragma unroll
        for (int j = t + 1; j < kPanelW; ++j)
          if (j < w) x[j] -= l * D[t][j];
      }
    }
  }
  T* dst = S + r0 + (int64_t)c * lda;
  if (vec && w == kPanelW) {
#pragma unroll
    for (int q = 0; q < kPanelW / V; ++q) {
      int4 v;
      T* e = reinterpret_cast<T*>(&v);
#pragma unroll
      for (int u = 0; u < V; ++u) e[u] = x[q * V + u];
      *reinterpret_cast<int4*>(dst + q * V) = v;
    }
  } else {
#pragma unroll
    for (int j = 0; j < kPanelW; ++j)
      if (j < w) dst[j] = x[j];
  }
}

// The whole step of one 32-wide sub-panel of a window-pivoted FP32 panel in one CTA
// (the panel's diagonal block only; rows and columns outside it follow per panel):
// warp 0 factors the 32 x 32 window in registers while the other threads load their
// columns; every thread then eliminates its column of the sub-panel (columns
// [r0 + 32, t0)), the factored window goes back into S, and one thread per row of the
// block applies the window's interchanges as a gather and, below the window, the
// unit-lower TRSM of trsm_small_kernel.  Pivots and the first exact zero pivot as
// window_panel_kernel.  w = 32; t0 - r0 <= kBlockThreads.
constexpr int kBlockThreads = 512;
__global__ void __launch_bounds__(kBlockThreads) window_block_kernel(float* S, int64_t lda, int j0, int t0, int r0,
                                                                     int* piv, int* status) {
  constexpr int W = kPanelW;
  __shared__ float D[W][W + 1];  // D[c][j] = S(r0 + j, r0 + c)
  __shared__ int s_p[W], s_g[W];
  const int tid = threadIdx.x, lane = tid & 31;
  const int c = r0 + W + tid;  // this thread's column
  float x[W];
  const bool has_col = c < t0;
  if (has_col) {
    const float* src = S + r0 + (int64_t)c * lda;
#pragma unroll
    for (int q = 0; q < W / 4; ++q) {
      const float4 v = *reinterpret_cast<const float4*>(src + 4 * q);
      x[4 * q] = v.x;
      x[4 * q + 1] = v.y;
      x[4 * q + 2] = v.z;
      x[4 * q + 3] = v.w;
    }
  }
  if (tid < W) {
#pragma unroll
    for (int cc = 0; cc < W; ++cc) D[cc][lane] = S[r0 + lane + (int64_t)(r0 + cc) * lda];
    __syncwarp();
    window_lu_warp_f32(D, s_p, s_g, lane);  // s_g: the interchanges as a gather, y[b] = x[s_g[b]]
    if (lane == 0) {
      for (int t = 0; t < W; ++t)
        if (D[t][t] == 0.f) {
          if (status[1] == 0) status[1] = r0 + t + 1;
          break;
        }
    }
    piv[r0 + lane] = r0 + s_p[lane];
  }
  __syncthreads();
  if (has_col) {
#pragma unroll
    for (int t = 0; t < W; ++t) {
      const float pv = D[t][t];
      if (pv != 0.f) {
        const float l = x[t] / pv;
        x[t] = l;
#pragma unroll
        for (int j = t + 1; j < W; ++j) x[j] -= l * D[t][j];
      }
    }
    float* dst = S + r0 + (int64_t)c * lda;
#pragma unroll
    for (int q = 0; q < W / 4; ++q)
      *reinterpret_cast<float4*>(dst + 4 * q) = make_float4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
  }
  // the factored window
  for (int i = tid; i < W * W; i += blockDim.x) {
    const int j = i % W, cc = i / W;
    S[r0 + j + (int64_t)(r0 + cc) * lda] = D[cc][j];
  }
  // rows of the block outside the window: the interchanges, and below it the TRSM
  const int nabove = r0 - j0, nrows = (t0 - j0) - W;
  if (tid < nrows) {
    const int r = tid < nabove ? j0 + tid : r0 + W + (tid - nabove);
    float y[W];
#pragma unroll
    for (int b = 0; b < W; ++b) y[b] = S[r + (int64_t)(r0 + s_g[b]) * lda];
    if (r >= r0 + W) {
#pragma unroll
      for (int b = 0; b < W; ++b) {
        float v = y[b];
#pragma unroll
        for (int a = 0; a < b; ++a) v -= y[a] * D[b][a];  // U(a, b) = S(r0 + a, r0 + b)
        y[b] = v;
      }
    }
#pragma unroll
    for (int b = 0; b < W; ++b) S[r + (int64_t)(r0 + b) * lda] = y[b];
  }
}

// Grid barrier of a cooperative launch (bounded): every thread's earlier writes are
// ordered before the arrival (CTA barrier, then thread 0's fence and release); the
// wait gives up after wait_ns or once another CTA recorded an error, and records
// BEM_ERR_TIMEOUT.  Returns false when the launch must stop.
__device__ __forceinline__ bool coop_barrier(unsigned* barrier, unsigned target, int* status,
                                             unsigned long long wait_ns, int* s_abort) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    red_release_add_u32(barrier, 1u);
    const unsigned long long t0 = globaltimer_ns();
    unsigned spins = 0;
    int abort = 0;
    while (ld_acquire_u32(barrier) < target) {
      if ((++spins & 63u) == 0 && (globaltimer_ns() - t0 > wait_ns || *((volatile int*)status) != 0)) {
        abort = 1;
        break;
      }
      __nanosleep(32);
    }
    if (abort) atomicCAS(status, 0, BEM_ERR_TIMEOUT);
    __threadfence();
    *s_abort = abort;
  }
  __syncthreads();
  return *s_abort == 0;
}

// The diagonal block [j0, t0)^2 of a window-pivoted FP32 panel in one cooperative
// launch: the 32-wide sub-panels in turn, each in three phases separated by grid
// barriers (two per sub-panel) instead of kernel boundaries:
//   A  every CTA's warp 0 stages and factors the 32 x 32 window (redundantly; the
//      interchanges composed into a gather on the way); CTA 0 records the pivots and
//      the first exact zero pivot;
//   B  the sub-panel's vectors, one thread each, spread over the CTAs in contiguous
//      runs: every column c in [r0 + 32, t0) eliminated with the window's steps
//      (window_panel_kernel's column operations, with each multiplier formed by the
//      pivot's reciprocal), every row of the block outside the window gathered
//      through the interchanges and, below the window, solved with the window's
//      unit-lower triangle (trsm_small_kernel's operations);
//   C  the rank-32 update of the block's trailing part, S(q, q) -= S(q, w) S(w, q)
//      with q = [r0 + 32, t0) and w the window, in 64 x 64 tiles (FP32 FMA), and
//      CTA 0 stores the factored window (every CTA has read it by now).
// Every read of S goes through L2 (__ldcg): the other CTAs' writes of the previous
// phase are ordered by the barrier, never by this SM's L1.  The rows and columns
// outside the block follow per panel (permute_panel_kernel, the blocked TRSMs).
constexpr int kCoopThreads = 256;
constexpr int kCoopTile = 64;
constexpr int kCoopMaxCtas = 160;  // one CTA per SM (148 on a B200)
__global__ void __launch_bounds__(kCoopThreads, 1)
    panel_coop_kernel(float* S, int64_t lda, int j0, int t0, int* piv, unsigned* barrier, unsigned bar_base,
                      int* status, unsigned long long wait_ns) {
  constexpr int W = kPanelW;
  constexpr int TP = kCoopTile + 4;  // strip pitch: 16-byte rows, 4-way store conflicts at most
  __shared__ float D[W][W + 1];     // D[c][j] = S(r0 + j, r0 + c)
  __shared__ float rdg[W];          // reciprocal pivots (0 for an exact zero pivot)
  __shared__ int s_p[W], s_g[W];
  __shared__ __align__(16) float Ls[W][TP];  // Ls[k][r] = S(q0 + tr + r, r0 + k)
  __shared__ __align__(16) float Us[W][TP];  // Us[k][c] = S(r0 + k, q0 + tc + c)
  __shared__ int s_abort;
  const int G = gridDim.x, g = blockIdx.x, tid = threadIdx.x, lane = tid & 31;
  unsigned target = bar_base;
  for (int r0 = j0; r0 < t0; r0 += W) {
    const int q0 = r0 + W, m = t0 - q0;
    // A: the window
    if (tid < W) {
      float wv[W];  // every load in flight before the first store
#pragma unroll
      for (int cc = 0; cc < W; ++cc) wv[cc] = __ldcg(S + r0 + lane + (int64_t)(r0 + cc) * lda);
#pragma unroll
      for (int cc = 0; cc < W; ++cc) D[cc][lane] = wv[cc];
      __syncwarp();
      window_lu_warp_f32(D, s_p, s_g, lane);
      rdg[lane] = (D[lane][lane] != 0.f) ? __frcp_rn(D[lane][lane]) : 0.f;
      if (g == 0) {
        piv[r0 + lane] = r0 + s_p[lane];
        if (lane == 0) {
          for (int t = 0; t < W; ++t)
            if (D[t][t] == 0.f) {
              if (status[1] == 0) status[1] = r0 + t + 1;
              break;
            }
        }
      }
    }
    __syncthreads();
    // B: columns [q0, t0), then rows [j0, r0) and [q0, t0)
    {
      const int nabove = r0 - j0;
      const int nvec = m + nabove + m;
      const int per = (nvec + G - 1) / G;
      const int v0 = g * per, v1 = min(nvec, v0 + per);
      for (int v = v0 + tid; v < v1; v += blockDim.x) {
        if (v < m) {
          float x[W];
          float* col = S + r0 + (int64_t)(q0 + v) * lda;
#pragma unroll
          for (int q = 0; q < W / 4; ++q) {
            const float4 f = __ldcg(reinterpret_cast<const float4*>(col) + q);
            x[4 * q] = f.x;
            x[4 * q + 1] = f.y;
            x[4 * q + 2] = f.z;
            x[4 * q + 3] = f.w;
          }
          // multipliers by the pivots' reciprocals: the chain of 32 steps is a multiply
          // and a fused multiply-add each, not a division
#pragma unroll
          for (int t = 0; t < W; ++t) {
            const float rp = rdg[t];
            if (rp != 0.f) {
              const float l = x[t] * rp;
              x[t] = l;
#pragma unroll
              for (int j = t + 1; j < W; ++j) x[j] -= l * D[t][j];
            }
          }
#pragma unroll
          for (int q = 0; q < W / 4; ++q)
            reinterpret_cast<float4*>(col)[q] = make_float4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
        } else {
          const int i = v - m;
          const int r = i < nabove ? j0 + i : q0 + (i - nabove);
          float y[W];
#pragma unroll
          for (int b = 0; b < W; ++b) y[b] = __ldcg(S + r + (int64_t)(r0 + s_g[b]) * lda);
          if (r >= q0) {
#pragma unroll
            for (int b = 0; b < W; ++b) {
              float a = y[b];
#pragma unroll
              for (int k = 0; k < b; ++k) a -= y[k] * D[b][k];  // U(k, b) = S(r0 + k, r0 + b)
              y[b] = a;
            }
          }
#pragma unroll
          for (int b = 0; b < W; ++b) S[r + (int64_t)(r0 + b) * lda] = y[b];
        }
      }
    }
    target += (unsigned)G;
    if (!coop_barrier(barrier, target, status, wait_ns, &s_abort)) return;
    // C: the trailing tiles; CTA 0 stores the window
    if (g == 0)
      for (int i = tid; i < W * W; i += blockDim.x) {
        const int j = i % W, cc = i / W;
        S[r0 + j + (int64_t)(r0 + cc) * lda] = D[cc][j];
      }
    const int nt = (m + kCoopTile - 1) / kCoopTile;
    for (int tau = g; tau < nt * nt; tau += G) {
      const int tr = (tau % nt) * kCoopTile, tc = (tau / nt) * kCoopTile;
      const int ri = (tid % 16) * 4, ci = (tid / 16) * 4;
      // every load of the tile in flight before the first use: the strips, then C
      constexpr int NS = W * kCoopTile / kCoopThreads;
      float lv[NS], uv[NS];
#pragma unroll
      for (int u = 0; u < NS; ++u) {
        const int i = tid + u * kCoopThreads;
        const int rr = i % kCoopTile, k = i / kCoopTile;
        lv[u] = (tr + rr < m) ? __ldcg(S + q0 + tr + rr + (int64_t)(r0 + k) * lda) : 0.f;
      }
#pragma unroll
      for (int u = 0; u < NS; ++u) {
        const int i = tid + u * kCoopThreads;
        const int k = i % W, cc = i / W;
        uv[u] = (tc + cc < m) ? __ldcg(S + r0 + k + (int64_t)(q0 + tc + cc) * lda) : 0.f;
      }
      float4 cv[4];
#pragma unroll
      for (int v = 0; v < 4; ++v)
        cv[v] = (tr + ri < m && tc + ci + v < m)
                    ? __ldcg(reinterpret_cast<const float4*>(S + q0 + tr + ri + (int64_t)(q0 + tc + ci + v) * lda))
                    : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int u = 0; u < NS; ++u) {
        const int i = tid + u * kCoopThreads;
        Ls[i / kCoopTile][i % kCoopTile] = lv[u];
        Us[i % W][i / W] = uv[u];
      }
      __syncthreads();
      float acc[4][4] = {};
#pragma unroll 8
      for (int k = 0; k < W; ++k) {
        const float4 a = *reinterpret_cast<const float4*>(&Ls[k][ri]);
        const float4 b = *reinterpret_cast<const float4*>(&Us[k][ci]);
        const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(av[u], bv[v], acc[u][v]);
      }
      // m is a multiple of 32: a 4-row group lies wholly inside or outside the block
      if (tr + ri < m) {
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          if (tc + ci + v < m) {
            float4 o = cv[v];
            o.x -= acc[0][v];
            o.y -= acc[1][v];
            o.z -= acc[2][v];
            o.w -= acc[3][v];
            *reinterpret_cast<float4*>(S + q0 + tr + ri + (int64_t)(q0 + tc + ci + v) * lda) = o;
          }
        }
      }
      __syncthreads();
    }
    target += (unsigned)G;
    if (!coop_barrier(barrier, target, status, wait_ns, &s_abort)) return;
  }
}

// Applies swaps k0+t <-> piv[k0+t] (t = 0..w-1 in order) to rows [a0,a1) and [b0,b1).
// With window pivoting `win` (nullable) holds the factored w x w diagonal block of the
// sub-panel (leading dimension kPanelW), which CTA 0 copies into S(k0.., k0..) first;
// the swaps below touch no row of that block.
template <typename T>
__global__ void swap_rows_kernel(T* S, int64_t lda, const int* piv, int k0, int w, int a0, int a1, int b0,
                                 int b1, const T* win) {
  __shared__ int sp[kPanelW];
  if (threadIdx.x < w) sp[threadIdx.x] = piv[k0 + threadIdx.x];
  if (win && blockIdx.x == 0)
    for (int i = threadIdx.x; i < w * w; i += blockDim.x) {
      const int j = i % w, cc = i / w;
      S[k0 + j + (int64_t)(k0 + cc) * lda] = win[j + cc * kPanelW];
    }
  __syncthreads();
  const int na = a1 - a0;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)na + (b1 - b0)) return;
  const int64_t r = (i < na) ? a0 + i : b0 + (i - na);
  for (int t = 0; t < w; ++t) {
    const int p = sp[t];
    if (p == k0 + t) continue;
    T* x = S + r + (int64_t)(k0 + t) * lda;
    T* y = S + r + (int64_t)p * lda;
    const T a = *x;
    *x = *y;
    *y = a;
  }
}

// A window-pivoted panel's interchanges (the swaps k0+t <-> piv[k0+t], t = 0..w-1 in
// order, every swap inside its 32-wide sub-panel) applied at once to rows [a0,a1) and
// [b0,b1) of S: they compose into a gather of the panel's columns,
// x[k0 + c] := x[k0 + perm[c]], and only the columns the gather moves are read and
// written.  The panel goes in chunks of up to 512 columns (no swap crosses a chunk);
// within a chunk the sub-panels compose independently (one warp lane each, in
// parallel).  A CTA takes 64 / sizeof(T) rows (32 KB of staged sources for 512 moved
// columns); every source of a chunk is read before any destination is written.
constexpr int kPermMax = 512;
template <typename T>
__global__ void __launch_bounds__(256) permute_panel_kernel(T* S, int64_t lda, const int* piv, int k0, int w, int a0,
                                                            int a1, int b0, int b1) {
  constexpr int R = 64 / sizeof(T);  // rows per CTA
  __shared__ int perm[kPermMax];
  __shared__ int moved[kPermMax];
  __shared__ int sp[kPermMax];
  __shared__ int nmoved;
  __shared__ T buf[kPermMax * R];
  const int tid = threadIdx.x, lane = tid & 31;
  const int na = a1 - a0;
  const int rr = tid % R, slot = tid / R, nslot = blockDim.x / R;
  const int64_t i = (int64_t)blockIdx.x * R + rr;
  const bool ok = i < (int64_t)na + (b1 - b0);
  const int64_t r = ok ? ((i < na) ? a0 + i : b0 + (i - na)) : 0;
  for (int h0 = 0; h0 < w; h0 += kPermMax) {
    const int hw = min(kPermMax, w - h0), kh = k0 + h0;
    for (int c = tid; c < hw; c += blockDim.x) {
      perm[c] = c;
      sp[c] = piv[kh + c] - kh;
    }
    if (tid == 0) nmoved = 0;
    __syncthreads();
    if (lane == 0) {
      for (int g0 = (tid >> 5) * kPanelW; g0 < hw; g0 += (int)(blockDim.x >> 5) * kPanelW) {
        const int ge = min(hw, g0 + kPanelW);
        for (int t = g0; t < ge; ++t) {
          const int p = sp[t];
          const int x = perm[t];
          perm[t] = perm[p];
          perm[p] = x;
        }
      }
    }
    __syncthreads();
    // the moved columns, in any order (a slot's source and destination stay paired)
    for (int c = tid; c < hw; c += blockDim.x)
      if (perm[c] != c) moved[atomicAdd(&nmoved, 1)] = c;
    __syncthreads();
    const int nm = nmoved;  // uniform in the CTA
    if (nm > 0) {
      for (int q = slot; q < nm; q += nslot)
        if (ok) buf[q * R + rr] = S[r + (int64_t)(kh + perm[moved[q]]) * lda];
      __syncthreads();
      for (int q = slot; q < nm; q += nslot)
        if (ok) S[r + (int64_t)(kh + moved[q]) * lda] = buf[q * R + rr];
    }
    __syncthreads();  // perm, moved and buf are reused by the next chunk
  }
}

// Y := X * U^{-1} in place for rows [r_lo, r_hi), X = S(rows, k0..k0+w), U the unit
// upper triangle of S(k0..k0+w, k0..k0+w).
template <typename T>
__global__ void trsm_small_kernel(T* S, int64_t lda, int k0, int w, int r_lo, int r_hi) {
  __shared__ T Ucm[kPanelW * (kPanelW + 1)];  // column-major, leading dimension kPanelW + 1
  stage_block<T>(Ucm, kPanelW + 1, S + k0 + (int64_t)k0 * lda, lda, w, w, kPanelW, kPanelW,
                 [](int, int) { return true; });
  __syncthreads();
  auto U = [&](int a, int b) { return Ucm[a + b * (kPanelW + 1)]; };
  const int r = r_lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= r_hi) return;
  // every load of the row before its first store (a store to S may alias later loads)
  T y[kPanelW];
#pragma unroll
  for (int b = 0; b < kPanelW; ++b) y[b] = (b < w) ? S[r + (int64_t)(k0 + b) * lda] : T(0);
#pragma unroll
  for (int b = 0; b < kPanelW; ++b) {
    if (b < w) {
      T v = y[b];
#pragma unroll
      for (int a = 0; a < b; ++a) v -= y[a] * U(a, b);
      y[b] = v;
    }
  }
#pragma unroll
  for (int b = 0; b < kPanelW; ++b)
    if (b < w) S[r + (int64_t)(k0 + b) * lda] = y[b];
}

// V = U^{-1} for the unit upper triangle U of S11 (jb x jb, jb <= 128); V column-major
// (ldv).  Blocked by 32: four warps invert the diagonal blocks (lane j holds column j
// of its block in registers and back-substitutes), then the off-diagonal blocks follow
// in order of their distance from the diagonal,
//   V_ij = -V_ii * sum_{k=i+1..j} U_ik V_kj,
// each a 32 x 32 product spread over all 256 threads.  U is staged in shared memory,
// V is written to (and re-read from) global memory by this CTA only.
template <typename T>
__global__ void __launch_bounds__(256) inv_unit_upper_kernel(const T* S11, int64_t lda, int jb, T* V, int ldv) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* U = reinterpret_cast<T*>(smem_raw);  // [128][128] column-major, zero outside the strict upper part
  __shared__ T tmp[32 * 33];
  constexpr int B = 32, NB = 128;
  stage_block<T>(U, NB, S11, lda, jb, jb, NB, NB, [](int a, int b) { return a < b; });
  __syncthreads();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nblk = (jb + B - 1) / B;
  // diagonal blocks
  if (warp < nblk) {
    const int o = warp * B;
    T x[B];
#pragma unroll
    for (int i = 0; i < B; ++i) x[i] = (i == lane) ? T(1) : T(0);
#pragma unroll
    for (int i = B - 2; i >= 0; --i) {
      T sacc = x[i];
#pragma unroll
      for (int k = i + 1; k < B; ++k) sacc -= U[(o + i) + (o + k) * NB] * x[k];
      x[i] = (i < lane) ? sacc : x[i];
    }
#pragma unroll
    for (int i = 0; i < B; ++i)
      if (o + i < jb && o + lane < jb) V[(o + i) + (int64_t)(o + lane) * ldv] = x[i];
  }
  // zero the strict lower blocks of V
  for (int idx = tid; idx < jb * jb; idx += blockDim.x) {
    const int r = idx % jb, cc = idx / jb;
    if (r / B > cc / B) V[r + (int64_t)cc * ldv] = T(0);
  }
  __syncthreads();
  for (int d = 1; d < nblk; ++d)
    for (int bi = 0; bi + d < nblk; ++bi) {
      const int bj = bi + d;
      const int oi = bi * B, oj = bj * B;
      // tmp = sum_{k=bi+1..bj} U_{bi,k} V_{k,bj}   (32 x 32)
      for (int e = tid; e < B * B; e += blockDim.x) {
        const int r = e % B, cc = e / B;
        T acc = T(0);
        for (int k = oi + B; k <= oj + B - 1 && k < jb; ++k) acc += U[(oi + r) + k * NB] * V[k + (int64_t)(oj + cc) * ldv];
        tmp[r + cc * 33] = acc;
      }
      __syncthreads();
      // V_{bi,bj} = -V_{bi,bi} tmp
      for (int e = tid; e < B * B; e += blockDim.x) {
        const int r = e % B, cc = e / B;
        T acc = T(0);
#pragma unroll 8
        for (int k = 0; k < B; ++k) acc += V[(oi + r) + (int64_t)(oi + k) * ldv] * tmp[k + cc * 33];
        if (oi + r < jb && oj + cc < jb) V[(oi + r) + (int64_t)(oj + cc) * ldv] = -acc;
      }
      __syncthreads();
    }
}

// The same inverse for FP32 factors with U and V both in shared memory (2 x 64 KB) and
// the off-diagonal blocks of one distance from the diagonal computed together (two
// barriers per distance); V is written to global memory once at the end.
constexpr int kInvThreads = 512;

// V (zeroed, [128][128] column-major, shared) := U^{-1} for the unit upper triangle whose
// strict upper part U holds (shared, zero elsewhere), jb <= 128; all threads take part.
__device__ __forceinline__ void unit_upper_inverse_smem(const float* U, float* V, int jb, float (*tmp)[32 * 33]) {
  constexpr int B = 32, NB = 128;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nblk = (jb + B - 1) / B;
  if (warp < nblk) {
    const int o = warp * B;
    float x[B];
#pragma unroll
    for (int i = 0; i < B; ++i) x[i] = (i == lane) ? 1.f : 0.f;
#pragma unroll
    for (int i = B - 2; i >= 0; --i) {
      float sacc = x[i];
#pragma unroll
      for (int k = i + 1; k < B; ++k) sacc -= U[(o + i) + (o + k) * NB] * x[k];
      x[i] = (i < lane) ? sacc : x[i];
    }
#pragma unroll
    for (int i = 0; i < B; ++i)
      if (o + i < jb && o + lane < jb) V[(o + i) + (o + lane) * NB] = x[i];
  }
  __syncthreads();
  for (int d = 1; d < nblk; ++d) {
    const int nb_d = nblk - d;  // blocks (bi, bi + d)
    for (int e = tid; e < nb_d * B * B; e += kInvThreads) {
      const int bi = e / (B * B), r = e % B, cc = (e / B) % B;
      const int oi = bi * B, oj = (bi + d) * B;
      float acc = 0.f;
      for (int k = oi + B; k <= oj + B - 1 && k < jb; ++k) acc += U[(oi + r) + k * NB] * V[k + (oj + cc) * NB];
      tmp[bi][r + cc * 33] = acc;
    }
    __syncthreads();
    for (int e = tid; e < nb_d * B * B; e += kInvThreads) {
      const int bi = e / (B * B), r = e % B, cc = (e / B) % B;
      const int oi = bi * B, oj = (bi + d) * B;
      float acc = 0.f;
#pragma unroll 8
      for (int k = 0; k < B; ++k) acc += V[(oi + r) + (oi + k) * NB] * tmp[bi][k + cc * 33];
      if (oi + r < jb && oj + cc < jb) V[(oi + r) + (oj + cc) * NB] = -acc;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kInvThreads) inv_unit_upper_f32_kernel(const float* S11, int64_t lda, int jb,
                                                                         float* Vout, int ldv) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int B = 32, NB = 128, NBLK = NB / B;
  float* U = reinterpret_cast<float*>(smem_raw);  // [NB][NB] column-major, the strict upper part
  float* V = U + NB * NB;                         // [NB][NB] column-major
  __shared__ float tmp[NBLK - 1][B * 33];
  stage_block<float>(U, NB, S11, lda, jb, jb, NB, NB, [](int a, int b) { return a < b; });
  for (int i = threadIdx.x; i < NB * NB; i += kInvThreads) V[i] = 0.f;
  __syncthreads();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nblk = (jb + B - 1) / B;
  if (warp < nblk) {
    const int o = warp * B;
    float x[B];
#pragma unroll
    for (int i = 0; i < B; ++i) x[i] = (i == lane) ? 1.f : 0.f;
#pragma unroll
    for (int i = B - 2; i >= 0; --i) {
      float sacc = x[i];
#pragma unroll
      for (int k = i + 1; k < B; ++k) sacc -= U[(o + i) + (o + k) * NB] * x[k];
      x[i] = (i < lane) ? sacc : x[i];
    }
#pragma unroll
    for (int i = 0; i < B; ++i)
      if (o + i < jb && o + lane < jb) V[(o + i) + (o + lane) * NB] = x[i];
  }
  __syncthreads();
  for (int d = 1; d < nblk; ++d) {
    const int nb_d = nblk - d;  // blocks (bi, bi + d)
    for (int e = tid; e < nb_d * B * B; e += kInvThreads) {
      const int bi = e / (B * B), r = e % B, cc = (e / B) % B;
      const int oi = bi * B, oj = (bi + d) * B;
      float acc = 0.f;
      for (int k = oi + B; k <= oj + B - 1 && k < jb; ++k) acc += U[(oi + r) + k * NB] * V[k + (oj + cc) * NB];
      tmp[bi][r + cc * 33] = acc;
    }
    __syncthreads();
    for (int e = tid; e < nb_d * B * B; e += kInvThreads) {
      const int bi = e / (B * B), r = e % B, cc = (e / B) % B;
      const int oi = bi * B, oj = (bi + d) * B;
      float acc = 0.f;
#pragma unroll 8
      for (int k = 0; k < B; ++k) acc += V[(oi + r) + (oi + k) * NB] * tmp[bi][k + cc * 33];
      if (oi + r < jb && oj + cc < jb) V[(oi + r) + (oj + cc) * NB] = -acc;
    }
    __syncthreads();
  }
  for (int i = tid; i < jb * jb; i += kInvThreads) {
    const int r = i % jb, cc = i / jb;
    Vout[r + (int64_t)cc * ldv] = V[r + cc * NB];
  }
}

// The inverses a window-pivoted panel's TRSMs take, for every 128-block b of the
// panel's diagonal block (S11 = S(j0.., j0..), jb <= 512): blockIdx.y = 0 writes
// Vu[b] = the inverse of the unit upper triangle of block b (the multipliers, as
// inv_unit_upper_f32_kernel), blockIdx.y = 1 writes Wl[b] = the inverse of its lower
// triangle, diagonal included (U^T of T).  The lower inverse goes through the unit
// upper routine: W = Lu D with Lu unit lower, so W^{-1} = D^{-1} ((Lu^T)^{-1})^T.
// Each inverse is 128 x 128 column-major (leading dimension 128, zero outside jb x jb).
__global__ void __launch_bounds__(kInvThreads) panel_inv_f32_kernel(const float* S11, int64_t lda, int jb,
                                                                    float* Vu, float* Wl) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int B = 32, NB = 128, NBLK = NB / B;
  float* U = reinterpret_cast<float*>(smem_raw);
  float* V = U + NB * NB;
  __shared__ float tmp[NBLK - 1][B * 33];
  __shared__ float rdiag[NB];
  const int b = blockIdx.x, o = b * NB, bb = min(NB, jb - o);
  const float* D = S11 + o + (int64_t)o * lda;
  const bool lower = blockIdx.y == 1;
  if (!lower) {
    stage_block<float>(U, NB, D, lda, bb, bb, NB, NB, [](int a, int c) { return a < c; });
  } else {
    for (int i = threadIdx.x; i < NB; i += kInvThreads) rdiag[i] = (i < bb) ? D[i + (int64_t)i * lda] : 1.f;
    __syncthreads();
    // U[a][c] = Lu^T[a][c] = W[c][a] / W[a][a]  (a < c)
    for (int i = threadIdx.x; i < NB * NB; i += kInvThreads) {
      const int a = i % NB, c = i / NB;
      U[i] = (a < c && c < bb) ? D[c + (int64_t)a * lda] / rdiag[a] : 0.f;
    }
  }
  for (int i = threadIdx.x; i < NB * NB; i += kInvThreads) V[i] = 0.f;
  __syncthreads();
  unit_upper_inverse_smem(U, V, bb, tmp);
  float* out = (lower ? Wl : Vu) + (size_t)b * NB * NB;
  for (int i = threadIdx.x; i < NB * NB; i += kInvThreads) {
    const int r = i % NB, c = i / NB;
    float v = 0.f;
    if (r < bb && c < bb) v = lower ? ((r >= c) ? V[c + r * NB] / rdiag[r] : 0.f) : V[r + c * NB];
    out[i] = v;
  }
}

// ---------------------------------------------------------------------------------
// GEMM (SIMT, register-tiled 128x128x8, 8x8 per thread)
// ---------------------------------------------------------------------------------
template <typename T, int MODE>
__global__ void __launch_bounds__(256) gemm_simt_kernel(int M, int N, int K, const T* __restrict__ A, int64_t lda,
                                                        const T* __restrict__ B, int64_t ldb, T* C, int64_t ldc) {
  constexpr int BM = 128, BN = 128, BK = 8;
  __shared__ T As[2][BK][BM];
  __shared__ T Bs[2][BK][BN];
  const int tid = threadIdx.x;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int tx = tid % 16, ty = tid / 16;  // 16 x 16 threads, 8x8 each
  T acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = T(0);
  // loaders: A tile 128 x 8 (4 per thread), B tile 8 x 128 (4 per thread)
  T ra[4], rb[4];
  auto load = [&](int k0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int idx = tid + 256 * i;
      const int am = idx % BM, ak = idx / BM;
      const int gm = m0 + am, gk = k0 + ak;
      ra[i] = (gm < M && gk < K) ? A[gm + (int64_t)gk * lda] : T(0);
      const int bk = idx % BK, bn = idx / BK;
      const int gk2 = k0 + bk, gn = n0 + bn;
      rb[i] = (gk2 < K && gn < N) ? B[gk2 + (int64_t)gn * ldb] : T(0);
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int idx = tid + 256 * i;
      As[buf][idx / BM][idx % BM] = ra[i];
      Bs[buf][idx % BK][idx / BK] = rb[i];
    }
  };
  load(0);
  store(0);
  __syncthreads();
  int buf = 0;
  for (int k0 = 0; k0 < K; k0 += BK) {
    const bool more = k0 + BK < K;
    if (more) load(k0 + BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      T a[8], b[8];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        a[i] = As[buf][kk][ty * 4 + i];
        a[4 + i] = As[buf][kk][64 + ty * 4 + i];
        b[i] = Bs[buf][kk][tx * 4 + i];
        b[4 + i] = Bs[buf][kk][64 + tx * 4 + i];
      }
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    if (more) {
      store(buf ^ 1);
      __syncthreads();
      buf ^= 1;
    }
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int gm = m0 + ((i < 4) ? ty * 4 + i : 64 + ty * 4 + (i - 4));
    T old[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int gn = n0 + ((j < 4) ? tx * 4 + j : 64 + tx * 4 + (j - 4));
      old[j] = (MODE == 0 && gm < M && gn < N) ? C[gm + (int64_t)gn * ldc] : T(0);
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int gn = n0 + ((j < 4) ? tx * 4 + j : 64 + tx * 4 + (j - 4));
      if (gm < M && gn < N) C[gm + (int64_t)gn * ldc] = (MODE == 0) ? old[j] - acc[i][j] : acc[i][j];
    }
  }
}

int gemm_dmma(bem_ctx* c, int M, int N, int K, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
              int64_t ldc, int mode);
int gemm_bf16(bem_ctx* c, int M, int N, int K, const float* A, int64_t lda, const float* B, int64_t ldb, float* C,
              int64_t ldc, int mode, int split);
bool gemm_tc_ok(const void* A, int64_t lda, const void* B, int64_t ldb, int elem);
bool umma_supported(int K);
int umma_reserve(bem_ctx* c, int M, int N, int K);
int gemm_umma_bf16(bem_ctx* c, int M, int N, int K, const float* A, int64_t lda, const float* B, int64_t ldb,
                   float* C, int64_t ldc, int nprod, bool store, int kmode);

// the FP32 trailing updates of this context run on tcgen05 (umma.cu)
static bool uses_umma(const bem_ctx* c) { return c->f32_gemm == 4 || c->f32_gemm == 2; }
// C as the tcgen05 epilogue's bulk tensor copies need it: 16-byte aligned base and column stride
static bool umma_c_ok(const void* C, int64_t ldc) {
  return (reinterpret_cast<uintptr_t>(C) & 15) == 0 && (ldc * 4) % 16 == 0;
}

template <typename T>
static int gemm_simt(bem_ctx* c, int M, int N, int K, const T* A, int64_t lda, const T* B, int64_t ldb, T* C,
                     int64_t ldc, int mode) {
  dim3 grid((N + 127) / 128, (M + 127) / 128);
  if (mode == 0)
    gemm_simt_kernel<T, 0><<<grid, 256, 0, c->stream>>>(M, N, K, A, lda, B, ldb, C, ldc);
  else
    gemm_simt_kernel<T, 1><<<grid, 256, 0, c->stream>>>(M, N, K, A, lda, B, ldb, C, ldc);
  BEM_LAUNCH_CHECK(c);
  return BEM_OK;
}

// FP64: DMMA tensor path; FP32: per-context choice (c->f32_gemm) of the BF16 tensor path
// with 3 (FP32-grade) or 1 (plain BF16) terms, or SIMT FP32.  With tcgen05 (f32_gemm 4
// or 2), GEMMs with K a multiple of 64, M >= 128 and N >= 256 run there with 3 terms
// (mode 0, C -= A B, and mode 1, C = A B); the trailing updates take trailing_gemm,
// which gives f32_gemm 2 its one-term update.  Misaligned operands take the SIMT kernel.
template <typename T>
int gemm(bem_ctx* c, int M, int N, int K, const T* A, int64_t lda, const T* B, int64_t ldb, T* C, int64_t ldc,
         int mode) {
  if (M <= 0 || N <= 0 || K <= 0) return BEM_OK;
  if ((M + 127) / 128 > 65535) return bem_fail(c, BEM_ERR_ARG, "gemm: M too large");
  const bool tc = gemm_tc_ok(A, lda, B, ldb, (int)sizeof(T));
  if (sizeof(T) == 8) {
    if (tc && c->f64_gemm == 1)
      return gemm_dmma(c, M, N, K, (const double*)A, lda, (const double*)B, ldb, (double*)C, ldc, mode);
  } else {
    if (uses_umma(c) && umma_supported(K) && M >= 128 && N >= 256 && umma_c_ok(C, ldc))
      return gemm_umma_bf16(c, M, N, K, (const float*)A, lda, (const float*)B, ldb, (float*)C, ldc, 3, mode == 1,
                            0);
    if (tc && (c->f32_gemm >= 1 && c->f32_gemm <= 4))
      return gemm_bf16(c, M, N, K, (const float*)A, lda, (const float*)B, ldb, (float*)C, ldc, mode,
                       c->f32_gemm == 1 ? 1 : 3);
  }
  return gemm_simt<T>(c, M, N, K, A, lda, B, ldb, C, ldc, mode);
}

// The trailing update C -= A B of an FP32 factorisation: one BF16 product on tcgen05 in
// the BF16 mode (f32_gemm 2), three otherwise.
static int trailing_gemm(bem_ctx* c, int M, int N, int K, const float* A, int64_t lda, const float* B, int64_t ldb,
                         float* C, int64_t ldc) {
  if (c->f32_gemm == 2 && umma_supported(K) && M >= 128 && N >= 256 && umma_c_ok(C, ldc))
    return gemm_umma_bf16(c, M, N, K, A, lda, B, ldb, C, ldc, 1, false, 0);
  return gemm<float>(c, M, N, K, A, lda, B, ldb, C, ldc, 0);
}

// Whether gemm_tri runs on tcgen05, whose kernel reads only the BF16 copies of its
// operands that the split kernels made before it: C may then be one of the operands.
static bool gemm_tri_in_place(const bem_ctx* c, int M, int N, int K, const float* C, int64_t ldc) {
  return uses_umma(c) && umma_supported(K) && M >= 128 && N >= 256 && umma_c_ok(C, ldc);
}

// C = A B with a triangular factor (kmode 1: A lower, kmode 2: B upper): on tcgen05 each
// tile skips the K chunks of the factor's zero part.
static int gemm_tri(bem_ctx* c, int M, int N, int K, const float* A, int64_t lda, const float* B, int64_t ldb,
                    float* C, int64_t ldc, int kmode) {
  if (gemm_tri_in_place(c, M, N, K, C, ldc)) return gemm_umma_bf16(c, M, N, K, A, lda, B, ldb, C, ldc, 3, true, kmode);
  return gemm<float>(c, M, N, K, A, lda, B, ldb, C, ldc, 1);
}

template int gemm<double>(bem_ctx*, int, int, int, const double*, int64_t, const double*, int64_t, double*,
                          int64_t, int);
template int gemm<float>(bem_ctx*, int, int, int, const float*, int64_t, const float*, int64_t, float*,
                         int64_t, int);

// ---------------------------------------------------------------------------------
// factorisation driver
// ---------------------------------------------------------------------------------
namespace {

// The barrier counter grows monotonically over a factorisation (zeroed once with the
// status words); each launch waits for its own arrivals on top of bar_base.
template <typename T>
int panel_launch(bem_ctx* c, const LUWorkspace& ws, T* S, int64_t lda, int n, int r0, int w, int* piv,
                 unsigned& bar_base) {
  static DeviceOnce checked;  // per instantiation (T) and device
  const int cols = n - r0;
  static const int cap = [] {  // BEM_PANEL_CTAS: at most this many CTAs per panel launch
    const char* e = getenv("BEM_PANEL_CTAS");
    return e ? std::max(1, atoi(e)) : INT_MAX;
  }();
  int G = std::min(std::min(std::min(c->sm_count, ws.gmax), cap), std::max(1, (cols + 63) / 64));
  int chunk = (cols + G - 1) / G;
  size_t smem = (size_t)chunk * kPitch * sizeof(T);
  if (smem > kPanelSmemMax) return bem_fail(c, BEM_ERR_ARG, "panel slice exceeds shared memory (matrix too large)");
  if (checked.pending()) {
    // one CTA per SM at the largest slice guarantees co-residency of every launch
    BEM_CUDA(c, cudaFuncSetAttribute(panel_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPanelSmemMax));
    int occ = 0;
    BEM_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, panel_kernel<T>, panel_threads<T>(), kPanelSmemMax));
    if (occ < 1) return bem_fail(c, BEM_ERR_CUDA, "panel kernel cannot be resident");
    checked.mark();
  }
  double* cv = ws.cand_val;
  int* ci = ws.cand_idx;
  T* cc = reinterpret_cast<T*>(ws.cand_col);
  T* dc = reinterpret_cast<T*>(ws.diag_col);
  unsigned* bar = ws.barrier;
  int* st = ws.status;
  unsigned bb = bar_base;
  unsigned long long wns = c->wait_ns;
  void* args[] = {&S, &lda, &n, &r0, &w, &chunk, &piv, &cv, &ci, &cc, &dc, &bar, &bb, &st, &wns};
  BEM_CUDA(c, cudaLaunchCooperativeKernel((void*)panel_kernel<T>, dim3(G), dim3(panel_threads<T>()), args, smem,
                                          c->stream));
  ++c->launches;
  bar_base += (unsigned)w * (unsigned)G;
  return BEM_OK;
}

// Window-pivoted sub-panel: one plain launch, one thread per column right of the window.
template <typename T>
int window_panel_launch(bem_ctx* c, const LUWorkspace& ws, T* S, int64_t lda, int n, int r0, int w, int* piv) {
  const int64_t cols = (int64_t)n - r0 - w;
  const unsigned G = (unsigned)std::max<int64_t>(1, (cols + 255) / 256);
  window_panel_kernel<T><<<G, 256, 0, c->stream>>>(S, lda, n, r0, w, piv, reinterpret_cast<T*>(ws.cand_col),
                                                   ws.status);
  BEM_LAUNCH_CHECK(c);
  return BEM_OK;
}

}  // namespace

// Optional phase timing of the factorisation (environment BEM_LU_PROFILE=1): CUDA
// events around every phase, summed per phase and printed to stderr at the end.
struct LUProfile {
  bool on = false;
  bem_ctx* c = nullptr;
  using Ev = LUGraph::Ev;  // phase, then indices a, b into c->ev_pool, then flops, bytes
  std::vector<Ev> ev;
  size_t used = 0;
  int cur = -1, start = -1;
  // events come from the context's pool (created once, reused by later factorisations)
  int take(cudaStream_t s) {
    if (used == c->ev_pool.size()) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return -1;
      c->ev_pool.push_back(e);
    }
    // External: inside a stream capture the record becomes a graph node (a plain
    // record there is only a capture dependency and cannot be timed)
    if (cudaEventRecordWithFlags(c->ev_pool[used], s, cudaEventRecordExternal) != cudaSuccess) return -1;
    return (int)used++;
  }
  // trailing-only mode times the trailing update of every 16th panel (events between
  // consecutive launches disturb the factorisation's timing; a sparse sample does not)
  bool trailing_only = false;
  int panel = 0;
  bool skip(int phase) const { return !on || (trailing_only && (phase != 4 || panel % 16 != 0)); }
  void begin(int phase, cudaStream_t s) {
    cur = phase;
    if (skip(phase)) return;
    start = take(s);
  }
  void end(cudaStream_t s, double flops = 0.0, double bytes = 0.0) {
    if (skip(cur)) return;
    const int b = take(s);
    if (start >= 0 && b >= 0) ev.push_back({cur, start, b, flops, bytes});
  }
  void report(bem_ctx* c, int n) {
    if (!on) return;
    double t[5] = {0, 0, 0, 0, 0}, fl = 0, by = 0;
    long long cnt = 0;
    for (auto& e : ev) {
      float ms = 0.f;
      // a failed query costs the sample only, never a later launch check
      if (cudaEventSynchronize(c->ev_pool[e.b]) != cudaSuccess ||
          cudaEventElapsedTime(&ms, c->ev_pool[e.a], c->ev_pool[e.b]) != cudaSuccess) {
        cudaGetLastError();
        ms = 0.f;
      }
      t[e.phase] += ms;
      if (e.phase == 4) {
        ++cnt;
        fl += e.flops;
        by += e.bytes;
      }
    }
    if (c->prof_timing) {
      c->prof.lu_panel_ms += t[0];
      c->prof.lu_swap_ms += t[1];
      c->prof.lu_panel_update_ms += t[2];
      c->prof.lu_trsm_ms += t[3];
      c->prof.lu_trailing_ms += t[4];
      c->prof.lu_trailing_launches += cnt;
      c->prof.lu_trailing_flops += fl;
      c->prof.lu_trailing_bytes += by;
    }
    if (getenv("BEM_LU_PROFILE"))
      fprintf(stderr, "[lu n=%d] panel %.1f ms  swaps %.1f ms  panel-update %.1f ms  trsm %.1f ms  trailing-gemm %.1f ms\n",
              n, t[0], t[1], t[2], t[3], t[4]);
  }
};

static size_t up256(size_t b) { return (b + 255) / 256 * 256; }

// blocks of the TRSM-inverse region: FP32 factors keep the 2 x 4 inverses of a
// window-pivoted 512-wide panel (panel_inv_f32_kernel), FP64 one block
static size_t inv_blocks(int elem, int nb) { return elem == 4 ? 2 * (size_t)((nb + kInvBlock - 1) / kInvBlock) : 1; }

static size_t finv_count(int elem, int nb) {
  return elem == 4 ? 2 * (size_t)nb * nb + 2 * (size_t)nb * kInvBlock : 0;
}

size_t lu_workspace_bytes(int n, int nb, int gmax, int elem) {
  const size_t ldy = ((size_t)n + 31) / 32 * 32;
  return up256(2 * (size_t)gmax * sizeof(double)) + up256(2 * (size_t)gmax * sizeof(int)) +
         up256(2 * (size_t)gmax * kPanelW * elem) + up256(2 * (size_t)kPanelW * elem) + up256(16) +
         up256(inv_blocks(elem, nb) * kInvBlock * kInvBlock * elem) + up256(finv_count(elem, nb) * elem) +
         up256(ldy * nb * elem);
}

LUWorkspace lu_workspace_carve(void* base, int n, int nb, int gmax, int elem) {
  unsigned char* p = static_cast<unsigned char*>(base);
  LUWorkspace w{};
  w.gmax = gmax;
  w.ldy = ((int64_t)n + 31) / 32 * 32;
  w.cand_val = reinterpret_cast<double*>(p);
  p += up256(2 * (size_t)gmax * sizeof(double));
  w.cand_idx = reinterpret_cast<int*>(p);
  p += up256(2 * (size_t)gmax * sizeof(int));
  w.cand_col = p;
  p += up256(2 * (size_t)gmax * kPanelW * elem);
  w.diag_col = p;
  p += up256(2 * (size_t)kPanelW * elem);
  w.barrier = reinterpret_cast<unsigned*>(p);
  w.status = reinterpret_cast<int*>(p + 8);
  p += up256(16);
  w.inv = p;
  p += up256(inv_blocks(elem, nb) * kInvBlock * kInvBlock * elem);
  w.finv = finv_count(elem, nb) ? p : nullptr;
  p += up256(finv_count(elem, nb) * elem);
  w.ybuf = p;
  return w;
}

size_t lu_solve_work_count(int n) { return ((size_t)n + 127) / 128 * 256 + 256; }

template <typename T>
int lu_prepare_inverses(bem_ctx* c, const T* S, int64_t lda, int n);

// x = P v with P = tau_0 tau_1 ... tau_{n-1} (tau_i swaps i and piv[i]) as a gather
// x[i] = v[perm[i]]; composed on the host once per factorisation
static int make_perm(bem_ctx* c, const int* d_piv, int n, int* d_perm) {
  std::vector<int> p(n), a(n);
  BEM_CUDA(c, cudaMemcpyAsync(p.data(), d_piv, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  for (int i = 0; i < n; ++i) a[i] = i;
  for (int i = n - 1; i >= 0; --i) std::swap(a[i], a[p[i]]);
  BEM_CUDA(c, cudaMemcpyAsync(d_perm, a.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  return BEM_OK;
}

static LUProfile make_profile(bem_ctx* c) {
  LUProfile prof;
  prof.c = c;
  prof.on = getenv("BEM_LU_PROFILE") != nullptr || c->prof_timing != BEM_PROF_COUNT;
  prof.trailing_only = c->prof_timing == BEM_PROF_TRAILING && getenv("BEM_LU_PROFILE") == nullptr;
  return prof;
}

// The factorisation's launches, in stream order with no host synchronisation (so that
// they can be captured as a graph).
template <typename T>
static int lu_factor_enqueue(bem_ctx* c, T* S, int64_t lda, int n, int* piv, int nb, const LUWorkspace& ws,
                             LUProfile& prof) {
  // barrier counter (offset 0) and status words (offset 8) of the workspace's sync slot
  BEM_CUDA(c, cudaMemsetAsync(ws.barrier, 0, 16, c->stream));
  unsigned bar_base = 0;
  if (sizeof(T) == 4 && uses_umma(c)) BEM_CUDA(c, cudaMemsetAsync(c->umma_err.p, 0, sizeof(int), c->stream));
  T* V = reinterpret_cast<T*>(ws.inv);
  T* Y = reinterpret_cast<T*>(ws.ybuf);
  const int64_t ldy = ws.ldy;
  // window pivoting (pivot search within each sub-panel's diagonal block) or partial
  // pivoting (over every remaining row of T)
  const bool window = c->lu_window;
  const size_t inv_smem = (size_t)kInvBlock * kInvBlock * sizeof(T);
  cudaFuncSetAttribute(inv_unit_upper_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)inv_smem);
  cudaFuncSetAttribute(inv_unit_upper_f32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(2 * kInvBlock * kInvBlock * sizeof(float)));
  cudaFuncSetAttribute(panel_inv_f32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(2 * kInvBlock * kInvBlock * sizeof(float)));
  int rc;
  // window-pivoted FP32 panels: the diagonal block in one cooperative launch
  // (panel_coop_kernel; BEM_PANEL_COOP=0 selects a launch pair per sub-panel)
  static const bool coop_env = [] {
    const char* e = getenv("BEM_PANEL_COOP");
    return !(e && e[0] == '0');
  }();
  const int coop_g = std::min(kCoopMaxCtas, c->sm_count);
  for (int j0 = 0; j0 < n; j0 += nb) {
    const int jb = std::min(nb, n - j0);
    prof.panel = j0 / nb;
    // window pivoting leaves the sub-panels' columns right of the panel (T rows below
    // its diagonal block) to one blocked TRSM per panel; partial pivoting needs them
    // eliminated sub-panel by sub-panel to search them for pivots
    const int cend = (window && sizeof(T) == 4) ? j0 + jb : n;
    const bool coop = coop_env && cend < n && sizeof(T) == 4 && jb % kPanelW == 0 && lda % 4 == 0 &&
                      (reinterpret_cast<uintptr_t>(S) & 15) == 0 && coop_g >= 1;
    if (coop) {
      prof.begin(0, c->stream);
      float* Sf = reinterpret_cast<float*>(S);
      int a_j0 = j0, a_t0 = j0 + jb;
      unsigned bb = bar_base;
      unsigned long long wns = c->wait_ns;
      int* st = ws.status;
      unsigned* bar = ws.barrier;
      void* args[] = {&Sf, const_cast<int64_t*>(&lda), &a_j0, &a_t0, &piv, &bar, &bb, &st, &wns};
      BEM_CUDA(c, cudaLaunchCooperativeKernel((void*)panel_coop_kernel, dim3(coop_g), dim3(kCoopThreads), args, 0,
                                              c->stream));
      ++c->launches;
      bar_base += 2u * (unsigned)(jb / kPanelW) * (unsigned)coop_g;
      prof.end(c->stream);
    }
    for (int r0 = j0; r0 < j0 + jb && !coop; r0 += kPanelW) {
      const int w = std::min(kPanelW, j0 + jb - r0);
      prof.begin(0, c->stream);
      if (cend < n && w == kPanelW && jb <= kBlockThreads && sizeof(T) == 4 && lda % 4 == 0 &&
          (reinterpret_cast<uintptr_t>(S) & 15) == 0) {
        // window-pivoted FP32 panel: the sub-panel's step in one CTA, then its GEMM
        window_block_kernel<<<1, kBlockThreads, 0, c->stream>>>(reinterpret_cast<float*>(S), lda, j0, j0 + jb, r0, piv,
                                                                 ws.status);
        BEM_LAUNCH_CHECK(c);
        prof.end(c->stream);
        const int q0 = r0 + w, q1 = j0 + jb;
        prof.begin(2, c->stream);
        if (q1 > q0 && (rc = gemm<T>(c, q1 - q0, cend - q0, w, S + q0 + (int64_t)r0 * lda, lda,
                                     S + r0 + (int64_t)q0 * lda, lda, S + q0 + (int64_t)q0 * lda, lda, 0)))
          return rc;
        prof.end(c->stream);
        continue;
      }
      if (window) {
        if ((rc = window_panel_launch<T>(c, ws, S, lda, cend, r0, w, piv))) return rc;
      } else if ((rc = panel_launch<T>(c, ws, S, lda, n, r0, w, piv, bar_base))) {
        return rc;
      }
      prof.end(c->stream);
      prof.begin(1, c->stream);
      // swaps on every other row of S: the earlier panels' multipliers (rows [0, r0),
      // so that the factors end up as T = P L U) and the trailing rows; with window
      // pivoting this launch also stores the factored window block
      // (window-pivoted FP32 panels: the panel's own rows here, the other rows once
      // per panel by permute_panel_kernel)
      const bool blk = cend < n;
      const int a0 = blk ? j0 : 0, a1 = r0, b0 = r0 + w, b1 = blk ? j0 + jb : n;
      const int64_t rows = (int64_t)(a1 - a0) + (b1 - b0);
      if (rows > 0 || window) {
        swap_rows_kernel<T><<<(unsigned)std::max<int64_t>(1, (rows + 255) / 256), 256, 0, c->stream>>>(
            S, lda, piv, r0, w, a0, a1, b0, b1, window ? reinterpret_cast<const T*>(ws.cand_col) : nullptr);
        BEM_LAUNCH_CHECK(c);
      }
      prof.end(c->stream);
      // update the panel rows below the sub-panel
      const int q0 = r0 + w, q1 = j0 + jb;
      prof.begin(2, c->stream);
      if (q1 > q0) {
        trsm_small_kernel<T><<<(q1 - q0 + 127) / 128, 128, 0, c->stream>>>(S, lda, r0, w, q0, q1);
        BEM_LAUNCH_CHECK(c);
        if ((rc = gemm<T>(c, q1 - q0, cend - q0, w, S + q0 + (int64_t)r0 * lda, lda, S + r0 + (int64_t)q0 * lda,
                          lda, S + q0 + (int64_t)q0 * lda, lda, 0)))
          return rc;
      }
      prof.end(c->stream);
    }
    const int t0 = j0 + jb;
    const bool blocked = cend < n;  // window-pivoted FP32 panel: blocked TRSMs below
    if (blocked) {
      prof.begin(1, c->stream);
      const int64_t rows = (int64_t)j0 + (n - t0);
      constexpr int R = 64 / (int)sizeof(T);
      permute_panel_kernel<T><<<(unsigned)((rows + R - 1) / R), 256, 0, c->stream>>>(S, lda, piv, j0, jb, 0, j0, t0, n);
      BEM_LAUNCH_CHECK(c);
      prof.end(c->stream);
    }
    if (t0 < n) {
      const int m = n - t0;
      const int nib = (nb + kInvBlock - 1) / kInvBlock;
      T* Vu = V;                                          // [nib][128 x 128]
      T* Wl = V + (size_t)(kInvBlock * kInvBlock) * nib;  // [nib][128 x 128]
      // blocked panels (FP32): jb x jb inverses of the unit upper and the lower triangle,
      // and a jb x 128 scratch for each
      T* XU = blocked ? reinterpret_cast<T*>(ws.finv) : nullptr;
      T* XL = blocked ? XU + (size_t)jb * jb : nullptr;
      T* Tu = blocked ? XL + (size_t)jb * jb : nullptr;
      T* Tl = blocked ? Tu + (size_t)jb * kInvBlock : nullptr;
      if (blocked) {
        // the panel's diagonal-block inverses: the 128 x 128 ones, then the two full
        // triangles' block column by block column (U unit upper, W lower, both of the
        // panel's diagonal block of S):
        //   XU_{<b,b} = -(XU_{<b,<b} U_{<b,b}) inv(U_bb),  XL_{b,<b} = -inv(W_bb) (W_{b,<b} XL_{<b,<b});
        // then the rest of the sub-panels' columns in one product, B = S(j0..t0, t0..n)
        // := W^{-1} B, through the TRSM buffer
        prof.begin(2, c->stream);
        const int nblk = (jb + kInvBlock - 1) / kInvBlock;
        panel_inv_f32_kernel<<<dim3(nblk, 2), kInvThreads, 2 * kInvBlock * kInvBlock * sizeof(float), c->stream>>>(
            reinterpret_cast<const float*>(S + j0 + (int64_t)j0 * lda), lda, jb, reinterpret_cast<float*>(Vu),
            reinterpret_cast<float*>(Wl));
        BEM_LAUNCH_CHECK(c);
        BEM_CUDA(c, cudaMemsetAsync(XU, 0, 2 * (size_t)jb * jb * sizeof(T), c->stream));
        // the two inverses are independent: XU's chain (no tcgen05 GEMM, whose operand
        // buffer is the context's) runs on the auxiliary stream, joined before the
        // block-row TRSM that needs it; XL's chain and the L21 product run here
        cudaStream_t main_stream = c->stream;
        const bool fork = c->aux_stream != nullptr;
        if (fork) {
          BEM_CUDA(c, cudaEventRecord(c->ev_fork, main_stream));
          BEM_CUDA(c, cudaStreamWaitEvent(c->aux_stream, c->ev_fork, 0));
          c->stream = c->aux_stream;
        }
        rc = 0;
        for (int b0 = 0; b0 < jb && rc == 0; b0 += kInvBlock) {
          const int bb = std::min(kInvBlock, jb - b0);
          const T* Vb = Vu + (size_t)(b0 / kInvBlock) * kInvBlock * kInvBlock;
          if (cudaMemcpy2DAsync(XU + b0 + (size_t)b0 * jb, jb * sizeof(T), Vb, kInvBlock * sizeof(T), bb * sizeof(T),
                                bb, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess) {
            rc = bem_fail(c, BEM_ERR_CUDA, "inverse assembly copy failed");
          } else if (b0 > 0) {
            rc = gemm<T>(c, b0, bb, b0, XU, jb, S + j0 + (int64_t)(j0 + b0) * lda, lda, Tu, jb, 1);
            if (rc == 0) rc = gemm<T>(c, b0, bb, bb, Tu, jb, Vb, kInvBlock, XU + (size_t)b0 * jb, jb, 0);
          }
        }
        if (fork) {
          if (rc == 0 && cudaEventRecord(c->ev_join, c->aux_stream) != cudaSuccess)
            rc = bem_fail(c, BEM_ERR_CUDA, "event record failed");
          c->stream = main_stream;
        }
        if (rc) return rc;
        for (int b0 = 0; b0 < jb; b0 += kInvBlock) {
          const int bb = std::min(kInvBlock, jb - b0);
          const T* Wb = Wl + (size_t)(b0 / kInvBlock) * kInvBlock * kInvBlock;
          BEM_CUDA(c, cudaMemcpy2DAsync(XL + b0 + (size_t)b0 * jb, jb * sizeof(T), Wb, kInvBlock * sizeof(T),
                                        bb * sizeof(T), bb, cudaMemcpyDeviceToDevice, c->stream));
          if (b0 == 0) continue;
          if ((rc = gemm<T>(c, bb, b0, b0, S + (j0 + b0) + (int64_t)j0 * lda, lda, XL, jb, Tl, kInvBlock, 1)) ||
              (rc = gemm<T>(c, bb, b0, bb, Wb, kInvBlock, Tl, kInvBlock, XL + b0, jb, 0)))
            return rc;
        }
        float* L21 = reinterpret_cast<float*>(S + j0 + (int64_t)t0 * lda);
        if (gemm_tri_in_place(c, jb, m, jb, L21, lda)) {  // written over its own operand
          if ((rc = gemm_tri(c, jb, m, jb, reinterpret_cast<const float*>(XL), jb, L21, lda, L21, lda, 1)))
            return rc;
        } else {
          if ((rc = gemm_tri(c, jb, m, jb, reinterpret_cast<const float*>(XL), jb, L21, lda,
                             reinterpret_cast<float*>(Y), jb, 1)))
            return rc;
          BEM_CUDA(c, cudaMemcpy2DAsync(L21, lda * sizeof(T), Y, jb * sizeof(T), jb * sizeof(T), m,
                                        cudaMemcpyDeviceToDevice, c->stream));
        }
        prof.end(c->stream);
      }
      prof.begin(3, c->stream);
      // the block row's solution Y = X U^{-1}: in a buffer (ldy), copied into S below, or
      // on tcgen05 written over X in S itself
      const T* Yr = Y;
      int64_t ldyr = ldy;
      if (blocked) {
        if (c->aux_stream) BEM_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_join, 0));
        // TRSM of the block row in one product, Y = X U^{-1}
        float* X = reinterpret_cast<float*>(S + t0 + (int64_t)j0 * lda);
        const bool in_place = gemm_tri_in_place(c, m, jb, jb, X, lda);
        if ((rc = gemm_tri(c, m, jb, jb, X, lda, reinterpret_cast<const float*>(XU), jb,
                           in_place ? X : reinterpret_cast<float*>(Y), in_place ? lda : ldy, 2)))
          return rc;
        if (in_place) {
          Yr = S + t0 + (int64_t)j0 * lda;
          ldyr = lda;
        }
      } else {
      // TRSM of the block row, Y = X U^{-1} with U the unit upper triangle of the panel's
      // diagonal block, in 128-wide column blocks: X_b -= Y_{<b} U_{<b,b}, Y_b = X_b inv(U_bb)
      for (int b0 = 0; b0 < jb; b0 += kInvBlock) {
        const int bb = std::min(kInvBlock, jb - b0);
        T* Xb = S + t0 + (int64_t)(j0 + b0) * lda;
        if (b0 > 0 &&
            (rc = gemm<T>(c, m, bb, b0, Y, ldy, S + j0 + (int64_t)(j0 + b0) * lda, lda, Xb, lda, 0)))
          return rc;
        if (sizeof(T) == 4)
          inv_unit_upper_f32_kernel<<<1, kInvThreads, 2 * kInvBlock * kInvBlock * sizeof(float), c->stream>>>(
              reinterpret_cast<const float*>(S + (j0 + b0) + (int64_t)(j0 + b0) * lda), lda, bb,
              reinterpret_cast<float*>(V), kInvBlock);
        else
          inv_unit_upper_kernel<T><<<1, 256, inv_smem, c->stream>>>(
              S + (j0 + b0) + (int64_t)(j0 + b0) * lda, lda, bb, V, kInvBlock);
        BEM_LAUNCH_CHECK(c);
        if ((rc = gemm<T>(c, m, bb, bb, Xb, lda, V, kInvBlock, Y + (int64_t)b0 * ldy, ldy, 1))) return rc;
      }
      }
      if (Yr == Y)
        BEM_CUDA(c, cudaMemcpy2DAsync(S + t0 + (int64_t)j0 * lda, lda * sizeof(T), Y, ldy * sizeof(T), m * sizeof(T),
                                      jb, cudaMemcpyDeviceToDevice, c->stream));
      prof.end(c->stream);
      prof.begin(4, c->stream);
      if constexpr (sizeof(T) == 4) {
        if ((rc = trailing_gemm(c, m, m, jb, Yr, ldyr, S + j0 + (int64_t)t0 * lda, lda, S + t0 + (int64_t)t0 * lda,
                                lda)))
          return rc;
      } else if ((rc = gemm<T>(c, m, m, jb, Yr, ldyr, S + j0 + (int64_t)t0 * lda, lda, S + t0 + (int64_t)t0 * lda,
                               lda, 0))) {
        return rc;
      }
      prof.end(c->stream, 2.0 * m * (double)m * jb, (2.0 * m * (double)m + 2.0 * m * (double)jb) * sizeof(T));
    }
  }
  return BEM_OK;
}

// After the launches: the phase profile, the status words and the gather form of P.
template <typename T>
static int lu_factor_finish(bem_ctx* c, int n, int* piv, int* perm, int* info, const LUWorkspace& ws,
                            LUProfile& prof) {
  prof.report(c, n);
  int st[2];
  BEM_CUDA(c, cudaMemcpyAsync(st, ws.status, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  if (st[0] != 0) return bem_fail(c, st[0], "panel grid barrier timed out");
  if (sizeof(T) == 4 && uses_umma(c)) {
    int ue = 0;
    BEM_CUDA(c, cudaMemcpy(&ue, c->umma_err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (ue != 0) return bem_fail(c, ue, "tcgen05 trailing update: an mbarrier wait timed out");
  }
  *info = st[1];
  if (*info == 0 && perm) return make_perm(c, piv, n, perm);
  return BEM_OK;
}

template <typename T>
int lu_factor_ws(bem_ctx* c, T* S, int64_t lda, int n, int* piv, int* perm, int nb, int* info,
                 const LUWorkspace& ws) {
  *info = 0;
  c->dinv_src = nullptr;  // the diagonal-block inverses belong to earlier factors
  if (sizeof(T) == 4 && uses_umma(c) && c->umma_err.count < 1) BEM_CUDA(c, c->umma_err.alloc(1));
  LUProfile prof = make_profile(c);
  const int rc = lu_factor_enqueue<T>(c, S, lda, n, piv, nb, ws, prof);
  if (rc) return rc;
  return lu_factor_finish<T>(c, n, piv, perm, info, ws, prof);
}

// The context's factorisation: workspace kept in the context, the launch sequence
// captured once per (factors, order, panel width, workspace, GEMM buffers, profile mode)
// and replayed, then the diagonal-block inverses of the solve.  Capture that the
// runtime refuses (or BEM_LU_GRAPH=0) leaves plain launches.
template <typename T>
int lu_factor(bem_ctx* c, T* S, int64_t lda, int n, int* piv, int* perm, int nb, int* info) {
  *info = 0;
  c->dinv_src = nullptr;
  const int ti = sizeof(T) == 8 ? 1 : 0;
  const int gmax = c->sm_count;
  const size_t bytes = lu_workspace_bytes(n, nb, gmax, sizeof(T));
  if (c->lu_scratch[ti].count < bytes) {
    c->lu_scratch[ti].release();
    BEM_CUDA(c, c->lu_scratch[ti].alloc(bytes));
  }
  const LUWorkspace ws = lu_workspace_carve(c->lu_scratch[ti].p, n, nb, gmax, sizeof(T));
  if (sizeof(T) == 4 && uses_umma(c)) {
    int rc0;
    // the largest operand pair: the trailing update's (M + N = 2 (n - nb)) or a blocked
    // TRSM's (M + N <= n)
    if (n > nb && (rc0 = umma_reserve(c, std::max(n, 2 * (n - nb)), 0, nb))) return rc0;
    if (c->umma_err.count < 1) BEM_CUDA(c, c->umma_err.alloc(1));
  }
  if (const char* e = getenv("BEM_LU_GRAPH"))
    if (atoi(e) == 0) c->lu_graph_off = true;
  LUProfile prof = make_profile(c);
  auto make_key = [&]() {
    return std::vector<long long>{(long long)(uintptr_t)S,  lda, n, nb, (long long)(uintptr_t)piv,
                                  (long long)(uintptr_t)ws.cand_val, (long long)(uintptr_t)c->umma_buf.p,
                                  (long long)c->umma_buf.count, (long long)(uintptr_t)c->umma_err.p,
                                  c->f32_gemm, c->f64_gemm, prof.on, prof.trailing_only, c->sm_count,
                                  c->lu_window ? 1 : 0};
  };
  int rc = BEM_OK;
  if (c->lu_graph_off) {
    rc = lu_factor_enqueue<T>(c, S, lda, n, piv, nb, ws, prof);
  } else {
    const std::vector<long long> key = make_key();
    LUGraph* hit = nullptr;
    for (auto& g : c->lu_graph[ti])
      if (g.exec && g.key == key) hit = &g;
    if (hit) {
      BEM_CUDA(c, cudaGraphLaunch(hit->exec, c->stream));
      c->launches += hit->launches;
      prof.ev = hit->ev;
    } else {
      LUGraph* slot = nullptr;
      for (auto& g : c->lu_graph[ti])
        if (!slot && !g.exec) slot = &g;
      if (!slot) {
        slot = &c->lu_graph[ti][c->lu_graph_next[ti]];
        c->lu_graph_next[ti] = (c->lu_graph_next[ti] + 1) % 4;
      }
      LUGraph& gr = *slot;
      gr.reset();
      const long long l0 = c->launches;
      cudaGraph_t g = nullptr;
      BEM_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
      rc = lu_factor_enqueue<T>(c, S, lda, n, piv, nb, ws, prof);
      cudaError_t e = cudaStreamEndCapture(c->stream, &g);
      cudaGraphExec_t ex = nullptr;
      if (rc == BEM_OK && e == cudaSuccess) e = cudaGraphInstantiate(&ex, g, 0);
      if (g) cudaGraphDestroy(g);
      if (rc == BEM_OK && e == cudaSuccess) {
        gr.exec = ex;
        gr.key = make_key();  // the trailing update may have grown its buffers while captured
        gr.ev = prof.ev;
        gr.launches = c->launches - l0;
        BEM_CUDA(c, cudaGraphLaunch(ex, c->stream));
      } else {
        // no capture: plain launches from now on
        if (getenv("BEM_LU_PROFILE"))
          fprintf(stderr, "[lu] graph capture unavailable (%s; %s): plain launches\n", cudaGetErrorString(e),
                  rc ? c->last_error.c_str() : "");
        if (ex) cudaGraphExecDestroy(ex);
        cudaGetLastError();
        c->lu_graph_off = true;
        c->launches = l0;
        prof = make_profile(c);
        rc = lu_factor_enqueue<T>(c, S, lda, n, piv, nb, ws, prof);
      }
    }
  }
  if (rc) return rc;
  rc = lu_factor_finish<T>(c, n, piv, perm, info, ws, prof);
  if (rc || *info != 0) return rc;
  return lu_prepare_inverses<T>(c, S, lda, n);
}

template int lu_factor<double>(bem_ctx*, double*, int64_t, int, int*, int*, int, int*);
template int lu_factor_ws<double>(bem_ctx*, double*, int64_t, int, int*, int*, int, int*, const LUWorkspace&);
template int lu_factor_ws<float>(bem_ctx*, float*, int64_t, int, int*, int*, int, int*, const LUWorkspace&);
template int lu_factor<float>(bem_ctx*, float*, int64_t, int, int*, int*, int, int*);

// ---------------------------------------------------------------------------------
// triangular solves
// ---------------------------------------------------------------------------------

// Triangular solves of the factors (see lu.cuh): forward with the lower triangle of S
// (non-unit diagonal), backward with the panels' multipliers and their interchanges.
// Diagonal blocks are solved by one warp from a shared-memory copy of the block: lane
// L holds unknowns L, L+32, L+64, L+96 in registers, and step c broadcasts the newest
// unknown from its owner lane (c % 32, register c / 32) with a shuffle.  The loops over
// the register slot and the owner lane are unrolled, so the owner and the slot are
// compile-time constants and each step's dependent chain is one shuffle, one multiply
// and one FMA; the shared-memory reads of the block's column do not depend on it.

// Solve the jb x jb lower (non-unit) block D (column-major, leading dimension
// kSolveBlock, zero outside jb x jb) for the unknowns w (in/out, shared); rdiag holds
// the reciprocals of the diagonal.
template <typename T>
__device__ void warp_lower_solve(const T* D, const double* rdiag, int jb, double* w) {
  const int lane = threadIdx.x & 31;
  double x[kSolveBlock / 32];
#pragma unroll
  for (int q = 0; q < kSolveBlock / 32; ++q) x[q] = (lane + 32 * q < jb) ? w[lane + 32 * q] : 0.0;
#pragma unroll
  for (int slot = 0; slot < kSolveBlock / 32; ++slot) {
#pragma unroll
    for (int o = 0; o < 32; ++o) {
      const int cidx = slot * 32 + o;
      if (cidx < jb) {
        const double xc = __shfl_sync(0xffffffffu, x[slot], o) * rdiag[cidx];
        if (lane == o) x[slot] = xc;
#pragma unroll
        for (int q = slot; q < kSolveBlock / 32; ++q) {
          const int r = lane + 32 * q;
          if (r > cidx) x[q] = fma(-(double)D[r + cidx * kSolveBlock], xc, x[q]);
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kSolveBlock / 32; ++q)
    if (lane + 32 * q < jb) w[lane + 32 * q] = x[q];
}

// the same for the strict upper (unit diagonal) block, from the last unknown down
template <typename T>
__device__ void warp_upper_unit_solve(const T* D, int jb, double* w) {
  const int lane = threadIdx.x & 31;
  double x[kSolveBlock / 32];
#pragma unroll
  for (int q = 0; q < kSolveBlock / 32; ++q) x[q] = (lane + 32 * q < jb) ? w[lane + 32 * q] : 0.0;
#pragma unroll
  for (int slot = kSolveBlock / 32 - 1; slot >= 0; --slot) {
#pragma unroll
    for (int o = 31; o >= 0; --o) {
      const int cidx = slot * 32 + o;
      if (cidx < jb) {
        const double xc = __shfl_sync(0xffffffffu, x[slot], o);
#pragma unroll
        for (int q = 0; q <= slot; ++q) {
          const int r = lane + 32 * q;
          if (r < cidx) x[q] = fma(-(double)D[r + cidx * kSolveBlock], xc, x[q]);
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kSolveBlock / 32; ++q)
    if (lane + 32 * q < jb) w[lane + 32 * q] = x[q];
}

// One sweep of blocked substitution over the 128-row blocks of S in one cooperative
// launch.  UPPER = false: forward with S's lower triangle (non-unit diagonal), blocks
// first to last; UPPER = true: backward with S's strict upper triangle (unit diagonal),
// blocks last to first.  Step s solves block k(s) and is owned by CTA s % G, which also
// owns the rows of that block: as soon as block k(s) is published (flags[s] = tag,
// release/acquire at gpu scope) every CTA subtracts S(its rows, block k(s)) * y_k(s)
// from its blocks' rows of b (128 x 128 tiles, contiguous column segments), the owner
// of step s+1 first, and that owner then solves and publishes block k(s+1) before it
// turns to its other blocks.  The dependent chain is one tile GEMV and one warp solve
// per block; the rest of the factor streams from HBM alongside.  Diagonal blocks are
// staged into shared memory one owned step ahead.  A wait that exceeds the context's
// wait limit (2 s by default) records BEM_ERR_TIMEOUT in *status and ends the CTA.
template <typename T, bool UPPER>
__global__ void __launch_bounds__(kSweepThreads, 1)
    sweep_kernel(const T* __restrict__ S, int64_t lda, int n, double* b, unsigned* flags, unsigned tag,
                 int* status, unsigned long long wait_ns) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* D = reinterpret_cast<T*>(smem_raw);  // [kSolveBlock][kSolveBlock] column-major
  __shared__ double ys[kSolveBlock];
  __shared__ double wn[kSolveBlock];
  __shared__ double rdiag[kSolveBlock];
  __shared__ double red[4][kSolveBlock];
  __shared__ int s_abort;
  const int t = threadIdx.x, G = gridDim.x, g = blockIdx.x;
  const int nblk = (n + kSolveBlock - 1) / kSolveBlock;
  auto blk0 = [&](int s) { return (UPPER ? nblk - 1 - s : s) * kSolveBlock; };
  auto stage_diag = [&](int s) {
    const int k0 = blk0(s), kb = min(kSolveBlock, n - k0);
    if (UPPER)
      stage_block<T>(D, kSolveBlock, S + k0 + (int64_t)k0 * lda, lda, kb, kb, kSolveBlock, kSolveBlock,
                     [](int r, int c) { return r < c; });
    else
      stage_block<T>(D, kSolveBlock, S + k0 + (int64_t)k0 * lda, lda, kb, kb, kSolveBlock, kSolveBlock,
                     [](int r, int c) { return r >= c; });
  };
  auto solve = [&](int s) {
    const int k0 = blk0(s), kb = min(kSolveBlock, n - k0);
    if (t < kb) wn[t] = b[k0 + t];
    if (!UPPER && t < kSolveBlock) rdiag[t] = (t < kb) ? 1.0 / (double)D[t + t * kSolveBlock] : 0.0;
    __syncthreads();
    if (t < 32) {
      if (UPPER)
        warp_upper_unit_solve<T>(D, kb, wn);
      else
        warp_lower_solve<T>(D, rdiag, kb, wn);
    }
    __syncthreads();
    if (t < kb) b[k0 + t] = wn[t];
    __syncthreads();
    if (t == 0) {
      __threadfence();
      st_release_u32(flags + s, tag);
    }
    if (s + G < nblk) stage_diag(s + G);  // D is free again: the next owned block
  };

  if (t == 0) s_abort = 0;
  if (g < nblk) stage_diag(g);
  __syncthreads();
  if (g == 0) solve(0);
  const int rl = t & (kSolveBlock - 1), q = t >> 7;
  for (int s = 0; s + 1 < nblk; ++s) {
    int s2 = s + 1 + ((g - (s + 1)) % G + G) % G;  // this CTA's first step after s
    if (s2 >= nblk) break;                          // no rows left to update
    if (t == 0 && s % G != g) {
      const unsigned long long t0 = globaltimer_ns();
      unsigned it = 0;
      while (ld_acquire_u32(flags + s) != tag) {
        if ((++it & 255u) == 0 && (globaltimer_ns() - t0 > wait_ns || *((volatile int*)status) != 0)) {
          atomicExch(status, BEM_ERR_TIMEOUT);
          s_abort = 1;
          break;
        }
      }
      __threadfence();
    }
    __syncthreads();
    if (s_abort) return;
    const int c0 = blk0(s), cb = min(kSolveBlock, n - c0);
    if (t < kSolveBlock) ys[t] = (t < cb) ? __ldcg(b + c0 + t) : 0.0;
    __syncthreads();
    for (; s2 < nblk; s2 += G) {
      const int r0 = blk0(s2), rb = min(kSolveBlock, n - r0);
      double acc = 0.0;
      // the row's current value travels with the tile's loads (only this thread writes it)
      const double bold = (q == 0 && rl < rb) ? b[r0 + rl] : 0.0;
      if (rl < rb) {
        const int cq = 32 * q;
        const T* p = S + (r0 + rl) + (int64_t)(c0 + cq) * lda;
        T a[32];
#pragma unroll
        for (int u = 0; u < 32; ++u) a[u] = (cq + u < cb) ? p[(int64_t)u * lda] : T(0);
#pragma unroll
        for (int u = 0; u < 32; ++u) acc = fma((double)a[u], ys[cq + u], acc);
      }
      red[q][rl] = acc;
      __syncthreads();
      if (q == 0 && rl < rb) b[r0 + rl] = bold - ((red[0][rl] + red[1][rl]) + (red[2][rl] + red[3][rl]));
      __syncthreads();
      if (s2 == s + 1) solve(s2);
    }
  }
}

__global__ void permute_kernel(int n, const int* __restrict__ perm, const double* __restrict__ v,
                               double* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = v[perm[i]];
}

// ---- block-inverse sweeps ------------------------------------------------------------
// The substitution of a 128 x 128 diagonal block is the sweeps' only sequential work.
// With the blocks' inverses computed once per factorisation it becomes one 128 x 128
// product, and the dependent chain per block is one publication, one tile product
// (its loads issued before the wait) and one inverse product.

constexpr int kInvPitch = kSolveBlock + 1;  // shared-memory pitch of the staged triangle

// Dinv[2 blk] = inverse of the lower triangle (diagonal included) of the diagonal block
// blk of S, Dinv[2 blk + 1] = inverse of its strict upper triangle plus the identity;
// each 128 x 128, column-major, FP64, zero outside the block's order.  Both are the
// inverse W of a unit upper triangle, blocked by 32 (the 32 x 32 diagonal blocks by
// back substitution in registers, then W_ij = -W_ii sum_{k=i+1..j} U_ik W_kj by
// distance from the diagonal): the upper one directly; for the lower one,
// D = N diag(D) with N unit lower, so D^{-1} = diag(D)^{-1} N^{-1} and N^{-1} = W^T
// for W = (N^T)^{-1}.  Grid (blocks, 2), blockIdx.y = 0 lower, 1 upper.
template <typename T>
__global__ void __launch_bounds__(256) diag_inv_kernel(const T* __restrict__ S, int64_t lda, int n,
                                                       double* __restrict__ Dinv) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* U = reinterpret_cast<double*>(smem_raw);  // [128][kInvPitch], the strict upper part
  __shared__ double dg[kSolveBlock];
  __shared__ double tmp[32 * 33];
  constexpr int B = 32, NB = kSolveBlock, P = kInvPitch;
  const int blk = blockIdx.x;
  const bool lower = blockIdx.y == 0;
  const int k0 = blk * NB, jb = min(NB, n - k0);
  const T* D = S + k0 + (int64_t)k0 * lda;
  double* V = Dinv + ((size_t)blk * 2 + blockIdx.y) * (NB * NB);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid < NB) dg[tid] = (tid < jb) ? (double)D[tid + (int64_t)tid * lda] : 1.0;
  __syncthreads();
  // U(a, b), a < b: S(a, b) for the upper inverse, S(b, a) / S(a, a) for the lower one;
  // the index runs along S's columns (contiguous) in both cases
  for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
    const int i = idx % NB, j = idx / NB;  // S(k0 + i, k0 + j)
    const double v = (i < jb && j < jb) ? (double)D[i + (int64_t)j * lda] : 0.0;
    if (lower) {
      if (j < i) U[j + i * P] = v / dg[j];
      else U[j + i * P] = 0.0;
    } else {
      U[i + j * P] = (i < j) ? v : 0.0;
    }
  }
  __syncthreads();
  const int nb32 = (jb + B - 1) / B;
  if (warp < nb32) {
    const int o = warp * B;
    double x[B];
#pragma unroll
    for (int i = 0; i < B; ++i) x[i] = (i == lane) ? 1.0 : 0.0;
#pragma unroll
    for (int i = B - 2; i >= 0; --i) {
      double s = x[i];
#pragma unroll
      for (int k = i + 1; k < B; ++k) s = fma(-U[(o + i) + (o + k) * P], x[k], s);
      x[i] = (i < lane) ? s : x[i];
    }
#pragma unroll
    for (int i = 0; i < B; ++i)
      if (o + i < jb && o + lane < jb) V[(o + i) + (o + lane) * NB] = x[i];
  }
  for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
    const int r = idx % NB, cc = idx / NB;
    if (r >= jb || cc >= jb || r / B > cc / B) V[idx] = 0.0;
  }
  __syncthreads();
  for (int d = 1; d < nb32; ++d)
    for (int bi = 0; bi + d < nb32; ++bi) {
      const int oi = bi * B, oj = (bi + d) * B;
      for (int e = tid; e < B * B; e += blockDim.x) {
        const int r = e % B, cc = e / B;
        double acc = 0.0;
        for (int k = oi + B; k < oj + B && k < jb; ++k) acc = fma(U[(oi + r) + k * P], V[k + (oj + cc) * NB], acc);
        tmp[r + cc * 33] = acc;
      }
      __syncthreads();
      for (int e = tid; e < B * B; e += blockDim.x) {
        const int r = e % B, cc = e / B;
        double acc = 0.0;
#pragma unroll 8
        for (int k = 0; k < B; ++k) acc = fma(V[(oi + r) + (oi + k) * NB], tmp[k + cc * 33], acc);
        if (oi + r < jb && oj + cc < jb) V[(oi + r) + (oj + cc) * NB] = -acc;
      }
      __syncthreads();
    }
  if (lower) {
    // V := diag(D)^{-1} W^T, pairwise in place
    for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
      const int i = idx % NB, j = idx / NB;
      if (i < j) {
        const double wij = V[i + j * NB], wji = V[j + i * NB];
        V[i + j * NB] = wji / dg[i];
        V[j + i * NB] = wij / dg[j];
      } else if (i == j) {
        V[i + i * NB] = (i < jb) ? 1.0 / dg[i] : 0.0;
      }
    }
  }
}

__device__ __forceinline__ void st_volatile_v2(unsigned long long* p, unsigned long long a, unsigned long long b) {
  asm volatile("st.volatile.global.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(a), "l"(b) : "memory");
}

__device__ __forceinline__ void ld_volatile_v2(const unsigned long long* p, unsigned long long& a,
                                               unsigned long long& b) {
  asm volatile("ld.volatile.global.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p) : "memory");
}

// One sweep over the 128-row blocks with the diagonal blocks' inverses.  UPPER as in
// sweep_kernel.  Step s solves block k(s) and is owned by CTA s % G, which keeps the
// partial right-hand sides w of its blocks in shared memory (w = b - the tiles of the
// blocks solved so far).  A solved block is published as 256 words {tag, 32 data bits}
// (two per unknown) in slots[256 s ..]: a reader polls the words themselves, so one
// L2 round trip both signals and delivers the block.  Every CTA loads its first tile of
// step s before it waits for y_s; the owner of step s+1 handles that tile first and
// then solves x = Dinv w from the inverse staged in shared memory one owned step ahead.
// A wait that exceeds the context's wait limit records BEM_ERR_TIMEOUT in *status and
// ends the CTA.  `withhold` (failure injection, -1 = none) is a step of the forward
// sweep that is solved but not published, so that the waits for it run out.
template <typename T, bool UPPER>
__global__ void __launch_bounds__(kSweepThreads, 1)
    sweep_inv_kernel(const T* __restrict__ S, int64_t lda, int n, const double* __restrict__ Dinv, double* b,
                     unsigned long long* slots, unsigned tag, int* status, unsigned long long wait_ns,
                     int withhold) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NB = kSolveBlock;
  constexpr bool kPrefetch = sizeof(T) == 4;  // double-buffered tile registers for FP32 factors
  double* Di = reinterpret_cast<double*>(smem_raw);  // [NB * NB] inverse of the next owned block
  double* wacc = Di + NB * NB;                        // [owned blocks][NB]
  __shared__ double ys[NB];
  __shared__ double red[4][NB];
  __shared__ int s_abort;
  const int t = threadIdx.x, G = gridDim.x, g = blockIdx.x;
  const int nblk = (n + NB - 1) / NB;
  const int rl = t & (NB - 1), q = t >> 7;
  auto bidx = [&](int s) { return UPPER ? nblk - 1 - s : s; };
  auto stage_inv = [&](int s) {
    const double2* src = reinterpret_cast<const double2*>(Dinv + ((size_t)bidx(s) * 2 + (UPPER ? 1 : 0)) * (NB * NB));
    double2* dst = reinterpret_cast<double2*>(Di);
    for (int i0 = 0; i0 < NB * NB / 2; i0 += 8 * kSweepThreads) {
      double2 v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = __ldcg(src + i0 + u * kSweepThreads + t);
#pragma unroll
      for (int u = 0; u < 8; ++u) dst[i0 + u * kSweepThreads + t] = v[u];
    }
  };
  auto load_tile = [&](T* a, int sx, int c0, int cb) {
    const int r0 = bidx(sx) * NB, rb = min(NB, n - r0);
    const int cq = 32 * q;
    const T* p = S + (r0 + rl) + (int64_t)(c0 + cq) * lda;
#pragma unroll
    for (int u = 0; u < 32; ++u) a[u] = (rl < rb && cq + u < cb) ? p[(int64_t)u * lda] : T(0);
  };
  const int nown = (g < nblk) ? (nblk - 1 - g) / G + 1 : 0;
  for (int i = t; i < nown * NB; i += blockDim.x) {
    const int k0 = bidx(g + (i / NB) * G) * NB, r = i % NB;
    wacc[i] = (k0 + r < n) ? b[k0 + r] : 0.0;
  }
  if (t == 0) s_abort = 0;
  if (nown > 0) stage_inv(g);
  __syncthreads();

  auto solve = [&](int s) {  // all threads; Di holds the inverse of block k(s)
    const int k0 = bidx(s) * NB, kb = min(NB, n - k0);
    const double* w = wacc + ((s - g) / G) * NB;
    double acc = 0.0;
#pragma unroll 8
    for (int u = 0; u < 32; ++u) acc = fma(Di[rl + (32 * q + u) * NB], w[32 * q + u], acc);
    red[q][rl] = acc;
    __syncthreads();
    if (t < kb) {
      const double x = (red[0][t] + red[1][t]) + (red[2][t] + red[3][t]);
      const unsigned long long hi = (unsigned long long)tag << 32;
      const unsigned long long bits = (unsigned long long)__double_as_longlong(x);
      if (UPPER || s != withhold)  // a withheld step (failure injection) is never published
        st_volatile_v2(slots + (size_t)s * 256 + 2 * t, hi | (bits & 0xffffffffull), hi | (bits >> 32));
      b[k0 + t] = x;
    }
    __syncthreads();  // Di and red are free again
    if (s + G < nblk) stage_inv(s + G);
  };

  if (g == 0) solve(0);
  for (int s = 0; s + 1 < nblk; ++s) {
    const int s2 = s + 1 + ((g - (s + 1)) % G + G) % G;  // this CTA's first step after s
    if (s2 >= nblk) break;                                // no rows left to update
    const int c0 = bidx(s) * NB, cb = min(NB, n - c0);
    T a[32];
    load_tile(a, s2, c0, cb);
    if (t < NB) {
      double y = 0.0;
      if (t < cb) {
        const unsigned long long* p = slots + (size_t)s * 256 + 2 * t;
        const unsigned long long t0 = globaltimer_ns();
        unsigned it = 0;
        unsigned long long w0, w1;
        for (;;) {
          ld_volatile_v2(p, w0, w1);
          if ((unsigned)(w0 >> 32) == tag && (unsigned)(w1 >> 32) == tag) break;
          if ((++it & 63u) == 0 &&
              (globaltimer_ns() - t0 > wait_ns || *((volatile int*)status) != 0)) {
            atomicCAS(status, 0, BEM_ERR_TIMEOUT);
            s_abort = 1;
            w0 = w1 = 0;
            break;
          }
        }
        y = __longlong_as_double((long long)((w1 << 32) | (w0 & 0xffffffffull)));
      }
      ys[t] = y;
    }
    __syncthreads();
    if (s_abort) return;
    for (int sx = s2; sx < nblk; sx += G) {
      const bool more = sx + G < nblk;
      T nx[32];
      if (kPrefetch && more) load_tile(nx, sx + G, c0, cb);
      double acc = 0.0;
#pragma unroll
      for (int u = 0; u < 32; ++u) acc = fma((double)a[u], ys[32 * q + u], acc);
      red[q][rl] = acc;
      __syncthreads();
      if (t < NB) wacc[((sx - g) / G) * NB + t] -= (red[0][t] + red[1][t]) + (red[2][t] + red[3][t]);
      __syncthreads();
      if (sx == s + 1) solve(sx);
      if (more) {
        if (kPrefetch) {
#pragma unroll
          for (int u = 0; u < 32; ++u) a[u] = nx[u];
        } else {
          load_tile(a, sx + G, c0, cb);
        }
      }
    }
  }
}

// ---- the transposed solve: S^T x = b with the same factors --------------------------
// S^T = T = P L U, so x = U^{-1} L^{-1} P^T b, where L_T(i, j) = S(j, i) (j < i, unit)
// and U_T(i, j) = S(j, i) (j >= i).  The sweeps read the factor transposed: a solved
// block j contributes S(block j rows, column i) . y_j to every target column i, one
// warp per column (coalesced 32-row segments); diagonal blocks are staged transposed
// with a padded leading dimension.
constexpr int kLdT = kSolveBlock + 1;

template <typename T>
__device__ void warp_lower_unit_solve_t(const T* D, int jb, double* w) {
  const int lane = threadIdx.x & 31;
  double x[kSolveBlock / 32];
#pragma unroll
  for (int q = 0; q < kSolveBlock / 32; ++q) x[q] = (lane + 32 * q < jb) ? w[lane + 32 * q] : 0.0;
#pragma unroll
  for (int slot = 0; slot < kSolveBlock / 32; ++slot) {
#pragma unroll
    for (int o = 0; o < 32; ++o) {
      const int cidx = slot * 32 + o;
      if (cidx < jb) {
        const double xc = __shfl_sync(0xffffffffu, x[slot], o);
#pragma unroll
        for (int q = slot; q < kSolveBlock / 32; ++q) {
          const int r = lane + 32 * q;
          if (r > cidx) x[q] = fma(-(double)D[r + cidx * kLdT], xc, x[q]);
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kSolveBlock / 32; ++q)
    if (lane + 32 * q < jb) w[lane + 32 * q] = x[q];
}

template <typename T>
__device__ void warp_upper_solve_t(const T* D, const double* rdiag, int jb, double* w) {
  const int lane = threadIdx.x & 31;
  double x[kSolveBlock / 32];
#pragma unroll
  for (int q = 0; q < kSolveBlock / 32; ++q) x[q] = (lane + 32 * q < jb) ? w[lane + 32 * q] : 0.0;
#pragma unroll
  for (int slot = kSolveBlock / 32 - 1; slot >= 0; --slot) {
#pragma unroll
    for (int o = 31; o >= 0; --o) {
      const int cidx = slot * 32 + o;
      if (cidx < jb) {
        const double xc = __shfl_sync(0xffffffffu, x[slot], o) * rdiag[cidx];
        if (lane == o) x[slot] = xc;
#pragma unroll
        for (int q = 0; q <= slot; ++q) {
          const int r = lane + 32 * q;
          if (r < cidx) x[q] = fma(-(double)D[r + cidx * kLdT], xc, x[q]);
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kSolveBlock / 32; ++q)
    if (lane + 32 * q < jb) w[lane + 32 * q] = x[q];
}

// UPPER = false: forward with L_T (blocks first to last); true: backward with U_T
template <typename T, bool UPPER>
__global__ void __launch_bounds__(kSweepThreads, 1)
    sweep_t_kernel(const T* __restrict__ S, int64_t lda, int n, double* b, unsigned* flags, unsigned tag,
                   int* status, unsigned long long wait_ns) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* D = reinterpret_cast<T*>(smem_raw);  // [kSolveBlock][kLdT]: D[r + c * kLdT] = T(k0 + r, k0 + c)
  __shared__ double ys[kSolveBlock];
  __shared__ double wn[kSolveBlock];
  __shared__ double rdiag[kSolveBlock];
  __shared__ int s_abort;
  const int t = threadIdx.x, G = gridDim.x, g = blockIdx.x, lane = t & 31, wp = t >> 5;
  const int nblk = (n + kSolveBlock - 1) / kSolveBlock;
  auto blk0 = [&](int s) { return (UPPER ? nblk - 1 - s : s) * kSolveBlock; };
  auto stage_diag = [&](int s) {
    const int k0 = blk0(s), kb = min(kSolveBlock, n - k0);
    for (int idx = t; idx < kSolveBlock * kSolveBlock; idx += kSweepThreads) {
      const int a = idx % kSolveBlock, c = idx / kSolveBlock;  // S(k0 + a, k0 + c) = T(k0 + c, k0 + a)
      const bool in = a < kb && c < kb && (UPPER ? (c <= a) : (c > a));
      D[c + a * kLdT] = in ? S[(k0 + a) + (int64_t)(k0 + c) * lda] : T(0);
    }
  };
  auto solve = [&](int s) {
    const int k0 = blk0(s), kb = min(kSolveBlock, n - k0);
    if (t < kb) wn[t] = b[k0 + t];
    if (UPPER && t < kSolveBlock) rdiag[t] = (t < kb) ? 1.0 / (double)D[t + t * kLdT] : 0.0;
    __syncthreads();
    if (t < 32) {
      if (UPPER)
        warp_upper_solve_t<T>(D, rdiag, kb, wn);
      else
        warp_lower_unit_solve_t<T>(D, kb, wn);
    }
    __syncthreads();
    if (t < kb) b[k0 + t] = wn[t];
    __syncthreads();
    if (t == 0) {
      __threadfence();
      st_release_u32(flags + s, tag);
    }
    if (s + G < nblk) stage_diag(s + G);
  };

  if (t == 0) s_abort = 0;
  if (g < nblk) stage_diag(g);
  __syncthreads();
  if (g == 0) solve(0);
  for (int s = 0; s + 1 < nblk; ++s) {
    int s2 = s + 1 + ((g - (s + 1)) % G + G) % G;
    if (s2 >= nblk) break;
    if (t == 0 && s % G != g) {
      const unsigned long long t0 = globaltimer_ns();
      unsigned it = 0;
      while (ld_acquire_u32(flags + s) != tag) {
        if ((++it & 255u) == 0 && (globaltimer_ns() - t0 > wait_ns || *((volatile int*)status) != 0)) {
          atomicExch(status, BEM_ERR_TIMEOUT);
          s_abort = 1;
          break;
        }
      }
      __threadfence();
    }
    __syncthreads();
    if (s_abort) return;
    const int c0 = blk0(s), cb = min(kSolveBlock, n - c0);
    if (t < kSolveBlock) ys[t] = (t < cb) ? __ldcg(b + c0 + t) : 0.0;
    __syncthreads();
    for (; s2 < nblk; s2 += G) {
      const int r0 = blk0(s2), rb = min(kSolveBlock, n - r0);
      // warp wp takes target columns r0 + wp, r0 + wp + 16, ...: dot of the solved rows
      for (int i = wp; i < rb; i += kSweepThreads / 32) {
        const T* p = S + c0 + (int64_t)(r0 + i) * lda;
        double acc = 0.0;
#pragma unroll
        for (int u = 0; u < kSolveBlock / 32; ++u) {
          const int j = lane + 32 * u;
          if (j < cb) acc = fma((double)p[j], ys[j], acc);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (lane == 0) b[r0 + i] -= acc;
      }
      __syncthreads();
      if (s2 == s + 1) solve(s2);
    }
  }
}

__global__ void scatter_kernel(int n, const int* __restrict__ perm, const double* __restrict__ v,
                               double* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[perm[i]] = v[i];
}

template <typename T, bool UPPER>
int sweep_t_launch(bem_ctx* c, const T* S, int64_t lda, int n, double* b, unsigned* flags, unsigned tag,
                   int* status) {
  static DeviceOnce ok;  // per instantiation and device
  const size_t dsm = (size_t)kSolveBlock * kLdT * sizeof(T);
  if (ok.pending()) {
    int per_sm = 0;
    BEM_CUDA(c, cudaFuncSetAttribute(sweep_t_kernel<T, UPPER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm));
    BEM_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_t_kernel<T, UPPER>, kSweepThreads, dsm));
    if (per_sm < 1) return bem_fail(c, BEM_ERR_CUDA, "transposed sweep kernel does not fit on an SM");
    ok.mark();
  }
  const int nblk = (n + kSolveBlock - 1) / kSolveBlock;
  const int G = std::min(nblk, c->sm_count);
  unsigned long long wns = c->wait_ns;
  void* args[] = {(void*)&S, (void*)&lda, (void*)&n, (void*)&b, (void*)&flags, (void*)&tag, (void*)&status,
                  (void*)&wns};
  BEM_CUDA(c, cudaLaunchCooperativeKernel((void*)sweep_t_kernel<T, UPPER>, dim3(G), dim3(kSweepThreads), args, dsm,
                                          c->stream));
  ++c->launches;
  return BEM_OK;
}

template <typename T, bool UPPER>
int sweep_launch(bem_ctx* c, const T* S, int64_t lda, int n, double* b, unsigned* flags, unsigned tag,
                 int* status) {
  static DeviceOnce ok;  // per instantiation and device
  const size_t dsm = (size_t)kSolveBlock * kSolveBlock * sizeof(T);
  if (ok.pending()) {
    int per_sm = 0;
    BEM_CUDA(c, cudaFuncSetAttribute(sweep_kernel<T, UPPER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm));
    BEM_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_kernel<T, UPPER>, kSweepThreads, dsm));
    if (per_sm < 1) return bem_fail(c, BEM_ERR_CUDA, "triangular sweep kernel does not fit on an SM");
    ok.mark();
  }
  const int nblk = (n + kSolveBlock - 1) / kSolveBlock;
  const int G = std::min(nblk, c->sm_count);  // one CTA per SM: the whole diagonal block in smem
  unsigned long long wns = c->wait_ns;
  void* args[] = {(void*)&S, (void*)&lda, (void*)&n, (void*)&b, (void*)&flags, (void*)&tag, (void*)&status,
                  (void*)&wns};
  BEM_CUDA(c, cudaLaunchCooperativeKernel((void*)sweep_kernel<T, UPPER>, dim3(G), dim3(kSweepThreads), args, dsm,
                                          c->stream));
  ++c->launches;
  return BEM_OK;
}

template <typename T>
int lu_solve_ws(bem_ctx* c, const T* S, int64_t lda, int n, const int* perm, double* b, double* work) {
  // work: [0, n) gather buffer, then the per-block flags and the status word
  const int nblk = (n + kSolveBlock - 1) / kSolveBlock;
  unsigned* flags = reinterpret_cast<unsigned*>(work + n);
  int* status = reinterpret_cast<int*>(flags + nblk);
  BEM_CUDA(c, cudaMemsetAsync(flags, 0, (nblk + 1) * sizeof(unsigned), c->stream));
  int rc;
  if ((rc = sweep_launch<T, false>(c, S, lda, n, b, flags, 1u, status))) return rc;
  if ((rc = sweep_launch<T, true>(c, S, lda, n, b, flags, 2u, status))) return rc;
  permute_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(n, perm, b, work);
  BEM_LAUNCH_CHECK(c);
  BEM_CUDA(c, cudaMemcpyAsync(b, work, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  int st = 0;
  BEM_CUDA(c, cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  if (st != 0) return bem_fail(c, st, "triangular solve: a wait for a solved block timed out");
  return BEM_OK;
}

// b := S^{-T} b with the factors of lu_factor (the transposed system, same factors)
template <typename T>
int lu_solve_t_ws(bem_ctx* c, const T* S, int64_t lda, int n, const int* perm, double* b, double* work) {
  const int nblk = (n + kSolveBlock - 1) / kSolveBlock;
  unsigned* flags = reinterpret_cast<unsigned*>(work + n);
  int* status = reinterpret_cast<int*>(flags + nblk);
  BEM_CUDA(c, cudaMemsetAsync(flags, 0, (nblk + 1) * sizeof(unsigned), c->stream));
  scatter_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(n, perm, b, work);  // P^T b
  BEM_LAUNCH_CHECK(c);
  int rc;
  if ((rc = sweep_t_launch<T, false>(c, S, lda, n, work, flags, 1u, status))) return rc;
  if ((rc = sweep_t_launch<T, true>(c, S, lda, n, work, flags, 2u, status))) return rc;
  BEM_CUDA(c, cudaMemcpyAsync(b, work, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  int st = 0;
  BEM_CUDA(c, cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  if (st != 0) return bem_fail(c, st, "transposed solve: a wait for a solved block timed out");
  return BEM_OK;
}

int lu_solve_t_fp64(bem_ctx* c, const double* LU, int64_t lda, int n, double* b) {
  const size_t need = lu_solve_work_count(n);
  if (c->work.count < need) {
    c->work.release();
    BEM_CUDA(c, c->work.alloc(need));
  }
  return lu_solve_t_ws<double>(c, LU, lda, n, c->perm.p, b, c->work.p);
}

// Inverses of the diagonal blocks of freshly computed factors, kept in the context for
// the block-inverse sweeps of lu_solve (2 x 128 KB per 128-row block).
template <typename T>
int lu_prepare_inverses(bem_ctx* c, const T* S, int64_t lda, int n) {
  c->dinv_src = nullptr;
  if (const char* e = getenv("BEM_SWEEP_INV"))  // 0: keep the substitution sweeps
    if (atoi(e) == 0) return BEM_OK;
  const int nblk = (n + kSolveBlock - 1) / kSolveBlock;
  const size_t need = (size_t)nblk * 2 * kSolveBlock * kSolveBlock;
  if (c->dinv.count < need) {
    c->dinv.release();
    BEM_CUDA(c, c->dinv.alloc(need));
  }
  const int smem = kSolveBlock * kInvPitch * (int)sizeof(double);
  static DeviceOnce attr;  // per instantiation and device
  if (attr.pending()) {
    BEM_CUDA(c, cudaFuncSetAttribute(diag_inv_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr.mark();
  }
  diag_inv_kernel<T><<<dim3(nblk, 2), 256, smem, c->stream>>>(S, lda, n, c->dinv.p);
  BEM_LAUNCH_CHECK(c);
  c->dinv_src = S;
  c->dinv_n = n;
  c->dinv_lda = lda;
  c->dinv_elem = (int)sizeof(T);
  return BEM_OK;
}

template <typename T, bool UPPER>
int sweep_inv_launch(bem_ctx* c, const T* S, int64_t lda, int n, double* b, unsigned long long* slots,
                     unsigned tag, int* status) {
  // per instantiation and device: the attribute is set once to the largest dynamic
  // shared memory the device allows next to the kernel's static arrays, so that no
  // later launch (of any order) needs to raise it
  static std::atomic<int> max_dyn[64];
  const int nblk = (n + kSolveBlock - 1) / kSolveBlock;
  const int G = std::min(nblk, c->sm_count);
  const int nown = (nblk + G - 1) / G;
  const size_t dsm = ((size_t)kSolveBlock * kSolveBlock + (size_t)nown * kSolveBlock) * sizeof(double);
  std::atomic<int>& lim = max_dyn[current_device()];
  if (lim.load() == 0) {
    cudaFuncAttributes fa{};
    int optin = 0;
    BEM_CUDA(c, cudaFuncGetAttributes(&fa, sweep_inv_kernel<T, UPPER>));
    BEM_CUDA(c, cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    const int mx = optin - (int)fa.sharedSizeBytes;
    BEM_CUDA(c, cudaFuncSetAttribute(sweep_inv_kernel<T, UPPER>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    int per_sm = 0;
    BEM_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_inv_kernel<T, UPPER>, kSweepThreads,
                                                              (size_t)mx));
    if (per_sm < 1) return bem_fail(c, BEM_ERR_CUDA, "block-inverse sweep kernel does not fit on an SM");
    lim.store(mx);
  }
  if (dsm > (size_t)lim.load()) return bem_fail(c, BEM_ERR_ARG, "block-inverse sweep: too many blocks per SM");
  const double* dinv = c->dinv.p;
  unsigned long long wns = c->wait_ns;
  int withhold = c->withhold_block;
  void* args[] = {(void*)&S,     (void*)&lda,    (void*)&n,   (void*)&dinv, (void*)&b,
                  (void*)&slots, (void*)&tag,    (void*)&status, (void*)&wns, (void*)&withhold};
  BEM_CUDA(c, cudaLaunchCooperativeKernel((void*)sweep_inv_kernel<T, UPPER>, dim3(G), dim3(kSweepThreads), args,
                                          dsm, c->stream));
  ++c->launches;
  return BEM_OK;
}

template <typename T>
int lu_solve(bem_ctx* c, const T* S, int64_t lda, int n, const int* perm, double* b) {
  const size_t need = lu_solve_work_count(n);
  if (c->work.count < need) {
    c->work.release();
    BEM_CUDA(c, c->work.alloc(need));
  }
  if (c->dinv_src != S || c->dinv_n != n || c->dinv_lda != lda || c->dinv_elem != (int)sizeof(T))
    return lu_solve_ws<T>(c, S, lda, n, perm, b, c->work.p);
  // block-inverse sweeps: slots [nblk][256] words, then the status word
  const int nblk = (n + kSolveBlock - 1) / kSolveBlock;
  const size_t words = (size_t)nblk * 256 + 2;
  if (c->slots.count < words) {
    c->slots.release();
    BEM_CUDA(c, c->slots.alloc(words));
  }
  unsigned long long* slots = c->slots.p;
  int* status = reinterpret_cast<int*>(slots + (size_t)nblk * 256);
  BEM_CUDA(c, cudaMemsetAsync(slots, 0, words * sizeof(unsigned long long), c->stream));
  int rc;
  if ((rc = sweep_inv_launch<T, false>(c, S, lda, n, b, slots, 1u, status))) return rc;
  if ((rc = sweep_inv_launch<T, true>(c, S, lda, n, b, slots, 2u, status))) return rc;
  double* work = c->work.p;
  permute_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(n, perm, b, work);
  BEM_LAUNCH_CHECK(c);
  BEM_CUDA(c, cudaMemcpyAsync(b, work, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  int st = 0;
  BEM_CUDA(c, cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  if (st != 0) return bem_fail(c, st, "triangular solve: a wait for a solved block timed out");
  return BEM_OK;
}

template int lu_solve<double>(bem_ctx*, const double*, int64_t, int, const int*, double*);
template int lu_solve_ws<double>(bem_ctx*, const double*, int64_t, int, const int*, double*, double*);
template int lu_solve<float>(bem_ctx*, const float*, int64_t, int, const int*, double*);

// ---------------------------------------------------------------------------------
// residual r = b - A x (FP64) with infinity norms
// ---------------------------------------------------------------------------------
constexpr int kResCols = 512;

__global__ void residual_part_kernel(const double* A, int64_t lda, int n, const double* x, double* part,
                                     double* apart, int want_anorm) {
  __shared__ double xs[kResCols];
  const int cs = blockIdx.y * kResCols;
  const int ce = min(n, cs + kResCols);
  for (int i = threadIdx.x; i < ce - cs; i += blockDim.x) xs[i] = x[cs + i];
  __syncthreads();
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0}, aabs = 0.0;
  const double* p = A + r + (int64_t)cs * lda;
  const int cnt = ce - cs;
  int cc = 0;
  for (; cc + 8 <= cnt; cc += 8) {
    double a[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) a[u] = p[(int64_t)(cc + u) * lda];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      acc[u] = fma(a[u], xs[cc + u], acc[u]);
      if (want_anorm) aabs += fabs(a[u]);
    }
  }
  for (; cc < cnt; ++cc) {
    const double a = p[(int64_t)cc * lda];
    acc[0] = fma(a, xs[cc], acc[0]);
    if (want_anorm) aabs += fabs(a);
  }
  part[(int64_t)blockIdx.y * n + r] = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
  if (want_anorm) apart[(int64_t)blockIdx.y * n + r] = aabs;
}

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  // non-negative doubles order like their bit patterns
  atomicMax(reinterpret_cast<unsigned long long*>(addr), __double_as_longlong(v));
}

__global__ void residual_finish_kernel(int n, int nchunk, const double* part, const double* apart, const double* b,
                                       const double* x, double* r, double* norms, int want_anorm) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double rv = 0.0, xv = 0.0, bv = 0.0, av = 0.0;
  if (i < n) {
    double s = 0.0, sa = 0.0;
    for (int k = 0; k < nchunk; ++k) {
      s += part[(int64_t)k * n + i];
      if (want_anorm) sa += apart[(int64_t)k * n + i];
    }
    const double ri = b[i] - s;
    r[i] = ri;
    rv = fabs(ri);
    xv = fabs(x[i]);
    bv = fabs(b[i]);
    av = sa;
  }
  for (int off = 16; off > 0; off >>= 1) {
    rv = fmax(rv, __shfl_xor_sync(0xffffffffu, rv, off));
    xv = fmax(xv, __shfl_xor_sync(0xffffffffu, xv, off));
    bv = fmax(bv, __shfl_xor_sync(0xffffffffu, bv, off));
    av = fmax(av, __shfl_xor_sync(0xffffffffu, av, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_nonneg(norms + 0, rv);
    atomic_max_nonneg(norms + 1, xv);
    atomic_max_nonneg(norms + 2, bv);
    if (want_anorm) atomic_max_nonneg(norms + 3, av);
  }
}

// The same residual with every product and sum carried as a double-double (an FP64
// value and its rounding error: the product's error by an FMA, the sums' by TwoSum),
// the residual b - A x rounded to FP64 once at the end.  Its error is ~1e-32 of |A||x|
// instead of ~n 1e-16, so that refinement can drive x to the solution of the stored
// FP64 system itself (its forward error no longer grows with the condition number).
// (explicitly rounded operations: no contraction into an FMA may merge them)
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}

__global__ void residual_part_dd_kernel(const double* A, int64_t lda, int n, const double* x, double* part_hi,
                                        double* part_lo, double* apart, int want_anorm) {
  __shared__ double xs[kResCols];
  const int cs = blockIdx.y * kResCols;
  const int ce = min(n, cs + kResCols);
  for (int i = threadIdx.x; i < ce - cs; i += blockDim.x) xs[i] = x[cs + i];
  __syncthreads();
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double hi[4] = {0, 0, 0, 0}, lo[4] = {0, 0, 0, 0}, aabs = 0.0;
  const double* p = A + r + (int64_t)cs * lda;
  const int cnt = ce - cs;
  int cc = 0;
  for (; cc + 8 <= cnt; cc += 8) {
    double a[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) a[u] = p[(int64_t)(cc + u) * lda];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const double pr = __dmul_rn(a[u], xs[cc + u]);
      const double pe = fma(a[u], xs[cc + u], -pr);
      double t, e;
      two_sum(hi[u & 3], pr, t, e);
      hi[u & 3] = t;
      lo[u & 3] += e + pe;
      if (want_anorm) aabs += fabs(a[u]);
    }
  }
  for (; cc < cnt; ++cc) {
    const double a = p[(int64_t)cc * lda];
    const double pr = __dmul_rn(a, xs[cc]);
    const double pe = fma(a, xs[cc], -pr);
    double t, e;
    two_sum(hi[0], pr, t, e);
    hi[0] = t;
    lo[0] += e + pe;
    if (want_anorm) aabs += fabs(a);
  }
  double sh = hi[0], sl = lo[0];
#pragma unroll
  for (int u = 1; u < 4; ++u) {
    double t, e;
    two_sum(sh, hi[u], t, e);
    sh = t;
    sl += e + lo[u];
  }
  part_hi[(int64_t)blockIdx.y * n + r] = sh;
  part_lo[(int64_t)blockIdx.y * n + r] = sl;
  if (want_anorm) apart[(int64_t)blockIdx.y * n + r] = aabs;
}

__global__ void residual_finish_dd_kernel(int n, int nchunk, const double* part_hi, const double* part_lo,
                                          const double* apart, const double* b, const double* x, double* r,
                                          double* norms, int want_anorm) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double rv = 0.0, xv = 0.0, bv = 0.0, av = 0.0;
  if (i < n) {
    double sh = 0.0, sl = 0.0, sa = 0.0;
    for (int k = 0; k < nchunk; ++k) {
      double t, e;
      two_sum(sh, part_hi[(int64_t)k * n + i], t, e);
      sh = t;
      sl += e + part_lo[(int64_t)k * n + i];
      if (want_anorm) sa += apart[(int64_t)k * n + i];
    }
    double t, e;
    two_sum(b[i], -sh, t, e);
    const double ri = t + (e - sl);
    r[i] = ri;
    rv = fabs(ri);
    xv = fabs(x[i]);
    bv = fabs(b[i]);
    av = sa;
  }
  for (int off = 16; off > 0; off >>= 1) {
    rv = fmax(rv, __shfl_xor_sync(0xffffffffu, rv, off));
    xv = fmax(xv, __shfl_xor_sync(0xffffffffu, xv, off));
    bv = fmax(bv, __shfl_xor_sync(0xffffffffu, bv, off));
    av = fmax(av, __shfl_xor_sync(0xffffffffu, av, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_nonneg(norms + 0, rv);
    atomic_max_nonneg(norms + 1, xv);
    atomic_max_nonneg(norms + 2, bv);
    if (want_anorm) atomic_max_nonneg(norms + 3, av);
  }
}

int residual_fp64(bem_ctx* c, const double* A, int64_t lda, int n, const double* x, const double* b, double* r,
                  double* norms, bool want_anorm, bool extended) {
  const int nchunk = (n + kResCols - 1) / kResCols;
  const size_t need = (size_t)nchunk * n * ((want_anorm ? 2 : 1) + (extended ? 1 : 0)) + 8;
  if (c->work.count < need) {
    c->work.release();
    BEM_CUDA(c, c->work.alloc(need));
  }
  double* part = c->work.p + 8;
  double* apart = part + (size_t)nchunk * n;
  double* part_lo = apart + (want_anorm ? (size_t)nchunk * n : 0);
  double* dn = c->work.p;
  BEM_CUDA(c, cudaMemsetAsync(dn, 0, 4 * sizeof(double), c->stream));
  dim3 grid((n + 255) / 256, nchunk);
  if (extended) {
    residual_part_dd_kernel<<<grid, 256, 0, c->stream>>>(A, lda, n, x, part, part_lo, apart, want_anorm ? 1 : 0);
    BEM_LAUNCH_CHECK(c);
    residual_finish_dd_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(n, nchunk, part, part_lo, apart, b, x, r, dn,
                                                                       want_anorm ? 1 : 0);
    BEM_LAUNCH_CHECK(c);
  } else {
    residual_part_kernel<<<grid, 256, 0, c->stream>>>(A, lda, n, x, part, apart, want_anorm ? 1 : 0);
    BEM_LAUNCH_CHECK(c);
    residual_finish_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(n, nchunk, part, apart, b, x, r, dn,
                                                                    want_anorm ? 1 : 0);
    BEM_LAUNCH_CHECK(c);
  }
  BEM_CUDA(c, cudaMemcpyAsync(norms, dn, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  return BEM_OK;
}

// ---------------------------------------------------------------------------------
// FP64 entry points used by context.cu
// ---------------------------------------------------------------------------------
constexpr int kNbFp64 = 512;  // panel width of the FP64 LU: the trailing DMMA update reaches 72 % of FP64 peak

int lu_factor_fp64(bem_ctx* c, double* A, int64_t lda, int n, int* d_piv, int* info, double* seconds) {
  cudaEvent_t e0, e1;
  BEM_CUDA(c, cudaEventCreate(&e0));
  BEM_CUDA(c, cudaEventCreate(&e1));
  BEM_CUDA(c, cudaEventRecord(e0, c->stream));
  BEM_CUDA(c, c->perm.alloc(n));
  int nb = kNbFp64;
  if (const char* e = getenv("BEM_LU_NB64")) {  // panel width override: 128, 256, 384 or 512
    const int v = atoi(e);
    if (v >= 128 && v <= 512 && v % 128 == 0) nb = v;
  }
  int rc = lu_factor<double>(c, A, lda, n, d_piv, c->perm.p, nb, info);
  BEM_CUDA(c, cudaEventRecord(e1, c->stream));
  BEM_CUDA(c, cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (seconds) *seconds = ms * 1e-3;
  return rc;
}

int lu_solve_fp64(bem_ctx* c, const double* LU, int64_t lda, int n, double* b) {
  return lu_solve<double>(c, LU, lda, n, c->perm.p, b);
}

}  // namespace bem
