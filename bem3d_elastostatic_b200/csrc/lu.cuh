// Dense LU with partial pivoting and the triangular solves, templated on the
// storage type of the factors (double for the DGESV replacement, float for the
// low-precision factorisation of the refinement solvers).
//
// Layout.  The matrix S is the reference's column-major A (lda >= n).  The
// factorisation is of T = S^T with row pivoting, i.e. column pivoting of S, so that
// every pivot swap and every panel load touches contiguous column segments of S:
//   T = P_1 L_1 P_2 L_2 ... P_K L_K U      (product form, one factor per NB panel)
// with U in the lower triangle of S (diagonal included) and the unit multipliers of
// panel k in the strict upper part of S's rows [j0, j0+NB).  Swaps of a panel are not
// applied to the multipliers of earlier panels (their rows of S), so the solve
// applies P_k panel by panel:
//   S x = b  ->  x = P_1 L_1^{-T} P_2 L_2^{-T} ... P_K L_K^{-T} U^{-T} b.
// LU of A^T with partial pivoting is as stable as that of A; info follows DGESV (the
// 1-based step of the first exactly zero pivot).
#pragma once

#include "common.cuh"

namespace bem {

constexpr int kPanelW = 32;  // columns of T factored by one cooperative panel launch

// Device scratch of one factorisation: the cooperative panel kernel's candidate
// exchange (double-buffered per-CTA candidates, the diagonal column, the grid-barrier
// counter and the status words) and the TRSM-by-inverse buffers.  lu_factor()
// allocates it per call; lu_factor_ws() takes it from the caller.
struct LUWorkspace {
  double* cand_val;   // [2][gmax]
  int* cand_idx;      // [2][gmax]
  void* cand_col;     // [2][gmax][kPanelW] of T
  void* diag_col;     // [2][kPanelW] of T
  unsigned* barrier;  // grid-barrier counter (zeroed before every panel launch)
  int* status;        // [0] error code, [1] info (zeroed at the start of a factorisation)
  void* inv;          // nb x nb of T
  void* ybuf;         // ldy x nb of T
  int64_t ldy;
  int gmax;           // most CTAs a panel launch may use
};

// bytes of an LUWorkspace for order n (rounded up per region to 256 bytes); carve()
// lays the regions out from base in that order
size_t lu_workspace_bytes(int n, int nb, int gmax, int elem);
LUWorkspace lu_workspace_carve(void* base, int n, int nb, int gmax, int elem);
// doubles of triangular-solve scratch for order n
size_t lu_solve_work_count(int n);

template <typename T>
int lu_factor_ws(bem_ctx* c, T* S, int64_t lda, int n, int* piv, int nb, int* info, const LUWorkspace& ws);
template <typename T>
int lu_solve_ws(bem_ctx* c, const T* S, int64_t lda, int n, const int* piv, int nb, double* b, double* work);

template <typename T>
int lu_factor(bem_ctx* c, T* S, int64_t lda, int n, int* piv, int nb, int* info);

template <typename T>
int lu_solve(bem_ctx* c, const T* S, int64_t lda, int n, const int* piv, int nb, double* b);

// y = b - A x (FP64 A, column-major) and the infinity norms of y; |A| row sums on request
int residual_fp64(bem_ctx* c, const double* A, int64_t lda, int n, const double* x, const double* b,
                  double* r, double* norms /* host: [0]=|r|inf [1]=|x|inf [2]=|b|inf [3]=|A|inf */,
                  bool want_anorm);

// C (M x N, ldc) op= A (M x K, lda) * B (K x N, ldb), column-major; op: 0 -=, 1 =.
template <typename T>
int gemm(bem_ctx* c, int M, int N, int K, const T* A, int64_t lda, const T* B, int64_t ldb, T* C,
         int64_t ldc, int mode);

}  // namespace bem
