// Dense LU with partial pivoting and the triangular solves, templated on the
// storage type of the factors (double for the DGESV replacement, float for the
// low-precision factorisation of the refinement solvers).
//
// Layout.  The matrix S is the reference's column-major A (lda >= n).  The
// factorisation is of T = S^T with row pivoting, i.e. column pivoting of S, so that
// every pivot swap and every panel load touches contiguous column segments of S:
//   T = P L U,   P = tau_0 tau_1 ... tau_{n-1}   (tau_i swaps rows i and piv[i])
// with U in the lower triangle of S (diagonal included) and the unit multipliers L in
// the strict upper triangle of S; every panel's swaps are applied to all other rows
// of S, the earlier panels' multipliers included (LAPACK's dgetrf convention for T).
// The solve is two substitution sweeps and one gather:
//   S x = b  ->  x = P L^{-T} U^{-T} b,   (P v)[i] = v[perm[i]].
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
  void* inv;          // the 128 x 128 diagonal-block inverses of a panel (T)
  void* finv;         // FP32 panels: the panel's two full triangle inverses (2 nb x nb)
                      // and their assembly's scratch (nb x 128), else null
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

// piv: the 0-based pivot rows of T; perm (n ints, nullable): the gather form of P
// that the solve takes, written when the factorisation succeeds (a host round trip)
template <typename T>
int lu_factor_ws(bem_ctx* c, T* S, int64_t lda, int n, int* piv, int* perm, int nb, int* info,
                 const LUWorkspace& ws);
// b (device, FP64) := S^{-1} b; work: lu_solve_work_count(n) doubles.  Synchronises
// the stream to read the sweeps' status word.
template <typename T>
int lu_solve_ws(bem_ctx* c, const T* S, int64_t lda, int n, const int* perm, double* b, double* work);

template <typename T>
int lu_factor(bem_ctx* c, T* S, int64_t lda, int n, int* piv, int* perm, int nb, int* info);

template <typename T>
int lu_solve(bem_ctx* c, const T* S, int64_t lda, int n, const int* perm, double* b);

// y = b - A x (FP64 A, column-major) and the infinity norms of y; |A| row sums on request;
// extended: products and sums carried as double-doubles (y rounded once)
int residual_fp64(bem_ctx* c, const double* A, int64_t lda, int n, const double* x, const double* b,
                  double* r, double* norms /* host: [0]=|r|inf [1]=|x|inf [2]=|b|inf [3]=|A|inf */,
                  bool want_anorm, bool extended = false);

// C (M x N, ldc) op= A (M x K, lda) * B (K x N, ldb), column-major; op: 0 -=, 1 =.
template <typename T>
int gemm(bem_ctx* c, int M, int N, int K, const T* A, int64_t lda, const T* B, int64_t ldb, T* C,
         int64_t ldc, int mode);

}  // namespace bem
