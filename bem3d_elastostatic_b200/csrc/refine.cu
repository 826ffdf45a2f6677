// Mixed-precision solve (FP32 factors + FP64 iterative refinement against the FP64
// A) and reorganize_solution (io_mod.f90:148-183).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <vector>

#include "lu.cuh"

namespace bem {

constexpr int kNbMixed = 256;  // panel width of the FP32 factorisation (halves the trailing C traffic)

__global__ void to_fp32_kernel(const double* A, int64_t lda, int n, float* A32) {
  const int64_t total = (int64_t)lda * n;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
    A32[i] = (float)A[i];
}

__global__ void axpy_kernel(int n, const double* d, double* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += d[i];
}

int solve_mixed(bem_ctx* c, int precision, double rel_tol, int max_iter, bem_solve_info* st, int* info) {
  const int n = 3 * c->n;
  const int64_t lda = c->lda;
  *info = 0;
  if (c->factored_fp64) return bem_fail(c, BEM_ERR_STATE, "A was overwritten by an FP64 factorisation");
  if (c->A32.count != (size_t)(lda * n)) {
    c->A32.release();
    cudaError_t e = c->A32.alloc((size_t)(lda * n));
    if (e != cudaSuccess) return bem_fail(c, BEM_ERR_OOM, "allocating the FP32 factor copy");
  }
  BEM_CUDA(c, c->piv.alloc(n));
  DBuf<double> r, d;
  BEM_CUDA(c, r.alloc(n));
  BEM_CUDA(c, d.alloc(n));
  {
    // one workspace for the triangular solves and the residual, sized once
    const size_t nchunk = ((size_t)n + 511) / 512;
    const size_t need = std::max(((size_t)n + 127) / 128 * 256 + 256, nchunk * n * 2 + 8);
    if (c->work.count < need) {
      c->work.release();
      BEM_CUDA(c, c->work.alloc(need));
    }
  }
  cudaEvent_t e0, e1, e2;
  BEM_CUDA(c, cudaEventCreate(&e0));
  BEM_CUDA(c, cudaEventCreate(&e1));
  BEM_CUDA(c, cudaEventCreate(&e2));
  BEM_CUDA(c, cudaEventRecord(e0, c->stream));
  to_fp32_kernel<<<c->sm_count * 8, 256, 0, c->stream>>>(c->A.p, lda, n, c->A32.p);
  BEM_LAUNCH_CHECK(c);
  const int saved = c->f32_gemm;
  if (c->f32_gemm_override >= 0)
    c->f32_gemm = c->f32_gemm_override;
  else
    c->f32_gemm = (precision == BEM_PREC_BF16_IR) ? 1 : 4;
  int rc = lu_factor<float>(c, c->A32.p, lda, n, c->piv.p, kNbMixed, info);
  c->f32_gemm = saved;
  if (rc) return rc;
  BEM_CUDA(c, cudaEventRecord(e1, c->stream));
  if (*info != 0) return BEM_OK;
  // x0 = LU^{-1} b, then x += LU^{-1} (b - A x)
  BEM_CUDA(c, cudaMemsetAsync(c->X.p, 0, n * sizeof(double), c->stream));
  BEM_CUDA(c, cudaMemcpyAsync(r.p, c->FI.p, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  double norms[4] = {0, 0, 0, 0};
  double anorm = -1.0, berr = 1.0, prev = 1e300;
  int it = 0;
  const bool ir_prof = getenv("BEM_IR_PROFILE") != nullptr;
  cudaEvent_t q0, q1, q2;
  if (ir_prof) {
    cudaEventCreate(&q0);
    cudaEventCreate(&q1);
    cudaEventCreate(&q2);
  }
  for (it = 1; it <= max_iter; ++it) {
    if (ir_prof) cudaEventRecord(q0, c->stream);
    BEM_CUDA(c, cudaMemcpyAsync(d.p, r.p, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    if ((rc = lu_solve<float>(c, c->A32.p, lda, n, c->piv.p, kNbMixed, d.p))) return rc;
    axpy_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(n, d.p, c->X.p);
    BEM_LAUNCH_CHECK(c);
    if (ir_prof) cudaEventRecord(q1, c->stream);
    if ((rc = residual_fp64(c, c->A.p, lda, n, c->X.p, c->FI.p, r.p, norms, anorm < 0))) return rc;
    if (ir_prof) {
      cudaEventRecord(q2, c->stream);
      cudaEventSynchronize(q2);
      float a = 0.f, b2 = 0.f;
      cudaEventElapsedTime(&a, q0, q1);
      cudaEventElapsedTime(&b2, q1, q2);
      fprintf(stderr, "[ir it=%d] lu-solve %.2f ms residual %.2f ms\n", it, a, b2);
    }
    if (anorm < 0) anorm = norms[3];
    berr = norms[0] / (anorm * norms[1] + norms[2]);
    if (!(berr == berr)) break;  // NaN: diverged
    if (berr <= rel_tol) break;
    if (berr > 0.5 * prev && it > 3) break;  // stagnation
    prev = berr;
  }
  BEM_CUDA(c, cudaEventRecord(e2, c->stream));
  BEM_CUDA(c, cudaEventSynchronize(e2));
  float f_ms = 0.f, r_ms = 0.f;
  cudaEventElapsedTime(&f_ms, e0, e1);
  cudaEventElapsedTime(&r_ms, e1, e2);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  if (st) {
    st->iterations = std::min(it, max_iter);
    st->restarts = 0;
    st->rel_residual = berr;
    st->factor_seconds = f_ms * 1e-3;
    st->refine_seconds = r_ms * 1e-3;
    st->gflops = f_ms > 0 ? (2.0 / 3.0) * (double)n * n * n / (f_ms * 1e-3) * 1e-9 : 0.0;
  }
  // Stagnation at the FP64 working-precision floor counts as converged: a requested
  // tolerance below ~1e-14 is met "to working precision".
  if (!(berr <= std::max(rel_tol, 1e-14)))
    return bem_fail(c, BEM_ERR_NOCONV, "refinement did not reach the tolerance");
  return BEM_OK;
}

// reorganize_solution: DFI(3k+ld, e) = x(3ik+ld) * mu where u is prescribed on the
// element, else the prescribed traction; FI(3i+ld) = prescribed u where an adjacent
// element prescribes it (first in ke order: the uknown/vp lookup), else x.
__global__ void reorganize_dfi_kernel(int ne, const int* nconec, const int* kconec, const int* kode,
                                      const double* bc, const double* X, double mu, double* DFI) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 27 * (int64_t)ne) return;
  const int e = (int)(i / 27), q = (int)(i % 27), k = q / 3, ld = q % 3;
  double v = 0.0;
  if (k < nconec[e]) {
    if (kode[3 * e + ld] == 0)
      v = X[3 * (int64_t)(kconec[k + 9 * e] - 1) + ld] * mu;
    else
      v = bc[i];
  }
  DFI[i] = v;
}

__global__ void reorganize_fi_kernel(int n3, const int* uknown, const double* vp, const double* X, double* FI) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) FI[i] = uknown[i] ? vp[i] : X[i];
}

int launch_reorganize(bem_ctx* c) {
  BEM_CUDA(c, c->DFI.alloc(27 * (size_t)c->ne));
  const int64_t nd = 27 * (int64_t)c->ne;
  reorganize_dfi_kernel<<<(unsigned)((nd + 255) / 256), 256, 0, c->stream>>>(c->ne, c->nconec.p, c->kconec.p,
                                                                             c->kode.p, c->bc.p, c->X.p, c->mat.mu,
                                                                             c->DFI.p);
  BEM_LAUNCH_CHECK(c);
  const int n3 = 3 * c->n;
  BEM_CUDA(c, c->U.alloc(n3));
  reorganize_fi_kernel<<<(n3 + 255) / 256, 256, 0, c->stream>>>(n3, c->uknown.p, c->vp.p, c->X.p, c->U.p);
  BEM_LAUNCH_CHECK(c);
  return BEM_OK;
}

}  // namespace bem
