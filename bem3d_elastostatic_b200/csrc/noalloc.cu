// bem_dgesv_noalloc: the dense FP64 solve on caller-owned device buffers without any
// device allocation.
//
// Some callers cannot allocate device memory at the point where they need a solve:
// a Fortran or C host that hands over pre-allocated device buffers from its own
// memory pool and forbids the library from growing the footprint; a time-stepping
// or adjoint loop that must not pay for cudaMalloc/cudaFree (both may synchronise the
// whole device); an application that runs under a fixed memory budget set at start
// up.  For them this entry point takes its scratch (the panel kernel's candidate
// exchange and grid-barrier words, the TRSM inverse, the TRSM buffer, the triangular
// sweeps' gather buffer and flags, and the pivot permutation) from one file-scope
// __device__ array of kNoAllocBytes (4.3 MiB), sized for systems of order up to
// kNoAllocMaxN = 4096.
//
// Rules that follow from the shared static array:
//   * every GPU that loads the library holds the array until the process exits;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current), so make that
//     first call before any stream capture;
//   * all calls share the array and it keeps the last call's contents: the barrier
//     counter and status words are cleared by every call, and calls that overlap on
//     the GPU (different streams or host threads) race on it and must be serialised
//     by the caller.
// The call synchronises `stream` (it reads the factorisation's status words and
// composes the pivot gather on the host).  Like bem_dgesv, the factors are those of
// A^T in A's storage and d_ipiv is dgetrf's pivot sequence of A^T (see lu.cuh): the
// solution of A X = B is exact LAPACK semantics, a reuse of dA/d_ipiv with dgetrs is
// not.  When the factorisation itself fails (a negative status) d_ipiv is undefined;
// otherwise it is 1-based on return, including an info > 0 return and a failed solve.
#include <algorithm>
#include <atomic>
#include <cstdio>

#include "lu.cuh"

namespace {

constexpr int kNoAllocMaxN = 4096;
constexpr int kNoAllocNb = 128;
constexpr int kNoAllocGmax = 160;  // >= the SM count of a B200 (148)
constexpr size_t up256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kFactorBytes = up256(2 * kNoAllocGmax * sizeof(double)) + up256(2 * kNoAllocGmax * sizeof(int)) +
                                up256(2 * (size_t)kNoAllocGmax * bem::kPanelW * 8) +
                                up256(2 * (size_t)bem::kPanelW * 8) + up256(16) +
                                up256((size_t)kNoAllocNb * kNoAllocNb * 8) +
                                up256((size_t)kNoAllocMaxN * kNoAllocNb * 8);
constexpr size_t kSolveDoubles = ((size_t)kNoAllocMaxN + 127) / 128 * 256 + 256;
constexpr size_t kPermBytes = up256((size_t)kNoAllocMaxN * sizeof(int));
constexpr size_t kNoAllocBytes = kFactorBytes + up256(kSolveDoubles * sizeof(double)) + kPermBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
// the array's device address per device (atomic: host threads may call on different
// devices at the same time; two threads that race on one device store the same value)
std::atomic<void*> g_scratch_addr[kMaxDevices];

__global__ void one_based_kernel(int n, int* ipiv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ipiv[i] += 1;
}

}  // namespace

extern "C" int bem_dgesv_noalloc(int n, int nrhs, double* dA, int lda, int* d_ipiv, double* dB, int ldb,
                                 int* info, void* stream) {
  if (n > kNoAllocMaxN) return BEM_ERR_TOO_LARGE;
  if (n <= 0 || nrhs < 0 || lda < n || ldb < n || !dA || !d_ipiv || (nrhs > 0 && !dB) || !info)
    return BEM_ERR_ARG;
  *info = 0;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return BEM_ERR_CUDA;
  if (!g_scratch_addr[dev].load(std::memory_order_acquire)) {
    // set-up, once per device with that device current: the host-side symbol is only
    // a stand-in, the kernels need the array's device address
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return BEM_ERR_CUDA;
    g_scratch_addr[dev].store(p, std::memory_order_release);
  }
  unsigned char* base = static_cast<unsigned char*>(g_scratch_addr[dev].load(std::memory_order_acquire));
  if (bem::lu_workspace_bytes(n, kNoAllocNb, kNoAllocGmax, sizeof(double)) > kFactorBytes) return BEM_ERR_TOO_LARGE;

  // a context on the stack: no device memory of its own (its buffers stay empty)
  bem_ctx c;
  c.device = dev;
  c.stream = static_cast<cudaStream_t>(stream);
  cudaDeviceGetAttribute(&c.sm_count, cudaDevAttrMultiProcessorCount, dev);
  // the candidate exchange of the panel launches is carved for kNoAllocGmax CTAs: every
  // grid sized from the SM count stays within it on a part with more SMs
  c.sm_count = std::min(c.sm_count, kNoAllocGmax);
  const bem::LUWorkspace ws = bem::lu_workspace_carve(base, n, kNoAllocNb, kNoAllocGmax, sizeof(double));
  double* solve_work = reinterpret_cast<double*>(base + kFactorBytes);
  int* perm = reinterpret_cast<int*>(base + kFactorBytes + up256(kSolveDoubles * sizeof(double)));
  int rc = bem::lu_factor_ws<double>(&c, dA, lda, n, d_ipiv, perm, kNoAllocNb, info, ws);
  if (rc) return rc;  // the factorisation failed: d_ipiv is undefined
  // from here on the pivots are complete: they are made 1-based on every return path
  if (*info == 0)
    for (int j = 0; j < nrhs && rc == 0; ++j)
      rc = bem::lu_solve_ws<double>(&c, dA, lda, n, perm, dB + (int64_t)j * ldb, solve_work);
  one_based_kernel<<<(n + 255) / 256, 256, 0, c.stream>>>(n, d_ipiv);
  if (cudaGetLastError() != cudaSuccess) return BEM_ERR_CUDA;
  return rc ? rc : *info;
}
