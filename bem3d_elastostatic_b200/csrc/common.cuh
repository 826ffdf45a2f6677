// Shared definitions of the B200 QUADESTH library: the context, status handling,
// quadrature constants and device helpers (shape functions, Kelvin constants).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#include "../../include/bem3d_b200.h"

namespace bem {

// assembly_mod.f90:6-19 — the reference's literal quadrature constants (15 and 10
// significant digits); parity needs these values, not freshly computed nodes.
constexpr double kGiQuad[6] = {0.238619186083197, -0.238619186083197, 0.661209386466265,
                               -0.661209386466265, 0.932469514203152, -0.932469514203152};
constexpr double kOmeQuad[6] = {0.467913934572691, 0.467913934572691, 0.360761573048139,
                                0.360761573048139, 0.171324492379170, 0.171324492379170};
constexpr double kRrTri[4] = {0.0694318422, 0.3300094782, 0.6699905218, 0.9305681558};
constexpr double kSsTri[4] = {0.0571041961, 0.2768430136, 0.5835904324, 0.8602401357};
constexpr double kOmeiTri[4] = {0.1739274226, 0.3260725774, 0.3260725774, 0.1739274226};
constexpr double kOmejTri[4] = {0.1355069134, 0.2034645680, 0.1298475476, 0.0311809709};
// data_mod.f90:7
constexpr double kPi = 3.14159265358979323846;

// Per-element packed quadrature table used by the assembly kernels: 36 Gauss points
// x {x, y, z, n1, n2, n3} followed by p12[36][9] = N_k * J * w_i * w_j
// (assembly_mod.f90:363-369).  540 doubles = 4320 bytes per element.
constexpr int kGp = 36;
constexpr int kTabGeo = 6 * kGp;
constexpr int kTabStride = kTabGeo + 9 * kGp;

// Element schedule for the conflict-free assembly: batches of up to kBatch elements
// that share no node.
constexpr int kBatch = 8;

struct Material {
  double mu, nu;
  double c3, c4, c5, c6;  // data_mod.f90:104-107
};

inline Material make_material(double mu, double nu) {
  Material m;
  m.mu = mu;
  m.nu = nu;
  m.c3 = 1.0 / (16.0 * kPi * (1.0 - nu) * mu);
  m.c4 = 3.0 - 4.0 * nu;
  m.c5 = -1.0 / (8.0 * kPi * (1.0 - nu));
  m.c6 = 1.0 - 2.0 * nu;
  return m;
}

// Device buffer with RAII release.
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t count = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    count = 0;
  }
  cudaError_t alloc(size_t n) {
    if (n == count && p) return cudaSuccess;
    release();
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    count = n;
    return cudaSuccess;
  }
  size_t bytes() const { return count * sizeof(T); }
};

// One-time set-up that CUDA keeps per device (kernel attributes, __constant__ tables),
// tracked per device so that a process driving several GPUs sets up each of them:
// `static DeviceOnce s; if (s.pending()) { ...; s.mark(); }` with the device current.
inline int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d & 63;
}
// The bits are atomic: host threads that set up different devices at the same time
// each keep their bit (a lost bit would only repeat the set-up, but a plain
// read-modify-write from several threads is a data race).
struct DeviceOnce {
  std::atomic<unsigned long long> bits{0};
  bool pending() const { return ((bits.load(std::memory_order_acquire) >> current_device()) & 1ull) == 0; }
  void mark() { bits.fetch_or(1ull << current_device(), std::memory_order_acq_rel); }
};

// A factorisation's launch sequence captured as a CUDA graph and replayed while every
// pointer and size it was captured with (the key) is unchanged, so that the ~10^4
// launches of a large factorisation neither wait on the host nor pay per-launch costs.
// The profile events the capture recorded are kept to be read after each replay.
struct LUGraph {
  cudaGraphExec_t exec = nullptr;
  std::vector<long long> key;
  struct Ev {
    int phase, a, b;
    double flops, bytes;
  };
  std::vector<Ev> ev;
  long long launches = 0;  // kernels per replay
  void reset() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    key.clear();
    ev.clear();
    launches = 0;
  }
  ~LUGraph() { reset(); }
};

}  // namespace bem

// The opaque context behind bem_ctx*.
struct bem_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  // a second stream for independent work inside a factorisation (forked from and joined
  // back to `stream` by the two events; null: everything on `stream`)
  cudaStream_t aux_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  std::string last_error;
  int sm_count = 148;

  // mesh (host copies kept for the adjacency-derived tables)
  int n = 0, ne = 0;
  std::vector<int> h_nconec, h_kconec, h_kode;
  std::vector<double> h_bc;
  std::vector<int> h_nesim, h_ke;  // io_mod.f90:125-135
  bool have_mesh = false, have_bc = false, have_material = false;
  bem::Material mat{};

  bem::DBuf<double> x, y, z;
  bem::DBuf<int> nconec, kconec, kode;
  bem::DBuf<double> bc;
  bem::DBuf<int> ke;     // (8, n), 1-based element numbers, as the reference
  bem::DBuf<int> nesim;  // (n)
  // column-swap lookup (assembly_mod.f90:149-161, 194-206): per (node, ld) whether an
  // adjacent element prescribes u there and the value it prescribes
  bem::DBuf<int> uknown;
  bem::DBuf<double> vp;
  // conflict-free element schedule
  bem::DBuf<int> batches;
  int nbatches = 0;
  bem::DBuf<int> pins;
  int npins = 0;

  // geometry (reference layout) and the packed assembly table
  bem::DBuf<double> eta1, eta2, eta3, xja, xg1, xg2, xg3, ff, tab;
  bem::DBuf<double> erec;  // per-element boundary records of the assembly (mode A)
  // split last wave of the assembly: host copy of the batch list, the pieces' node
  // slots (built for tail_parts pieces, 0 = not built) and their scratch
  std::vector<int> h_batches;
  int tail_parts = 0, tail_cols = 0;
  bem::DBuf<int> tail_slot;
  bem::DBuf<double> tail_scr, tail_fd;
  bool have_geometry = false;

  // system
  bem::DBuf<double> A, FI, X, U, DFI;  // FI: rhs; X: solution; U, DFI: reorganized u, t
  int64_t lda = 0;
  int64_t nsys = 0;          // order of the system in A (3n after ghmat8, any n after set_system)
  bool mesh_system = false;  // A and FI come from ghmat8 on the current mesh
  bool have_system = false, have_solution = false, factored_fp64 = false;

  // LU / refinement workspace
  bem::DBuf<float> A32;
  bem::DBuf<int> piv;
  bem::DBuf<int> perm;  // gather form of the pivots of the latest factorisation (solve side)
  bem::DBuf<double> work;
  bem::DBuf<float> work32;
  bem::DBuf<unsigned int> sync;
  bem::DBuf<int> status;
  bem::DBuf<double> rowscale, colscale;
  // refinement vectors (residual, correction) and timing events, kept: allocation and
  // release next to a 10^10-byte system stalled the host for up to 0.7 s per solve
  bem::DBuf<double> ir_r, ir_d, ir_dmax;
  bem::DBuf<double> gm_V, gm_h, gm_part, gm_zero;  // GMRES-IR basis and reduction buffers
  bem::DBuf<double> A64f;     // FP64 factor copy of BEM_PREC_FP64_IR
  bool ext_residual = true;  // BEM_OPT_RESIDUAL: refinement residuals in double-double
  cudaEvent_t solve_ev[3] = {nullptr, nullptr, nullptr};
  // FP64 inverses of the 128 x 128 diagonal blocks of the latest factorisation (for the
  // block-inverse sweeps) and the sweeps' publication slots; dinv_src/n/lda/elem name
  // the factors the inverses belong to (cleared by every new factorisation)
  bem::DBuf<double> dinv;
  bem::DBuf<unsigned long long> slots;
  const void* dinv_src = nullptr;
  int dinv_n = 0, dinv_elem = 0;
  int64_t dinv_lda = 0;
  // factorisation workspace (kept, so that captured factorisations can be replayed)
  // and the captured factorisations, one per factor type (0 FP32, 1 FP64)
  bem::DBuf<unsigned char> lu_scratch[2];
  bem::LUGraph lu_graph[2][4];  // up to four captured variants per factor type
  int lu_graph_next[2] = {0, 0};  // the slot a new capture replaces when all are taken
  bool lu_graph_off = false;  // set when capture is unavailable (or BEM_LU_GRAPH=0)
  // GEMM flavour of the LU trailing update: f64_gemm 1 = DMMA tensor path, 0 = SIMT;
  // f32_gemm 4 = BF16 x3 split on tcgen05 for the trailing update (mma.sync elsewhere),
  // 3 = BF16 x3 split on mma.sync, 1 = plain BF16 (mma.sync), 0 = SIMT FP32
  int f64_gemm = 1;
  int f32_gemm = 4;
  // pivoting of the next factorisation: true = the pivot search of each 32-wide
  // sub-panel restricted to its diagonal block (the mixed-precision modes, with a
  // fallback to partial pivoting), false = partial pivoting (DGESV)
  bool lu_window = false;
  int pivot_pref = BEM_PIVOT_WINDOW;  // BEM_OPT_PIVOTING
  // bounded device waits (BEM_OPT_WAIT_LIMIT_MS), in ns, and the test-only withheld
  // sweep block (BEM_OPT_WITHHOLD_BLOCK, -1 = none)
  unsigned long long wait_ns = 2000000000ull;
  int withhold_block = -1;
  int panel_width = 0;  // FP32 factorisation panel width of the *_IR modes (0: the mode's own)
  int f32_gemm_override = -1;  // BEM_F32_GEMM environment override (0, 1, 3)
  // tcgen05 trailing update: BF16 hi/lo operand copies and its error word
  bem::DBuf<unsigned long long> ip_counters;  // internal points: far and near evaluations
  bem::DBuf<unsigned char> umma_buf;
  bem::DBuf<int> umma_err;
  // profiling (bem_profile_begin/end)
  long long launches = 0;
  int prof_timing = 0;
  bem_profile prof{};
  std::vector<cudaEvent_t> ev_pool;  // timing events of the LU phase profile, reused
  ~bem_ctx() {
    for (auto& t : lu_graph)
      for (auto& g : t) g.reset();
    for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : solve_ev)
      if (e) cudaEventDestroy(e);
  }
};

// Status helpers (host).
int bem_fail(bem_ctx* c, int code, const std::string& what);
int bem_cuda_fail(bem_ctx* c, cudaError_t e, const char* where);

#define BEM_CUDA(ctx, call)                                          \
  do {                                                               \
    cudaError_t _e = (call);                                         \
    if (_e != cudaSuccess) return bem_cuda_fail((ctx), _e, #call);   \
  } while (0)

#define BEM_LAUNCH_CHECK(ctx)                                               \
  do {                                                                      \
    ++(ctx)->launches;                                                      \
    cudaError_t _e = cudaGetLastError();                                    \
    if (_e != cudaSuccess) return bem_cuda_fail((ctx), _e, "kernel launch"); \
  } while (0)

// Internal (C++) entry points implemented in the .cu files.
namespace bem {
int launch_geometry(bem_ctx* c);
int launch_geometry_arrays(cudaStream_t stream, int ne, const double* x, const double* y, const double* z,
                           const int* nconec, const int* kconec, double* ref, double* tab);
int launch_ghmat8(bem_ctx* c, int precision);
int launch_hg(bem_ctx* c, int in0, int in1, double* dH, int64_t ldh, double* dG,
              int64_t ldg);
int lu_factor_fp64(bem_ctx* c, double* A, int64_t lda, int n, int* d_piv, int* info,
                   double* seconds);
int lu_solve_fp64(bem_ctx* c, const double* LU, int64_t lda, int n, double* b);
// the transposed system A^T y = b with the factors of lu_factor_fp64
int lu_solve_t_fp64(bem_ctx* c, const double* LU, int64_t lda, int n, double* b);
int solve_mixed(bem_ctx* c, int precision, double rel_tol, int max_iter,
                bem_solve_info* stats, int* info);
int launch_reorganize(bem_ctx* c);
int launch_boundary_stresses(bem_ctx* c, double* se, double* sn, double* pr, double* vm);
int launch_adjoint_gradient(bem_ctx* c, double* lam, double* grad, double* gmat);
int launch_internal_points(bem_ctx* c, int l, const double* cx, const double* cy,
                           const double* cz, double* u, double* s, double* pr, double* vm,
                           int flags);
}  // namespace bem
