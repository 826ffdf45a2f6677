/*
 * bem3d_b200.h — C ABI of the B200-native (sm_100a) QUADESTH boundary-element hot path.
 *
 * Every entry point takes plain pointers and sizes and returns an int status.  The
 * reference exposes its hot path as Fortran module procedures working on module
 * globals (data_mod.f90:37-52); each function below names the procedure it stands
 * in for.  A Fortran caller binds them with ISO_C_BINDING (include/assembly_gpu_mod.f90
 * holds the interface block); Python binds them with ctypes
 * (bem3d_elastostatic_b200/_lib.py).
 *
 * Data contract (identical to the reference's globals):
 *   x, y, z       (n) node coordinates
 *   nconec        (ne) nodes per element: 9 = quad9, 6 = tri6
 *   kconec        (9, ne) column-major, 1-based node numbers
 *   kode          (3*ne) per element and component: 0 = displacement prescribed,
 *                 1 = traction prescribed
 *   bc            (27, ne) column-major, value of component ld at local node k is
 *                 bc(3*(k-1)+ld, e)
 *   A             (3n, 3n) column-major, leading dimension lda
 *   FI            (3n); DFI (27, ne)
 *   u_int (3,l), sigma_int (6,l) ordered xx,yy,zz,xy,yz,zx, prin (3,l), vm (l)
 *
 * Status: 0 = success; > 0 = the LU met an exactly zero pivot at that 1-based step
 * (the DGESV info convention); < 0 = one of the BEM_ERR_* codes.  Host pointers may be
 * NULL where marked "nullable": the data then stays resident on the device.
 * One CUDA stream per context; a context is not re-entrant.
 */
#ifndef BEM3D_B200_H
#define BEM3D_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bem_ctx bem_ctx;

#define BEM_OK 0
#define BEM_ERR_ARG (-1)      /* bad argument or size */
#define BEM_ERR_CUDA (-2)     /* a CUDA call failed */
#define BEM_ERR_OOM (-3)      /* device allocation failed */
#define BEM_ERR_TIMEOUT (-4)  /* a bounded device wait ran out (grid barrier) */
#define BEM_ERR_STATE (-5)    /* called out of order (e.g. solve before ghmat8) */
#define BEM_ERR_MESH (-6)     /* a node lies in more than 8 elements, bad connectivity */
#define BEM_ERR_NOCONV (-7)   /* refinement did not reach the requested tolerance */
#define BEM_ERR_TOO_LARGE (-8) /* order above the limit of bem_dgesv_noalloc (4096) */

/* Solve precision modes (bem_solve). */
#define BEM_PREC_FP64 0      /* FP64 LU with partial pivoting: the DGESV replacement */
#define BEM_PREC_FP32_IR 1   /* FP32 LU whose trailing update runs on the tensor cores as a
                                three-term BF16 split (FP32-grade products, FP32
                                accumulation) + FP64 iterative refinement */
#define BEM_PREC_BF16_IR 2   /* LU of an equilibrated FP32 copy (power-of-two row and column
                                scales) whose trailing updates run on the tcgen05 tensor
                                cores as one BF16 product with FP32 accumulation (the
                                panel and TRSM GEMMs keep the three-term split), + GMRES-IR
                                in FP64 with that LU as preconditioner */

#define BEM_PREC_FP64_IR 3   /* FP64 LU (partial pivoting) of a copy of A, + refinement with
                                extended-precision residuals: the solution of the stored
                                FP64 system to FP64 rounding, whatever its conditioning
                                (LAPACK's extra-precise refinement, xGERFSX, in kind) */

/* Assembly precision modes (bem_ghmat8). */
#define BEM_ASM_FP64 0  /* every element integral in FP64 (parity with the reference) */
#define BEM_ASM_FP32_FAR 1 /* far-field integrals in FP32, near-singular and singular in FP64 */

/* Internal-point flags (bem_internal_points). */
#define BEM_IP_KELVIN_CONSISTENT 1 /* use T*_ij u_j in the displacement identity; clear =
                                      the reference's stress_mod.f90:838-843 form */

/* Pivoting of the low-precision factorisation of the *_IR modes (BEM_OPT_PIVOTING).
 * BEM_PREC_FP64 always pivots partially (DGESV). */
#define BEM_PIVOT_WINDOW 1  /* default: the pivot search of each 32-wide sub-panel is
                               restricted to its 32 x 32 diagonal block (a warp-level
                               search, no grid-wide exchange per pivot); a zero pivot or a
                               refinement that does not converge repeats the solve with
                               partial pivoting */
#define BEM_PIVOT_PARTIAL 0 /* partial pivoting over every remaining row */

typedef struct {
  int iterations;        /* refinement sweeps (IR) or GMRES iterations */
  int restarts;          /* GMRES restarts */
  double rel_residual;   /* ||b - A x|| / (||A||_inf ||x|| + ||b||), FP64 */
  double factor_seconds; /* device time of the factorisation */
  double refine_seconds; /* device time of the refinement */
  double gflops;         /* 2/3 N^3 / factor_seconds */
  int pivoting;          /* BEM_PIVOT_* of the factorisation that produced the solution */
  int fallbacks;         /* window-pivoted attempts repeated with partial pivoting */
} bem_solve_info;

/* Context ------------------------------------------------------------------------ */
int bem_ctx_create(bem_ctx** ctx, int device);
int bem_ctx_destroy(bem_ctx* ctx);
const char* bem_last_error(const bem_ctx* ctx);
/* sync the context's stream; returns a pending asynchronous error, if any */
int bem_sync(bem_ctx* ctx);
/* the context's CUDA stream (a cudaStream_t), for callers that time or order work */
int bem_get_stream(bem_ctx* ctx, void** stream);

/* Context options (no counterpart in the reference).
 *   BEM_OPT_PIVOTING        BEM_PIVOT_WINDOW (default) or BEM_PIVOT_PARTIAL for the
 *                           factorisations of the *_IR solve modes
 *   BEM_OPT_WAIT_LIMIT_MS   limit of every bounded device wait of the context's kernels
 *                           (grid barriers, triangular-sweep publications, tcgen05
 *                           mbarriers), 1..60000 ms, default 2000; a wait that runs out
 *                           ends its kernel and the call returns BEM_ERR_TIMEOUT
 *   BEM_OPT_RESIDUAL        1 (default): the refinement of the *_IR modes computes its
 *                           residuals b - A x in double-double (exact products, TwoSum
 *                           accumulation, one rounding) and iterates until the backward
 *                           error meets rel_tol and the last correction is below
 *                           max(rel_tol, 4 u) relative to x (u the unit roundoff), so at
 *                           the default tolerances the solution carries FP64 rounding
 *                           only; 0: FP64 residuals, stopping on the backward error
 *   BEM_OPT_WITHHOLD_BLOCK  failure injection for tests: the block-inverse triangular
 *                           sweep of the next solves does not publish this 128-row block
 *                           (-1, the default, publishes all), so that the waits for it run
 *                           out and the solve returns BEM_ERR_TIMEOUT with the context
 *                           still usable
 *   BEM_OPT_PANEL_WIDTH     panel width of the FP32 factorisations of the *_IR modes: a
 *                           multiple of 128 up to 1024, or 0 (default) for the mode's
 *                           own (1024 for BEM_PREC_BF16_IR, 512 for BEM_PREC_FP32_IR) */
#define BEM_OPT_PIVOTING 1
#define BEM_OPT_WAIT_LIMIT_MS 2
#define BEM_OPT_WITHHOLD_BLOCK 3
#define BEM_OPT_RESIDUAL 4
#define BEM_OPT_PANEL_WIDTH 5
int bem_set_option(bem_ctx* ctx, int option, int64_t value);

/* Input: replaces input_data (io_mod.f90:36-146) and update_material_constants
 * (data_mod.f90:97-108).  Node -> element adjacency (io_mod.f90:125-135) is built here;
 * a node in more than 8 elements is rejected (BEM_ERR_MESH). */
int bem_set_mesh(bem_ctx* ctx, int n, int ne, const double* x, const double* y,
                 const double* z, const int* nconec, const int* kconec);
int bem_set_material(bem_ctx* ctx, double mu, double nu);
int bem_set_bc(bem_ctx* ctx, const int* kode, const double* bc);
/* Pinned displacement DOFs (0-based 3*(node-1)+comp) held at 0: row := unit row,
 * rhs := 0 after assembly.  No counterpart in the reference (supports there are per
 * element); used by the uniaxial-cube and sphere workloads. */
int bem_set_pins(bem_ctx* ctx, int npins, const int* dofs);

/* precompute_element_geometry (assembly_mod.f90:28-51) with etaxja (:225-337).
 * Optional host copies of the tables in the reference's layout (nullable each):
 * eta1..3, xja, xg1..3 as (36, ne), ff as (9, 36, ne). */
int bem_precompute_geometry(bem_ctx* ctx);
int bem_get_geometry(bem_ctx* ctx, double* eta1, double* eta2, double* eta3, double* xja,
                     double* xg1, double* xg2, double* xg3, double* ff);

/* ghmat8 (assembly_mod.f90:53-223): assembles A and FI on the device (column swap,
 * rigid-body diagonal).  A_out/FI_out (nullable) receive host copies; lda >= 3n. */
int bem_ghmat8(bem_ctx* ctx, int asm_precision, double* A_out, int64_t lda, double* FI_out);

/* A dense system of any order n (A column-major with leading dimension lda >= n, and
 * its right-hand side FI), copied to the device in place of an assembled one, for
 * bem_solve: the reference's solve_linear_system(A_mat, B_vec, n_size)
 * (solver_mod.f90:17) takes any system.  The phases that need the mesh's system
 * (bem_reorganize, stresses, adjoint) refuse it (BEM_ERR_STATE). */
int bem_set_system(bem_ctx* ctx, int n, const double* A, int64_t lda, const double* FI);

/* Rows [r0, r1) of the assembled A (into A_rows, (r1 - r0) x 3n, leading dimension
 * ld >= r1 - r0) and of FI (FI_rows, nullable), copied from the device: a slice for
 * parity checks at orders whose A does not fit in host memory.  No counterpart in the
 * reference.  A must not have been overwritten by a BEM_PREC_FP64 factorisation (the
 * *_IR modes factor a copy). */
int bem_get_rows(bem_ctx* ctx, int r0, int r1, double* A_rows, int64_t ld, double* FI_rows);

/* H (3n x 3n, rigid-body diagonal included) and G (3n x 27ne) for collocation nodes
 * [in0, in1) — the two products ghmat8 combines, for entrywise parity checks. */
int bem_get_hg(bem_ctx* ctx, int in0, int in1, double* H, int64_t ldh, double* G,
               int64_t ldg);

/* solve_linear_system (solver_mod.f90:17-36): solves A x = FI in place on the device.
 * BEM_PREC_FP64 factors A itself (as DGESV overwrites it); the *_IR modes factor a
 * lower-precision copy and refine against the FP64 A to rel_tol.  *info follows DGESV
 * (0, or the 1-based step of an exactly zero pivot).  FI_inout (nullable) receives the
 * solution on the host.  stats (nullable) receives iteration counts and timings. */
int bem_solve(bem_ctx* ctx, int precision, double rel_tol, int max_iter, double* FI_inout,
              int* info, bem_solve_info* stats);

/* LAPACK dgesv drop-in on host buffers (solver_mod.f90:28): A (n x n, lda) is
 * overwritten by its factors, B (n x nrhs, ldb) by the solution; ipiv receives the
 * 1-based pivot sequence of the factorisation (pivoting over the rows of A^T: see the
 * header of lu.cu).  Runs on the context's device. */
int bem_dgesv(bem_ctx* ctx, int n, int nrhs, double* A, int lda, int* ipiv, double* B,
              int ldb, int* info);

/* No counterpart in the reference.  The dgesv solve on caller-owned DEVICE buffers
 * that performs no device allocation, for callers that cannot allocate at the point
 * of the solve (a host that owns all device memory through its own pool, a loop that
 * must not pay for cudaMalloc/cudaFree synchronisation, a fixed memory budget).  Its
 * scratch is one static 4.3 MiB device array per GPU, which limits n to 4096
 * (larger n returns BEM_ERR_TOO_LARGE).  As in bem_dgesv, dA (n x n, lda) is
 * overwritten by the factors of A^T in A's storage and d_ipiv (n ints) by dgetrf's
 * 1-based pivot sequence of A^T (pivoting over the rows of A^T: see the header of
 * lu.cu), so dA/d_ipiv are not dgetrs input for A; dB (n x nrhs, ldb) receives the
 * solution of A X = B and *info (host) follows DGESV.  d_ipiv is undefined when the
 * call returns an error before the factorisation completed.  Work is queued on
 * `stream` (a cudaStream_t, 0 = legacy default stream); the call synchronises that
 * stream to read the factorisation's status.  The first call on a device sets up the
 * array's device address: make it before any stream capture.  All calls share the
 * array: calls that overlap on the GPU race and must be serialised. */
int bem_dgesv_noalloc(int n, int nrhs, double* dA, int lda, int* d_ipiv, double* dB, int ldb,
                      int* info, void* stream);

/* reorganize_solution (io_mod.f90:148-183): FI -> nodal displacements u (3n),
 * DFI (27, ne) element-nodal tractions.  Host outputs nullable. */
int bem_reorganize(bem_ctx* ctx, double* FI_out, double* DFI_out);

/* Adjoint (no counterpart in the reference).  bem_solve_transposed solves A^T y = g
 * (g: host, 3n, overwritten by y) with the factors of the last BEM_PREC_FP64 bem_solve.
 * bem_adjoint_gradient returns, for lambda (host, 3n), the derivative of
 * R = lambda^T (FI - A x) at the current solution x with respect to the node
 * coordinates, grad_xyz (3n: x, y, z of node 1, ...), and to the material, grad_mat
 * ([d/dmu, d/dnu]), without forming dA/dX.  With lambda = A^{-T} dJ/dx this is the
 * implicit part of dJ/dX for any objective J(x, X); pinned rows carry no geometry and
 * their lambda is ignored.  9-node elements. */
int bem_solve_transposed(bem_ctx* ctx, double* g);
int bem_adjoint_gradient(bem_ctx* ctx, const double* lambda, double* grad_xyz, double* grad_mat);

/* compute_boundary_stresses (stress_mod.f90:119-406): traction-recovery stresses at
 * every node of every element, sigma_elem (6, 9, ne) (nullable), their average over
 * each node's elements, sigma_node (6, n), and the nodal principal (3, n) and von
 * Mises (n) stresses; order xx, yy, zz, xy, yz, zx.  Needs a solved system (it
 * reorganizes the current solution itself). */
int bem_boundary_stresses(bem_ctx* ctx, double* sigma_elem, double* sigma_node,
                          double* prin, double* vm);

/* compute_internal_points (stress_mod.f90:511-886): Somigliana displacement and stress
 * with calc_principal_and_vm (:299-359) at l points.  flags: BEM_IP_*. */
int bem_internal_points(bem_ctx* ctx, int l, const double* cx, const double* cy,
                        const double* cz, double* u_int, double* sigma_int, double* prin,
                        double* vm, int flags);

/* Batches of small systems (no counterpart in the reference, which solves one system
 * per run).  Each system is a boundary mesh of its own (size, material, supports) with
 * nrhs load cases: nrhs sets of prescribed values bc (27 x ne each, consecutive), the
 * same kode.  The systems are assembled together (one geometry launch, one persistent
 * work-queue launch for the regular pairs, one for the singular ones) and solved
 * together (one CTA per system: LU, substitution for all load cases, FP64 residual),
 * the solve captured once in a CUDA graph.  A node's prescribed displacement must be
 * the same in every element that prescribes it (BEM_ERR_MESH otherwise). */
typedef struct bem_batch bem_batch;

typedef struct {
  int systems;                 /* systems in the batch */
  int sweeps;                  /* refinement sweeps in the solve graph (0 for FP64) */
  int converged;               /* systems whose backward error reached tol */
  int singular;                /* systems with an exactly zero pivot */
  double max_backward_error;   /* over the systems and their load cases */
  double solve_seconds;        /* device time of the whole solve (factor + sweeps) */
  int lu_threads;              /* CTA size of the per-system LU picked by the autotuner */
  float lu_ms_256, lu_ms_512;  /* the autotuner's timings of one batch LU */
} bem_batch_info;

int bem_batch_create(bem_batch** batch, int device);
int bem_batch_destroy(bem_batch* batch);
const char* bem_batch_last_error(const bem_batch* batch);
/* adds one system (arguments as bem_set_mesh / bem_set_material / bem_set_bc /
 * bem_set_pins; bc holds nrhs load cases, nrhs <= 8 and the same for every system);
 * returns the system's index (>= 0) or an error (< 0) */
int bem_batch_add(bem_batch* batch, int n, int ne, const double* x, const double* y,
                  const double* z, const int* nconec, const int* kconec, double mu, double nu,
                  const int* kode, int nrhs, const double* bc, int npins, const int* pins);
/* geometry, H and G, then A and FI of every system */
int bem_batch_assemble(bem_batch* batch);
/* solve every system for all its load cases: BEM_PREC_FP64 (FP64 LU) or
 * BEM_PREC_FP32_IR (FP32 LU, then max_iter FP64 refinement sweeps; a system stops
 * once its backward error is <= tol or a sweep gains less than 10 %).  Order <= 25,600. */
int bem_batch_solve(bem_batch* batch, int precision, double tol, int max_iter,
                    bem_batch_info* info);
/* system i: its solution x (3n x nrhs, column-major), its A (3n x 3n) and FI (3n x nrhs) */
int bem_batch_get_solution(bem_batch* batch, int i, double* x);
int bem_batch_get_system(bem_batch* batch, int i, double* A, double* FI);
/* kernels the batch launched so far (graph launches counted by their kernels) */
long long bem_batch_launches(const bem_batch* batch);

/* Profiling of the library's own kernels.  bem_profile_begin zeroes the counters;
 * with timing = BEM_PROF_PHASES the LU phases are bracketed by CUDA events on the
 * context's stream (the stream every kernel of the context runs on); with
 * BEM_PROF_TRAILING only the trailing updates of every 16th panel are (a sample with
 * little disturbance of the run: events between all launches slow it down).  bem_profile_end syncs the stream and reports.  Trailing flops/bytes are the algorithmic work of the trailing-update
 * GEMMs: 2*m*m*nb flops and the C read+write plus one read of each operand. */
#define BEM_PROF_COUNT 0     /* launch counts only */
#define BEM_PROF_PHASES 1    /* every LU phase timed */
#define BEM_PROF_TRAILING 2  /* a sample of the trailing updates timed */

typedef struct {
  long long kernel_launches;    /* kernels this context launched */
  double lu_panel_ms;           /* cooperative panel factorisation */
  double lu_swap_ms;            /* row interchanges outside the panel */
  double lu_panel_update_ms;    /* TRSM + GEMM inside the panel */
  double lu_trsm_ms;            /* TRSM of the block row (inverse + GEMM) */
  double lu_trailing_ms;        /* trailing-matrix GEMM */
  long long lu_trailing_launches;
  double lu_trailing_flops;
  double lu_trailing_bytes;
  /* internal points (every bem_internal_points* call while profiling): points, points
   * with a near element, and the kernel evaluations (point x table point) of the far
   * (element Gauss points) and near (40 x 40) quadratures */
  long long ip_points;
  long long ip_near_points;
  double ip_far_evals;
  double ip_near_evals;
} bem_profile;
int bem_profile_begin(bem_ctx* ctx, int timing);
int bem_profile_end(bem_ctx* ctx, bem_profile* out);

/* Device-resident variants for callers that keep data in HBM (the Python layer and
 * the benchmark).  Pointers are device addresses. */
int bem_device_state(bem_ctx* ctx, double** A, int64_t* lda, double** FI, double** DFI);
int bem_internal_points_device(bem_ctx* ctx, int l, const double* d_cx, const double* d_cy,
                               const double* d_cz, double* d_u_int, double* d_sigma_int,
                               double* d_prin, double* d_vm, int flags);

#ifdef __cplusplus
}
#endif

#endif /* BEM3D_B200_H */
