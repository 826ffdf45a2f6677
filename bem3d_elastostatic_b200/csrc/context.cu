// C ABI of the library (include/bem3d_b200.h): context, input, phase entry points.
//
// The host work here is set-up of the kind the reference does while reading its
// input: the node -> element adjacency nesim/ke (io_mod.f90:125-135), the per
// (node, component) "displacement prescribed by a neighbour" lookup that ghmat8
// recomputes inside its hot loop (assembly_mod.f90:149-161, 194-206), and the
// conflict-free element schedule of the assembly kernel.  All numerics run on the GPU.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "common.cuh"

int bem_fail(bem_ctx* c, int code, const std::string& what) {
  if (c) c->last_error = what;
  return code;
}

int bem_cuda_fail(bem_ctx* c, cudaError_t e, const char* where) {
  std::string s = std::string(where) + ": " + cudaGetErrorString(e);
  if (c) c->last_error = s;
  return (e == cudaErrorMemoryAllocation) ? BEM_ERR_OOM : BEM_ERR_CUDA;
}

namespace {

// Greedy schedule: elements in index order (spatially coherent for structured
// meshes) go into the first of the recent not-full batches that holds none of their
// nodes, else open a new batch.  Elements of one batch therefore share no node.
void build_batches(int n, int ne, const std::vector<int>& nconec, const std::vector<int>& kconec,
                   std::vector<int>& out, int& nb) {
  std::vector<std::vector<int>> batches;
  std::vector<std::vector<int>> node_batches(n);  // batches touching each node (<= 8)
  std::vector<int> open;                          // not-full batches, newest last
  const size_t window = 32;
  for (int e = 0; e < ne; ++e) {
    int chosen = -1;
    for (int b : open) {
      bool clash = false;
      for (int m = 0; m < nconec[e] && !clash; ++m)
        for (int t : node_batches[kconec[m + 9 * e] - 1])
          if (t == b) {
            clash = true;
            break;
          }
      if (!clash) {
        chosen = b;
        break;
      }
    }
    if (chosen < 0) {
      chosen = (int)batches.size();
      batches.emplace_back();
      open.push_back(chosen);
      if (open.size() > window) open.erase(open.begin());
    }
    batches[chosen].push_back(e);
    for (int m = 0; m < nconec[e]; ++m) node_batches[kconec[m + 9 * e] - 1].push_back(chosen);
    if ((int)batches[chosen].size() == bem::kBatch)
      open.erase(std::remove(open.begin(), open.end(), chosen), open.end());
  }
  nb = (int)batches.size();
  out.assign((size_t)nb * bem::kBatch, -1);
  for (int b = 0; b < nb; ++b)
    for (size_t i = 0; i < batches[b].size(); ++i) out[(size_t)b * bem::kBatch + i] = batches[b][i];
}

template <typename T>
int upload(bem_ctx* c, bem::DBuf<T>& d, const T* h, size_t count) {
  BEM_CUDA(c, d.alloc(count));
  if (count) BEM_CUDA(c, cudaMemcpyAsync(d.p, h, count * sizeof(T), cudaMemcpyHostToDevice, c->stream));
  return BEM_OK;
}

int build_lookup(bem_ctx* c) {
  // per (node, ld): first element in ke order prescribing u there (assembly_mod.f90:149-161)
  const int n = c->n;
  std::vector<int> uk(3 * (size_t)n, 0);
  std::vector<double> vp(3 * (size_t)n, 0.0);
  for (int in = 0; in < n; ++in)
    for (int ld = 0; ld < 3; ++ld) {
      for (int i = 0; i < std::min(c->h_nesim[in], 8); ++i) {
        const int e = c->h_ke[i + 8 * (size_t)in] - 1;
        if (c->h_kode[3 * (size_t)e + ld] == 0) {
          for (int m = 0; m < c->h_nconec[e]; ++m)
            if (c->h_kconec[m + 9 * (size_t)e] - 1 == in) {
              vp[3 * (size_t)in + ld] = c->h_bc[3 * m + ld + 27 * (size_t)e];
              uk[3 * (size_t)in + ld] = 1;
              break;
            }
          if (uk[3 * (size_t)in + ld]) break;
        }
      }
    }
  int rc = upload(c, c->uknown, uk.data(), uk.size());
  if (rc) return rc;
  rc = upload(c, c->vp, vp.data(), vp.size());
  if (rc) return rc;
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  return BEM_OK;
}

}  // namespace

extern "C" {

int bem_ctx_create(bem_ctx** out, int device) {
  if (!out) return BEM_ERR_ARG;
  *out = nullptr;
  bem_ctx* c = new bem_ctx();
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return BEM_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (const char* v = getenv("BEM_F32_GEMM")) c->f32_gemm_override = atoi(v);
  if (const char* v = getenv("BEM_F64_GEMM")) c->f64_gemm = atoi(v);
  *out = c;
  return BEM_OK;
}

int bem_ctx_destroy(bem_ctx* c) {
  if (!c) return BEM_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  cudaStreamSynchronize(c->aux_stream);
  cudaEventDestroy(c->ev_fork);
  cudaEventDestroy(c->ev_join);
  cudaStreamDestroy(c->aux_stream);
  cudaStreamDestroy(c->stream);
  delete c;  // DBuf destructors free device memory
  return BEM_OK;
}

const char* bem_last_error(const bem_ctx* c) { return c ? c->last_error.c_str() : "null context"; }

int bem_sync(bem_ctx* c) {
  if (!c) return BEM_ERR_ARG;
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  return BEM_OK;
}

int bem_get_stream(bem_ctx* c, void** stream) {
  if (!c || !stream) return BEM_ERR_ARG;
  *stream = (void*)c->stream;
  return BEM_OK;
}

int bem_set_option(bem_ctx* c, int option, int64_t value) {
  if (!c) return BEM_ERR_ARG;
  switch (option) {
    case BEM_OPT_PIVOTING:
      if (value != BEM_PIVOT_WINDOW && value != BEM_PIVOT_PARTIAL)
        return bem_fail(c, BEM_ERR_ARG, "set_option: pivoting must be BEM_PIVOT_WINDOW or BEM_PIVOT_PARTIAL");
      c->pivot_pref = (int)value;
      return BEM_OK;
    case BEM_OPT_WAIT_LIMIT_MS:
      if (value < 1 || value > 60000) return bem_fail(c, BEM_ERR_ARG, "set_option: wait limit must be 1..60000 ms");
      c->wait_ns = (unsigned long long)value * 1000000ull;
      return BEM_OK;
    case BEM_OPT_RESIDUAL:
      if (value != 0 && value != 1) return bem_fail(c, BEM_ERR_ARG, "set_option: residual must be 0 or 1");
      c->ext_residual = value == 1;
      return BEM_OK;
    case BEM_OPT_PANEL_WIDTH:
      if (value != 0 && (value < 128 || value > 1024 || value % 128 != 0))
        return bem_fail(c, BEM_ERR_ARG, "set_option: panel width must be 0 or a multiple of 128 up to 1024");
      c->panel_width = (int)value;
      return BEM_OK;
    case BEM_OPT_WITHHOLD_BLOCK:
      if (value < -1 || value > INT32_MAX) return bem_fail(c, BEM_ERR_ARG, "set_option: bad block index");
      c->withhold_block = (int)value;
      return BEM_OK;
    default:
      return bem_fail(c, BEM_ERR_ARG, "set_option: unknown option");
  }
}

int bem_set_mesh(bem_ctx* c, int n, int ne, const double* x, const double* y, const double* z,
                 const int* nconec, const int* kconec) {
  if (!c || n <= 0 || ne <= 0 || !x || !y || !z || !nconec || !kconec)
    return bem_fail(c, BEM_ERR_ARG, "set_mesh: bad arguments");
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(x[i]) || !std::isfinite(y[i]) || !std::isfinite(z[i]))
      return bem_fail(c, BEM_ERR_ARG, "set_mesh: a node coordinate is not finite");
  BEM_CUDA(c, cudaSetDevice(c->device));
  c->h_nconec.assign(nconec, nconec + ne);
  c->h_kconec.assign(kconec, kconec + 9 * (size_t)ne);
  for (int e = 0; e < ne; ++e) {
    if (nconec[e] != 9 && nconec[e] != 6) return bem_fail(c, BEM_ERR_MESH, "nconec must be 6 or 9");
    for (int m = 0; m < nconec[e]; ++m) {
      const int k = kconec[m + 9 * (size_t)e];
      if (k < 1 || k > n) return bem_fail(c, BEM_ERR_MESH, "kconec references a node out of range");
    }
    for (int m = nconec[e]; m < 9; ++m) c->h_kconec[m + 9 * (size_t)e] = 1;
  }
  // io_mod.f90:125-135 (ke capped at 8 entries; more is an error here — the
  // reference would read past ke's column)
  c->h_nesim.assign(n, 0);
  c->h_ke.assign(8 * (size_t)n, 0);
  for (int e = 0; e < ne; ++e)
    for (int m = 0; m < nconec[e]; ++m) {
      const int in = kconec[m + 9 * (size_t)e] - 1;
      int& cnt = c->h_nesim[in];
      ++cnt;
      if (cnt > 8) return bem_fail(c, BEM_ERR_MESH, "a node lies in more than 8 elements");
      c->h_ke[(cnt - 1) + 8 * (size_t)in] = e + 1;
    }
  c->n = n;
  c->ne = ne;
  int rc;
  if ((rc = upload(c, c->x, x, n)) || (rc = upload(c, c->y, y, n)) || (rc = upload(c, c->z, z, n)) ||
      (rc = upload(c, c->nconec, nconec, ne)) ||
      (rc = upload(c, c->kconec, c->h_kconec.data(), 9 * (size_t)ne)) ||
      (rc = upload(c, c->nesim, c->h_nesim.data(), n)) ||
      (rc = upload(c, c->ke, c->h_ke.data(), 8 * (size_t)n)))
    return rc;
  std::vector<int> sched;
  build_batches(n, ne, c->h_nconec, c->h_kconec, sched, c->nbatches);
  if ((rc = upload(c, c->batches, sched.data(), sched.size()))) return rc;
  c->h_batches = sched;
  c->tail_parts = 0;
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  c->have_mesh = true;
  c->have_bc = false;
  c->have_geometry = false;
  c->have_system = false;
  c->have_solution = false;
  c->npins = 0;
  return BEM_OK;
}

int bem_set_material(bem_ctx* c, double mu, double nu) {
  if (!c || !(mu > 0.0) || !(nu < 0.5) || !(nu > -1.0))
    return bem_fail(c, BEM_ERR_ARG, "set_material: need mu > 0 and -1 < nu < 0.5");
  c->mat = bem::make_material(mu, nu);
  c->have_material = true;
  c->have_system = false;
  return BEM_OK;
}

int bem_set_bc(bem_ctx* c, const int* kode, const double* bc) {
  if (!c || !kode || !bc) return bem_fail(c, BEM_ERR_ARG, "set_bc: null pointer");
  if (!c->have_mesh) return bem_fail(c, BEM_ERR_STATE, "set_bc before set_mesh");
  BEM_CUDA(c, cudaSetDevice(c->device));
  c->h_kode.assign(kode, kode + 3 * (size_t)c->ne);
  c->h_bc.assign(bc, bc + 27 * (size_t)c->ne);
  int rc;
  if ((rc = upload(c, c->kode, kode, 3 * (size_t)c->ne)) ||
      (rc = upload(c, c->bc, bc, 27 * (size_t)c->ne)))
    return rc;
  if ((rc = build_lookup(c))) return rc;
  c->have_bc = true;
  c->have_system = false;
  return BEM_OK;
}

int bem_set_pins(bem_ctx* c, int npins, const int* dofs) {
  if (!c || npins < 0 || (npins > 0 && !dofs)) return bem_fail(c, BEM_ERR_ARG, "set_pins: bad arguments");
  if (!c->have_mesh) return bem_fail(c, BEM_ERR_STATE, "set_pins before set_mesh");
  for (int i = 0; i < npins; ++i)
    if (dofs[i] < 0 || dofs[i] >= 3 * c->n) return bem_fail(c, BEM_ERR_ARG, "set_pins: dof out of range");
  BEM_CUDA(c, cudaSetDevice(c->device));
  c->npins = npins;
  if (npins) {
    int rc = upload(c, c->pins, dofs, npins);
    if (rc) return rc;
    BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  }
  c->have_system = false;
  return BEM_OK;
}

int bem_precompute_geometry(bem_ctx* c) {
  if (!c) return BEM_ERR_ARG;
  BEM_CUDA(c, cudaSetDevice(c->device));
  return bem::launch_geometry(c);
}

int bem_get_geometry(bem_ctx* c, double* eta1, double* eta2, double* eta3, double* xja, double* xg1,
                     double* xg2, double* xg3, double* ff) {
  if (!c) return BEM_ERR_ARG;
  if (!c->have_geometry) return bem_fail(c, BEM_ERR_STATE, "geometry not computed");
  BEM_CUDA(c, cudaSetDevice(c->device));
  double* outs[8] = {eta1, eta2, eta3, xja, xg1, xg2, xg3, ff};
  bem::DBuf<double>* ins[8] = {&c->eta1, &c->eta2, &c->eta3, &c->xja, &c->xg1, &c->xg2, &c->xg3, &c->ff};
  for (int i = 0; i < 8; ++i)
    if (outs[i])
      BEM_CUDA(c, cudaMemcpyAsync(outs[i], ins[i]->p, ins[i]->bytes(), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  return BEM_OK;
}

int bem_ghmat8(bem_ctx* c, int asm_precision, double* A_out, int64_t lda_out, double* FI_out) {
  if (!c) return BEM_ERR_ARG;
  BEM_CUDA(c, cudaSetDevice(c->device));
  const int64_t N = 3 * (int64_t)c->n;
  if (A_out && lda_out < N) return bem_fail(c, BEM_ERR_ARG, "ghmat8: lda < 3n");
  c->dinv_src = nullptr;  // A is overwritten: inverses of earlier factors are stale
  int rc = bem::launch_ghmat8(c, asm_precision);
  if (rc) return rc;
  if (A_out)
    BEM_CUDA(c, cudaMemcpy2DAsync(A_out, lda_out * sizeof(double), c->A.p, c->lda * sizeof(double),
                                  N * sizeof(double), N, cudaMemcpyDeviceToHost, c->stream));
  if (FI_out)
    BEM_CUDA(c, cudaMemcpyAsync(FI_out, c->FI.p, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  return BEM_OK;
}

int bem_set_system(bem_ctx* c, int n, const double* A, int64_t lda_in, const double* FI) {
  if (!c || !A || !FI || n <= 0 || lda_in < n) return bem_fail(c, BEM_ERR_ARG, "set_system: bad arguments");
  BEM_CUDA(c, cudaSetDevice(c->device));
  const int64_t lda = ((int64_t)n + 31) / 32 * 32;
  if (c->A.count != (size_t)(lda * n)) {
    c->A.release();
    if (c->A.alloc((size_t)(lda * n)) != cudaSuccess) return bem_fail(c, BEM_ERR_OOM, "set_system: allocating A");
  }
  c->lda = lda;
  BEM_CUDA(c, c->FI.alloc(n));
  BEM_CUDA(c, cudaMemsetAsync(c->A.p, 0, c->A.bytes(), c->stream));  // the padding rows stay zero
  BEM_CUDA(c, cudaMemcpy2DAsync(c->A.p, lda * sizeof(double), A, lda_in * sizeof(double), (size_t)n * sizeof(double),
                                n, cudaMemcpyHostToDevice, c->stream));
  BEM_CUDA(c, cudaMemcpyAsync(c->FI.p, FI, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  c->dinv_src = nullptr;
  c->nsys = n;
  c->have_system = true;
  c->mesh_system = false;
  c->have_solution = false;
  c->factored_fp64 = false;
  return BEM_OK;
}

int bem_get_rows(bem_ctx* c, int r0, int r1, double* A_rows, int64_t ld, double* FI_rows) {
  if (!c || !A_rows) return bem_fail(c, BEM_ERR_ARG, "get_rows: null argument");
  const int64_t N = c->nsys;
  if (r0 < 0 || r1 > N || r1 <= r0 || ld < r1 - r0) return bem_fail(c, BEM_ERR_ARG, "get_rows: bad row range");
  if (!c->have_system) return bem_fail(c, BEM_ERR_STATE, "get_rows before ghmat8");
  if (c->factored_fp64) return bem_fail(c, BEM_ERR_STATE, "get_rows: A was overwritten by its FP64 factors");
  BEM_CUDA(c, cudaSetDevice(c->device));
  BEM_CUDA(c, cudaMemcpy2DAsync(A_rows, ld * sizeof(double), c->A.p + r0, c->lda * sizeof(double),
                                (size_t)(r1 - r0) * sizeof(double), N, cudaMemcpyDeviceToHost, c->stream));
  if (FI_rows)
    BEM_CUDA(c, cudaMemcpyAsync(FI_rows, c->FI.p + r0, (size_t)(r1 - r0) * sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  return BEM_OK;
}

int bem_get_hg(bem_ctx* c, int in0, int in1, double* H, int64_t ldh, double* G, int64_t ldg) {
  if (!c || !H || !G || in0 < 0 || in1 > c->n || in1 <= in0)
    return bem_fail(c, BEM_ERR_ARG, "get_hg: bad row range");
  const int64_t nr = 3 * (int64_t)(in1 - in0);
  if (ldh < nr || ldg < nr) return bem_fail(c, BEM_ERR_ARG, "get_hg: leading dimension too small");
  BEM_CUDA(c, cudaSetDevice(c->device));
  const int64_t N = 3 * (int64_t)c->n, NG = 27 * (int64_t)c->ne;
  bem::DBuf<double> dH, dG;
  BEM_CUDA(c, dH.alloc((size_t)(nr * N)));
  BEM_CUDA(c, dG.alloc((size_t)(nr * NG)));
  BEM_CUDA(c, cudaMemsetAsync(dH.p, 0, dH.bytes(), c->stream));
  BEM_CUDA(c, cudaMemsetAsync(dG.p, 0, dG.bytes(), c->stream));
  int rc = bem::launch_hg(c, in0, in1, dH.p, nr, dG.p, nr);
  if (rc) return rc;
  BEM_CUDA(c, cudaMemcpy2DAsync(H, ldh * sizeof(double), dH.p, nr * sizeof(double), nr * sizeof(double), N,
                                cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaMemcpy2DAsync(G, ldg * sizeof(double), dG.p, nr * sizeof(double), nr * sizeof(double), NG,
                                cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  return BEM_OK;
}

int bem_solve(bem_ctx* c, int precision, double rel_tol, int max_iter, double* FI_inout, int* info,
              bem_solve_info* stats) {
  if (!c || !info) return bem_fail(c, BEM_ERR_ARG, "solve: null argument");
  if (!c->have_system) return bem_fail(c, BEM_ERR_STATE, "solve before ghmat8");
  BEM_CUDA(c, cudaSetDevice(c->device));
  *info = 0;
  const int64_t N = c->nsys;
  bem_solve_info st{};
  int rc;
  BEM_CUDA(c, c->X.alloc(N));
  if (precision == BEM_PREC_FP64) {
    if (c->factored_fp64) return bem_fail(c, BEM_ERR_STATE, "A already factored; assemble again");
    BEM_CUDA(c, c->piv.alloc(N));
    double secs = 0.0;
    rc = bem::lu_factor_fp64(c, c->A.p, c->lda, (int)N, c->piv.p, info, &secs);
    if (rc) return rc;
    c->factored_fp64 = true;
    st.factor_seconds = secs;
    st.gflops = secs > 0 ? (2.0 / 3.0) * (double)N * N * N / secs * 1e-9 : 0.0;
    if (*info != 0) return *info;  // DGESV: singular U, no solution
    BEM_CUDA(c, cudaMemcpyAsync(c->X.p, c->FI.p, N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    rc = bem::lu_solve_fp64(c, c->A.p, c->lda, (int)N, c->X.p);
    if (rc) return rc;
  } else if (precision == BEM_PREC_FP32_IR || precision == BEM_PREC_BF16_IR || precision == BEM_PREC_FP64_IR) {
    rc = bem::solve_mixed(c, precision, rel_tol > 0 ? rel_tol : 1e-12, max_iter > 0 ? max_iter : 50, &st,
                          info);
    if (stats) *stats = st;
    if (rc) return rc;
    if (*info != 0) return *info;
  } else {
    return bem_fail(c, BEM_ERR_ARG, "unknown solve precision");
  }
  if (FI_inout)
    BEM_CUDA(c, cudaMemcpyAsync(FI_inout, c->X.p, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  c->have_solution = true;
  if (stats) *stats = st;
  return BEM_OK;
}

int bem_dgesv(bem_ctx* c, int n, int nrhs, double* A, int lda, int* ipiv, double* B, int ldb, int* info) {
  if (!c || !A || !ipiv || !B || !info || n <= 0 || nrhs < 0 || lda < n || ldb < n)
    return bem_fail(c, BEM_ERR_ARG, "dgesv: bad arguments");
  BEM_CUDA(c, cudaSetDevice(c->device));
  *info = 0;
  const int64_t ld = ((int64_t)n + 31) / 32 * 32;
  bem::DBuf<double> dA, dB;
  bem::DBuf<int> dp;
  if (dA.alloc((size_t)(ld * n)) != cudaSuccess) return bem_fail(c, BEM_ERR_OOM, "dgesv: allocating A");
  BEM_CUDA(c, dB.alloc((size_t)ld * std::max(nrhs, 1)));
  BEM_CUDA(c, dp.alloc(n));
  BEM_CUDA(c, cudaMemcpy2DAsync(dA.p, ld * sizeof(double), A, (size_t)lda * sizeof(double), n * sizeof(double), n,
                                cudaMemcpyHostToDevice, c->stream));
  if (nrhs > 0)
    BEM_CUDA(c, cudaMemcpy2DAsync(dB.p, ld * sizeof(double), B, (size_t)ldb * sizeof(double), n * sizeof(double),
                                  nrhs, cudaMemcpyHostToDevice, c->stream));
  double secs = 0.0;
  int rc = bem::lu_factor_fp64(c, dA.p, ld, n, dp.p, info, &secs);
  if (rc) return rc;
  if (*info == 0)
    for (int j = 0; j < nrhs; ++j)
      if ((rc = bem::lu_solve_fp64(c, dA.p, ld, n, dB.p + (int64_t)j * ld))) return rc;
  std::vector<int> hp(n);
  BEM_CUDA(c, cudaMemcpyAsync(hp.data(), dp.p, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaMemcpy2DAsync(A, (size_t)lda * sizeof(double), dA.p, ld * sizeof(double), n * sizeof(double), n,
                                cudaMemcpyDeviceToHost, c->stream));
  if (nrhs > 0 && *info == 0)
    BEM_CUDA(c, cudaMemcpy2DAsync(B, (size_t)ldb * sizeof(double), dB.p, ld * sizeof(double), n * sizeof(double),
                                  nrhs, cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  for (int i = 0; i < n; ++i) ipiv[i] = hp[i] + 1;
  return *info;
}

int bem_reorganize(bem_ctx* c, double* FI_out, double* DFI_out) {
  if (!c) return BEM_ERR_ARG;
  if (!c->have_solution) return bem_fail(c, BEM_ERR_STATE, "reorganize before solve");
  if (!c->mesh_system) return bem_fail(c, BEM_ERR_STATE, "reorganize: the system was not assembled by ghmat8");
  BEM_CUDA(c, cudaSetDevice(c->device));
  int rc = bem::launch_reorganize(c);
  if (rc) return rc;
  if (FI_out)
    BEM_CUDA(c, cudaMemcpyAsync(FI_out, c->U.p, 3 * (size_t)c->n * sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream));
  if (DFI_out)
    BEM_CUDA(c, cudaMemcpyAsync(DFI_out, c->DFI.p, 27 * (size_t)c->ne * sizeof(double),
                                cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  return BEM_OK;
}

int bem_boundary_stresses(bem_ctx* c, double* sigma_elem, double* sigma_node, double* prin, double* vm) {
  if (!c) return BEM_ERR_ARG;
  if (!sigma_node || !prin || !vm) return bem_fail(c, BEM_ERR_ARG, "boundary_stresses: null output");
  if (!c->have_solution) return bem_fail(c, BEM_ERR_STATE, "boundary stresses before solve");
  if (!c->mesh_system) return bem_fail(c, BEM_ERR_STATE, "boundary stresses: the system was not assembled by ghmat8");
  BEM_CUDA(c, cudaSetDevice(c->device));
  // u and t of the current solution (cheap: two small kernels)
  int rc = bem::launch_reorganize(c);
  if (rc) return rc;
  const size_t ne = c->ne, n = c->n;
  bem::DBuf<double> d;
  BEM_CUDA(c, d.alloc(54 * ne + 10 * n));
  double *se = d.p, *sn = se + 54 * ne, *pr = sn + 6 * n, *v = pr + 3 * n;
  if ((rc = bem::launch_boundary_stresses(c, se, sn, pr, v))) return rc;
  if (sigma_elem)
    BEM_CUDA(c, cudaMemcpyAsync(sigma_elem, se, 54 * ne * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaMemcpyAsync(sigma_node, sn, 6 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaMemcpyAsync(prin, pr, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaMemcpyAsync(vm, v, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  return BEM_OK;
}

int bem_solve_transposed(bem_ctx* c, double* g) {
  if (!c || !g) return BEM_ERR_ARG;
  if (!c->factored_fp64 || !c->have_solution)
    return bem_fail(c, BEM_ERR_STATE, "solve_transposed needs a solve with BEM_PREC_FP64 first");
  BEM_CUDA(c, cudaSetDevice(c->device));
  const size_t N = (size_t)c->nsys;
  bem::DBuf<double> d;
  BEM_CUDA(c, d.alloc(N));
  BEM_CUDA(c, cudaMemcpyAsync(d.p, g, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  int rc = bem::lu_solve_t_fp64(c, c->A.p, c->lda, (int)N, d.p);
  if (rc) return rc;
  BEM_CUDA(c, cudaMemcpyAsync(g, d.p, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  return BEM_OK;
}

int bem_adjoint_gradient(bem_ctx* c, const double* lambda, double* grad_xyz, double* grad_mat) {
  if (!c || !lambda || !grad_xyz || !grad_mat) return BEM_ERR_ARG;
  if (!c->have_solution || !c->have_geometry) return bem_fail(c, BEM_ERR_STATE, "adjoint_gradient before solve");
  if (!c->mesh_system) return bem_fail(c, BEM_ERR_STATE, "adjoint_gradient: the system was not assembled by ghmat8");
  BEM_CUDA(c, cudaSetDevice(c->device));
  int rc = bem::launch_reorganize(c);  // u and t of the current solution
  if (rc) return rc;
  const size_t N = 3 * (size_t)c->n;
  bem::DBuf<double> d;
  BEM_CUDA(c, d.alloc(2 * N + 2));
  BEM_CUDA(c, cudaMemcpyAsync(d.p, lambda, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if ((rc = bem::launch_adjoint_gradient(c, d.p, d.p + N, d.p + 2 * N))) return rc;
  BEM_CUDA(c, cudaMemcpyAsync(grad_xyz, d.p + N, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaMemcpyAsync(grad_mat, d.p + 2 * N, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  return BEM_OK;
}

int bem_internal_points_device(bem_ctx* c, int l, const double* cx, const double* cy, const double* cz,
                               double* u, double* s, double* pr, double* vm, int flags) {
  if (!c || l < 0) return BEM_ERR_ARG;
  if (l == 0) return BEM_OK;
  if (!cx || !cy || !cz || !u || !s || !pr || !vm) return bem_fail(c, BEM_ERR_ARG, "internal_points: null");
  BEM_CUDA(c, cudaSetDevice(c->device));
  return bem::launch_internal_points(c, l, cx, cy, cz, u, s, pr, vm, flags);
}

int bem_internal_points(bem_ctx* c, int l, const double* cx, const double* cy, const double* cz, double* u,
                        double* s, double* pr, double* vm, int flags) {
  if (!c || l < 0) return BEM_ERR_ARG;
  if (l == 0) return BEM_OK;
  if (!cx || !cy || !cz || !u || !s || !pr || !vm) return bem_fail(c, BEM_ERR_ARG, "internal_points: null");
  BEM_CUDA(c, cudaSetDevice(c->device));
  bem::DBuf<double> d;
  BEM_CUDA(c, d.alloc(16 * (size_t)l));
  double* p = d.p;
  double *dx = p, *dy = p + l, *dz = p + 2 * (size_t)l, *du = p + 3 * (size_t)l, *ds = p + 6 * (size_t)l,
         *dp = p + 12 * (size_t)l, *dv = p + 15 * (size_t)l;
  BEM_CUDA(c, cudaMemcpyAsync(dx, cx, l * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  BEM_CUDA(c, cudaMemcpyAsync(dy, cy, l * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  BEM_CUDA(c, cudaMemcpyAsync(dz, cz, l * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  int rc = bem::launch_internal_points(c, l, dx, dy, dz, du, ds, dp, dv, flags);
  if (rc) return rc;
  BEM_CUDA(c, cudaMemcpyAsync(u, du, 3 * (size_t)l * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaMemcpyAsync(s, ds, 6 * (size_t)l * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaMemcpyAsync(pr, dp, 3 * (size_t)l * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaMemcpyAsync(vm, dv, (size_t)l * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  return BEM_OK;
}

int bem_profile_begin(bem_ctx* c, int timing) {
  if (!c) return BEM_ERR_ARG;
  c->launches = 0;
  c->prof = bem_profile{};
  if (timing < BEM_PROF_COUNT || timing > BEM_PROF_TRAILING) return BEM_ERR_ARG;
  c->prof_timing = timing;
  return BEM_OK;
}

int bem_profile_end(bem_ctx* c, bem_profile* out) {
  if (!c) return BEM_ERR_ARG;
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  c->prof.kernel_launches = c->launches;
  if (out) *out = c->prof;
  c->prof_timing = 0;
  return BEM_OK;
}

int bem_device_state(bem_ctx* c, double** A, int64_t* lda, double** FI, double** DFI) {
  if (!c) return BEM_ERR_ARG;
  if (A) *A = c->A.p;
  if (lda) *lda = c->lda;
  if (FI) *FI = c->FI.p;
  if (DFI) *DFI = c->DFI.p;
  return BEM_OK;
}

}  // extern "C"
