// precompute_element_geometry / etaxja (assembly_mod.f90:28-51, 225-337) on the GPU.
//
// One thread per (element, Gauss point).  This translation unit is compiled with
// --fmad=false so every product and sum rounds exactly as the reference's FP64
// Fortran does: the tables (Gauss-point coordinates, Jacobians, unit normals, shape
// functions and the weighted shape functions p12) are bitwise equal to the oracle's.
#include "common.cuh"
#include "shape.cuh"

namespace bem {

__constant__ double c_gi_quad[6];
__constant__ double c_ome_quad[6];
__constant__ double c_rr_tri[4];
__constant__ double c_ss_tri[4];
__constant__ double c_omei_tri[4];
__constant__ double c_omej_tri[4];

__global__ void etaxja_kernel(int ne, const double* __restrict__ x, const double* __restrict__ y,
                              const double* __restrict__ z, const int* __restrict__ nconec,
                              const int* __restrict__ kconec, double* eta1, double* eta2,
                              double* eta3, double* xja, double* xg1, double* xg2, double* xg3,
                              double* ff, double* tab, int* bad) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)ne * kGp) return;
  const int e = (int)(gid / kGp);
  const int q = (int)(gid % kGp);
  const int ncone = nconec[e];
  const int npg = (ncone < 9) ? 4 : 6;
  const int64_t kk = (int64_t)q + (int64_t)kGp * e;
  double* T = tab + (int64_t)e * kTabStride;
  if (q >= npg * npg) {
    // unused points of a tri6 element stay zero (etaxja zeroes all 36 first)
    eta1[kk] = eta2[kk] = eta3[kk] = xja[kk] = 0.0;
    xg1[kk] = xg2[kk] = xg3[kk] = 0.0;
    for (int m = 0; m < 9; ++m) ff[m + 9 * kk] = 0.0;
    for (int v = 0; v < 6; ++v) T[6 * q + v] = 0.0;
    for (int m = 0; m < 9; ++m) T[kTabGeo + 9 * q + m] = 0.0;
    return;
  }
  const int i = q / npg, j = q % npg;
  double xj1[9], xj2[9], xj3[9];
  for (int m = 0; m < 9; ++m) {
    if (m < ncone) {
      const int k = kconec[m + 9 * e] - 1;
      xj1[m] = x[k];
      xj2[m] = y[k];
      xj3[m] = z[k];
    } else {
      xj1[m] = xj2[m] = xj3[m] = 0.0;
    }
  }
  double g1, g2, wij;
  if (ncone == 9) {
    g1 = c_gi_quad[i];
    g2 = c_gi_quad[j];
  } else {
    g1 = c_ss_tri[j];
    g2 = c_rr_tri[i] * (1.0 - c_ss_tri[j]);
  }
  double f[9], fd1[9], fd2[9];
  shape_fn<double>(ncone, g1, g2, f, fd1, fd2);
  double a = 0.0, b = 0.0, c = 0.0;
  for (int ik = 0; ik < ncone; ++ik) {
    a = a + f[ik] * xj1[ik];
    b = b + f[ik] * xj2[ik];
    c = c + f[ik] * xj3[ik];
  }
  double J, n1, n2, n3;
  jacobian_dc<double>(ncone, fd1, fd2, xj1, xj2, xj3, J, n1, n2, n3);
  // a zero (or non-finite) Jacobian makes the unit normal a division by zero
  // (assembly_mod.f90:331-334): the element is degenerate
  if (bad && !(J > 0.0 && J < INFINITY && a - a == 0.0 && b - b == 0.0 && c - c == 0.0)) atomicExch(bad, 1);
  eta1[kk] = n1;
  eta2[kk] = n2;
  eta3[kk] = n3;
  xja[kk] = J;
  xg1[kk] = a;
  xg2[kk] = b;
  xg3[kk] = c;
  for (int m = 0; m < 9; ++m) ff[m + 9 * kk] = (m < ncone) ? f[m] : 0.0;
  T[6 * q + 0] = a;
  T[6 * q + 1] = b;
  T[6 * q + 2] = c;
  T[6 * q + 3] = n1;
  T[6 * q + 4] = n2;
  T[6 * q + 5] = n3;
  // p12 (assembly_mod.f90:363-369): ((N_k * J) * w_i) * w_j
  for (int m = 0; m < 9; ++m) {
    double p = 0.0;
    if (m < ncone) {
      if (ncone == 9)
        p = f[m] * J * c_ome_quad[i] * c_ome_quad[j];
      else
        p = f[m] * J * c_omei_tri[i] * c_omej_tri[j];
    }
    T[kTabGeo + 9 * q + m] = p;
  }
  (void)wij;
}

int upload_quadrature_constants() {
  if (cudaMemcpyToSymbol(c_gi_quad, kGiQuad, sizeof(kGiQuad)) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_ome_quad, kOmeQuad, sizeof(kOmeQuad)) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_rr_tri, kRrTri, sizeof(kRrTri)) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_ss_tri, kSsTri, sizeof(kSsTri)) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_omei_tri, kOmeiTri, sizeof(kOmeiTri)) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_omej_tri, kOmejTri, sizeof(kOmejTri)) != cudaSuccess) return -1;
  return 0;
}

int launch_geometry(bem_ctx* c) {
  if (!c->have_mesh) return bem_fail(c, BEM_ERR_STATE, "precompute_geometry before set_mesh");
  static DeviceOnce constants;  // __constant__ tables are per device
  if (constants.pending()) {
    if (upload_quadrature_constants() != 0) return bem_fail(c, BEM_ERR_CUDA, "uploading quadrature constants");
    constants.mark();
  }
  const size_t ng = (size_t)kGp * c->ne;
  for (auto* b : {&c->eta1, &c->eta2, &c->eta3, &c->xja, &c->xg1, &c->xg2, &c->xg3})
    BEM_CUDA(c, b->alloc(ng));
  BEM_CUDA(c, c->ff.alloc(9 * ng));
  BEM_CUDA(c, c->tab.alloc((size_t)kTabStride * c->ne));
  const int threads = 128;
  const int64_t blocks = ((int64_t)ng + threads - 1) / threads;
  if (c->status.count < 1) BEM_CUDA(c, c->status.alloc(1));
  BEM_CUDA(c, cudaMemsetAsync(c->status.p, 0, sizeof(int), c->stream));
  etaxja_kernel<<<(unsigned)blocks, threads, 0, c->stream>>>(
      c->ne, c->x.p, c->y.p, c->z.p, c->nconec.p, c->kconec.p, c->eta1.p, c->eta2.p, c->eta3.p,
      c->xja.p, c->xg1.p, c->xg2.p, c->xg3.p, c->ff.p, c->tab.p, c->status.p);
  BEM_LAUNCH_CHECK(c);
  int bad = 0;
  BEM_CUDA(c, cudaMemcpyAsync(&bad, c->status.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  if (bad) {
    c->have_geometry = false;
    return bem_fail(c, BEM_ERR_MESH, "degenerate element: zero or non-finite Jacobian at a Gauss point");
  }
  c->have_geometry = true;
  return BEM_OK;
}


// The same for raw arrays (the systems of a batch, with global node numbers in
// kconec): ref receives the reference-layout tables (16 x 36 x ne doubles: eta1..3,
// xja, xg1..3, then ff), tab the packed table (kTabStride x ne).
int launch_geometry_arrays(cudaStream_t stream, int ne, const double* x, const double* y, const double* z,
                           const int* nconec, const int* kconec, double* ref, double* tab) {
  if (upload_quadrature_constants() != 0) return BEM_ERR_CUDA;
  const size_t ng = (size_t)kGp * ne;
  const int threads = 128;
  const int64_t blocks = ((int64_t)ng + threads - 1) / threads;
  etaxja_kernel<<<(unsigned)blocks, threads, 0, stream>>>(ne, x, y, z, nconec, kconec, ref, ref + ng,
                                                          ref + 2 * ng, ref + 3 * ng, ref + 4 * ng,
                                                          ref + 5 * ng, ref + 6 * ng, ref + 7 * ng, tab, nullptr);
  return cudaGetLastError() == cudaSuccess ? BEM_OK : BEM_ERR_CUDA;
}

}  // namespace bem
