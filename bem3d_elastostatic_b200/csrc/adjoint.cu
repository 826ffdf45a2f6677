// Backward assembly for the adjoint: the derivative of R = lambda^T (FI - A x) with
// respect to the node coordinates and the material (mu, nu), at fixed lambda and x,
// without forming dA/dX.
//
// With u (3n) and t (27 ne) the reorganized solution, FI - A x = -(H u - G t) row by
// row (the column swap only moves known values to the right-hand side; pinned rows
// carry no geometry and are excluded by zeroing their lambda), and with the rigid-body
// diagonal H_ii = -sum_{j != i} H_ij:
//   R = - sum_i sum_e integral_e [ lambda_i . T*(x_i, y) (u(y) - u_i)
//                                 - lambda_i . U*(x_i, y) t(y) ] dGamma(y),
// integrated with the reference's own discrete rules (6 x 6 Gauss points for regular
// pairs, locin8's collapsed sub-triangles for singular pairs).  Each Gauss point
// contributes W phi with W = J w; its derivative goes
//   * to every element node k through the point y (shape value N_k) and through the
//     surface normal a1 x a2 (d(a1 x a2) = dX_k x (N_k,1 a2 - N_k,2 a1)),
//   * to the collocation node through -r,
//   * to nu through c3..c6, and to mu through the prescribed tractions only (an
//     unknown traction is mu x, and mu G does not depend on mu).
// 9-node quadrilateral elements.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "shape.cuh"

namespace bem {
namespace {

constexpr int kRec = 18;  // per (element, Gauss point): y, a1, a2, u(y), t(y), prescribed t(y)

__constant__ double c_f[36][9], c_d1[36][9], c_d2[36][9], c_w[36];
__constant__ double c_gi6[6], c_om6[6];

struct Kelvin {
  double c3, c4, c5, c6, mu, nu;
};

// phi at one point and its partial derivatives: g_r = d phi / d r, g_n = d phi / d n,
// and the scalar derivatives in nu and mu
__device__ __forceinline__ void point_terms(const Kelvin& K, const double* rv, const double* n, const double* lam,
                                            const double* du, const double* t, const double* td, double& phi,
                                            double* g_r, double* g_n, double& p_nu, double& p_mu) {
  const double r = sqrt(rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2]);
  const double ri = 1.0 / r;
  const double rh[3] = {rv[0] * ri, rv[1] * ri, rv[2] * ri};
  auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  // U* part: phi_U = -(c3 / r) (c4 A + a bt)
  const double A = dot(lam, t), a = dot(lam, rh), bt = dot(t, rh);
  const double Ad = dot(lam, td), btd = dot(td, rh);
  const double phiU = -K.c3 * ri * (K.c4 * A + a * bt);
  // T* part: phi_T = (c5 / r^2) F
  const double B = dot(lam, du), q = dot(du, rh), m = dot(rh, n), ln = dot(lam, n), dn = dot(du, n);
  const double base = K.c6 * B + 3.0 * a * q;
  const double F = m * base + K.c6 * (ln * q - dn * a);
  const double c5r2 = K.c5 * ri * ri;
  phi = phiU + c5r2 * F;
  double gF[3];
  for (int d = 0; d < 3; ++d)
    gF[d] = n[d] * base + m * 3.0 * (q * lam[d] + a * du[d]) + K.c6 * (ln * du[d] - dn * lam[d]);
  const double rgF = dot(rh, gF);
  const double cU = -K.c3 * ri * ri, cT = c5r2 * ri;
  for (int d = 0; d < 3; ++d) {
    g_r[d] = cU * (bt * lam[d] + a * t[d] - (K.c4 * A + 3.0 * a * bt) * rh[d]) +
             cT * (-2.0 * F * rh[d] + gF[d] - rgF * rh[d]);
    g_n[d] = c5r2 * (rh[d] * base + K.c6 * (q * lam[d] - a * du[d]));
  }
  const double inv1 = 1.0 / (1.0 - K.nu);
  p_nu = -K.c3 * inv1 * ri * (K.c4 * A + a * bt) + K.c3 * ri * 4.0 * A + K.c5 * inv1 * ri * ri * F -
         2.0 * c5r2 * (m * B + ln * q - dn * a);
  p_mu = K.c3 * ri / K.mu * (K.c4 * Ad + a * btd);
}

// the point's contributions: node gradients gk (element nodes, 9 x 3) and the
// collocation-node gradient gx, scaled by w
__device__ __forceinline__ void accumulate(const double* fq, const double* d1q, const double* d2q,
                                           const double* a1, const double* a2, double w, double J,
                                           const double* n, double phi, const double* g_r, const double* g_n,
                                           double (*gk)[3], double* gx) {
  const double gnn = g_n[0] * n[0] + g_n[1] * n[1] + g_n[2] * n[2];
  double s[3], rr[3];
  for (int d = 0; d < 3; ++d) {
    s[d] = w * (phi * n[d] + g_n[d] - gnn * n[d]);  // w (phi n + (I - n n^T) g_n)
    rr[d] = w * J * g_r[d];
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    double v[3];
    for (int d = 0; d < 3; ++d) v[d] = d1q[k] * a2[d] - d2q[k] * a1[d];
    gk[k][0] += v[1] * s[2] - v[2] * s[1] + fq[k] * rr[0];
    gk[k][1] += v[2] * s[0] - v[0] * s[2] + fq[k] * rr[1];
    gk[k][2] += v[0] * s[1] - v[1] * s[0] + fq[k] * rr[2];
  }
  for (int d = 0; d < 3; ++d) gx[d] -= rr[d];
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// per (element, Gauss point): y, a1, a2, u(y), t(y), prescribed t(y)
__global__ void adj_table_kernel(int ne, const int* __restrict__ kconec, const int* __restrict__ kode,
                                 const double* __restrict__ x, const double* __restrict__ y,
                                 const double* __restrict__ z, const double* __restrict__ U,
                                 const double* __restrict__ DFI, double* __restrict__ tab) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)ne * 36) return;
  const int e = (int)(gid / 36), q = (int)(gid % 36);
  double o[kRec];
  for (int c = 0; c < kRec; ++c) o[c] = 0.0;
  for (int k = 0; k < 9; ++k) {
    const int nd = kconec[k + 9 * e] - 1;
    const double X[3] = {x[nd], y[nd], z[nd]};
    for (int d = 0; d < 3; ++d) {
      o[d] += c_f[q][k] * X[d];
      o[3 + d] += c_d1[q][k] * X[d];
      o[6 + d] += c_d2[q][k] * X[d];
      o[9 + d] += c_f[q][k] * U[3 * nd + d];
      const double tv = DFI[3 * k + d + 27 * (int64_t)e];
      o[12 + d] += c_f[q][k] * tv;
      if (kode[3 * e + d] != 0) o[15 + d] += c_f[q][k] * tv;
    }
  }
  for (int c = 0; c < kRec; ++c) tab[(int64_t)gid * kRec + c] = o[c];
}

// regular pairs: CTA = 32 collocation nodes (lanes) x 8 warps over the elements
__global__ void __launch_bounds__(256) adj_regular_kernel(int n, int ne, const int* __restrict__ kconec,
                                                          const double* __restrict__ x,
                                                          const double* __restrict__ y,
                                                          const double* __restrict__ z,
                                                          const double* __restrict__ U,
                                                          const double* __restrict__ lam,
                                                          const double* __restrict__ tab, Kelvin K,
                                                          double* grad, double* gmat) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * 32 + lane;
  const bool active = i < n;
  const int ii = active ? i : 0;
  const double xi[3] = {x[ii], y[ii], z[ii]};
  const double ui[3] = {U[3 * ii], U[3 * ii + 1], U[3 * ii + 2]};
  const double li[3] = {active ? lam[3 * ii] : 0.0, active ? lam[3 * ii + 1] : 0.0, active ? lam[3 * ii + 2] : 0.0};
  double gx[3] = {0.0, 0.0, 0.0}, snu = 0.0, smu = 0.0;
  for (int e = w; e < ne; e += 8) {
    int kc[9];
    bool sing = false;
    for (int k = 0; k < 9; ++k) {
      kc[k] = __ldg(kconec + k + 9 * e) - 1;
      sing |= kc[k] == ii;
    }
    const bool on = active && !sing;
    double gk[9][3];
    for (int k = 0; k < 9; ++k) gk[k][0] = gk[k][1] = gk[k][2] = 0.0;
    if (on) {
      const double* T = tab + (int64_t)e * 36 * kRec;
#pragma unroll 1
      for (int q = 0; q < 36; ++q) {
        const double* o = T + q * kRec;
        const double a1[3] = {__ldg(o + 3), __ldg(o + 4), __ldg(o + 5)};
        const double a2[3] = {__ldg(o + 6), __ldg(o + 7), __ldg(o + 8)};
        const double cr[3] = {a1[1] * a2[2] - a1[2] * a2[1], a1[2] * a2[0] - a1[0] * a2[2],
                              a1[0] * a2[1] - a1[1] * a2[0]};
        const double J = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        const double nn[3] = {cr[0] / J, cr[1] / J, cr[2] / J};
        const double rv[3] = {__ldg(o + 0) - xi[0], __ldg(o + 1) - xi[1], __ldg(o + 2) - xi[2]};
        const double du[3] = {__ldg(o + 9) - ui[0], __ldg(o + 10) - ui[1], __ldg(o + 11) - ui[2]};
        const double tq[3] = {__ldg(o + 12), __ldg(o + 13), __ldg(o + 14)};
        const double td[3] = {__ldg(o + 15), __ldg(o + 16), __ldg(o + 17)};
        double phi, g_r[3], g_n[3], pn, pm;
        point_terms(K, rv, nn, li, du, tq, td, phi, g_r, g_n, pn, pm);
        const double wq = c_w[q];
        accumulate(c_f[q], c_d1[q], c_d2[q], a1, a2, wq, J, nn, phi, g_r, g_n, gk, gx);
        snu += wq * J * pn;
        smu += wq * J * pm;
      }
    }
    // the element nodes' gradients: this warp's 32 collocation nodes summed first
#pragma unroll
    for (int k = 0; k < 9; ++k)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double v = warp_sum(gk[k][d]);
        if (lane == 0 && v != 0.0) atomicAdd(grad + 3 * kc[k] + d, -v);
      }
  }
  if (active)
    for (int d = 0; d < 3; ++d) atomicAdd(grad + 3 * i + d, -gx[d]);
  snu = warp_sum(snu);
  smu = warp_sum(smu);
  if (lane == 0) {
    atomicAdd(gmat + 0, -smu);
    atomicAdd(gmat + 1, -snu);
  }
}

// the sub-triangles of locin8 (assembly_mod.f90:399-489) for local node nodo of a quad9
__device__ int sub_tris9(int nodo, double v1[4][3], double v2[4][3], double area[4]) {
  const double gi1[9] = {-1.0, 0.0, 1.0, 1.0, 1.0, 0.0, -1.0, -1.0, 0.0};
  const double gi2[9] = {-1.0, -1.0, -1.0, 0.0, 1.0, 1.0, 1.0, 0.0, 0.0};
  auto G1 = [&](int p) { return gi1[(p - 1) % 8]; };
  auto G2 = [&](int p) { return gi2[(p - 1) % 8]; };
  int cnt = 0;
  if (nodo == 9) {
    for (int k = 1; k <= 4; ++k) {
      const int m = 2 * k - 1;
      v1[cnt][0] = gi1[8];
      v2[cnt][0] = gi2[8];
      v1[cnt][1] = G1(m);
      v2[cnt][1] = G2(m);
      v1[cnt][2] = G1(m + 2);
      v2[cnt][2] = G2(m + 2);
      area[cnt++] = 1.0;
    }
  } else if (nodo % 2 == 1) {
    for (int k = 1; k <= 2; ++k) {
      const int m = 2 * k;
      v1[cnt][0] = gi1[nodo - 1];
      v2[cnt][0] = gi2[nodo - 1];
      v1[cnt][1] = G1(nodo + m);
      v2[cnt][1] = G2(nodo + m);
      v1[cnt][2] = G1(nodo + m + 2);
      v2[cnt][2] = G2(nodo + m + 2);
      area[cnt++] = 2.0;
    }
  } else {
    for (int k = 1; k <= 3; ++k) {
      const int m = 2 * k - 1;
      const double a1[3] = {gi1[nodo - 1], G1(nodo + m), G1(nodo + m + 2)};
      const double a2[3] = {gi2[nodo - 1], G2(nodo + m), G2(nodo + m + 2)};
      for (int t = 0; t < 3; ++t) {
        v1[cnt][t] = a1[t];
        v2[cnt][t] = a2[t];
      }
      area[cnt++] = 0.5 * (a1[1] * a2[2] + a1[0] * a2[1] + a1[2] * a2[0] - a1[1] * a2[0] - a1[2] * a2[1] -
                           a1[0] * a2[2]);
    }
  }
  return cnt;
}

// singular pairs: one warp per (node, adjacent element); lanes over the sub-triangle points
__global__ void __launch_bounds__(128) adj_singular_kernel(int n, const int* __restrict__ nesim,
                                                           const int* __restrict__ ke,
                                                           const int* __restrict__ kconec,
                                                           const int* __restrict__ kode,
                                                           const double* __restrict__ x,
                                                           const double* __restrict__ y,
                                                           const double* __restrict__ z,
                                                           const double* __restrict__ U,
                                                           const double* __restrict__ DFI,
                                                           const double* __restrict__ lam, Kelvin K,
                                                           double* grad, double* gmat) {
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int item = blockIdx.x * 4 + wib;  // (node, j-th element)
  const int i = item / 8, jj = item % 8;
  if (i >= n || jj >= min(nesim[i], 8)) return;  // warp-uniform
  const int e = ke[jj + 8 * i] - 1;
  int kc[9], nodo = 0;
  double X[9][3], Ue[9][3], Te[9][3];
  for (int k = 0; k < 9; ++k) {
    kc[k] = kconec[k + 9 * e] - 1;
    if (kc[k] == i && nodo == 0) nodo = k + 1;
    X[k][0] = x[kc[k]];
    X[k][1] = y[kc[k]];
    X[k][2] = z[kc[k]];
    for (int d = 0; d < 3; ++d) {
      Ue[k][d] = U[3 * kc[k] + d];
      Te[k][d] = DFI[3 * k + d + 27 * (int64_t)e];
    }
  }
  const bool tdat[3] = {kode[3 * e] != 0, kode[3 * e + 1] != 0, kode[3 * e + 2] != 0};
  const double li[3] = {lam[3 * i], lam[3 * i + 1], lam[3 * i + 2]};
  const double xi[3] = {x[i], y[i], z[i]};
  const double ui[3] = {U[3 * i], U[3 * i + 1], U[3 * i + 2]};
  double v1[4][3], v2[4][3], area[4];
  const int ntri = sub_tris9(nodo, v1, v2, area);
  double gk[9][3], gx[3] = {0.0, 0.0, 0.0}, snu = 0.0, smu = 0.0;
  for (int k = 0; k < 9; ++k) gk[k][0] = gk[k][1] = gk[k][2] = 0.0;
  for (int p = lane; p < ntri * 36; p += 32) {
    const int tri = p / 36, qi = (p % 36) / 6, qj = p % 6;
    const double s1 = 0.5 * (c_gi6[qi] + 1.0), s2 = 0.5 * (c_gi6[qj] + 1.0);
    const double g1 = (1.0 - s1) * v1[tri][0] + s1 * (1.0 - s2) * v1[tri][1] + s1 * s2 * v1[tri][2];
    const double g2 = (1.0 - s1) * v2[tri][0] + s1 * (1.0 - s2) * v2[tri][1] + s1 * s2 * v2[tri][2];
    const double wq = (c_gi6[qi] + 1.0) * area[tri] * 0.25 * c_om6[qi] * c_om6[qj];
    double f[9], d1[9], d2[9];
    shape_fn<double>(9, g1, g2, f, d1, d2);
    double yp[3] = {0, 0, 0}, a1[3] = {0, 0, 0}, a2[3] = {0, 0, 0}, uq[3] = {0, 0, 0}, tq[3] = {0, 0, 0},
           td[3] = {0, 0, 0};
    for (int k = 0; k < 9; ++k)
      for (int d = 0; d < 3; ++d) {
        yp[d] += f[k] * X[k][d];
        a1[d] += d1[k] * X[k][d];
        a2[d] += d2[k] * X[k][d];
        uq[d] += f[k] * Ue[k][d];
        tq[d] += f[k] * Te[k][d];
        if (tdat[d]) td[d] += f[k] * Te[k][d];
      }
    const double cr[3] = {a1[1] * a2[2] - a1[2] * a2[1], a1[2] * a2[0] - a1[0] * a2[2], a1[0] * a2[1] - a1[1] * a2[0]};
    const double J = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    const double nn[3] = {cr[0] / J, cr[1] / J, cr[2] / J};
    const double rv[3] = {yp[0] - xi[0], yp[1] - xi[1], yp[2] - xi[2]};
    const double du[3] = {uq[0] - ui[0], uq[1] - ui[1], uq[2] - ui[2]};
    double phi, g_r[3], g_n[3], pn, pm;
    point_terms(K, rv, nn, li, du, tq, td, phi, g_r, g_n, pn, pm);
    accumulate(f, d1, d2, a1, a2, wq, J, nn, phi, g_r, g_n, gk, gx);
    snu += wq * J * pn;
    smu += wq * J * pm;
  }
  // the collocation node is the element's node nodo
  for (int d = 0; d < 3; ++d) gk[nodo - 1][d] += gx[d];
#pragma unroll
  for (int k = 0; k < 9; ++k)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double v = warp_sum(gk[k][d]);
      if (lane == 0 && v != 0.0) atomicAdd(grad + 3 * kc[k] + d, -v);
    }
  snu = warp_sum(snu);
  smu = warp_sum(smu);
  if (lane == 0) {
    atomicAdd(gmat + 0, -smu);
    atomicAdd(gmat + 1, -snu);
  }
}

__global__ void zero_pins_kernel(const int* pins, int npins, double* lam) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < npins) lam[pins[p]] = 0.0;
}

int upload_tables() {
  static DeviceOnce done;  // per device: __constant__ tables
  if (!done.pending()) return BEM_OK;
  double f[36][9], d1[36][9], d2[36][9], w[36];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      const int q = 6 * i + j;
      shape_fn<double>(9, kGiQuad[i], kGiQuad[j], f[q], d1[q], d2[q]);
      w[q] = kOmeQuad[i] * kOmeQuad[j];
    }
  if (cudaMemcpyToSymbol(c_f, f, sizeof(f)) != cudaSuccess || cudaMemcpyToSymbol(c_d1, d1, sizeof(d1)) != cudaSuccess ||
      cudaMemcpyToSymbol(c_d2, d2, sizeof(d2)) != cudaSuccess || cudaMemcpyToSymbol(c_w, w, sizeof(w)) != cudaSuccess ||
      cudaMemcpyToSymbol(c_gi6, kGiQuad, sizeof(kGiQuad)) != cudaSuccess ||
      cudaMemcpyToSymbol(c_om6, kOmeQuad, sizeof(kOmeQuad)) != cudaSuccess)
    return BEM_ERR_CUDA;
  done.mark();
  return BEM_OK;
}

}  // namespace

// grad (3n) and gmat ([d/dmu, d/dnu]) of R = lambda^T (FI - A x) at the current
// (reorganized) solution; lambda (3n) on the device, its pinned entries are zeroed
int launch_adjoint_gradient(bem_ctx* c, double* lam, double* grad, double* gmat) {
  for (int e = 0; e < c->ne; ++e)
    if (c->h_nconec[e] != 9) return bem_fail(c, BEM_ERR_ARG, "the adjoint supports 9-node elements only");
  int rc = upload_tables();
  if (rc) return bem_fail(c, rc, "uploading the adjoint tables");
  const Material& M = c->mat;
  const Kelvin K{M.c3, M.c4, M.c5, M.c6, M.mu, M.nu};
  DBuf<double> tab;
  BEM_CUDA(c, tab.alloc((size_t)c->ne * 36 * kRec));
  if (c->npins > 0) {
    zero_pins_kernel<<<(c->npins + 127) / 128, 128, 0, c->stream>>>(c->pins.p, c->npins, lam);
    BEM_LAUNCH_CHECK(c);
  }
  BEM_CUDA(c, cudaMemsetAsync(grad, 0, 3 * (size_t)c->n * sizeof(double), c->stream));
  BEM_CUDA(c, cudaMemsetAsync(gmat, 0, 2 * sizeof(double), c->stream));
  const int64_t nt = 36 * (int64_t)c->ne;
  adj_table_kernel<<<(unsigned)((nt + 127) / 128), 128, 0, c->stream>>>(c->ne, c->kconec.p, c->kode.p, c->x.p,
                                                                         c->y.p, c->z.p, c->U.p, c->DFI.p, tab.p);
  BEM_LAUNCH_CHECK(c);
  adj_regular_kernel<<<(c->n + 31) / 32, 256, 0, c->stream>>>(c->n, c->ne, c->kconec.p, c->x.p, c->y.p, c->z.p,
                                                               c->U.p, lam, tab.p, K, grad, gmat);
  BEM_LAUNCH_CHECK(c);
  adj_singular_kernel<<<(8 * c->n + 3) / 4, 128, 0, c->stream>>>(c->n, c->nesim.p, c->ke.p, c->kconec.p, c->kode.p,
                                                                  c->x.p, c->y.p, c->z.p, c->U.p, c->DFI.p, lam, K,
                                                                  grad, gmat);
  BEM_LAUNCH_CHECK(c);
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  return BEM_OK;
}

}  // namespace bem
