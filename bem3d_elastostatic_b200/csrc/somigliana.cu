// compute_internal_points (stress_mod.f90:511-886) on the GPU: Somigliana
// displacement and stress identities at internal points, with the reference's
// two-tier quadrature (the element's own 6x6 / 4x4 table when the point is farther
// than 3.5 element radii from its centroid, a 40x40 Gauss-Legendre table otherwise)
// and calc_principal_and_vm (:299-359).
//
// Kernels
//   far_table / near_table  pre-weighted Gauss-point tables (:580-726), 12 doubles per
//                           point: x, y, z, n1, n2, n3, u*w (3), t*w (3)
//   far_kernel              persistent: each CTA takes tiles of 256 x P internal points
//                           (P = 4, 2 or 1 points per thread, whichever keeps every SM
//                           busy) and streams every element's table through a
//                           double-buffered shared-memory ring (cp.async, 8 elements per
//                           chunk) that it reads as broadcasts, so each staged table point
//                           feeds 256 P points; near elements are skipped and the point
//                           is flagged
//   near_kernel             one warp per flagged point: its near elements' 1600 points
//                           split over the lanes, a fixed-order warp reduction, then the
//                           principal stresses
//   finish_kernel           principal stresses of the points with no near element
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "shape.cuh"
#include "stress.cuh"

namespace bem {

constexpr int kNearN = 40;
constexpr int kNear = kNearN * kNearN;
constexpr int kRec = 12;  // doubles per table point
constexpr int kChunk = 8;  // elements staged per shared-memory chunk (27.6 KB)

__constant__ double c_xgl[kNearN];
__constant__ double c_wgl[kNearN];
__constant__ double c_ome6[6];
__constant__ double c_omei4[4];
__constant__ double c_omej4[4];

// gauss_legendre_1d (stress_mod.f90:475-503): Newton iteration on P_n from the
// Chebyshev-like first guess, to |dz| <= 1e-15.
static void gauss_legendre(int n, double* x, double* w) {
  const int m = (n + 1) / 2;
  for (int i = 1; i <= m; ++i) {
    double z = std::cos(kPi * ((double)i - 0.25) / ((double)n + 0.5));
    double p1 = 0, p2 = 0, p3 = 0, pp = 0;
    for (int it = 0; it < 100; ++it) {
      p1 = 1.0;
      p2 = 0.0;
      for (int j = 1; j <= n; ++j) {
        p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      const double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) <= 1.0e-15) break;
    }
    x[i - 1] = -z;
    x[n - i] = z;
    w[i - 1] = 2.0 / ((1.0 - z * z) * pp * pp);
    w[n - i] = w[i - 1];
  }
}

// element centroid and near threshold 3.5^2 * max |node - centroid|^2 (:584-604)
__global__ void einfo_kernel(int ne, const double* x, const double* y, const double* z, const int* nconec,
                             const int* kconec, double* einfo) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int nc = nconec[e];
  double xj[9], yj[9], zj[9], cx = 0, cy = 0, cz = 0;
  for (int m = 0; m < nc; ++m) {
    const int k = kconec[m + 9 * e] - 1;
    xj[m] = x[k];
    yj[m] = y[k];
    zj[m] = z[k];
    cx += xj[m];
    cy += yj[m];
    cz += zj[m];
  }
  cx /= nc;
  cy /= nc;
  cz /= nc;
  double d2 = 0.0;
  for (int m = 0; m < nc; ++m) {
    const double dx = xj[m] - cx, dy = yj[m] - cy, dz = zj[m] - cz;
    d2 = fmax(d2, dx * dx + dy * dy + dz * dz);
  }
  einfo[4 * e + 0] = cx;
  einfo[4 * e + 1] = cy;
  einfo[4 * e + 2] = cz;
  einfo[4 * e + 3] = (3.5 * 3.5) * d2;
}

// far table (:606-650), fixed stride of 36 points per element
__global__ void far_table_kernel(int ne, const int* nconec, const int* kconec, const double* eta1,
                                 const double* eta2, const double* eta3, const double* xja, const double* xg1,
                                 const double* xg2, const double* xg3, const double* ff, const double* U,
                                 const double* DFI, double* far) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)ne * kGp) return;
  const int e = (int)(gid / kGp), q = (int)(gid % kGp);
  const int nc = nconec[e];
  const int npg = (nc == 9) ? 6 : 4;
  double* P = far + gid * kRec;
  if (q >= npg * npg) {
    for (int v = 0; v < kRec; ++v) P[v] = 0.0;
    return;
  }
  const int i = q / npg, j = q % npg;
  const double wg = (nc == 9) ? c_ome6[i] * c_ome6[j] * xja[gid] : c_omei4[i] * c_omej4[j] * xja[gid];
  double ug[3] = {0, 0, 0}, tg[3] = {0, 0, 0};
  for (int m = 0; m < nc; ++m) {
    const int64_t ik = kconec[m + 9 * e] - 1;
    const double f = ff[m + 9 * gid];
    for (int c = 0; c < 3; ++c) {
      ug[c] += f * U[3 * ik + c];
      tg[c] += f * DFI[3 * m + c + 27 * (int64_t)e];
    }
  }
  P[0] = xg1[gid];
  P[1] = xg2[gid];
  P[2] = xg3[gid];
  P[3] = eta1[gid];
  P[4] = eta2[gid];
  P[5] = eta3[gid];
  for (int c = 0; c < 3; ++c) {
    P[6 + c] = ug[c] * wg;
    P[9 + c] = tg[c] * wg;
  }
}

// near table (:654-726): 40 x 40 Gauss-Legendre, Duffy map on tri6
__global__ void near_table_kernel(int ne, const double* x, const double* y, const double* z, const int* nconec,
                                  const int* kconec, const double* U, const double* DFI, double* near) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)ne * kNear) return;
  const int e = (int)(gid / kNear), q = (int)(gid % kNear), i = q / kNearN, j = q % kNearN;
  const int nc = nconec[e];
  double g1, g2, tj;
  if (nc == 9) {
    g1 = c_xgl[i];
    g2 = c_xgl[j];
    tj = 1.0;
  } else {
    g1 = 0.5 * (1.0 + c_xgl[i]);
    g2 = 0.25 * (1.0 - c_xgl[i]) * (1.0 + c_xgl[j]);
    tj = 0.125 * (1.0 - c_xgl[i]);
  }
  double f[9], fd1[9], fd2[9];
  shape_fn<double>(nc, g1, g2, f, fd1, fd2);
  double xg[3] = {0, 0, 0}, d1[3] = {0, 0, 0}, d2[3] = {0, 0, 0}, ug[3] = {0, 0, 0}, tg[3] = {0, 0, 0};
  for (int m = 0; m < nc; ++m) {
    const int64_t ik = kconec[m + 9 * e] - 1;
    const double p[3] = {x[ik], y[ik], z[ik]};
    for (int c = 0; c < 3; ++c) {
      xg[c] += f[m] * p[c];
      d1[c] += fd1[m] * p[c];
      d2[c] += fd2[m] * p[c];
      ug[c] += f[m] * U[3 * ik + c];
      tg[c] += f[m] * DFI[3 * m + c + 27 * (int64_t)e];
    }
  }
  const double c0 = d1[1] * d2[2] - d1[2] * d2[1];
  const double c1 = d1[2] * d2[0] - d1[0] * d2[2];
  const double c2 = d1[0] * d2[1] - d1[1] * d2[0];
  const double jac = sqrt(c0 * c0 + c1 * c1 + c2 * c2);
  const double wg = c_wgl[i] * c_wgl[j] * tj * jac;
  double* P = near + gid * kRec;
  P[0] = xg[0];
  P[1] = xg[1];
  P[2] = xg[2];
  P[3] = c0 / jac;
  P[4] = c1 / jac;
  P[5] = c2 / jac;
  for (int c = 0; c < 3; ++c) {
    P[6 + c] = ug[c] * wg;
    P[9 + c] = tg[c] * wg;
  }
}

struct SomConst {
  double nu, c4, c6, pr4, cU, cT, cD, cS, asg;
};

// accumulate_somigliana_range body (:807-885) for one table point
__device__ __forceinline__ void somigliana_point(const SomConst& K, const double* P, double xx, double yy,
                                                 double zz, double* ua, double* sa) {
  const double rx = P[0] - xx, ry = P[1] - yy, rz = P[2] - zz;
  const double ir = rsqrt(rx * rx + ry * ry + rz * rz);
  const double ir2 = ir * ir, ir3 = ir2 * ir;
  const double rd1 = rx * ir, rd2 = ry * ir, rd3 = rz * ir;
  const double n1 = P[3], n2 = P[4], n3 = P[5];
  const double rdn = rd1 * n1 + rd2 * n2 + rd3 * n3;
  const double tu1 = P[6], tu2 = P[7], tu3 = P[8];
  const double tt1 = P[9], tt2 = P[10], tt3 = P[11];
  const double rdt = rd1 * tt1 + rd2 * tt2 + rd3 * tt3;
  const double rdu = rd1 * tu1 + rd2 * tu2 + rd3 * tu3;
  const double nuv = n1 * tu1 + n2 * tu2 + n3 * tu3;
  const double c4 = K.c4, c6 = K.c6, nu = K.nu, pr4 = K.pr4;
  const double fU = K.cU * ir, fT = K.cT * ir2, ac6 = K.asg * c6;
  ua[0] += fU * (c4 * tt1 + rd1 * rdt) - fT * (rdn * (c6 * tu1 + 3.0 * rd1 * rdu) + ac6 * (nuv * rd1 - n1 * rdu));
  ua[1] += fU * (c4 * tt2 + rd2 * rdt) - fT * (rdn * (c6 * tu2 + 3.0 * rd2 * rdu) + ac6 * (nuv * rd2 - n2 * rdu));
  ua[2] += fU * (c4 * tt3 + rd3 * rdt) - fT * (rdn * (c6 * tu3 + 3.0 * rd3 * rdu) + ac6 * (nuv * rd3 - n3 * rdu));
  const double fD = K.cD * ir2, fS = K.cS * ir3;
  const double Dxx = fD * (c6 * (2.0 * tt1 * rd1 - rdt) + 3.0 * rd1 * rd1 * rdt);
  const double Dyy = fD * (c6 * (2.0 * tt2 * rd2 - rdt) + 3.0 * rd2 * rd2 * rdt);
  const double Dzz = fD * (c6 * (2.0 * tt3 * rd3 - rdt) + 3.0 * rd3 * rd3 * rdt);
  const double Dxy = fD * (c6 * (tt1 * rd2 + tt2 * rd1) + 3.0 * rd1 * rd2 * rdt);
  const double Dyz = fD * (c6 * (tt2 * rd3 + tt3 * rd2) + 3.0 * rd2 * rd3 * rdt);
  const double Dzx = fD * (c6 * (tt3 * rd1 + tt1 * rd3) + 3.0 * rd3 * rd1 * rdt);
  const double Sxx = fS * (3.0 * rdn * (c6 * rdu + 2.0 * nu * tu1 * rd1 - 5.0 * rd1 * rd1 * rdu) +
                           6.0 * nu * rdu * n1 * rd1 + c6 * (3.0 * nuv * rd1 * rd1 + 2.0 * n1 * tu1) - pr4 * nuv);
  const double Syy = fS * (3.0 * rdn * (c6 * rdu + 2.0 * nu * tu2 * rd2 - 5.0 * rd2 * rd2 * rdu) +
                           6.0 * nu * rdu * n2 * rd2 + c6 * (3.0 * nuv * rd2 * rd2 + 2.0 * n2 * tu2) - pr4 * nuv);
  const double Szz = fS * (3.0 * rdn * (c6 * rdu + 2.0 * nu * tu3 * rd3 - 5.0 * rd3 * rd3 * rdu) +
                           6.0 * nu * rdu * n3 * rd3 + c6 * (3.0 * nuv * rd3 * rd3 + 2.0 * n3 * tu3) - pr4 * nuv);
  const double Sxy = fS * (3.0 * rdn * (nu * (tu1 * rd2 + tu2 * rd1) - 5.0 * rd1 * rd2 * rdu) +
                           3.0 * nu * rdu * (n1 * rd2 + n2 * rd1) + c6 * (3.0 * nuv * rd1 * rd2 + n1 * tu2 + n2 * tu1));
  const double Syz = fS * (3.0 * rdn * (nu * (tu2 * rd3 + tu3 * rd2) - 5.0 * rd2 * rd3 * rdu) +
                           3.0 * nu * rdu * (n2 * rd3 + n3 * rd2) + c6 * (3.0 * nuv * rd2 * rd3 + n2 * tu3 + n3 * tu2));
  const double Szx = fS * (3.0 * rdn * (nu * (tu3 * rd1 + tu1 * rd3) - 5.0 * rd3 * rd1 * rdu) +
                           3.0 * nu * rdu * (n3 * rd1 + n1 * rd3) + c6 * (3.0 * nuv * rd3 * rd1 + n3 * tu1 + n1 * tu3));
  sa[0] += Dxx - Sxx;
  sa[1] += Dyy - Syy;
  sa[2] += Dzz - Szz;
  sa[3] += Dxy - Sxy;
  sa[4] += Dyz - Syz;
  sa[5] += Dzx - Szx;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}

constexpr int kFarThreads = 256;
constexpr int kChunkDoubles = kChunk * kGp * kRec;  // one staged chunk of element tables
constexpr size_t kFarSmem = 2 * (size_t)(kChunkDoubles + kChunk * 4) * sizeof(double);

// Far pass over tiles of kFarThreads * P points (point p of thread t: tile base +
// p * kFarThreads + t, so every load of a point array is coalesced).  counters[0]
// accumulates the table points evaluated (far Gauss points x internal points).
template <int P>
__global__ void __launch_bounds__(kFarThreads, 1)
    far_kernel(int l, const double* __restrict__ cx, const double* __restrict__ cy, const double* __restrict__ cz,
               int ne, const int* __restrict__ nconec, const double* __restrict__ einfo,
               const double* __restrict__ far, SomConst K, double* part, int* nearflag,
               unsigned long long* counters) {
  extern __shared__ __align__(16) double far_smem[];
  double* s_tab = far_smem;                      // [2][kChunkDoubles]
  double* s_info = far_smem + 2 * kChunkDoubles;  // [2][kChunk][4]
  __shared__ int s_npt[2][kChunk];
  constexpr int T = kFarThreads * P;
  const int tid = threadIdx.x;
  const int ntiles = (l + T - 1) / T;
  const int nchunks = (ne + kChunk - 1) / kChunk;
  unsigned long long evals = 0;
  auto stage = [&](int ch, int buf) {  // issue the copies of chunk ch into buffer buf
    const int e0 = ch * kChunk, ce = min(kChunk, ne - e0);
    const double* src = far + (int64_t)e0 * kGp * kRec;
    double* dst = s_tab + buf * kChunkDoubles;
    for (int i = tid; i < ce * kGp * kRec / 2; i += kFarThreads) cp_async16(dst + 2 * i, src + 2 * i);
    const double* isrc = einfo + 4 * (int64_t)e0;
    double* idst = s_info + buf * kChunk * 4;
    for (int i = tid; i < ce * 2; i += kFarThreads) cp_async16(idst + 2 * i, isrc + 2 * i);
    if (tid < ce) s_npt[buf][tid] = (nconec[e0 + tid] == 9) ? 36 : 16;
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    double xx[P], yy[P], zz[P], ua[P][3], sa[P][6];
    bool act[P];
    int has_near[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const int ip = tile * T + p * kFarThreads + tid;
      act[p] = ip < l;
      xx[p] = act[p] ? cx[ip] : 0.0;
      yy[p] = act[p] ? cy[ip] : 0.0;
      zz[p] = act[p] ? cz[ip] : 0.0;
      has_near[p] = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c) ua[p][c] = 0.0;
#pragma unroll
      for (int c = 0; c < 6; ++c) sa[p][c] = 0.0;
    }
    __syncthreads();  // the previous tile's last chunk is no longer read
    stage(0, 0);
    for (int ch = 0; ch < nchunks; ++ch) {
      const int buf = ch & 1;
      if (ch + 1 < nchunks) {
        stage(ch + 1, buf ^ 1);
        asm volatile("cp.async.wait_group 1;" ::: "memory");
      } else {
        asm volatile("cp.async.wait_group 0;" ::: "memory");
      }
      __syncthreads();
      const int ce = min(kChunk, ne - ch * kChunk);
      const double* tab = s_tab + buf * kChunkDoubles;
      const double* inf = s_info + buf * kChunk * 4;
      for (int ee = 0; ee < ce; ++ee) {
        bool farp[P];
        bool any = false;
#pragma unroll
        for (int p = 0; p < P; ++p) {
          const double dx = xx[p] - inf[4 * ee], dy = yy[p] - inf[4 * ee + 1], dz = zz[p] - inf[4 * ee + 2];
          farp[p] = act[p] && (dx * dx + dy * dy + dz * dz > inf[4 * ee + 3]);
          if (act[p] && !farp[p]) has_near[p] = 1;
          any |= farp[p];
        }
        if (!any) continue;
        const int np = s_npt[buf][ee];
        const double* Pt = tab + ee * kGp * kRec;
        for (int q = 0; q < np; ++q) {
#pragma unroll
          for (int p = 0; p < P; ++p)
            if (farp[p]) somigliana_point(K, Pt + q * kRec, xx[p], yy[p], zz[p], ua[p], sa[p]);
        }
#pragma unroll
        for (int p = 0; p < P; ++p) evals += farp[p] ? (unsigned long long)np : 0ull;
      }
      __syncthreads();  // buffer buf is refilled by the next iteration's stage
    }
#pragma unroll
    for (int p = 0; p < P; ++p) {
      if (!act[p]) continue;
      const int64_t ip = (int64_t)tile * T + p * kFarThreads + tid;
      for (int c = 0; c < 3; ++c) part[9 * ip + c] = ua[p][c];
      for (int c = 0; c < 6; ++c) part[9 * ip + 3 + c] = sa[p][c];
      nearflag[ip] = has_near[p];
    }
  }
  // one addition per warp
  for (int off = 16; off > 0; off >>= 1) evals += __shfl_xor_sync(0xffffffffu, evals, off);
  if ((tid & 31) == 0 && evals) atomicAdd(counters, evals);
}

__global__ void near_list_kernel(int l, const int* nearflag, int* list, int* count) {
  const int ip = blockIdx.x * blockDim.x + threadIdx.x;
  if (ip < l && nearflag[ip]) list[atomicAdd(count, 1)] = ip;
}

__global__ void __launch_bounds__(128) near_kernel(int nlist, const int* list, const double* cx, const double* cy,
                                                   const double* cz, int ne, const double* einfo, const double* near,
                                                   SomConst K, const double* part, double* u, double* s, double* pr,
                                                   double* vm, unsigned long long* counters) {
  const int wid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (wid >= nlist) return;
  const int ip = list[wid];
  const double xx = cx[ip], yy = cy[ip], zz = cz[ip];
  double ua[3] = {0, 0, 0}, sa[6] = {0, 0, 0, 0, 0, 0};
  unsigned long long evals = 0;
  for (int e = 0; e < ne; ++e) {
    const double dx = xx - einfo[4 * e], dy = yy - einfo[4 * e + 1], dz = zz - einfo[4 * e + 2];
    if (dx * dx + dy * dy + dz * dz > einfo[4 * e + 3]) continue;
    const double* T = near + (int64_t)e * kNear * kRec;
    for (int q = lane; q < kNear; q += 32) somigliana_point(K, T + (int64_t)q * kRec, xx, yy, zz, ua, sa);
    evals += kNear;
  }
  if (lane == 0 && evals) atomicAdd(counters + 1, evals);
  for (int off = 16; off > 0; off >>= 1) {
    for (int c = 0; c < 3; ++c) ua[c] += __shfl_xor_sync(0xffffffffu, ua[c], off);
    for (int c = 0; c < 6; ++c) sa[c] += __shfl_xor_sync(0xffffffffu, sa[c], off);
  }
  if (lane != 0) return;
  double uu[3], ss[6];
  for (int c = 0; c < 3; ++c) uu[c] = part[9 * (int64_t)ip + c] + ua[c];
  for (int c = 0; c < 6; ++c) ss[c] = part[9 * (int64_t)ip + 3 + c] + sa[c];
  for (int c = 0; c < 3; ++c) u[3 * (int64_t)ip + c] = uu[c];
  for (int c = 0; c < 6; ++c) s[6 * (int64_t)ip + c] = ss[c];
  principal_vm(ss, pr + 3 * (int64_t)ip, vm + ip);
}

__global__ void finish_kernel(int l, const int* nearflag, const double* part, double* u, double* s, double* pr,
                              double* vm) {
  const int ip = blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= l || nearflag[ip]) return;
  double ss[6];
  for (int c = 0; c < 3; ++c) u[3 * (int64_t)ip + c] = part[9 * (int64_t)ip + c];
  for (int c = 0; c < 6; ++c) {
    ss[c] = part[9 * (int64_t)ip + 3 + c];
    s[6 * (int64_t)ip + c] = ss[c];
  }
  principal_vm(ss, pr + 3 * (int64_t)ip, vm + ip);
}

int launch_internal_points(bem_ctx* c, int l, const double* cx, const double* cy, const double* cz, double* u,
                           double* s, double* pr, double* vm, int flags) {
  if (!c->have_geometry || c->DFI.count == 0 || c->U.count == 0)
    return bem_fail(c, BEM_ERR_STATE, "internal_points needs geometry and a reorganized solution");
  double xgl[kNearN], wgl[kNearN];
  gauss_legendre(kNearN, xgl, wgl);
  BEM_CUDA(c, cudaMemcpyToSymbol(c_xgl, xgl, sizeof(xgl)));
  BEM_CUDA(c, cudaMemcpyToSymbol(c_wgl, wgl, sizeof(wgl)));
  BEM_CUDA(c, cudaMemcpyToSymbol(c_ome6, kOmeQuad, sizeof(kOmeQuad)));
  BEM_CUDA(c, cudaMemcpyToSymbol(c_omei4, kOmeiTri, sizeof(kOmeiTri)));
  BEM_CUDA(c, cudaMemcpyToSymbol(c_omej4, kOmejTri, sizeof(kOmejTri)));
  const int ne = c->ne;
  DBuf<double> einfo, far, near, part;
  DBuf<int> flag, list;
  BEM_CUDA(c, einfo.alloc(4 * (size_t)ne));
  BEM_CUDA(c, far.alloc((size_t)ne * kGp * kRec));
  if (near.alloc((size_t)ne * kNear * kRec) != cudaSuccess)
    return bem_fail(c, BEM_ERR_OOM, "allocating the 40x40 near-field table");
  BEM_CUDA(c, part.alloc(9 * (size_t)l));
  BEM_CUDA(c, flag.alloc((size_t)l + 1));
  BEM_CUDA(c, list.alloc((size_t)l));
  einfo_kernel<<<(ne + 127) / 128, 128, 0, c->stream>>>(ne, c->x.p, c->y.p, c->z.p, c->nconec.p, c->kconec.p,
                                                        einfo.p);
  BEM_LAUNCH_CHECK(c);
  const int64_t nf = (int64_t)ne * kGp;
  far_table_kernel<<<(unsigned)((nf + 127) / 128), 128, 0, c->stream>>>(
      ne, c->nconec.p, c->kconec.p, c->eta1.p, c->eta2.p, c->eta3.p, c->xja.p, c->xg1.p, c->xg2.p, c->xg3.p,
      c->ff.p, c->U.p, c->DFI.p, far.p);
  BEM_LAUNCH_CHECK(c);
  const int64_t nn = (int64_t)ne * kNear;
  near_table_kernel<<<(unsigned)((nn + 127) / 128), 128, 0, c->stream>>>(ne, c->x.p, c->y.p, c->z.p, c->nconec.p,
                                                                          c->kconec.p, c->U.p, c->DFI.p, near.p);
  BEM_LAUNCH_CHECK(c);
  const double nu = c->mat.nu, mu = c->mat.mu;
  SomConst K;
  K.nu = nu;
  K.c4 = 3.0 - 4.0 * nu;
  K.c6 = 1.0 - 2.0 * nu;
  K.pr4 = 1.0 - 4.0 * nu;
  K.cU = 1.0 / (16.0 * kPi * (1.0 - nu) * mu);
  K.cT = -1.0 / (8.0 * kPi * (1.0 - nu));
  K.cD = 1.0 / (8.0 * kPi * (1.0 - nu));
  K.cS = mu / (4.0 * kPi * (1.0 - nu));
  K.asg = (flags & BEM_IP_KELVIN_CONSISTENT) ? -1.0 : 1.0;
  if (c->ip_counters.count < 2) BEM_CUDA(c, c->ip_counters.alloc(2));
  BEM_CUDA(c, cudaMemsetAsync(c->ip_counters.p, 0, 2 * sizeof(unsigned long long), c->stream));
  {
    static DeviceOnce attr;  // the double-buffered chunk ring is above the 48 KB default
    if (attr.pending()) {
      BEM_CUDA(c, cudaFuncSetAttribute(far_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFarSmem));
      BEM_CUDA(c, cudaFuncSetAttribute(far_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFarSmem));
      BEM_CUDA(c, cudaFuncSetAttribute(far_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFarSmem));
      attr.mark();
    }
    // the most points per thread that still gives every SM at least four tiles
    const int grid = c->sm_count;
    const int P = ((int64_t)l >= 4LL * grid * 4 * kFarThreads) ? 4 : ((int64_t)l >= 4LL * grid * 2 * kFarThreads) ? 2 : 1;
    const int ntiles = (int)((l + (int64_t)P * kFarThreads - 1) / ((int64_t)P * kFarThreads));
    const int G = std::min(grid, ntiles);
    if (P == 4)
      far_kernel<4><<<G, kFarThreads, kFarSmem, c->stream>>>(l, cx, cy, cz, ne, c->nconec.p, einfo.p, far.p, K,
                                                             part.p, flag.p, c->ip_counters.p);
    else if (P == 2)
      far_kernel<2><<<G, kFarThreads, kFarSmem, c->stream>>>(l, cx, cy, cz, ne, c->nconec.p, einfo.p, far.p, K,
                                                             part.p, flag.p, c->ip_counters.p);
    else
      far_kernel<1><<<G, kFarThreads, kFarSmem, c->stream>>>(l, cx, cy, cz, ne, c->nconec.p, einfo.p, far.p, K,
                                                             part.p, flag.p, c->ip_counters.p);
    BEM_LAUNCH_CHECK(c);
  }
  int* count = flag.p + l;
  BEM_CUDA(c, cudaMemsetAsync(count, 0, sizeof(int), c->stream));
  near_list_kernel<<<(l + 255) / 256, 256, 0, c->stream>>>(l, flag.p, list.p, count);
  BEM_LAUNCH_CHECK(c);
  int nlist = 0;
  BEM_CUDA(c, cudaMemcpyAsync(&nlist, count, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  if (nlist > 0) {
    near_kernel<<<(nlist + 3) / 4, 128, 0, c->stream>>>(nlist, list.p, cx, cy, cz, ne, einfo.p, near.p, K, part.p, u,
                                                        s, pr, vm, c->ip_counters.p);
    BEM_LAUNCH_CHECK(c);
  }
  finish_kernel<<<(l + 255) / 256, 256, 0, c->stream>>>(l, flag.p, part.p, u, s, pr, vm);
  BEM_LAUNCH_CHECK(c);
  unsigned long long cnt[2] = {0, 0};
  BEM_CUDA(c, cudaMemcpyAsync(cnt, c->ip_counters.p, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream));
  BEM_CUDA(c, cudaStreamSynchronize(c->stream));
  c->prof.ip_points += l;
  c->prof.ip_near_points += nlist;
  c->prof.ip_far_evals += (double)cnt[0];
  c->prof.ip_near_evals += (double)cnt[1];
  return BEM_OK;
}

}  // namespace bem
