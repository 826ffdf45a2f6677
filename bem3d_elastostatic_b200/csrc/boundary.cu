// compute_boundary_stresses (stress_mod.f90:365-406) on the GPU: the traction-recovery
// stresses at every node of every boundary element, their average at each node over
// its elements, and the nodal principal and von Mises stresses.
//
//   elem_kernel   one thread per (element, element node): the local triad and the
//                 surface map at the node (axes_cos_lagrange, :119-168), the in-plane
//                 strains from the element's displacements, the out-of-plane stresses
//                 from its traction, plane Hooke's law and the rotation back to global
//                 axes (boundary_stresses_elem, :174-297)
//   node_kernel   one thread per node: the average over its first min(nesim, 8)
//                 elements in the adjacency order of io_mod.f90:125-135 (a fixed
//                 order, so the result is deterministic), then calc_principal_and_vm
//
// Compiled with --fmad=false and in the reference's operation order, like the
// geometry kernel.
#include "common.cuh"
#include "shape.cuh"
#include "stress.cuh"

namespace bem {

namespace {

__global__ void elem_kernel(int ne, const int* __restrict__ nconec, const int* __restrict__ kconec,
                            const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, const double* __restrict__ U,
                            const double* __restrict__ DFI, double rge, double xnu, double* __restrict__ se) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= 9 * (int64_t)ne) return;
  const int e = (int)(tid / 9), k = (int)(tid % 9);
  const int ncone = nconec[e];
  double* o = se + 6 * tid;
  if (k >= ncone) {
    for (int c = 0; c < 6; ++c) o[c] = 0.0;
    return;
  }
  // node parametric coordinates (stress_mod.f90:216-223)
  const double q1[9] = {-1.0, 0.0, 1.0, 1.0, 1.0, 0.0, -1.0, -1.0, 0.0};
  const double q2[9] = {-1.0, -1.0, -1.0, 0.0, 1.0, 1.0, 1.0, 0.0, 0.0};
  const double t1[6] = {1.0, 0.0, 0.0, 0.5, 0.0, 0.5};
  const double t2[6] = {0.0, 1.0, 0.0, 0.5, 0.5, 0.0};
  const double g1 = ncone == 9 ? q1[k] : t1[k], g2 = ncone == 9 ? q2[k] : t2[k];
  double ff[9], fd1[9], fd2[9];
  shape_fn<double>(ncone, g1, g2, ff, fd1, fd2);

  // axes_cos_lagrange
  double a1[3] = {0.0, 0.0, 0.0}, a2[3] = {0.0, 0.0, 0.0};
  for (int a = 0; a < ncone; ++a) {
    const int ik = kconec[a + 9 * e] - 1;
    const double c[3] = {x[ik], y[ik], z[ik]};
    for (int i = 0; i < 3; ++i) {
      a1[i] = a1[i] + fd1[a] * c[i];
      a2[i] = a2[i] + fd2[a] * c[i];
    }
  }
  const double v1 = sqrt(a1[0] * a1[0] + a1[1] * a1[1] + a1[2] * a1[2]);
  const double v2 = sqrt(a2[0] * a2[0] + a2[1] * a2[1] + a2[2] * a2[2]);
  const double a3[3] = {a1[1] * a2[2] - a1[2] * a2[1], a1[2] * a2[0] - a1[0] * a2[2],
                        a1[0] * a2[1] - a1[1] * a2[0]};
  const double jcb = sqrt(a3[0] * a3[0] + a3[1] * a3[1] + a3[2] * a3[2]);
  double L[3][3];
  for (int i = 0; i < 3; ++i) {
    L[2][i] = a3[i] / jcb;
    L[0][i] = a1[i] / v1;
  }
  L[1][0] = L[2][1] * L[0][2] - L[2][2] * L[0][1];
  L[1][1] = L[2][2] * L[0][0] - L[2][0] * L[0][2];
  L[1][2] = L[2][0] * L[0][1] - L[2][1] * L[0][0];
  double cos_th = (a1[0] * a2[0] + a1[1] * a2[1] + a1[2] * a2[2]) / (v1 * v2);
  if (cos_th > 1.0) cos_th = 1.0;
  if (cos_th < -1.0) cos_th = -1.0;
  double sin_th = sqrt(fmax(0.0, 1.0 - cos_th * cos_th));
  if (sin_th < 1.0e-12) sin_th = 1.0e-12;
  const double cl11 = 1.0 / v1, cl12 = -cos_th / (v1 * sin_th), cl21 = 0.0, cl22 = 1.0 / (v2 * sin_th);

  // local displacement gradients at node k
  double u1_1 = 0.0, u2_2 = 0.0, u1_2 = 0.0, u2_1 = 0.0;
  for (int a = 0; a < ncone; ++a) {
    const int ik = kconec[a + 9 * e] - 1;
    const double u[3] = {U[3 * ik], U[3 * ik + 1], U[3 * ik + 2]};
    const double dn1 = cl11 * fd1[a] + cl21 * fd2[a];
    const double dn2 = cl12 * fd1[a] + cl22 * fd2[a];
    const double ul1 = L[0][0] * u[0] + L[0][1] * u[1] + L[0][2] * u[2];
    const double ul2 = L[1][0] * u[0] + L[1][1] * u[1] + L[1][2] * u[2];
    u1_1 = u1_1 + dn1 * ul1;
    u2_2 = u2_2 + dn2 * ul2;
    u1_2 = u1_2 + dn2 * ul1;
    u2_1 = u2_1 + dn1 * ul2;
  }
  const double eps11 = u1_1, eps22 = u2_2, eps12 = 0.5 * (u1_2 + u2_1);
  const double* t = DFI + 27 * (int64_t)e + 3 * k;
  double tl[3];
  for (int i = 0; i < 3; ++i) tl[i] = L[i][0] * t[0] + L[i][1] * t[1] + L[i][2] * t[2];

  // local stress: Cauchy's formula out of plane, plane Hooke's law in plane
  const double c_eps = 2.0 * rge / (1.0 - xnu);
  const double c_nu = 2.0 * rge * xnu / (1.0 - xnu);
  const double c_sig3 = xnu / (1.0 - xnu);
  double S[3][3];
  S[0][2] = tl[0];
  S[2][0] = S[0][2];
  S[1][2] = tl[1];
  S[2][1] = S[1][2];
  S[2][2] = tl[2];
  S[0][0] = c_eps * eps11 + c_nu * eps22 + c_sig3 * S[2][2];
  S[1][1] = c_eps * eps22 + c_nu * eps11 + c_sig3 * S[2][2];
  S[0][1] = 2.0 * rge * eps12;
  S[1][0] = S[0][1];
  // global stress L^T (S L)
  double T[3][3], G[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) T[i][j] = S[i][0] * L[0][j] + S[i][1] * L[1][j] + S[i][2] * L[2][j];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) G[i][j] = L[0][i] * T[0][j] + L[1][i] * T[1][j] + L[2][i] * T[2][j];
  o[0] = G[0][0];
  o[1] = G[1][1];
  o[2] = G[2][2];
  o[3] = 0.5 * (G[0][1] + G[1][0]);
  o[4] = 0.5 * (G[1][2] + G[2][1]);
  o[5] = 0.5 * (G[2][0] + G[0][2]);
}

__global__ void node_kernel(int n, const int* __restrict__ nesim, const int* __restrict__ ke,
                            const int* __restrict__ nconec, const int* __restrict__ kconec,
                            const double* __restrict__ se, double* __restrict__ sn, double* __restrict__ pr,
                            double* __restrict__ vm) {
  const int in = blockIdx.x * blockDim.x + threadIdx.x;
  if (in >= n) return;
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const int ns = min(nesim[in], 8);
  if (ns > 0) {
    for (int j = 0; j < ns; ++j) {
      const int e = ke[j + 8 * in] - 1;
      for (int k = 0; k < nconec[e]; ++k)
        if (kconec[k + 9 * e] - 1 == in) {
          for (int c = 0; c < 6; ++c) acc[c] = acc[c] + se[c + 6 * (k + 9 * (int64_t)e)];
          break;
        }
    }
    for (int c = 0; c < 6; ++c) acc[c] = acc[c] / (double)ns;
  }
  for (int c = 0; c < 6; ++c) sn[c + 6 * (int64_t)in] = acc[c];
  principal_vm(acc, pr + 3 * (int64_t)in, vm + in);
}

}  // namespace

// sigma_elem (6, 9, ne), sigma_node (6, n), prin (3, n), vm (n): device buffers
int launch_boundary_stresses(bem_ctx* c, double* se, double* sn, double* pr, double* vm) {
  if (c->DFI.count == 0 || c->U.count == 0)
    return bem_fail(c, BEM_ERR_STATE, "boundary stresses need a reorganized solution");
  const int64_t nt = 9 * (int64_t)c->ne;
  elem_kernel<<<(unsigned)((nt + 127) / 128), 128, 0, c->stream>>>(c->ne, c->nconec.p, c->kconec.p, c->x.p, c->y.p,
                                                                    c->z.p, c->U.p, c->DFI.p, c->mat.mu,
                                                                    c->mat.nu, se);
  BEM_LAUNCH_CHECK(c);
  node_kernel<<<(c->n + 127) / 128, 128, 0, c->stream>>>(c->n, c->nesim.p, c->ke.p, c->nconec.p, c->kconec.p, se,
                                                         sn, pr, vm);
  BEM_LAUNCH_CHECK(c);
  return BEM_OK;
}

}  // namespace bem
