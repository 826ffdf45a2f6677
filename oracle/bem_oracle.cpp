// ORACLE — test infrastructure only, never the product path.
//
// A plain C++17 + OpenMP restatement of the QUADESTH (e-albuquerque/BEM3D_elastostatic)
// boundary-element hot path, written to reproduce the reference's FP64 results
// operation for operation.  Only the tests, the smoke check and the CPU-baseline
// leg of the benchmark load this library; the CUDA product never calls it.
//
// Parity pin: the reference's own output `internal_points.dat` for its shipped
// input `cube8.dat` (both committed as tests/golden/cube8_golden.npz) is
// reproduced to its printed 7 significant digits (tests/test_oracle_golden.py).
//
// Conventions follow the Fortran module globals exactly:
//   kconec(9, ne)  column-major, node numbers 1-based      -> kconec[m + 9*e]
//   nconec(ne)     6 (tri6) or 9 (quad9)
//   kode(3*ne)     0 = displacement prescribed, 1 = traction prescribed -> kode[3*e + ld]
//   bc(27, ne)     prescribed values, index 3*(k-1)+ld     -> bc[3*k + ld + 27*e]
//   A(3n, 3n)      column-major with leading dimension lda
//   geometry tables all_*(36, ne) and all_ff(9, 36, ne), column-major.
// Compile with -O2 -ffp-contract=off (no FMA contraction, no reassociation) so the
// arithmetic matches gfortran -O3 on baseline x86-64.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// assembly_mod.f90:6-19 — literal quadrature constants (15 and 10 significant digits).
const double gi_quad[6] = {0.238619186083197, -0.238619186083197, 0.661209386466265,
                           -0.661209386466265, 0.932469514203152, -0.932469514203152};
const double ome_quad[6] = {0.467913934572691, 0.467913934572691, 0.360761573048139,
                            0.360761573048139, 0.171324492379170, 0.171324492379170};
const double rr_tri[4] = {0.0694318422, 0.3300094782, 0.6699905218, 0.9305681558};
const double ss_tri[4] = {0.0571041961, 0.2768430136, 0.5835904324, 0.8602401357};
const double omei_tri[4] = {0.1739274226, 0.3260725774, 0.3260725774, 0.1739274226};
const double omej_tri[4] = {0.1355069134, 0.2034645680, 0.1298475476, 0.0311809709};

// data_mod.f90:7
const double PI = 3.14159265358979323846;

struct Consts {
  double c3, c4, c5, c6;
};

// data_mod.f90:97-108 (update_material_constants) — rge (mu) given.
Consts make_consts(double mu, double nu) {
  Consts c;
  c.c3 = 1.0 / (16.0 * PI * (1.0 - nu) * mu);
  c.c4 = 3.0 - 4.0 * nu;
  c.c5 = -1.0 / (8.0 * PI * (1.0 - nu));
  c.c6 = 1.0 - 2.0 * nu;
  return c;
}

// Shape functions and intrinsic derivatives; assembly_mod.f90:247-302 and
// stress_mod.f90:32-112 (identical formulas).  Fortran g**2 is g*g.
void shape(int ncone, double g1, double g2, double* f, double* fd1, double* fd2) {
  if (ncone == 9) {
    f[0] = 0.25 * g1 * g2 * (g1 - 1.0) * (g2 - 1.0);
    f[1] = 0.5 * (1.0 - g1 * g1) * g2 * (g2 - 1.0);
    f[2] = 0.25 * g1 * g2 * (g1 + 1.0) * (g2 - 1.0);
    f[3] = 0.5 * g1 * (g1 + 1.0) * (1.0 - g2 * g2);
    f[4] = 0.25 * g1 * g2 * (g1 + 1.0) * (g2 + 1.0);
    f[5] = 0.5 * (1.0 - g1 * g1) * g2 * (g2 + 1.0);
    f[6] = 0.25 * g1 * g2 * (g1 - 1.0) * (g2 + 1.0);
    f[7] = 0.5 * g1 * (g1 - 1.0) * (1.0 - g2 * g2);
    f[8] = (1.0 - g1 * g1) * (1.0 - g2 * g2);

    fd1[0] = 0.25 * g2 * (g2 - 1.0) * (2.0 * g1 - 1.0);
    fd1[1] = -g1 * g2 * (g2 - 1.0);
    fd1[2] = 0.25 * g2 * (g2 - 1.0) * (2.0 * g1 + 1.0);
    fd1[3] = 0.5 * (1.0 - g2 * g2) * (2.0 * g1 + 1.0);
    fd1[4] = 0.25 * g2 * (g2 + 1.0) * (2.0 * g1 + 1.0);
    fd1[5] = -g1 * g2 * (g2 + 1.0);
    fd1[6] = 0.25 * g2 * (g2 + 1.0) * (2.0 * g1 - 1.0);
    fd1[7] = 0.5 * (1.0 - g2 * g2) * (2.0 * g1 - 1.0);
    fd1[8] = -2.0 * g1 * (1.0 - g2 * g2);

    fd2[0] = 0.25 * g1 * (g1 - 1.0) * (2.0 * g2 - 1.0);
    fd2[1] = 0.5 * (1.0 - g1 * g1) * (2.0 * g2 - 1.0);
    fd2[2] = 0.25 * g1 * (g1 + 1.0) * (2.0 * g2 - 1.0);
    fd2[3] = -g1 * g2 * (g1 + 1.0);
    fd2[4] = 0.25 * g1 * (g1 + 1.0) * (2.0 * g2 + 1.0);
    fd2[5] = 0.5 * (1.0 - g1 * g1) * (2.0 * g2 + 1.0);
    fd2[6] = 0.25 * g1 * (g1 - 1.0) * (2.0 * g2 + 1.0);
    fd2[7] = -g1 * g2 * (g1 - 1.0);
    fd2[8] = -2.0 * g2 * (1.0 - g1 * g1);
  } else {
    const double g3 = 1.0 - g1 - g2;
    f[0] = g1 * (2.0 * g1 - 1.0);
    f[1] = g2 * (2.0 * g2 - 1.0);
    f[2] = g3 * (2.0 * g3 - 1.0);
    f[3] = 4.0 * g1 * g2;
    f[4] = 4.0 * g2 * g3;
    f[5] = 4.0 * g3 * g1;
    fd1[0] = 4.0 * g1 - 1.0;
    fd1[1] = 0.0;
    fd1[2] = 1.0 - 4.0 * g3;
    fd1[3] = 4.0 * g2;
    fd1[4] = -4.0 * g2;
    fd1[5] = 4.0 * (g3 - g1);
    fd2[0] = 0.0;
    fd2[1] = 4.0 * g2 - 1.0;
    fd2[2] = 1.0 - 4.0 * g3;
    fd2[3] = 4.0 * g1;
    fd2[4] = 4.0 * (g3 - g2);
    fd2[5] = -4.0 * g1;
    for (int m = 6; m < 9; ++m) f[m] = fd1[m] = fd2[m] = 0.0;
  }
}

// Jacobian/normal by the dc - dct double sum: assembly_mod.f90:311-334 (also 566-589).
void jac_normal(int ncone, const double* fd1, const double* fd2, const double* xj1,
                const double* xj2, const double* xj3, double* xja, double* e1, double* e2,
                double* e3) {
  double aux[9], bux[9], cux[9];
  for (int jk = 0; jk < ncone; ++jk) {
    aux[jk] = 0.0;
    bux[jk] = 0.0;
    cux[jk] = 0.0;
    for (int ik = 0; ik < ncone; ++ik) {
      const double dc = fd1[ik] * fd2[jk];
      const double dct = fd2[ik] * fd1[jk];
      aux[jk] = aux[jk] + xj2[ik] * (dc - dct);
      bux[jk] = bux[jk] + xj3[ik] * (dc - dct);
      cux[jk] = cux[jk] + xj1[ik] * (dc - dct);
    }
  }
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (int jk = 0; jk < ncone; ++jk) s1 = s1 + aux[jk] * xj3[jk];
  for (int jk = 0; jk < ncone; ++jk) s2 = s2 + bux[jk] * xj1[jk];
  for (int jk = 0; jk < ncone; ++jk) s3 = s3 + cux[jk] * xj2[jk];
  *xja = std::sqrt(s1 * s1 + s2 * s2 + s3 * s3);
  *e1 = s1 / *xja;
  *e2 = s2 / *xja;
  *e3 = s3 / *xja;
}

// funkelvin: assembly_mod.f90:618-650.  u(jj,ii) -> u[jj + 3*ii].
void funkelvin(const Consts& C, double* u, double* t, double xp, double yp, double zp,
               const double* eta, double xg, double yg, double zg) {
  const double r1 = xg - xp, r2 = yg - yp, r3 = zg - zp;
  const double r = std::sqrt(r1 * r1 + r2 * r2 + r3 * r3);
  const double rdn = (r1 * eta[0] + r2 * eta[1] + r3 * eta[2]) / r;
  const double rd[3] = {r1 / r, r2 / r, r3 / r};
  const double c3r = C.c3 / r;
  const double c5r2 = C.c5 / (r * r);
  for (int ii = 0; ii < 3; ++ii)
    for (int jj = 0; jj < 3; ++jj) {
      const double d = (ii == jj) ? 1.0 : 0.0;
      u[jj + 3 * ii] = (C.c4 * d + rd[ii] * rd[jj]) * c3r;
      t[jj + 3 * ii] = c5r2 * (rdn * (C.c6 * d + 3.0 * rd[ii] * rd[jj]) +
                               C.c6 * (eta[jj] * rd[ii] - eta[ii] * rd[jj]));
    }
}

struct Geo {
  const double *eta1, *eta2, *eta3, *xja, *xg1, *xg2, *xg3, *ff;
};

// extin8: assembly_mod.f90:339-384.  h,g are (3,27) column-major: h[jj + 3*ind].
void extin8(const Consts& C, const Geo& G, int e, const double* xi, double* h, double* g,
            int ncone) {
  for (int q = 0; q < 81; ++q) h[q] = g[q] = 0.0;
  const int npg = (ncone < 9) ? 4 : 6;
  for (int i = 0; i < npg; ++i)
    for (int j = 0; j < npg; ++j) {
      const int k = npg * i + j;
      const int kk36 = k + 36 * e;
      const double eta[3] = {G.eta1[kk36], G.eta2[kk36], G.eta3[kk36]};
      double p12[9];
      for (int ik = 0; ik < ncone; ++ik) {
        const double f = G.ff[ik + 9 * kk36];
        if (ncone == 9)
          p12[ik] = f * G.xja[kk36] * ome_quad[i] * ome_quad[j];
        else
          p12[ik] = f * G.xja[kk36] * omei_tri[i] * omej_tri[j];
      }
      double u[9], t[9];
      funkelvin(C, u, t, xi[0], xi[1], xi[2], eta, G.xg1[kk36], G.xg2[kk36], G.xg3[kk36]);
      for (int kk = 0; kk < ncone; ++kk)
        for (int ii = 0; ii < 3; ++ii)
          for (int jj = 0; jj < 3; ++jj) {
            const int ind = 3 * kk + ii;
            g[jj + 3 * ind] = g[jj + 3 * ind] + u[jj + 3 * ii] * p12[kk];
            h[jj + 3 * ind] = h[jj + 3 * ind] + t[jj + 3 * ii] * p12[kk];
          }
    }
}

// triloc8: assembly_mod.f90:492-616.  v1/v2 hold the parent coordinates of the
// three sub-triangle vertices (first vertex = the collocation node).
void triloc8(const Consts& C, const double* xi, const double* xj1, const double* xj2,
             const double* xj3, double* h, double* g, double area, const double* v1,
             const double* v2, int ncone) {
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      const double ss1 = 0.5 * (gi_quad[i] + 1.0);
      const double ss2 = 0.5 * (gi_quad[j] + 1.0);
      const double g1 = (1.0 - ss1) * v1[0] + ss1 * (1.0 - ss2) * v1[1] + ss1 * ss2 * v1[2];
      const double g2 = (1.0 - ss1) * v2[0] + ss1 * (1.0 - ss2) * v2[1] + ss1 * ss2 * v2[2];
      double f[9], fd1[9], fd2[9];
      shape(ncone, g1, g2, f, fd1, fd2);
      double xja, eta[3];
      jac_normal(ncone, fd1, fd2, xj1, xj2, xj3, &xja, &eta[0], &eta[1], &eta[2]);
      double xp[3] = {0.0, 0.0, 0.0};
      for (int ik = 0; ik < ncone; ++ik) {
        xp[0] = xp[0] + f[ik] * xj1[ik];
        xp[1] = xp[1] + f[ik] * xj2[ik];
        xp[2] = xp[2] + f[ik] * xj3[ik];
      }
      double p12[9];
      for (int ik = 0; ik < ncone; ++ik)
        p12[ik] = f[ik] * xja * (gi_quad[i] + 1.0) * area * 0.25 * ome_quad[i] * ome_quad[j];
      double u[9], t[9];
      funkelvin(C, u, t, xi[0], xi[1], xi[2], eta, xp[0], xp[1], xp[2]);
      for (int kk = 0; kk < ncone; ++kk)
        for (int ii = 0; ii < 3; ++ii)
          for (int jj = 0; jj < 3; ++jj) {
            const int ind = 3 * kk + ii;
            g[jj + 3 * ind] = g[jj + 3 * ind] + u[jj + 3 * ii] * p12[kk];
            h[jj + 3 * ind] = h[jj + 3 * ind] + t[jj + 3 * ii] * p12[kk];
          }
    }
}

// locin8: assembly_mod.f90:386-490.  nodo is 1-based as in the reference.
void locin8(const Consts& C, const double* xj1, const double* xj2, const double* xj3,
            double* h, double* g, int nodo, int ncone) {
  for (int q = 0; q < 81; ++q) h[q] = g[q] = 0.0;
  double v1[3], v2[3], xi[3];
  if (ncone == 9) {
    const double gi1[9] = {-1.0, 0.0, 1.0, 1.0, 1.0, 0.0, -1.0, -1.0, 0.0};
    const double gi2[9] = {-1.0, -1.0, -1.0, 0.0, 1.0, 1.0, 1.0, 0.0, 0.0};
    double gii1[15], gii2[15];
    for (int q = 0; q < 8; ++q) {
      gii1[q] = gi1[q];
      gii2[q] = gi2[q];
    }
    for (int q = 0; q < 7; ++q) {
      gii1[8 + q] = gi1[q];
      gii2[8 + q] = gi2[q];
    }
    // 1-based helpers
    auto G1 = [&](int p) { return gii1[p - 1]; };
    auto G2 = [&](int p) { return gii2[p - 1]; };
    v1[0] = gi1[nodo - 1];
    v2[0] = gi2[nodo - 1];
    xi[0] = xj1[nodo - 1];
    xi[1] = xj2[nodo - 1];
    xi[2] = xj3[nodo - 1];
    if (nodo == 1 || nodo == 3 || nodo == 5 || nodo == 7) {
      const double area = 2.0;
      for (int k = 1; k <= 2; ++k) {
        const int m = 2 * k;
        v1[1] = G1(nodo + m);
        v2[1] = G2(nodo + m);
        v1[2] = G1(nodo + m + 2);
        v2[2] = G2(nodo + m + 2);
        triloc8(C, xi, xj1, xj2, xj3, h, g, area, v1, v2, 9);
      }
    } else if (nodo == 2 || nodo == 4 || nodo == 6 || nodo == 8) {
      for (int k = 1; k <= 3; ++k) {
        const int m = 2 * k - 1;
        v1[1] = G1(nodo + m);
        v2[1] = G2(nodo + m);
        v1[2] = G1(nodo + m + 2);
        v2[2] = G2(nodo + m + 2);
        const double area = 0.5 * (v1[1] * v2[2] + v1[0] * v2[1] + v1[2] * v2[0] -
                                   v1[1] * v2[0] - v1[2] * v2[1] - v1[0] * v2[2]);
        triloc8(C, xi, xj1, xj2, xj3, h, g, area, v1, v2, 9);
      }
    } else {
      const double area = 1.0;
      for (int k = 1; k <= 4; ++k) {
        const int m = 2 * k - 1;
        v1[1] = G1(m);
        v2[1] = G2(m);
        v1[2] = G1(m + 2);
        v2[2] = G2(m + 2);
        triloc8(C, xi, xj1, xj2, xj3, h, g, area, v1, v2, 9);
      }
    }
  } else {
    const double gi1[6] = {1.0, 0.0, 0.0, 0.5, 0.0, 0.5};
    const double gi2[6] = {0.0, 1.0, 0.0, 0.5, 0.5, 0.0};
    v1[0] = gi1[nodo - 1];
    v2[0] = gi2[nodo - 1];
    xi[0] = xj1[nodo - 1];
    xi[1] = xj2[nodo - 1];
    xi[2] = xj3[nodo - 1];
    auto tri = [&](int a, int b, double area) {
      v1[1] = gi1[a - 1];
      v2[1] = gi2[a - 1];
      v1[2] = gi1[b - 1];
      v2[2] = gi2[b - 1];
      triloc8(C, xi, xj1, xj2, xj3, h, g, area, v1, v2, 6);
    };
    switch (nodo) {
      case 1: tri(2, 3, 0.5); break;
      case 2: tri(3, 1, 0.5); break;
      case 3: tri(1, 2, 0.5); break;
      case 4: tri(2, 3, 0.25); tri(3, 1, 0.25); break;
      case 5: tri(3, 1, 0.25); tri(1, 2, 0.25); break;
      case 6: tri(1, 2, 0.25); tri(2, 3, 0.25); break;
      default: break;
    }
  }
}

}  // namespace

extern "C" {

typedef struct {
  int n, ne;
  const double *x, *y, *z;
  const int* nconec;  // (ne)
  const int* kconec;  // (9, ne), 1-based node numbers
  const int* kode;    // (3*ne)
  const double* bc;   // (27, ne)
  double mu, nu;
} orc_mesh;

// Node -> element adjacency nesim/ke, io_mod.f90:125-135 (ke capped at 8).
// Returns the largest nesim seen (the caller rejects > 8).
int orc_adjacency(const orc_mesh* M, int* nesim, int* ke) {
  for (int i = 0; i < M->n; ++i) nesim[i] = 0;
  int mx = 0;
  for (int e = 0; e < M->ne; ++e)
    for (int j = 0; j < M->nconec[e]; ++j) {
      const int in = M->kconec[j + 9 * e] - 1;
      nesim[in] += 1;
      if (nesim[in] <= 8) ke[(nesim[in] - 1) + 8 * in] = e + 1;
      if (nesim[in] > mx) mx = nesim[in];
    }
  return mx;
}

// precompute_element_geometry / etaxja: assembly_mod.f90:28-51, 225-337.
int orc_geometry(const orc_mesh* M, double* eta1, double* eta2, double* eta3, double* xja,
                 double* xg1, double* xg2, double* xg3, double* ff) {
  const int ne = M->ne;
#pragma omp parallel for schedule(static)
  for (int e = 0; e < ne; ++e) {
    const int ncone = M->nconec[e];
    double xj1[9] = {0}, xj2[9] = {0}, xj3[9] = {0};
    for (int m = 0; m < ncone; ++m) {
      const int k = M->kconec[m + 9 * e] - 1;
      xj1[m] = M->x[k];
      xj2[m] = M->y[k];
      xj3[m] = M->z[k];
    }
    for (int q = 0; q < 36; ++q) {
      const int kk = q + 36 * e;
      eta1[kk] = eta2[kk] = eta3[kk] = xja[kk] = 0.0;
      xg1[kk] = xg2[kk] = xg3[kk] = 0.0;
      for (int m = 0; m < 9; ++m) ff[m + 9 * kk] = 0.0;
    }
    const int npg = (ncone < 9) ? 4 : 6;
    for (int i = 0; i < npg; ++i)
      for (int j = 0; j < npg; ++j) {
        const int k = npg * i + j;
        const int kk = k + 36 * e;
        double g1, g2;
        if (ncone == 9) {
          g1 = gi_quad[i];
          g2 = gi_quad[j];
        } else {
          g1 = ss_tri[j];
          g2 = rr_tri[i] * (1.0 - ss_tri[j]);
        }
        double f[9], fd1[9], fd2[9];
        shape(ncone, g1, g2, f, fd1, fd2);
        for (int m = 0; m < ncone; ++m) ff[m + 9 * kk] = f[m];
        double a = 0.0, b = 0.0, c = 0.0;
        for (int ik = 0; ik < ncone; ++ik) {
          a = a + f[ik] * xj1[ik];
          b = b + f[ik] * xj2[ik];
          c = c + f[ik] * xj3[ik];
        }
        xg1[kk] = a;
        xg2[kk] = b;
        xg3[kk] = c;
        jac_normal(ncone, fd1, fd2, xj1, xj2, xj3, &xja[kk], &eta1[kk], &eta2[kk], &eta3[kk]);
      }
  }
  return 0;
}

typedef struct {
  const double *eta1, *eta2, *eta3, *xja, *xg1, *xg2, *xg3, *ff;
} orc_geo;

static int lookup_vp(const orc_mesh* M, const int* nesim, const int* ke, int ik0, int ld,
                     double* vp) {
  // assembly_mod.f90:149-161 (ik0 0-based, ld 0-based)
  for (int i = 0; i < nesim[ik0]; ++i) {
    const int e = ke[i + 8 * ik0] - 1;
    if (M->kode[3 * e + ld] == 0) {
      for (int m = 0; m < M->nconec[e]; ++m)
        if (M->kconec[m + 9 * e] - 1 == ik0) {
          *vp = M->bc[3 * m + ld + 27 * e];
          return 1;
        }
    }
  }
  return 0;
}

// ghmat8: assembly_mod.f90:53-223, restricted to collocation nodes [in0, in1) (0-based).
// A receives rows 3*(in-in0)+jj with leading dimension lda (3n columns); FI receives
// 3*(in1-in0) entries.  Both are zeroed here first (assembly_mod.f90:61-62).
// Returns 0, or -1 if some node lies in more than 8 elements.
int orc_ghmat8(const orc_mesh* M, const orc_geo* Gp, int in0, int in1, double* A, int64_t lda,
               double* FI) {
  const int n = M->n, ne = M->ne;
  std::vector<int> nesim(n), ke(8 * (size_t)n, 0);
  if (orc_adjacency(M, nesim.data(), ke.data()) > 8) return -1;
  const Consts C = make_consts(M->mu, M->nu);
  Geo G{Gp->eta1, Gp->eta2, Gp->eta3, Gp->xja, Gp->xg1, Gp->xg2, Gp->xg3, Gp->ff};
  const int nrow = 3 * (in1 - in0);
  for (int64_t c = 0; c < 3 * (int64_t)n; ++c)
    for (int r = 0; r < nrow; ++r) A[r + c * lda] = 0.0;
  for (int r = 0; r < nrow; ++r) FI[r] = 0.0;
  const double rge = M->mu;

#pragma omp parallel for schedule(dynamic)
  for (int in = in0; in < in1; ++in) {
    const int ro = 3 * (in - in0);
    const double xi[3] = {M->x[in], M->y[in], M->z[in]};
    double h[81], g[81];
    for (int e = 0; e < ne; ++e) {
      const int ncone = M->nconec[e];
      double xj1[9] = {0}, xj2[9] = {0}, xj3[9] = {0};
      for (int m = 0; m < ncone; ++m) {
        const int k = M->kconec[m + 9 * e] - 1;
        xj1[m] = M->x[k];
        xj2[m] = M->y[k];
        xj3[m] = M->z[k];
      }
      int nodo = 0;
      for (int i = 0; i < ncone; ++i)
        if (in == M->kconec[i + 9 * e] - 1) {
          nodo = i + 1;
          break;
        }
      if (nodo > 0)
        locin8(C, xj1, xj2, xj3, h, g, nodo, ncone);
      else
        extin8(C, G, e, xi, h, g, ncone);

      double d1[9] = {0}, d2[9] = {0};  // d(i,j) -> d[i + 3*j]
      if (nodo == 0) {
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i < 3; ++i)
            for (int k = 0; k < ncone; ++k) d1[i + 3 * j] = d1[i + 3 * j] - h[i + 3 * (3 * k + j)];
      } else {
        for (int j = 0; j < 3; ++j)
          for (int i = 0; i < 3; ++i)
            for (int k = 0; k < ncone; ++k)
              if (k != nodo - 1) d2[i + 3 * j] = d2[i + 3 * j] - h[i + 3 * (3 * k + j)];
      }

      for (int ld = 0; ld < 3; ++ld) {
        if (M->kode[3 * e + ld] == 0) {
          for (int k = 0; k < ncone; ++k) {
            const int ik = M->kconec[k + 9 * e] - 1;
            const int64_t col = 3 * (int64_t)ik + ld;
            const int ind = 3 * k + ld;
            const double bcv = M->bc[ind + 27 * e];
            for (int r = 0; r < 3; ++r)
              A[ro + r + col * lda] = A[ro + r + col * lda] - g[r + 3 * ind] * rge;
            if (in != ik) {
              for (int r = 0; r < 3; ++r) FI[ro + r] = FI[ro + r] - h[r + 3 * ind] * bcv;
            } else {
              for (int r = 0; r < 3; ++r) FI[ro + r] = FI[ro + r] - d2[r + 3 * ld] * bcv;
            }
          }
        } else {
          for (int k = 0; k < ncone; ++k) {
            const int ik = M->kconec[k + 9 * e] - 1;
            const int ind = 3 * k + ld;
            const double bcv = M->bc[ind + 27 * e];
            double vp = 0.0;
            const int kode0 = lookup_vp(M, nesim.data(), ke.data(), ik, ld, &vp);
            if (kode0 == 0) {
              for (int r = 0; r < 3; ++r) FI[ro + r] = FI[ro + r] + g[r + 3 * ind] * bcv;
              if (in != ik) {
                const int64_t col = 3 * (int64_t)ik + ld;
                for (int r = 0; r < 3; ++r)
                  A[ro + r + col * lda] = A[ro + r + col * lda] + h[r + 3 * ind];
              } else {
                const int64_t col = 3 * (int64_t)in + ld;
                for (int r = 0; r < 3; ++r)
                  A[ro + r + col * lda] = A[ro + r + col * lda] + d2[r + 3 * ld];
              }
            } else {
              if (in != ik) {
                for (int r = 0; r < 3; ++r)
                  FI[ro + r] = FI[ro + r] + g[r + 3 * ind] * bcv - h[r + 3 * ind] * vp;
              } else {
                for (int r = 0; r < 3; ++r)
                  FI[ro + r] = FI[ro + r] + g[r + 3 * ind] * bcv - d2[r + 3 * ld] * vp;
              }
            }
          }
        }
      }

      if (nodo == 0) {
        for (int ld = 0; ld < 3; ++ld) {
          double vp = 0.0;
          const int kode0 = lookup_vp(M, nesim.data(), ke.data(), in, ld, &vp);
          if (kode0 == 0) {
            const int64_t col = 3 * (int64_t)in + ld;
            for (int r = 0; r < 3; ++r)
              A[ro + r + col * lda] = A[ro + r + col * lda] + d1[r + 3 * ld];
          } else {
            for (int r = 0; r < 3; ++r) FI[ro + r] = FI[ro + r] - d1[r + 3 * ld] * vp;
          }
        }
      }
    }
  }
  return 0;
}

// H and G as separate products (the reference never forms them; they are the
// blocks ghmat8 combines).  Rows for collocation nodes [in0, in1):
//   H (3*(in1-in0), 3n): off-diagonal blocks sum h_elem over the elements holding
//   the column node; the diagonal 3x3 block is the rigid-body sum of d1 and d2
//   (assembly_mod.f90:100-123), i.e. -sum_{j != i} H_ij.
//   G (3*(in1-in0), 27*ne): G(row, 27*e + 3k + ii) = g_elem(row, 3k+ii) of element e.
int orc_hg(const orc_mesh* M, const orc_geo* Gp, int in0, int in1, double* H, int64_t ldh,
           double* Gm, int64_t ldg) {
  const int n = M->n, ne = M->ne;
  const Consts C = make_consts(M->mu, M->nu);
  Geo G{Gp->eta1, Gp->eta2, Gp->eta3, Gp->xja, Gp->xg1, Gp->xg2, Gp->xg3, Gp->ff};
  const int nrow = 3 * (in1 - in0);
  for (int64_t c = 0; c < 3 * (int64_t)n; ++c)
    for (int r = 0; r < nrow; ++r) H[r + c * ldh] = 0.0;
  for (int64_t c = 0; c < 27 * (int64_t)ne; ++c)
    for (int r = 0; r < nrow; ++r) Gm[r + c * ldg] = 0.0;
#pragma omp parallel for schedule(dynamic)
  for (int in = in0; in < in1; ++in) {
    const int ro = 3 * (in - in0);
    const double xi[3] = {M->x[in], M->y[in], M->z[in]};
    double h[81], g[81];
    for (int e = 0; e < ne; ++e) {
      const int ncone = M->nconec[e];
      double xj1[9] = {0}, xj2[9] = {0}, xj3[9] = {0};
      for (int m = 0; m < ncone; ++m) {
        const int k = M->kconec[m + 9 * e] - 1;
        xj1[m] = M->x[k];
        xj2[m] = M->y[k];
        xj3[m] = M->z[k];
      }
      int nodo = 0;
      for (int i = 0; i < ncone; ++i)
        if (in == M->kconec[i + 9 * e] - 1) {
          nodo = i + 1;
          break;
        }
      if (nodo > 0)
        locin8(C, xj1, xj2, xj3, h, g, nodo, ncone);
      else
        extin8(C, G, e, xi, h, g, ncone);
      for (int ind = 0; ind < 3 * ncone; ++ind)
        for (int r = 0; r < 3; ++r) Gm[ro + r + (27 * (int64_t)e + ind) * ldg] = g[r + 3 * ind];
      for (int k = 0; k < ncone; ++k) {
        if (k == nodo - 1) continue;
        const int ik = M->kconec[k + 9 * e] - 1;
        for (int ii = 0; ii < 3; ++ii) {
          const int64_t col = 3 * (int64_t)ik + ii;
          for (int r = 0; r < 3; ++r) H[ro + r + col * ldh] += h[r + 3 * (3 * k + ii)];
        }
      }
      // rigid-body diagonal, same d1/d2 sums as ghmat8
      double d[9] = {0};
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i)
          for (int k = 0; k < ncone; ++k)
            if (k != nodo - 1) d[i + 3 * j] = d[i + 3 * j] - h[i + 3 * (3 * k + j)];
      for (int ld = 0; ld < 3; ++ld) {
        const int64_t col = 3 * (int64_t)in + ld;
        for (int r = 0; r < 3; ++r) H[ro + r + col * ldh] += d[r + 3 * ld];
      }
    }
  }
  return 0;
}

// reorganize_solution: io_mod.f90:148-183.  FI (3n) in: solution x, out: u.
int orc_reorganize(const orc_mesh* M, double* FI, double* DFI) {
  const int n = M->n, ne = M->ne;
  std::vector<int> nesim(n), ke(8 * (size_t)n, 0);
  if (orc_adjacency(M, nesim.data(), ke.data()) > 8) return -1;
  for (int e = 0; e < ne; ++e)
    for (int ld = 0; ld < 3; ++ld) {
      if (M->kode[3 * e + ld] == 0) {
        for (int k = 0; k < M->nconec[e]; ++k) {
          const int ik = M->kconec[k + 9 * e] - 1;
          DFI[3 * k + ld + 27 * e] = FI[3 * ik + ld] * M->mu;
        }
      } else {
        for (int k = 0; k < M->nconec[e]; ++k)
          DFI[3 * k + ld + 27 * e] = M->bc[3 * k + ld + 27 * e];
      }
    }
  for (int in = 0; in < n; ++in)
    for (int ld = 0; ld < 3; ++ld)
      for (int j = 0; j < nesim[in]; ++j) {
        const int e = ke[j + 8 * in] - 1;
        if (M->kode[3 * e + ld] == 0) {
          for (int m = 0; m < M->nconec[e]; ++m)
            if (in == M->kconec[m + 9 * e] - 1) {
              FI[3 * in + ld] = M->bc[3 * m + ld + 27 * e];
              break;
            }
          break;
        }
      }
  return 0;
}

// gauss_legendre_1d: stress_mod.f90:475-503.
void orc_gauss_legendre(int n_pts, double* x_gl, double* w_gl) {
  const int m_half = (n_pts + 1) / 2;
  for (int i = 1; i <= m_half; ++i) {
    double z = std::cos(PI * ((double)i - 0.25) / ((double)n_pts + 0.5));
    double p1 = 0, p2 = 0, p3 = 0, pp = 0;
    for (int iter = 1; iter <= 100; ++iter) {
      p1 = 1.0;
      p2 = 0.0;
      for (int j = 1; j <= n_pts; ++j) {
        p3 = p2;
        p2 = p1;
        p1 = ((2.0 * (double)j - 1.0) * z * p2 - (double)(j - 1) * p3) / (double)j;
      }
      pp = (double)n_pts * (z * p1 - p2) / (z * z - 1.0);
      const double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) <= 1.0e-15) break;
    }
    x_gl[i - 1] = -z;
    x_gl[n_pts - i] = z;
    w_gl[i - 1] = 2.0 / ((1.0 - z * z) * pp * pp);
    w_gl[n_pts - i] = w_gl[i - 1];
  }
}

// calc_principal_and_vm: stress_mod.f90:299-359.
void orc_principal(const double* sig, double* prin, double* vm) {
  const double sxx = sig[0], syy = sig[1], szz = sig[2], sxy = sig[3], syz = sig[4],
               szx = sig[5];
  const double tol = 1.0e-20;
  *vm = std::sqrt(0.5 * ((sxx - syy) * (sxx - syy) + (syy - szz) * (syy - szz) +
                         (szz - sxx) * (szz - sxx) + 6.0 * (sxy * sxy + syz * syz + szx * szx)));
  const double i1 = sxx + syy + szz;
  const double q = i1 / 3.0;
  const double pxx = sxx - q, pyy = syy - q, pzz = szz - q;
  const double j2 = 0.5 * (pxx * pxx + pyy * pyy + pzz * pzz) + sxy * sxy + syz * syz + szx * szx;
  if (j2 <= tol * (i1 * i1 + 1.0)) {
    prin[0] = prin[1] = prin[2] = q;
    return;
  }
  const double j3 = pxx * (pyy * pzz - syz * syz) - sxy * (sxy * pzz - syz * szx) +
                    szx * (sxy * syz - pyy * szx);
  const double r = std::sqrt(4.0 * j2 / 3.0);
  double c3p = 4.0 * j3 / (r * r * r);
  if (c3p > 1.0) c3p = 1.0;
  if (c3p < -1.0) c3p = -1.0;
  const double phi = std::acos(c3p) / 3.0;
  prin[0] = q + r * std::cos(phi);
  prin[2] = q + r * std::cos(phi + 2.0 * PI / 3.0);
  prin[1] = 3.0 * q - prin[0] - prin[2];
  double tmp;
  if (prin[0] < prin[1]) { tmp = prin[0]; prin[0] = prin[1]; prin[1] = tmp; }
  if (prin[1] < prin[2]) { tmp = prin[1]; prin[1] = prin[2]; prin[2] = tmp; }
  if (prin[0] < prin[1]) { tmp = prin[0]; prin[0] = prin[1]; prin[1] = tmp; }
}

// axes_cos_lagrange: stress_mod.f90:119-168.  Orthonormal triad L (rows e1, e2, e3)
// and the intrinsic-to-local map CL at a point of an element.
static void axes_cos(int ncone, const double* fd1, const double* fd2, const double* cx, const double* cy,
                     const double* cz, double L[3][3], double CL[2][2]) {
  double g1[3] = {0, 0, 0}, g2[3] = {0, 0, 0}, g3[3];
  for (int a = 0; a < ncone; ++a) {
    const double c[3] = {cx[a], cy[a], cz[a]};
    for (int i = 0; i < 3; ++i) {
      g1[i] = g1[i] + fd1[a] * c[i];
      g2[i] = g2[i] + fd2[a] * c[i];
    }
  }
  const double v1 = std::sqrt(g1[0] * g1[0] + g1[1] * g1[1] + g1[2] * g1[2]);
  const double v2 = std::sqrt(g2[0] * g2[0] + g2[1] * g2[1] + g2[2] * g2[2]);
  g3[0] = g1[1] * g2[2] - g1[2] * g2[1];
  g3[1] = g1[2] * g2[0] - g1[0] * g2[2];
  g3[2] = g1[0] * g2[1] - g1[1] * g2[0];
  const double jcb = std::sqrt(g3[0] * g3[0] + g3[1] * g3[1] + g3[2] * g3[2]);
  for (int i = 0; i < 3; ++i) {
    L[2][i] = g3[i] / jcb;
    L[0][i] = g1[i] / v1;
  }
  L[1][0] = L[2][1] * L[0][2] - L[2][2] * L[0][1];
  L[1][1] = L[2][2] * L[0][0] - L[2][0] * L[0][2];
  L[1][2] = L[2][0] * L[0][1] - L[2][1] * L[0][0];
  double cos_th = (g1[0] * g2[0] + g1[1] * g2[1] + g1[2] * g2[2]) / (v1 * v2);
  if (cos_th > 1.0) cos_th = 1.0;
  if (cos_th < -1.0) cos_th = -1.0;
  double sin_th = std::sqrt(std::max(0.0, 1.0 - cos_th * cos_th));
  if (sin_th < 1.0e-12) sin_th = 1.0e-12;
  CL[0][0] = 1.0 / v1;
  CL[0][1] = -cos_th / (v1 * sin_th);
  CL[1][0] = 0.0;
  CL[1][1] = 1.0 / (v2 * sin_th);
}

// compute_boundary_stresses with boundary_stresses_elem: stress_mod.f90:174-297,
// 365-406.  FI: nodal displacements, DFI(27, ne): element-nodal tractions (after
// reorganize_solution).  Outputs: sigma_elem(6, 9, ne) (nullable), sigma_node(6, n),
// prin(3, n), vm(n).  Stress order xx, yy, zz, xy, yz, zx.
int orc_boundary_stresses(const orc_mesh* M, const double* FI, const double* DFI, double* sigma_elem,
                          double* sigma_node, double* prin, double* vm) {
  const int n = M->n, ne = M->ne;
  std::vector<int> nesim(n), ke(8 * (size_t)n, 0);
  if (orc_adjacency(M, nesim.data(), ke.data()) > 8) return -1;
  std::vector<double> se(54 * (size_t)ne, 0.0);
  const double rge = M->mu, xnu = M->nu;
  const double c_eps = 2.0 * rge / (1.0 - xnu);
  const double c_nu = 2.0 * rge * xnu / (1.0 - xnu);
  const double c_sig3 = xnu / (1.0 - xnu);
  const double q1[9] = {-1.0, 0.0, 1.0, 1.0, 1.0, 0.0, -1.0, -1.0, 0.0};
  const double q2[9] = {-1.0, -1.0, -1.0, 0.0, 1.0, 1.0, 1.0, 0.0, 0.0};
  const double t1[6] = {1.0, 0.0, 0.0, 0.5, 0.0, 0.5};
  const double t2[6] = {0.0, 1.0, 0.0, 0.5, 0.5, 0.0};
#pragma omp parallel for schedule(dynamic)
  for (int e = 0; e < ne; ++e) {
    const int ncone = M->nconec[e];
    double cx[9], cy[9], cz[9], ue[3][9], te[3][9];
    for (int a = 0; a < ncone; ++a) {
      const int ik = M->kconec[a + 9 * e] - 1;
      cx[a] = M->x[ik];
      cy[a] = M->y[ik];
      cz[a] = M->z[ik];
      for (int i = 0; i < 3; ++i) {
        ue[i][a] = FI[3 * ik + i];
        te[i][a] = DFI[3 * a + i + 27 * e];
      }
    }
    for (int k = 0; k < ncone; ++k) {
      const double g1 = ncone == 9 ? q1[k] : t1[k], g2 = ncone == 9 ? q2[k] : t2[k];
      double ff[9], fd1[9], fd2[9], L[3][3], CL[2][2];
      shape(ncone, g1, g2, ff, fd1, fd2);
      axes_cos(ncone, fd1, fd2, cx, cy, cz, L, CL);
      double u1_1 = 0.0, u2_2 = 0.0, u1_2 = 0.0, u2_1 = 0.0;
      for (int a = 0; a < ncone; ++a) {
        const double dn1 = CL[0][0] * fd1[a] + CL[1][0] * fd2[a];
        const double dn2 = CL[0][1] * fd1[a] + CL[1][1] * fd2[a];
        const double ul1 = L[0][0] * ue[0][a] + L[0][1] * ue[1][a] + L[0][2] * ue[2][a];
        const double ul2 = L[1][0] * ue[0][a] + L[1][1] * ue[1][a] + L[1][2] * ue[2][a];
        u1_1 = u1_1 + dn1 * ul1;
        u2_2 = u2_2 + dn2 * ul2;
        u1_2 = u1_2 + dn2 * ul1;
        u2_1 = u2_1 + dn1 * ul2;
      }
      const double eps11 = u1_1, eps22 = u2_2, eps12 = 0.5 * (u1_2 + u2_1);
      double tl[3];
      for (int i = 0; i < 3; ++i) tl[i] = L[i][0] * te[0][k] + L[i][1] * te[1][k] + L[i][2] * te[2][k];
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
      // S_glob = L^T (S_loc L)
      double T[3][3], Gm[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) T[i][j] = S[i][0] * L[0][j] + S[i][1] * L[1][j] + S[i][2] * L[2][j];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Gm[i][j] = L[0][i] * T[0][j] + L[1][i] * T[1][j] + L[2][i] * T[2][j];
      double* o = &se[6 * (k + 9 * (size_t)e)];
      o[0] = Gm[0][0];
      o[1] = Gm[1][1];
      o[2] = Gm[2][2];
      o[3] = 0.5 * (Gm[0][1] + Gm[1][0]);
      o[4] = 0.5 * (Gm[1][2] + Gm[2][1]);
      o[5] = 0.5 * (Gm[2][0] + Gm[0][2]);
    }
  }
  for (int in = 0; in < n; ++in) {
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const int ns = std::min(nesim[in], 8);
    if (ns > 0) {
      for (int j = 0; j < ns; ++j) {
        const int e = ke[j + 8 * in] - 1;
        for (int k = 0; k < M->nconec[e]; ++k)
          if (M->kconec[k + 9 * e] - 1 == in) {
            for (int c = 0; c < 6; ++c) acc[c] = acc[c] + se[c + 6 * (k + 9 * (size_t)e)];
            break;
          }
      }
      for (int c = 0; c < 6; ++c) acc[c] = acc[c] / (double)ns;
    }
    for (int c = 0; c < 6; ++c) sigma_node[c + 6 * (size_t)in] = acc[c];
    orc_principal(acc, prin + 3 * (size_t)in, vm + in);
  }
  if (sigma_elem)
    for (size_t i = 0; i < se.size(); ++i) sigma_elem[i] = se[i];
  return 0;
}

// compute_internal_points: stress_mod.f90:511-781 with accumulate_somigliana_range
// (:788-886), for points [p0, p1) (0-based).  FI holds the nodal displacements
// and DFI(27, ne) the element-nodal tractions (after reorganize_solution).
// Outputs are indexed by point: u_int(3,l), sigma_int(6,l), prin(3,l), vm(l).
// flags bit 0: use T*_ij u_j with the antisymmetric part of funkelvin
// (assembly_mod.f90:646-647) in the displacement identity.  The reference's
// stress_mod.f90:838-843 uses the transposed antisymmetric part, which leaves
// internal displacements wrong for general loading; bit 0 clear reproduces it.
int orc_internal_points(const orc_mesh* M, const orc_geo* Gp, const double* FI,
                        const double* DFI, int l, const double* cx, const double* cy,
                        const double* cz, int p0, int p1, double* u_int, double* sigma_int,
                        double* prin, double* vm, int flags) {
  const double asg = (flags & 1) ? -1.0 : 1.0;
  const int ne = M->ne;
  const int NG = 40;
  const double rge = M->mu;
  double xgl[NG], wgl[NG];
  orc_gauss_legendre(NG, xgl, wgl);
  std::vector<double> elc(3 * (size_t)ne), thr(ne);
  std::vector<int> fs(ne), fe(ne);
  int tot_far = 0;
  for (int e = 0; e < ne; ++e) tot_far += (M->nconec[e] == 9) ? 36 : 16;
  const size_t tot_near = (size_t)ne * NG * NG;
  // far and near tables: x,y,z,nx,ny,nz,u*w(3),t*w(3) -> 12 doubles per point
  std::vector<double> gfar(12 * (size_t)tot_far), fn(12 * tot_near);
  int igp = 0;
  for (int e = 0; e < ne; ++e) {
    const int ncone = M->nconec[e];
    double xj1[9], xj2[9], xj3[9];
    double ex = 0.0, ey = 0.0, ez = 0.0;
    for (int m = 0; m < ncone; ++m) {
      const int ik = M->kconec[m + 9 * e] - 1;
      xj1[m] = M->x[ik];
      xj2[m] = M->y[ik];
      xj3[m] = M->z[ik];
      ex = ex + xj1[m];
      ey = ey + xj2[m];
      ez = ez + xj3[m];
    }
    ex = ex / (double)ncone;
    ey = ey / (double)ncone;
    ez = ez / (double)ncone;
    elc[3 * e] = ex;
    elc[3 * e + 1] = ey;
    elc[3 * e + 2] = ez;
    double dmax2 = 0.0;
    for (int m = 0; m < ncone; ++m) {
      const double dx = xj1[m] - ex, dy = xj2[m] - ey, dz = xj3[m] - ez;
      const double d2 = dx * dx + dy * dy + dz * dz;
      dmax2 = (dmax2 > d2) ? dmax2 : d2;
    }
    thr[e] = (3.5 * 3.5) * dmax2;
    const int npg = (ncone == 9) ? 6 : 4;
    fs[e] = igp;
    for (int i = 0; i < npg; ++i)
      for (int j = 0; j < npg; ++j) {
        const int k = npg * i + j;
        const int kk = k + 36 * e;
        const double wg = (ncone == 9) ? ome_quad[i] * ome_quad[j] * Gp->xja[kk]
                                       : omei_tri[i] * omej_tri[j] * Gp->xja[kk];
        double* P = &gfar[12 * (size_t)igp];
        P[0] = Gp->xg1[kk];
        P[1] = Gp->xg2[kk];
        P[2] = Gp->xg3[kk];
        P[3] = Gp->eta1[kk];
        P[4] = Gp->eta2[kk];
        P[5] = Gp->eta3[kk];
        double ug[3] = {0, 0, 0}, tg[3] = {0, 0, 0};
        for (int m = 0; m < ncone; ++m) {
          const int ik = M->kconec[m + 9 * e] - 1;
          const double fv = Gp->ff[m + 9 * kk];
          ug[0] = ug[0] + fv * FI[3 * ik];
          ug[1] = ug[1] + fv * FI[3 * ik + 1];
          ug[2] = ug[2] + fv * FI[3 * ik + 2];
          tg[0] = tg[0] + fv * DFI[3 * m + 27 * e];
          tg[1] = tg[1] + fv * DFI[3 * m + 1 + 27 * e];
          tg[2] = tg[2] + fv * DFI[3 * m + 2 + 27 * e];
        }
        P[6] = ug[0] * wg;
        P[7] = ug[1] * wg;
        P[8] = ug[2] * wg;
        P[9] = tg[0] * wg;
        P[10] = tg[1] * wg;
        P[11] = tg[2] * wg;
        ++igp;
      }
    fe[e] = igp;
  }
#pragma omp parallel for schedule(static)
  for (int e = 0; e < ne; ++e) {
    const int ncone = M->nconec[e];
    double xj1[9], xj2[9], xj3[9];
    for (int m = 0; m < ncone; ++m) {
      const int ik = M->kconec[m + 9 * e] - 1;
      xj1[m] = M->x[ik];
      xj2[m] = M->y[ik];
      xj3[m] = M->z[ik];
    }
    for (int i = 0; i < NG; ++i)
      for (int j = 0; j < NG; ++j) {
        const size_t q = (size_t)e * NG * NG + (size_t)i * NG + j;
        double g1, g2, tj;
        if (ncone == 9) {
          g1 = xgl[i];
          g2 = xgl[j];
          tj = 1.0;
        } else {
          g1 = 0.5 * (1.0 + xgl[i]);
          g2 = 0.25 * (1.0 - xgl[i]) * (1.0 + xgl[j]);
          tj = 0.125 * (1.0 - xgl[i]);
        }
        double f[9], fd1[9], fd2[9];
        shape(ncone, g1, g2, f, fd1, fd2);
        double xg[3] = {0, 0, 0}, dx1[3] = {0, 0, 0}, dx2[3] = {0, 0, 0}, ug[3] = {0, 0, 0},
               tg[3] = {0, 0, 0};
        for (int m = 0; m < ncone; ++m) {
          const int ik = M->kconec[m + 9 * e] - 1;
          const double fv = f[m];
          xg[0] = xg[0] + fv * xj1[m];
          xg[1] = xg[1] + fv * xj2[m];
          xg[2] = xg[2] + fv * xj3[m];
          dx1[0] = dx1[0] + fd1[m] * xj1[m];
          dx1[1] = dx1[1] + fd1[m] * xj2[m];
          dx1[2] = dx1[2] + fd1[m] * xj3[m];
          dx2[0] = dx2[0] + fd2[m] * xj1[m];
          dx2[1] = dx2[1] + fd2[m] * xj2[m];
          dx2[2] = dx2[2] + fd2[m] * xj3[m];
          ug[0] = ug[0] + fv * FI[3 * ik];
          ug[1] = ug[1] + fv * FI[3 * ik + 1];
          ug[2] = ug[2] + fv * FI[3 * ik + 2];
          tg[0] = tg[0] + fv * DFI[3 * m + 27 * e];
          tg[1] = tg[1] + fv * DFI[3 * m + 1 + 27 * e];
          tg[2] = tg[2] + fv * DFI[3 * m + 2 + 27 * e];
        }
        const double cv0 = dx1[1] * dx2[2] - dx1[2] * dx2[1];
        const double cv1 = dx1[2] * dx2[0] - dx1[0] * dx2[2];
        const double cv2 = dx1[0] * dx2[1] - dx1[1] * dx2[0];
        const double jac = std::sqrt(cv0 * cv0 + cv1 * cv1 + cv2 * cv2);
        const double wg = wgl[i] * wgl[j] * tj * jac;
        double* P = &fn[12 * q];
        P[0] = xg[0];
        P[1] = xg[1];
        P[2] = xg[2];
        P[3] = cv0 / jac;
        P[4] = cv1 / jac;
        P[5] = cv2 / jac;
        P[6] = ug[0] * wg;
        P[7] = ug[1] * wg;
        P[8] = ug[2] * wg;
        P[9] = tg[0] * wg;
        P[10] = tg[1] * wg;
        P[11] = tg[2] * wg;
      }
  }
  const double nu = M->nu;
  const double c4 = 3.0 - 4.0 * nu, c6 = 1.0 - 2.0 * nu, pr4 = 1.0 - 4.0 * nu;
  const double cU = 1.0 / (16.0 * PI * (1.0 - nu) * rge);
  const double cT = -1.0 / (8.0 * PI * (1.0 - nu));
  const double cD = 1.0 / (8.0 * PI * (1.0 - nu));
  const double cS = rge / (4.0 * PI * (1.0 - nu));
  (void)l;
#pragma omp parallel for schedule(guided)
  for (int ip = p0; ip < p1; ++ip) {
    const double xx = cx[ip], yy = cy[ip], zz = cz[ip];
    double ua[3] = {0, 0, 0}, sa[6] = {0, 0, 0, 0, 0, 0};
    for (int e = 0; e < ne; ++e) {
      const double ddx = xx - elc[3 * e], ddy = yy - elc[3 * e + 1], ddz = zz - elc[3 * e + 2];
      const double dc2 = ddx * ddx + ddy * ddy + ddz * ddz;
      const double* tab;
      size_t g0, g1;
      if (dc2 > thr[e]) {
        tab = gfar.data();
        g0 = fs[e];
        g1 = fe[e];
      } else {
        tab = fn.data();
        g0 = (size_t)e * NG * NG;
        g1 = g0 + NG * NG;
      }
      for (size_t q = g0; q < g1; ++q) {
        const double* P = &tab[12 * q];
        const double rx = P[0] - xx, ry = P[1] - yy, rz = P[2] - zz;
        const double r2 = rx * rx + ry * ry + rz * rz;
        const double r = std::sqrt(r2);
        const double ir = 1.0 / r;
        const double ir2 = ir * ir;
        const double ir3 = ir2 * ir;
        const double rd1 = rx * ir, rd2 = ry * ir, rd3 = rz * ir;
        const double n1 = P[3], n2 = P[4], n3 = P[5];
        const double rdn = rd1 * n1 + rd2 * n2 + rd3 * n3;
        const double tu1 = P[6], tu2 = P[7], tu3 = P[8];
        const double tt1 = P[9], tt2 = P[10], tt3 = P[11];
        const double rdt = rd1 * tt1 + rd2 * tt2 + rd3 * tt3;
        const double rdu = rd1 * tu1 + rd2 * tu2 + rd3 * tu3;
        const double nuv = n1 * tu1 + n2 * tu2 + n3 * tu3;
        const double fU = cU * ir, fT = cT * ir2;
        ua[0] = ua[0] + fU * (c4 * tt1 + rd1 * rdt) -
                fT * (rdn * (c6 * tu1 + 3.0 * rd1 * rdu) + asg * c6 * (nuv * rd1 - n1 * rdu));
        ua[1] = ua[1] + fU * (c4 * tt2 + rd2 * rdt) -
                fT * (rdn * (c6 * tu2 + 3.0 * rd2 * rdu) + asg * c6 * (nuv * rd2 - n2 * rdu));
        ua[2] = ua[2] + fU * (c4 * tt3 + rd3 * rdt) -
                fT * (rdn * (c6 * tu3 + 3.0 * rd3 * rdu) + asg * c6 * (nuv * rd3 - n3 * rdu));
        const double fD = cD * ir2, fS = cS * ir3;
        const double Dxx = fD * (c6 * (2.0 * tt1 * rd1 - rdt) + 3.0 * rd1 * rd1 * rdt);
        const double Dyy = fD * (c6 * (2.0 * tt2 * rd2 - rdt) + 3.0 * rd2 * rd2 * rdt);
        const double Dzz = fD * (c6 * (2.0 * tt3 * rd3 - rdt) + 3.0 * rd3 * rd3 * rdt);
        const double Dxy = fD * (c6 * (tt1 * rd2 + tt2 * rd1) + 3.0 * rd1 * rd2 * rdt);
        const double Dyz = fD * (c6 * (tt2 * rd3 + tt3 * rd2) + 3.0 * rd2 * rd3 * rdt);
        const double Dzx = fD * (c6 * (tt3 * rd1 + tt1 * rd3) + 3.0 * rd3 * rd1 * rdt);
        const double Sxx =
            fS * (3.0 * rdn * (c6 * rdu + 2.0 * nu * tu1 * rd1 - 5.0 * rd1 * rd1 * rdu) +
                  6.0 * nu * rdu * n1 * rd1 + c6 * (3.0 * nuv * rd1 * rd1 + 2.0 * n1 * tu1) -
                  pr4 * nuv);
        const double Syy =
            fS * (3.0 * rdn * (c6 * rdu + 2.0 * nu * tu2 * rd2 - 5.0 * rd2 * rd2 * rdu) +
                  6.0 * nu * rdu * n2 * rd2 + c6 * (3.0 * nuv * rd2 * rd2 + 2.0 * n2 * tu2) -
                  pr4 * nuv);
        const double Szz =
            fS * (3.0 * rdn * (c6 * rdu + 2.0 * nu * tu3 * rd3 - 5.0 * rd3 * rd3 * rdu) +
                  6.0 * nu * rdu * n3 * rd3 + c6 * (3.0 * nuv * rd3 * rd3 + 2.0 * n3 * tu3) -
                  pr4 * nuv);
        const double Sxy = fS * (3.0 * rdn * (nu * (tu1 * rd2 + tu2 * rd1) - 5.0 * rd1 * rd2 * rdu) +
                                 3.0 * nu * rdu * (n1 * rd2 + n2 * rd1) +
                                 c6 * (3.0 * nuv * rd1 * rd2 + n1 * tu2 + n2 * tu1));
        const double Syz = fS * (3.0 * rdn * (nu * (tu2 * rd3 + tu3 * rd2) - 5.0 * rd2 * rd3 * rdu) +
                                 3.0 * nu * rdu * (n2 * rd3 + n3 * rd2) +
                                 c6 * (3.0 * nuv * rd2 * rd3 + n2 * tu3 + n3 * tu2));
        const double Szx = fS * (3.0 * rdn * (nu * (tu3 * rd1 + tu1 * rd3) - 5.0 * rd3 * rd1 * rdu) +
                                 3.0 * nu * rdu * (n3 * rd1 + n1 * rd3) +
                                 c6 * (3.0 * nuv * rd3 * rd1 + n3 * tu1 + n1 * tu3));
        sa[0] = sa[0] + (Dxx - Sxx);
        sa[1] = sa[1] + (Dyy - Syy);
        sa[2] = sa[2] + (Dzz - Szz);
        sa[3] = sa[3] + (Dxy - Sxy);
        sa[4] = sa[4] + (Dyz - Syz);
        sa[5] = sa[5] + (Dzx - Szx);
      }
    }
    const int o = ip - p0;
    for (int c = 0; c < 3; ++c) u_int[3 * o + c] = ua[c];
    for (int c = 0; c < 6; ++c) sigma_int[6 * o + c] = sa[c];
    orc_principal(sa, &prin[3 * o], &vm[o]);
  }
  return 0;
}

}  // extern "C"
