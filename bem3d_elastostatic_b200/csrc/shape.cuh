// Device shape functions of the 9-node Lagrangian quadrilateral and the 6-node
// triangle, with their intrinsic derivatives (assembly_mod.f90:247-302,
// stress_mod.f90:32-112), and the surface Jacobian / unit normal.
#pragma once

namespace bem {

// quad9 node order: 1:(-1,-1) 2:(0,-1) 3:(1,-1) 4:(1,0) 5:(1,1) 6:(0,1) 7:(-1,1)
// 8:(-1,0) 9:(0,0); tri6: 1:(1,0,0) 2:(0,1,0) 3:(0,0,1) 4..6 mid-sides.
template <typename T>
__host__ __device__ __forceinline__ void shape_fn(int ncone, T g1, T g2, T* f, T* fd1, T* fd2) {
  const T one = T(1), two = T(2), half = T(0.5), qtr = T(0.25), four = T(4);
  if (ncone == 9) {
    f[0] = qtr * g1 * g2 * (g1 - one) * (g2 - one);
    f[1] = half * (one - g1 * g1) * g2 * (g2 - one);
    f[2] = qtr * g1 * g2 * (g1 + one) * (g2 - one);
    f[3] = half * g1 * (g1 + one) * (one - g2 * g2);
    f[4] = qtr * g1 * g2 * (g1 + one) * (g2 + one);
    f[5] = half * (one - g1 * g1) * g2 * (g2 + one);
    f[6] = qtr * g1 * g2 * (g1 - one) * (g2 + one);
    f[7] = half * g1 * (g1 - one) * (one - g2 * g2);
    f[8] = (one - g1 * g1) * (one - g2 * g2);
    fd1[0] = qtr * g2 * (g2 - one) * (two * g1 - one);
    fd1[1] = -g1 * g2 * (g2 - one);
    fd1[2] = qtr * g2 * (g2 - one) * (two * g1 + one);
    fd1[3] = half * (one - g2 * g2) * (two * g1 + one);
    fd1[4] = qtr * g2 * (g2 + one) * (two * g1 + one);
    fd1[5] = -g1 * g2 * (g2 + one);
    fd1[6] = qtr * g2 * (g2 + one) * (two * g1 - one);
    fd1[7] = half * (one - g2 * g2) * (two * g1 - one);
    fd1[8] = -two * g1 * (one - g2 * g2);
    fd2[0] = qtr * g1 * (g1 - one) * (two * g2 - one);
    fd2[1] = half * (one - g1 * g1) * (two * g2 - one);
    fd2[2] = qtr * g1 * (g1 + one) * (two * g2 - one);
    fd2[3] = -g1 * g2 * (g1 + one);
    fd2[4] = qtr * g1 * (g1 + one) * (two * g2 + one);
    fd2[5] = half * (one - g1 * g1) * (two * g2 + one);
    fd2[6] = qtr * g1 * (g1 - one) * (two * g2 + one);
    fd2[7] = -g1 * g2 * (g1 - one);
    fd2[8] = -two * g2 * (one - g1 * g1);
  } else {
    const T g3 = one - g1 - g2;
    f[0] = g1 * (two * g1 - one);
    f[1] = g2 * (two * g2 - one);
    f[2] = g3 * (two * g3 - one);
    f[3] = four * g1 * g2;
    f[4] = four * g2 * g3;
    f[5] = four * g3 * g1;
    fd1[0] = four * g1 - one;
    fd1[1] = T(0);
    fd1[2] = one - four * g3;
    fd1[3] = four * g2;
    fd1[4] = -four * g2;
    fd1[5] = four * (g3 - g1);
    fd2[0] = T(0);
    fd2[1] = four * g2 - one;
    fd2[2] = one - four * g3;
    fd2[3] = four * g1;
    fd2[4] = four * (g3 - g2);
    fd2[5] = -four * g1;
    f[6] = f[7] = f[8] = T(0);
    fd1[6] = fd1[7] = fd1[8] = T(0);
    fd2[6] = fd2[7] = fd2[8] = T(0);
  }
}

// Jacobian and unit normal by the reference's dc - dct double sum
// (assembly_mod.f90:311-334): s = (dx/dxi1) x (dx/dxi2) expanded node by node.
template <typename T>
__device__ __forceinline__ void jacobian_dc(int ncone, const T* fd1, const T* fd2,
                                            const T* xj1, const T* xj2, const T* xj3,
                                            T& xja, T& e1, T& e2, T& e3) {
  T s1 = T(0), s2 = T(0), s3 = T(0);
  for (int jk = 0; jk < ncone; ++jk) {
    T aux = T(0), bux = T(0), cux = T(0);
    for (int ik = 0; ik < ncone; ++ik) {
      const T d = fd1[ik] * fd2[jk] - fd2[ik] * fd1[jk];
      aux = aux + xj2[ik] * d;
      bux = bux + xj3[ik] * d;
      cux = cux + xj1[ik] * d;
    }
    s1 = s1 + aux * xj3[jk];
    s2 = s2 + bux * xj1[jk];
    s3 = s3 + cux * xj2[jk];
  }
  xja = sqrt(s1 * s1 + s2 * s2 + s3 * s3);
  e1 = s1 / xja;
  e2 = s2 / xja;
  e3 = s3 / xja;
}

}  // namespace bem
