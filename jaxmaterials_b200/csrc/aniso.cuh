// Anisotropic stiffness (the derivation of doc/linear_elasticity.tex:372-402 and
// doc/anisotropic.py): the 21 independent entries C_0..C_20 of the symmetric 6 x 6 Voigt
// matrix, numbered as in doc/anisotropic.py:150-185 (diagonal first, then the upper
// triangle row by row), Voigt order (xx, yy, zz, xy, xz, yz) with tensor shear strains.
//
// Stress: sigma_a = sum_b C_ab w_b eps_b, w = (1, 1, 1, 2, 2, 2).
// Gamma^0 for a reference stiffness C^0 and the unit wave vector xi: acoustic matrix
// K_ki = C^0_{kjil} xi_j xi_l, N = K^-1, u = N (tau xi), (Gamma^0 tau)_kl = (xi_k u_l +
// xi_l u_k) / 2 (the symmetrised N xi xi of doc/anisotropic.py:98-128); the update uses
// r = -Gamma^0 tau. For an isotropic C^0 this is the closed form of fourier.py:115-186.
#pragma once

namespace lsb {

// entry number of Voigt pair (a, b)
__host__ __device__ __forceinline__ int c21_index(int a, int b) {
  if (a > b) {
    const int t = a;
    a = b;
    b = t;
  }
  if (a == b) return a;
  // off-diagonal pairs numbered 6..20 in the order (0,1), (0,2), (1,2), (0,3), (0,4), (0,5),
  // (1,3), (1,4), (1,5), (2,3), (2,4), (2,5), (3,4), (3,5), (4,5)
  constexpr int tab[6][6] = {{0, 6, 7, 9, 10, 11},    {6, 1, 8, 12, 13, 14},
                             {7, 8, 2, 15, 16, 17},   {9, 12, 15, 3, 18, 19},
                             {10, 13, 16, 18, 4, 20}, {11, 14, 17, 19, 20, 5}};
  return tab[a][b];
}

// Voigt index of the tensor pair (p, q)
__host__ __device__ __forceinline__ int voigt_of(int p, int q) {
  if (p == q) return p;
  const int s = p + q;  // (0,1) -> 1, (0,2) -> 2, (1,2) -> 3
  return s == 1 ? 3 : (s == 2 ? 4 : 5);
}

// sigma = C eps for one voxel; c(k) returns entry k.
template <typename T, typename F>
__host__ __device__ __forceinline__ void aniso_stress(F c, const T e[6], T s[6]) {
  const T we[6] = {e[0], e[1], e[2], (T)2 * e[3], (T)2 * e[4], (T)2 * e[5]};
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    T acc = (T)0;
#pragma unroll
    for (int b = 0; b < 6; ++b) acc += c(c21_index(a, b)) * we[b];
    s[a] = acc;
  }
}

// The symmetric N = K^-1 (n00, n11, n22, n12, n02, n01) for unit xi; false when K is
// singular (no usable reference medium).
__host__ __device__ __forceinline__ bool aniso_inverse_acoustic(const double* c0, const double z[3],
                                                               double n[6]) {
  double K[3][3];
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < 3; ++i) {
      double acc = 0.0;
      for (int j = 0; j < 3; ++j)
        for (int l = 0; l < 3; ++l) acc += c0[c21_index(voigt_of(k, j), voigt_of(i, l))] * z[j] * z[l];
      K[k][i] = acc;
    }
  const double a00 = K[1][1] * K[2][2] - K[1][2] * K[2][1];
  const double a01 = K[0][2] * K[2][1] - K[0][1] * K[2][2];
  const double a02 = K[0][1] * K[1][2] - K[0][2] * K[1][1];
  const double det = K[0][0] * a00 + K[1][0] * a01 + K[2][0] * a02;
  if (!(fabs(det) > 0.0)) return false;
  const double id = 1.0 / det;
  n[0] = a00 * id;
  n[1] = (K[0][0] * K[2][2] - K[0][2] * K[2][0]) * id;
  n[2] = (K[0][0] * K[1][1] - K[0][1] * K[1][0]) * id;
  n[3] = (K[0][2] * K[1][0] - K[0][0] * K[1][2]) * id;  // (1,2)
  n[4] = a02 * id;                                       // (0,2)
  n[5] = a01 * id;                                       // (0,1)
  return true;
}

// r = -Gamma^0 tau (Voigt, tensor shear) for real tau, N from aniso_inverse_acoustic.
template <typename T>
__host__ __device__ __forceinline__ void aniso_gamma(const T n[6], const T z[3], const T t[6], T r[6]) {
  // tau xi
  const T v0 = t[0] * z[0] + t[3] * z[1] + t[4] * z[2];
  const T v1 = t[3] * z[0] + t[1] * z[1] + t[5] * z[2];
  const T v2 = t[4] * z[0] + t[5] * z[1] + t[2] * z[2];
  // u = N v
  const T u0 = n[0] * v0 + n[5] * v1 + n[4] * v2;
  const T u1 = n[5] * v0 + n[1] * v1 + n[3] * v2;
  const T u2 = n[4] * v0 + n[3] * v1 + n[2] * v2;
  r[0] = -(z[0] * u0);
  r[1] = -(z[1] * u1);
  r[2] = -(z[2] * u2);
  r[3] = -(T)0.5 * (z[0] * u1 + z[1] * u0);
  r[4] = -(T)0.5 * (z[0] * u2 + z[2] * u0);
  r[5] = -(T)0.5 * (z[1] * u2 + z[2] * u1);
}

}  // namespace lsb
