// Pointwise laws of the damage extension (src/jaxmaterials/solver/lippmann_schwinger.py:
// 36-100): the strain's spectral split into tension and compression parts, the degraded
// stress and the tensile energy. Voigt components (v0..v5) sit in the strain tensor as
// [[v0, v5, v4], [v5, v1, v3], [v4, v3, v2]] (src/jaxmaterials/utilities.py:65-85) and
// the stress leaves in the same places.
//
// Eigenvalues of the symmetric 3 x 3 tensor by the trigonometric solution of its
// characteristic cubic (O. K. Smith, Comm. ACM 4 (1961) 168): with q = tr/3, p^2 =
// |T - qI|^2 / 6, r = det((T - qI)/p) / 2 in [-1, 1] and phi = acos(r) / 3, the
// eigenvalues are q + 2p cos(phi), q + 2p cos(phi + 2 pi / 3) and the third from the
// trace. Only the part with eigenvalues of one sign is assembled from an eigenvector (of
// an eigenvalue that the sign separates from the other two, so it is simple): that vector
// is the largest cross product of two rows of T - lambda I; the other part is T minus it.
#pragma once

namespace lsb {

template <typename T>
struct Sym3 {
  T a, b, c;     // diagonal 00, 11, 22
  T d, e, f;     // 12, 02, 01
};

template <typename T>
__host__ __device__ __forceinline__ Sym3<T> sym_from_voigt(const T v[6]) {
  return Sym3<T>{v[0], v[1], v[2], v[3], v[4], v[5]};
}

// Eigenvalues l0 >= l1 >= l2.
template <typename T>
__host__ __device__ __forceinline__ void sym_eigenvalues(const Sym3<T>& m, T& l0, T& l1, T& l2) {
  const T q = (m.a + m.b + m.c) / (T)3;
  const T off = m.d * m.d + m.e * m.e + m.f * m.f;
  const T da = m.a - q, db = m.b - q, dc = m.c - q;
  const T p2 = (da * da + db * db + dc * dc + (T)2 * off) / (T)6;
  if (!(p2 > (T)0)) {
    l0 = l1 = l2 = q;
    return;
  }
  const T p = sqrt(p2);
  const T ip = (T)1 / p;
  const T ba = da * ip, bb = db * ip, bc = dc * ip, bd = m.d * ip, be = m.e * ip, bf = m.f * ip;
  // det of [[ba, bf, be], [bf, bb, bd], [be, bd, bc]]
  T r = (ba * (bb * bc - bd * bd) - bf * (bf * bc - bd * be) + be * (bf * bd - bb * be)) / (T)2;
  r = r < (T)-1 ? (T)-1 : (r > (T)1 ? (T)1 : r);
  const T phi = acos(r) / (T)3;
  const T two_pi_3 = (T)2.0943951023931954923;
  l0 = q + (T)2 * p * cos(phi);
  l2 = q + (T)2 * p * cos(phi + two_pi_3);
  l1 = (T)3 * q - l0 - l2;
}

// Unit eigenvector of the simple eigenvalue lam; false when no row pair gives a usable
// direction (lam then coincides with another eigenvalue to round-off).
template <typename T>
__host__ __device__ __forceinline__ bool sym_eigenvector(const Sym3<T>& m, T lam, T n[3]) {
  const T r0[3] = {m.a - lam, m.f, m.e};
  const T r1[3] = {m.f, m.b - lam, m.d};
  const T r2[3] = {m.e, m.d, m.c - lam};
  T c[3][3];
  const T* rows[3][2] = {{r0, r1}, {r0, r2}, {r1, r2}};
  T best = (T)0;
  int bi = -1;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const T* u = rows[i][0];
    const T* w = rows[i][1];
    c[i][0] = u[1] * w[2] - u[2] * w[1];
    c[i][1] = u[2] * w[0] - u[0] * w[2];
    c[i][2] = u[0] * w[1] - u[1] * w[0];
    const T nn = c[i][0] * c[i][0] + c[i][1] * c[i][1] + c[i][2] * c[i][2];
    if (nn > best) {
      best = nn;
      bi = i;
    }
  }
  if (bi < 0) return false;
  const T s = (T)1 / sqrt(best);
#pragma unroll
  for (int k = 0; k < 3; ++k) n[k] = c[bi][k] * s;
  return true;
}

// n^T m n
template <typename T>
__host__ __device__ __forceinline__ T rayleigh(const Sym3<T>& m, const T n[3]) {
  return m.a * n[0] * n[0] + m.b * n[1] * n[1] + m.c * n[2] * n[2] +
         (T)2 * (m.d * n[1] * n[2] + m.e * n[0] * n[2] + m.f * n[0] * n[1]);
}

// Eigenpair of the simple eigenvalue near lam, refined once: the Rayleigh quotient of the
// first vector (accurate to the square of its error) gives a second vector and the final
// value. The trigonometric eigenvalues lose digits when two eigenvalues nearly coincide.
template <typename T>
__host__ __device__ __forceinline__ bool refined_pair(const Sym3<T>& m, T& lam, T n[3]) {
  if (!sym_eigenvector(m, lam, n)) return false;
  lam = rayleigh(m, n);
  T n2[3];
  if (sym_eigenvector(m, lam, n2)) {
    n[0] = n2[0];
    n[1] = n2[1];
    n[2] = n2[2];
    lam = rayleigh(m, n);
  }
  return true;
}

// Tension part (eigenvalues clipped below at 0) of m, as a Sym3; compression = m - tension.
template <typename T>
__host__ __device__ __forceinline__ Sym3<T> tension_part(const Sym3<T>& m) {
  T l0, l1, l2;
  sym_eigenvalues(m, l0, l1, l2);
  const Sym3<T> zero{0, 0, 0, 0, 0, 0};
  if (l2 >= (T)0) return m;      // no negative eigenvalue
  if (l0 <= (T)0) return zero;   // no positive eigenvalue
  T n[3];
  if (l1 <= (T)0) {  // one positive eigenvalue: tension = l0 n n^T
    if (!refined_pair(m, l0, n)) return zero;
    if (l0 <= (T)0) return zero;
    return Sym3<T>{l0 * n[0] * n[0], l0 * n[1] * n[1], l0 * n[2] * n[2],
                   l0 * n[1] * n[2], l0 * n[0] * n[2], l0 * n[0] * n[1]};
  }
  // two positive eigenvalues: tension = m - l2 n n^T
  if (!refined_pair(m, l2, n)) return m;
  if (l2 >= (T)0) return m;
  return Sym3<T>{m.a - l2 * n[0] * n[0], m.b - l2 * n[1] * n[1], m.c - l2 * n[2] * n[2],
                 m.d - l2 * n[1] * n[2], m.e - l2 * n[0] * n[2], m.f - l2 * n[0] * n[1]};
}

// sigma = g sigma+ + sigma-, sigma+- = lambda <tr eps>+- I + 2 mu eps+-,
// g = (1 - d)^2 + k (lippmann_schwinger.py:36-75).
template <typename T>
__host__ __device__ __forceinline__ void damaged_stress(const T e[6], T lam, T mu, T g, T s[6]) {
  const Sym3<T> m = sym_from_voigt(e);
  const Sym3<T> tp = tension_part(m);
  const T tr = m.a + m.b + m.c;
  const T trp = tr > (T)0 ? tr : (T)0, trm = tr < (T)0 ? tr : (T)0;
  const T ep[6] = {tp.a, tp.b, tp.c, tp.d, tp.e, tp.f};
  const T tmu = (T)2 * mu;
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    const T em = e[c] - ep[c];
    const T sp = (c < 3 ? lam * trp : (T)0) + tmu * ep[c];
    const T sm = (c < 3 ? lam * trm : (T)0) + tmu * em;
    s[c] = g * sp + sm;
  }
}

// psi+ = 1/2 lambda <tr eps>+^2 + mu sum_i <l_i>+^2 (lippmann_schwinger.py:78-100).
template <typename T>
__host__ __device__ __forceinline__ T tensile_energy(const T e[6], T lam, T mu) {
  const Sym3<T> m = sym_from_voigt(e);
  T l0, l1, l2;
  sym_eigenvalues(m, l0, l1, l2);
  const T tr = m.a + m.b + m.c;
  const T trp = tr > (T)0 ? tr : (T)0;
  const T p0 = l0 > (T)0 ? l0 : (T)0, p1 = l1 > (T)0 ? l1 : (T)0, p2 = l2 > (T)0 ? l2 : (T)0;
  return (T)0.5 * lam * trp * trp + mu * (p0 * p0 + p1 * p1 + p2 * p2);
}

}  // namespace lsb
