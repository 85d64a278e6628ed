// Block-cooperative mixed-radix FFTs on lines held in shared memory, for float2 or
// double2 complex values.
//
// A "line set" is nlines complex lines of length n at buf[line * ls + e * es].
// All threads of the block call fft_lines() together (it contains __syncthreads()).
// Each radix-R stage is the Stockham autosort step: butterfly j of a line reads
// x[j + r n/R] (r < R), multiplies by the twiddle exp(-2 pi i r k / (Ns R)) with
// k = j mod Ns, applies the length-R DFT and writes y[(j/Ns) Ns R + k + r Ns].
// Stages run in place: every thread first computes all of its outputs into registers,
// the block synchronises, then the outputs are stored. The caller sizes the block so
// that nthreads * VPT >= nlines * n (VPT = complex values held per thread).
//
// Radices 2, 3, 4, 5 and 8 have unrolled butterflies; any other prime factor p is a
// direct length-p DFT stage in which each thread produces single outputs.
// Only the forward transform (exp(-i...)) is implemented; inverse transforms are
// obtained by conjugating the input and the output.
// LF selects the work-item order: false = consecutive threads walk along a line
// (lines contiguous, es == 1), true = consecutive threads walk across lines (ls == 1).
#pragma once

#include "ls_types.cuh"

namespace lsb {

template <typename C>
__device__ __forceinline__ C mk(decltype(C::x) x, decltype(C::x) y) {
  C r;
  r.x = x;
  r.y = y;
  return r;
}
template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by -i
template <typename C>
__device__ __forceinline__ C cmul_mi(C a) { return mk<C>(a.y, -a.x); }

template <int R>
struct Bfly;

template <>
struct Bfly<2> {
  template <typename C>
  static __device__ __forceinline__ void run(C* v) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <>
struct Bfly<4> {
  template <typename C>
  static __device__ __forceinline__ void run(C* v) {
    C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    C t2 = cadd(v[1], v[3]), t3 = cmul_mi(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};

template <>
struct Bfly<8> {
  template <typename C>
  static __device__ __forceinline__ void run(C* v) {
    using R = decltype(C::x);
    const R h = (R)0.70710678118654752440;
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    Bfly<4>::run(e);
    Bfly<4>::run(o);
    // o[k] *= exp(-2 pi i k / 8)
    o[1] = mk<C>(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
    o[2] = cmul_mi(o[2]);
    o[3] = mk<C>(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[k] = cadd(e[k], o[k]);
      v[k + 4] = csub(e[k], o[k]);
    }
  }
};

// 16-point DFT as 4 x 4 with the twiddles exp(-2 pi i k / 16) in between.
template <>
struct Bfly<16> {
  template <typename C>
  static __device__ __forceinline__ void run(C* v) {
    using R = decltype(C::x);
    const R c = (R)0.92387953251128675613;  // cos(pi/8)
    const R s = (R)0.38268343236508977173;  // sin(pi/8)
    const R h = (R)0.70710678118654752440;  // cos(pi/4)
    C a[4][4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
#pragma unroll
      for (int e = 0; e < 4; ++e) a[p][e] = v[p + 4 * e];
      Bfly<4>::run(a[p]);
    }
    // a[p][k] *= W16^(p k)
    a[1][1] = mk<C>(c * a[1][1].x + s * a[1][1].y, c * a[1][1].y - s * a[1][1].x);   // W^1
    a[1][2] = mk<C>(h * (a[1][2].x + a[1][2].y), h * (a[1][2].y - a[1][2].x));       // W^2
    a[1][3] = mk<C>(s * a[1][3].x + c * a[1][3].y, s * a[1][3].y - c * a[1][3].x);   // W^3
    a[2][1] = mk<C>(h * (a[2][1].x + a[2][1].y), h * (a[2][1].y - a[2][1].x));       // W^2
    a[2][2] = cmul_mi(a[2][2]);                                                       // W^4
    a[2][3] = mk<C>(h * (a[2][3].y - a[2][3].x), -h * (a[2][3].x + a[2][3].y));      // W^6
    a[3][1] = mk<C>(s * a[3][1].x + c * a[3][1].y, s * a[3][1].y - c * a[3][1].x);   // W^3
    a[3][2] = mk<C>(h * (a[3][2].y - a[3][2].x), -h * (a[3][2].x + a[3][2].y));      // W^6
    a[3][3] = mk<C>(-c * a[3][3].x - s * a[3][3].y, s * a[3][3].x - c * a[3][3].y);  // W^9
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      C b[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
      Bfly<4>::run(b);
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = b[k2];
    }
  }
};

template <>
struct Bfly<3> {
  template <typename C>
  static __device__ __forceinline__ void run(C* v) {
    using R = decltype(C::x);
    const R s = (R)0.86602540378443864676;  // sin(2 pi / 3)
    C b = cadd(v[1], v[2]);
    C d = csub(v[1], v[2]);
    C t = mk<C>(v[0].x - (R)0.5 * b.x, v[0].y - (R)0.5 * b.y);
    C u = mk<C>(s * d.y, -s * d.x);  // -i s d
    v[0] = cadd(v[0], b);
    v[1] = cadd(t, u);
    v[2] = csub(t, u);
  }
};

// 6-point DFT as 2 x 3: DFT over e of v[p + 2e] (p = 0, 1), twiddle exp(-2 pi i p k / 6),
// then DFT over p, giving X[k1 + 3 k2].
template <>
struct Bfly<6> {
  template <typename C>
  static __device__ __forceinline__ void run(C* v) {
    using R = decltype(C::x);
    const R h = (R)0.5, s = (R)0.86602540378443864676;  // cos, sin(pi/3)
    C a[3] = {v[0], v[2], v[4]};
    C b[3] = {v[1], v[3], v[5]};
    Bfly<3>::run(a);
    Bfly<3>::run(b);
    b[1] = mk<C>(h * b[1].x + s * b[1].y, h * b[1].y - s * b[1].x);    // exp(-i pi/3)
    b[2] = mk<C>(-h * b[2].x + s * b[2].y, -h * b[2].y - s * b[2].x);  // exp(-2 i pi/3)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      v[k] = cadd(a[k], b[k]);
      v[k + 3] = csub(a[k], b[k]);
    }
  }
};

template <>
struct Bfly<5> {
  template <typename C>
  static __device__ __forceinline__ void run(C* v) {
    using R = decltype(C::x);
    const R c1 = (R)0.30901699437494742410;   // cos(2 pi/5)
    const R c2 = (R)-0.80901699437494742410;  // cos(4 pi/5)
    const R s1 = (R)0.95105651629515357212;   // sin(2 pi/5)
    const R s2 = (R)0.58778525229247312917;   // sin(4 pi/5)
    C b1 = cadd(v[1], v[4]), b2 = cadd(v[2], v[3]);
    C d1 = csub(v[1], v[4]), d2 = csub(v[2], v[3]);
    C a0 = v[0];
    C p1 = mk<C>(a0.x + c1 * b1.x + c2 * b2.x, a0.y + c1 * b1.y + c2 * b2.y);
    C p2 = mk<C>(a0.x + c2 * b1.x + c1 * b2.x, a0.y + c2 * b1.y + c1 * b2.y);
    C q1 = mk<C>(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y);
    C q2 = mk<C>(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y);
    v[0] = mk<C>(a0.x + b1.x + b2.x, a0.y + b1.y + b2.y);
    v[1] = cadd(p1, cmul_mi(q1));
    v[4] = csub(p1, cmul_mi(q1));
    v[2] = cadd(p2, cmul_mi(q2));
    v[3] = csub(p2, cmul_mi(q2));
  }
};

// One Stockham stage with an unrolled radix-R butterfly.
template <int R, int VPT, bool LF, typename C>
__device__ __forceinline__ void stage_bfly(C* buf, int nlines, int es, int ls, int n, int Ns,
                                           const C* __restrict__ tw) {
  constexpr int IT = VPT / R > 0 ? VPT / R : 1;
  const int nb = n / R;
  const int total = nlines * nb;
  const int tws = n / (Ns * R);
  const int tid = threadIdx.x, nt = blockDim.x;
  C v[IT][R];
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    int w = tid + it * nt;
    if (w < total) {
      int line, j;
      if (LF) { j = w / nlines; line = w - j * nlines; } else { line = w / nb; j = w - line * nb; }
      int k = j % Ns;
      const C* L = buf + (size_t)line * ls;
#pragma unroll
      for (int r = 0; r < R; ++r) v[it][r] = L[(j + r * nb) * es];
      if (Ns > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) v[it][r] = cmul(v[it][r], tw[k * r * tws]);
      }
      Bfly<R>::run(v[it]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    int w = tid + it * nt;
    if (w < total) {
      int line, j;
      if (LF) { j = w / nlines; line = w - j * nlines; } else { line = w / nb; j = w - line * nb; }
      int k = j % Ns;
      int base = (j / Ns) * Ns * R + k;
      C* L = buf + (size_t)line * ls;
#pragma unroll
      for (int r = 0; r < R; ++r) L[(base + r * Ns) * es] = v[it][r];
    }
  }
  __syncthreads();
}

// One Stockham stage of arbitrary radix R: each work item produces one output.
template <int VPT, bool LF, typename C>
__device__ __forceinline__ void stage_generic(C* buf, int nlines, int es, int ls, int n, int Ns,
                                              int R, const C* __restrict__ tw) {
  const int nb = n / R;
  const int total = nlines * n;
  const int tws = n / (Ns * R);
  const int tid = threadIdx.x, nt = blockDim.x;
  C o[VPT];
#pragma unroll
  for (int it = 0; it < VPT; ++it) {
    int w = tid + it * nt;
    if (w < total) {
      int line, e;
      if (LF) { e = w / nlines; line = w - e * nlines; } else { line = w / n; e = w - line * n; }
      int k = e % Ns;
      int q = (e / Ns) % R;
      int j = (e / (Ns * R)) * Ns + k;
      const C* L = buf + (size_t)line * ls;
      C acc = mk<C>(0, 0);
      int rq = 0;  // (r * q) mod R
      for (int r = 0; r < R; ++r) {
        C x = L[(j + r * nb) * es];
        if (r > 0) x = cmul(x, tw[k * r * tws]);
        C wv = tw[rq * nb];
        acc = mk<C>(acc.x + x.x * wv.x - x.y * wv.y, acc.y + x.x * wv.y + x.y * wv.x);
        rq += q;
        if (rq >= R) rq -= R;
      }
      o[it] = acc;
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < VPT; ++it) {
    int w = tid + it * nt;
    if (w < total) {
      int line, e;
      if (LF) { e = w / nlines; line = w - e * nlines; } else { line = w / n; e = w - line * n; }
      buf[(size_t)line * ls + e * es] = o[it];
    }
  }
  __syncthreads();
}

// Forward (exp(-i...)) unnormalised FFT of every line in the set; tw = twiddle table of
// the plan in the precision of C.
template <int VPT, bool LF, typename C>
__device__ void fft_lines(C* buf, int nlines, int es, int ls, const Plan1D& p, const C* tw) {
  int Ns = 1;
  for (int s = 0; s < p.nst; ++s) {
    const int R = p.radix[s];
    switch (R) {
      case 2: stage_bfly<2, VPT, LF>(buf, nlines, es, ls, p.n, Ns, tw); break;
      case 3: stage_bfly<3, VPT, LF>(buf, nlines, es, ls, p.n, Ns, tw); break;
      case 4: stage_bfly<4, VPT, LF>(buf, nlines, es, ls, p.n, Ns, tw); break;
      case 5: stage_bfly<5, VPT, LF>(buf, nlines, es, ls, p.n, Ns, tw); break;
      case 8: stage_bfly<8, VPT, LF>(buf, nlines, es, ls, p.n, Ns, tw); break;
      default: stage_generic<VPT, LF>(buf, nlines, es, ls, p.n, Ns, R, tw); break;
    }
    Ns *= R;
  }
}

// Smallest block size (multiple of 32) that satisfies nthreads * (VPT/R) * R >= n_elems
// for every stage of the plan and nthreads * VPT >= n_elems for generic stages.
__host__ inline int threads_for(const Plan1D& p, long long n_elems, int vpt) {
  long long need = 32;
  for (int s = 0; s < p.nst; ++s) {
    int R = p.radix[s];
    if (R == 2 || R == 3 || R == 4 || R == 5 || R == 8) {
      long long per = vpt / R > 0 ? vpt / R : 1;  // butterflies per thread
      long long nb = n_elems / R;
      long long t = (nb + per - 1) / per;
      if (t > need) need = t;
    } else {
      long long t = (n_elems + vpt - 1) / vpt;
      if (t > need) need = t;
    }
  }
  return (int)((need + 31) / 32 * 32);
}

}  // namespace lsb
