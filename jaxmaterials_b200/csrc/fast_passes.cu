// FP32 passes for power-of-two axis lengths (16..256) with compile-time sizes.
//
// Each 1-D transform of length N = E * P is a four-step FFT spread over P threads:
// thread p holds x[p + P e] (e < E), does the E-point DFT in registers, multiplies by
// exp(-2 pi i p k1 / N), writes its E values to shared memory transposed, and after one
// barrier each thread gathers P values of one k1 and finishes with the P-point DFT,
// producing X[k1 + E k2]. One shared-memory round trip per transform, no runtime index
// division, and the y and x passes read and write global memory in coalesced rows.
// Semantics are those of the generic passes in ls_kernels.cu (same layouts, shift of the
// forward transform, criterion partials, Gamma^0), which remain the path for every other
// size and for FP64 fields.
#include <cmath>

#include <cooperative_groups.h>

#include "aniso.cuh"
#include "damage.cuh"
#include "fast_passes.cuh"
#include "fft_smem.cuh"

namespace lsb {
namespace fast {

template <int N>
struct Split;
template <>
struct Split<16> { static constexpr int E = 4, P = 4; };
template <>
struct Split<32> { static constexpr int E = 8, P = 4; };
template <>
struct Split<64> { static constexpr int E = 8, P = 8; };
template <>
struct Split<128> { static constexpr int E = 16, P = 8; };
template <>
struct Split<256> { static constexpr int E = 16, P = 16; };
template <>
struct Split<48> { static constexpr int E = 16, P = 3; };
template <>
struct Split<96> { static constexpr int E = 16, P = 6; };

// Step B work per thread: the E DFTs of length P are dealt round-robin (k1 = p + P j);
// when P does not divide E the last round is partial.
template <int N>
__host__ __device__ constexpr int rounds() { return (Split<N>::E + Split<N>::P - 1) / Split<N>::P; }

__device__ __forceinline__ float2 conj2(float2 a) { return make_float2(a.x, -a.y); }

__device__ __forceinline__ bool active32(const InstanceState& s) { return !s.done && s.phase == 0; }

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// Bounded wait on a one-shot mbarrier (phase 0). Returns false if the copies did not
// complete within the limit.
__device__ __forceinline__ bool mbar_wait(unsigned mbar) {
  for (long long spin = 0; spin < (1LL << 24); ++spin) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done) : "r"(mbar), "r"(0u) : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(mbar) : "memory");
}

// Step A of the four-step transform: DFT over e of v[e] = x[p + P e], then the twiddle.
template <int N, int E = Split<N>::E>
__device__ __forceinline__ void step_a(float2* v, int p, const float2* __restrict__ tw) {
  Bfly<E>::run(v);
  if (p > 0) {
#pragma unroll
    for (int k1 = 1; k1 < E; ++k1) v[k1] = cmul(v[k1], __ldg(tw + p * k1));
  }
}

// Step A with the twiddles read from a shared-memory copy of the table.
template <int N, int E>
__device__ __forceinline__ void step_a_smem(float2* v, int p, const float2* tw) {
  Bfly<E>::run(v);
  if (p > 0) {
#pragma unroll
    for (int k1 = 1; k1 < E; ++k1) v[k1] = cmul(v[k1], tw[p * k1]);
  }
}

// ----------------------------------------------------------------------------- tiled layout
// The tiled spectrum layout (grids with nx <= 128 and nz/2+1 = 8 k + 1, ny = 8 k'), written
// by the forward y pass and read by the inverse y pass, and in place by this x pass: per
// instance and component,
//   full tiles   [j][ky][x][t]   kz = 8 j + t, j < NF = (nz/2+1 - 1) / 8
//   tail         [ky / 8][x][ky % 8]   the z Nyquist column kz = nz/2
// (tile_offset below). Every tile of the x pass is then one contiguous chunk of 8 nx complex
// values per component, fetched with one bulk copy.
constexpr int kTW = 8;

__host__ __device__ __forceinline__ size_t tile_offset(int nx, int ny, int nf, int x, int ky, int kz) {
  if (kz < nf * kTW) return ((size_t)((kz / kTW) * ny + ky) * nx + x) * kTW + (kz % kTW);
  return (size_t)ny * nf * nx * kTW + ((size_t)(ky / kTW) * nx + x) * kTW + (ky % kTW);
}

// ----------------------------------------------------------------------------- y pass
// Block = (16 kz columns, x, instance * 6 + component); thread (p, t), t fastest. When
// nz/2+1 = 16 k + 1 (every even extent here but 16 and 48), the last column (the z
// Nyquist plane) is not given a 16-column tile of its own per x: tile k instead takes that
// column for 16 consecutive x.
// kz columns per y-pass block (the x pass's column count is chosen per grid at run time,
// see x_cols).
#ifndef LSB_Y_COLS
#define LSB_Y_COLS 16
#endif
constexpr int kYT = LSB_Y_COLS;
// kz columns per y-pass block for extent N and variant YV: variant 0 is 8 at 128 (16
// threads per column, eight resident blocks per SM; measured -3% against 16 columns, 32
// columns +14%) and kYT elsewhere; variant 1 the other of 8 and 16. The autotuner times
// both (the results are the same: a column's transform does not depend on YT).
template <int N, int YV = 0>
__host__ __device__ constexpr int y_cols() { return (N == 128) != (YV == 1) ? 8 : kYT; }

// Split of the y transform (may differ from the x/z split): 128 = 8 x 16 puts 16 threads
// on a column and halves the values each thread holds (measured -13% at 128^3 against
// 16 x 8; the shorter extents are fastest with their x/z split).
template <int N>
struct YSplit { static constexpr int E = Split<N>::E, P = Split<N>::P; };
template <>
struct YSplit<128> { static constexpr int E = 8, P = 16; };
template <int N, int YV = 0>
__host__ __device__ constexpr int y_threads() { return y_cols<N, YV>() * YSplit<N>::P; }
template <int N, int YV = 0>
__host__ __device__ constexpr int y_min_blocks() {
  // (256: three blocks, so that its 16 values per thread fit without spilling)
  return N == 256 ? 3 : 1024 / (32 * ((y_threads<N, YV>() + 31) / 32));
}

// TILED: the x-pass side of the transform is the tiled layout in `tspec` (see xpass_tiled):
// the forward pass reads `spec` (cuFFT layout) and writes `tspec`, the inverse pass reads
// `tspec` and writes `spec`. Otherwise both sides are `spec`, transformed in place.
// (the tiled form keeps a second base pointer and index terms; LSB_YT_MINB_NUM / 4 of the
// in-place form's resident blocks: 4/4 measured fastest at 128^3, 0.141 against 0.151 ms
// at 3/4, despite a few bytes of spill)
#ifndef LSB_YT_MINB_NUM
#define LSB_YT_MINB_NUM 4
#endif
template <int NY, int YV = 0>
__host__ __device__ constexpr int yt_min_blocks() {
  // (other extents: half the in-place form's blocks; at 48 and 96, whose threads hold 16
  // values, the full count spilled and made the pass 2-3x slower)
  return NY == 128 ? LSB_YT_MINB_NUM * y_min_blocks<NY, YV>() / 4
                   : (y_min_blocks<NY, YV>() / 2 > 2 ? y_min_blocks<NY, YV>() / 2 : 2);
}
template <int NY, bool TILED, int YV>
__global__ void __launch_bounds__(y_threads<NY, YV>(), TILED ? yt_min_blocks<NY, YV>() : y_min_blocks<NY, YV>())
    ypass_fast(GridDesc g, int inverse,
                                                               float2* __restrict__ spec,
                                                               float2* __restrict__ tspec,
                                                               const InstanceState* __restrict__ st) {
  constexpr int E = YSplit<NY>::E, P = YSplit<NY>::P, NJ = (E + P - 1) / P;
  constexpr int YT = y_cols<NY, YV>();
  // rows k1 of the transposed layout padded to RS = 8 (mod 16) values, so that the two rows
  // a half-warp reads in step B (lanes: YT columns t of consecutive k1) fall in disjoint
  // bank halves (unpadded, P YT = 128 at 128 put them in the same banks)
  constexpr int RS = P * YT + (8 - (P * YT) % 16 + 16) % 16;
  __shared__ float2 buf[E * RS];
  const int bc = blockIdx.z;
  if (!active32(st[bc / 6])) return;
  const int t = threadIdx.x % YT, p = threadIdx.x / YT;
  const int nzh = g.nzh;
  // grid: (kz tiles, x) for the in-place form; (x, kz tiles) for the tiled form, so that
  // consecutive blocks write neighbouring tile rows
  const int bx = TILED ? (int)blockIdx.y : (int)blockIdx.x;
  const int by = TILED ? (int)blockIdx.x : (int)blockIdx.y;
  int kz, x;
  bool valid;
  if (nzh % YT == 1 && bx == nzh / YT) {
    if (by * YT >= g.nx) return;
    kz = nzh - 1;
    x = by * YT + t;
    valid = x < g.nx;
  } else {
    kz = bx * YT + t;
    x = by;
    valid = kz < nzh;
  }
  float2* base = spec + ((size_t)bc * g.nx + x) * (size_t)NY * nzh + kz;
  // tiled side: element ky of this column sits at tb + (ky >> sh) * ta + (ky & mk)
  // (tile_offset: full columns step by a tile row per ky, the Nyquist column by 8 ky groups)
  const int nf = (nzh - 1) / kTW;
  const bool ncol = kz >= nf * kTW;
  float2* tb = tspec + (size_t)bc * g.nm + tile_offset(g.nx, NY, nf, x, 0, kz);
  const int sh = ncol ? 3 : 0, mk = ncol ? kTW - 1 : 0;
  const int ta = g.nx * kTW;
  auto tptr = [&](int ky) { return tb + (size_t)((ky >> sh) * ta + (ky & mk)); };
  const float2* tw = g.py.tw;
  float2 v[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int ky = p + P * e;
    float2 a = make_float2(0.f, 0.f);
    if (valid) a = (TILED && inverse) ? *tptr(ky) : base[(size_t)ky * nzh];
    v[e] = inverse ? conj2(a) : a;
  }
  step_a<NY, E>(v, p, tw);
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) buf[k1 * RS + p * YT + t] = v[k1];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    const int k1 = p + P * j;
    if (k1 >= E) break;
    float2 w[P];
#pragma unroll
    for (int q = 0; q < P; ++q) w[q] = buf[k1 * RS + q * YT + t];
    Bfly<P>::run(w);
    if (valid) {
#pragma unroll
      for (int k2 = 0; k2 < P; ++k2) {
        const int ky = k1 + E * k2;
        const float2 o = inverse ? conj2(w[k2]) : w[k2];
        if (TILED && !inverse) *tptr(ky) = o;
        else base[(size_t)ky * nzh] = o;
      }
    }
  }
}

// ----------------------------------------------------------------------------- x pass
// Block = (TX kz columns, ky, instance); thread (c, p, t) with t fastest. Component c owns
// a shared-memory region holding either the natural layout [kx][t] or the transposed
// layout [k1][p][t] with rows of P*T + T values (the padding makes the column reads of
// the second step conflict-free).
template <int NX>
__host__ __device__ constexpr int x_cols() { return NX <= 48 ? 16 : (NX == 256 ? 4 : 8); }
// Split of the x transform (may differ from the z split).
template <int N>
struct XSplit { static constexpr int E = Split<N>::E, P = Split<N>::P; };
// Tile variants of the x pass: 0 = x_cols columns per block (two resident blocks per SM),
// 1 = half as many (four resident blocks); the solver times both on its first solve and
// keeps the faster (lsb::fast::launch_xpass `variant`).
// (variant 1 only where its block is still whole warps: the block reduction shuffles
// over full warps)
template <int NX, int V>
__host__ __device__ constexpr int x_cols_v() {
  return (V == 1 && NX != 256 && NX != 16 && (6 * XSplit<NX>::P * (x_cols<NX>() / 2)) % 32 == 0)
             ? x_cols<NX>() / 2 : x_cols<NX>();
}
template <int NX, int V>
__host__ __device__ constexpr int x_min_blocks() { return x_cols_v<NX, V>() < x_cols<NX>() ? 4 : 2; }
template <int NX, int T, typename SP = XSplit<NX>>
__host__ __device__ constexpr int x_row() { return SP::P * T + T; }
template <int NX, int T, typename SP = XSplit<NX>>
__host__ __device__ constexpr int x_region() {
  return SP::E * x_row<NX, T, SP>() > NX * T ? SP::E * x_row<NX, T, SP>() : NX * T;
}

// Pieces of the x pass shared by its two forms (strided rows of the cuFFT layout, and
// contiguous tiles of the tiled layout). One block owns T columns (kz or ky varies with
// the column index tt) and all NX rows of the six components; component c's shared region
// `tr` holds either the natural layout [kx][t] or the transposed layout [k1][p][t].

// Forward x DFT of this thread's column values v (natural order x = p + P e): step A,
// transpose, step B; leaves X[kx] in the natural layout of tr.
template <int NX, int T, typename SP = XSplit<NX>>
__device__ __forceinline__ void x_forward(float2* tr, float2* v, int p, int t, const float2* stw) {
  constexpr int E = SP::E, P = SP::P, RS = x_row<NX, T, SP>(), NJ = (E + P - 1) / P;
  step_a_smem<NX, E>(v, p, stw);
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) tr[k1 * RS + p * T + t] = v[k1];
  __syncthreads();
  float2 o[NJ * P];  // outputs X[k1 + E k2] for k1 = p + P j: o[j * P + k2]
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    const int k1 = p + P * j;
    if (k1 >= E) break;
    float2 w[P];
#pragma unroll
    for (int q = 0; q < P; ++q) w[q] = tr[k1 * RS + q * T + t];
    Bfly<P>::run(w);
#pragma unroll
    for (int k2 = 0; k2 < P; ++k2) o[j * P + k2] = w[k2];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NJ; ++j)
    if (p + P * j < E) {
#pragma unroll
      for (int k2 = 0; k2 < P; ++k2) tr[((p + P * j) + E * k2) * T + t] = o[j * P + k2];
    }
  __syncthreads();
}

// Wave-vector factors of a block's columns and rows, in shared memory:
// tilde(xi)_d = (2 n_d / L_d) * sin/cos products (fourier.py:9-58), tabulated in FP64 and
// kept as FP32 for the isotropic Gamma^0 (whose operator is applied in FP32), as FP64 as
// well for the anisotropic one (its per-mode acoustic inverse is FP64).
template <int NX, int T, bool ANI>
struct XWave {
  float f[3][T];
  float sx[NX], cx[NX];
  double df[3][ANI ? T : 1];
  double dsx[ANI ? NX : 1], dcx[ANI ? NX : 1];
  // threads tid < T fill the column factors, all threads the row tables
  template <typename CY, typename CZ>
  __device__ __forceinline__ void fill(const GridDesc& g, CY col_ky, CZ col_kz) {
    const int tid = threadIdx.x;
    if (tid < T) {
      const int kzz = col_kz(tid) < g.nzh ? col_kz(tid) : 0;
      const int kyy = col_ky(tid);
      const double c0 = (2.0 * g.nx / g.Lx) * g.cy[kyy] * g.cz[kzz];
      const double c1 = (2.0 * g.ny / g.Ly) * g.sy[kyy] * g.cz[kzz];
      const double c2 = (2.0 * g.nz / g.Lz) * g.cy[kyy] * g.sz[kzz];
      f[0][tid] = (float)c0;
      f[1][tid] = (float)c1;
      f[2][tid] = (float)c2;
      if constexpr (ANI) {
        df[0][tid] = c0;
        df[1][tid] = c1;
        df[2][tid] = c2;
      }
    }
    for (int i = tid; i < NX; i += blockDim.x) {
      sx[i] = (float)g.sx[i];
      cx[i] = (float)g.cx[i];
      if constexpr (ANI) {
        dsx[i] = g.sx[i];
        dcx[i] = g.cx[i];
      }
    }
  }
};

// Per mode of the block's tile (all six components in the regions of buf): the
// Hermitian-weighted |xi~ . sigma_hat|^2 (FP32 per mode, summed in FP64; returned, this
// thread's share), the FP64 zero mode, and r_hat = -Gamma^0 sigma_hat written back
// conjugated for the inverse transform. col_ky / col_kz map a column index to its (ky, kz).
// The isotropic form computes the wave vector and its norm in FP32 from the FP64 tables:
// the operator it feeds is FP32, and the FP32 |xi|^2 differs from the FP64 one by
// rounding (relative 1e-7; a component that underflows FP32 is below 1e-7 of another one
// or the mode is below the guard either way), so the guard |xi|^2 < 1e-24 takes the same
// modes in both except within that rounding of the threshold.
template <int NX, int T, int REG, bool ANI, typename CY, typename CZ>
__device__ __forceinline__ double x_modes(float2* buf, const XWave<NX, T, ANI>& wv,
                                          const GridDesc& g, const Medium& md,
                                          InstanceState* st, int b, CY col_ky, CZ col_kz) {
  const int tid = threadIdx.x;
  const int nzh = g.nzh;
  const float c_a = md.c_a, c_b = md.c_b;
  double acc = 0.0;
  for (int idx = tid; idx < NX * T; idx += blockDim.x) {
    const int kx = idx / T, tt = idx % T;
    const int kzz = col_kz(tt);
    if (kzz >= nzh) continue;
    float2 s[6];
#pragma unroll
    for (int cc = 0; cc < 6; ++cc) s[cc] = buf[(size_t)cc * REG + kx * T + tt];
    const float f0 = wv.sx[kx] * wv.f[0][tt];
    const float f1 = wv.cx[kx] * wv.f[1][tt];
    const float f2 = wv.cx[kx] * wv.f[2][tt];
    {
      float2 d0 = make_float2(f0 * s[0].x + f1 * s[3].x + f2 * s[4].x, f0 * s[0].y + f1 * s[3].y + f2 * s[4].y);
      float2 d1 = make_float2(f0 * s[3].x + f1 * s[1].x + f2 * s[5].x, f0 * s[3].y + f1 * s[1].y + f2 * s[5].y);
      float2 d2 = make_float2(f0 * s[4].x + f1 * s[5].x + f2 * s[2].x, f0 * s[4].y + f1 * s[5].y + f2 * s[2].y);
      const float m2 = d0.x * d0.x + d0.y * d0.y + d1.x * d1.x + d1.y * d1.y + d2.x * d2.x + d2.y * d2.y;
      acc += ((kzz == 0 || 2 * kzz == g.nz) ? 1.0 : 2.0) * (double)m2;
    }
    if (kx == 0 && col_ky(tt) == 0 && kzz == 0) {
#pragma unroll
      for (int cc = 0; cc < 6; ++cc) {
        st[b].sig0[2 * cc] = (double)s[cc].x + (double)g.nv * st[b].shift[cc];
        st[b].sig0[2 * cc + 1] = (double)s[cc].y;
      }
    }
    if constexpr (ANI) {
      // normalised wave vector: |xi| < 1e-12 (|xi|^2 < 1e-24) is replaced by 1 (fourier.py:84)
      const double x0 = wv.dsx[kx] * wv.df[0][tt];
      const double x1 = wv.dcx[kx] * wv.df[1][tt];
      const double x2 = wv.dcx[kx] * wv.df[2][tt];
      const double n2 = x0 * x0 + x1 * x1 + x2 * x2;
      const double inv = n2 < 1.0e-24 ? 1.0 : rsqrt(n2);
      // r = -Gamma^0 tau through the inverse acoustic matrix (FP64 per mode); modes without a
      // direction get r = 0
      const double zd[3] = {x0 * inv, x1 * inv, x2 * inv};
      double nd[6];
      float o[2][6];
      if (!(n2 < 1.0e-24) &&
          aniso_inverse_acoustic(g.c0 + (size_t)(b / g.lame_group) * 21, zd, nd)) {
        const float zt[3] = {(float)zd[0], (float)zd[1], (float)zd[2]};
        float nt[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) nt[k] = (float)nd[k];
#pragma unroll
        for (int part = 0; part < 2; ++part) {
          float tv[6];
#pragma unroll
          for (int cc = 0; cc < 6; ++cc) tv[cc] = part ? s[cc].y : s[cc].x;
          aniso_gamma<float>(nt, zt, tv, o[part]);
        }
      } else {
#pragma unroll
        for (int cc = 0; cc < 6; ++cc) o[0][cc] = o[1][cc] = 0.f;
      }
#pragma unroll
      for (int cc = 0; cc < 6; ++cc) buf[(size_t)cc * REG + kx * T + tt] = make_float2(o[0][cc], -o[1][cc]);
      continue;
    }
    // normalised wave vector: |xi| < 1e-12 (|xi|^2 < 1e-24) is replaced by 1 (fourier.py:84)
    const float n2 = f0 * f0 + f1 * f1 + f2 * f2;
    const float inv = n2 < 1.0e-24f ? 1.f : rsqrtf(n2);
    const float z0 = f0 * inv, z1 = f1 * inv, z2 = f2 * inv;
    const float z00 = z0 * z0, z11 = z1 * z1, z22 = z2 * z2;
    const float z01 = z0 * z1, z02 = z0 * z2, z12 = z1 * z2;
    float r[2][6];
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      float t0 = part ? s[0].y : s[0].x, t1 = part ? s[1].y : s[1].x, t2 = part ? s[2].y : s[2].x;
      float t3 = part ? s[3].y : s[3].x, t4 = part ? s[4].y : s[4].x, t5 = part ? s[5].y : s[5].x;
      float rho = z00 * t0 + z11 * t1 + z22 * t2 + 2.f * (z01 * t3 + z02 * t4 + z12 * t5);
      float a0 = z0 * (z0 * t0 + z2 * t4 + z1 * t3);
      float a1 = z1 * (z1 * t1 + z2 * t5 + z0 * t3);
      float a2 = z2 * (z2 * t2 + z1 * t5 + z0 * t4);
      float a3 = 0.5f * (z01 * (t0 + t1) + (z00 + z11) * t3 + z2 * (z0 * t5 + z1 * t4));
      float a4 = 0.5f * (z02 * (t0 + t2) + (z00 + z22) * t4 + z1 * (z0 * t5 + z2 * t3));
      float a5 = 0.5f * (z12 * (t1 + t2) + (z11 + z22) * t5 + z0 * (z1 * t4 + z2 * t3));
      r[part][0] = c_a * a0 + c_b * rho * z00;
      r[part][1] = c_a * a1 + c_b * rho * z11;
      r[part][2] = c_a * a2 + c_b * rho * z22;
      r[part][3] = c_a * a3 + c_b * rho * z01;
      r[part][4] = c_a * a4 + c_b * rho * z02;
      r[part][5] = c_a * a5 + c_b * rho * z12;
    }
#pragma unroll
    for (int cc = 0; cc < 6; ++cc) buf[(size_t)cc * REG + kx * T + tt] = make_float2(r[0][cc], -r[1][cc]);
  }
  __syncthreads();
  return acc;
}

// Inverse x DFT (forward transform of the conjugate held in tr, natural layout): step A,
// transpose, step B; out(k, w) receives the conjugated output for row k = k1 + E k2.
template <int NX, int T, typename SP, typename OUT>
__device__ __forceinline__ void x_inverse(float2* tr, int p, int t, const float2* stw, OUT out) {
  constexpr int E = SP::E, P = SP::P, RS = x_row<NX, T, SP>();
  float2 v[E];
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = tr[(p + P * e) * T + t];
  step_a_smem<NX, E>(v, p, stw);
  __syncthreads();
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) tr[k1 * RS + p * T + t] = v[k1];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < (E + P - 1) / P; ++j) {
    const int k1 = p + P * j;
    if (k1 >= E) break;
    float2 w[P];
#pragma unroll
    for (int q = 0; q < P; ++q) w[q] = tr[k1 * RS + q * T + t];
    Bfly<P>::run(w);
#pragma unroll
    for (int k2 = 0; k2 < P; ++k2) out(k1 + E * k2, conj2(w[k2]));
  }
}

// Deterministic block reduction of the residual partial into *out (thread 0 writes).
__device__ __forceinline__ void x_block_sum(double acc, double* red, double* out) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((tid & 31) == 0) red[tid >> 5] = acc;
  __syncthreads();
  if (tid < 32) {
    double w = (tid < (int)(blockDim.x + 31) / 32) ? red[tid] : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) w += __shfl_xor_sync(0xffffffffu, w, off);
    if (tid == 0) *out = w;
  }
}

// ANI: Gamma^0 of an anisotropic reference stiffness (aniso.cuh) instead of the isotropic
// closed form.
template <int NX, int V, bool ANI>
__global__ void __launch_bounds__(6 * XSplit<NX>::P * x_cols_v<NX, V>(), x_min_blocks<NX, V>()) xpass_fast(
    GridDesc g, float2* __restrict__ spec, const Medium* __restrict__ med,
    InstanceState* __restrict__ st, double* __restrict__ partials) {
  constexpr int E = XSplit<NX>::E, P = XSplit<NX>::P, T = x_cols_v<NX, V>(), REG = x_region<NX, T>();
  static_assert((6 * P * T) % 32 == 0, "the x pass reduces over whole warps");
  extern __shared__ __align__(16) unsigned char xfraw[];
  float2* buf = reinterpret_cast<float2*>(xfraw);  // 6 regions of REG values
  __shared__ double red[32];
  // shared-memory copies of the x twiddles and wave-vector tables (read per element / mode;
  // from shared memory the x pass is 6% faster at 128^3 than from the L1/global path)
  __shared__ float2 stw[NX];  // exp(-2 pi i k / NX)
  __shared__ XWave<NX, T, ANI> wv;
  const int b = blockIdx.z;
  if (!active32(st[b])) return;
  const int tid = threadIdx.x;
  const int t = tid % T, p = (tid / T) % P, c = tid / (T * P);
  const int nzh = g.nzh;
  // With nz/2+1 = T k + 1 the last tile takes the z Nyquist column for T consecutive ky
  // instead of one column per ky (as the y pass); its surplus blocks only report a zero
  // partial.
  const bool tail = nzh % T == 1 && (int)blockIdx.x == nzh / T;
  if (tail && (int)blockIdx.y * T >= g.ny) {
    if (tid == 0) partials[(size_t)b * gridDim.x * gridDim.y + blockIdx.y * gridDim.x + blockIdx.x] = 0.0;
    return;
  }
  auto col_ky = [&](int tt) { return tail ? (int)blockIdx.y * T + tt : (int)blockIdx.y; };
  auto col_kz = [&](int tt) { return tail ? nzh - 1 : (int)blockIdx.x * T + tt; };
  const int ky = col_ky(t);
  const int kz = col_kz(t);
  const bool valid = kz < nzh;
  const size_t xstride = (size_t)g.ny * nzh;
  float2* gcol = spec + (size_t)b * 6 * g.nm + (size_t)c * g.nm + (size_t)ky * nzh + kz;
  const float2* tw = g.px.tw;
  float2* tr = buf + (size_t)c * REG;   // this component's region

  wv.fill(g, col_ky, col_kz);

  // forward: load, step A, transpose
  float2 v[E];
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = valid ? gcol[(size_t)(p + P * e) * xstride] : make_float2(0.f, 0.f);
  for (int i = tid; i < NX; i += blockDim.x) stw[i] = tw[i];
  __syncthreads();
  x_forward<NX, T>(tr, v, p, t, stw);
  const double acc = x_modes<NX, T, REG, ANI>(buf, wv, g, med[b / g.lame_group], st, b, col_ky, col_kz);
  x_inverse<NX, T, XSplit<NX>>(tr, p, t, stw, [&](int k, float2 w) {
    if (valid) gcol[(size_t)k * xstride] = w;
  });
  x_block_sum(acc, red, partials + (size_t)b * gridDim.x * gridDim.y + blockIdx.y * gridDim.x + blockIdx.x);
}

// ----------------------------------------------------------------------------- tiled x pass
// Split of the tiled x pass's transform: that of the strided pass, except 48 = 8 x 6 (six
// threads per column, so that 6 components x 8 columns make whole warps).
template <int N>
struct XTSplit { static constexpr int E = XSplit<N>::E, P = XSplit<N>::P; };
template <>
struct XTSplit<48> { static constexpr int E = 8, P = 6; };
template <int NX>
__host__ __device__ constexpr int xt_threads() { return 6 * XTSplit<NX>::P * kTW; }
// (three 384-thread blocks per SM: 0.193 against 0.208 ms with two at 128^3)
#ifndef LSB_XT_MINB
#define LSB_XT_MINB 3
#endif
template <int NX>
__host__ __device__ constexpr int xt_min_blocks() { return xt_threads<NX>() <= 192 ? 4 : LSB_XT_MINB; }

// Block = one tile (full tile of ky, or a tail group of 8 ky) of one instance; thread
// (c, p, t) with t fastest.
template <int NX, bool ANI>
__global__ void __launch_bounds__(xt_threads<NX>(), xt_min_blocks<NX>()) xpass_tiled(
    GridDesc g, float2* __restrict__ spec, const Medium* __restrict__ med,
    InstanceState* __restrict__ st, double* __restrict__ partials) {
  using SP = XTSplit<NX>;
  constexpr int E = SP::E, P = SP::P, T = kTW, REG = x_region<NX, T, SP>();
  static_assert((6 * P * T) % 32 == 0, "the x pass reduces over whole warps");
  extern __shared__ __align__(128) unsigned char xtraw[];
  float2* buf = reinterpret_cast<float2*>(xtraw);  // 6 regions of REG values
  __shared__ double red[32];
  __shared__ float2 stw[NX];
  __shared__ XWave<NX, T, ANI> wv;
  __shared__ __align__(8) unsigned long long mbar_word;
  const int b = blockIdx.y;
  if (!active32(st[b])) return;
  const int tid = threadIdx.x;
  const int t = tid % T, p = (tid / T) % P, c = tid / (T * P);
  const int nzh = g.nzh, nf = (nzh - 1) / T;
  const int tile = blockIdx.x;
  const bool tail = tile >= g.ny * nf;
  const int ky_full = tail ? 0 : tile % g.ny, j = tail ? 0 : tile / g.ny, grp = tail ? tile - g.ny * nf : 0;
  auto col_ky = [&](int tt) { return tail ? grp * T + tt : ky_full; };
  auto col_kz = [&](int tt) { return tail ? nzh - 1 : j * T + tt; };
  const size_t chunk = tail ? (size_t)g.ny * nf * NX * T + (size_t)grp * NX * T
                            : (size_t)(j * g.ny + ky_full) * NX * T;
  float2* sb = spec + (size_t)b * 6 * g.nm;
  float2* tr = buf + (size_t)c * REG;
  const unsigned mbar = smem_u32(&mbar_word);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    constexpr unsigned bytes = NX * T * 8;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(mbar), "r"(6 * bytes) : "memory");
    for (int cc = 0; cc < 6; ++cc) bulk_g2s(buf + (size_t)cc * REG, sb + (size_t)cc * g.nm + chunk, bytes, mbar);
  }
  wv.fill(g, col_ky, col_kz);
  for (int i = tid; i < NX; i += blockDim.x) stw[i] = g.px.tw[i];
  if (!mbar_wait(mbar)) {
    // the copies did not land in time: report, leave the instance stopped, and wait once
    // more (bounded) before the shared memory is released
    if (tid == 0) {
      st[b].status = kTimeout;
      st[b].done = 1;
    }
    if (!mbar_wait(mbar) && tid == 0) st[b].copies_lost = 1;
    if (tid == 0) partials[(size_t)b * gridDim.x + tile] = 0.0;
    return;
  }
  __syncthreads();
  float2 v[E];
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = tr[(p + P * e) * T + t];
  __syncthreads();
  x_forward<NX, T, SP>(tr, v, p, t, stw);
  const double acc = x_modes<NX, T, REG, ANI>(buf, wv, g, med[b / g.lame_group], st, b, col_ky, col_kz);
  float2* gout = sb + (size_t)c * g.nm + chunk;
  x_inverse<NX, T, SP>(tr, p, t, stw, [&](int k, float2 w) { gout[(size_t)k * T + t] = w; });
  x_block_sum(acc, red, partials + (size_t)b * gridDim.x + tile);
}

// ----------------------------------------------------------------------------- z pass
// Block = L (x, y) lines = 3L complex pair lines; thread (line q, p), p fastest.
// The block's inputs (spectrum rows, strain rows, lambda/mu rows) are contiguous chunks;
// one thread issues them as TMA bulk copies into shared memory (completion on an
// mbarrier), so all of a block's loads are in flight at once, and the resident blocks of
// an SM overlap one block's loads with the others' transforms.
template <int NZ>
__host__ __device__ constexpr int z_lines() {
  // 96 threads (72 for P = 3, 6): small blocks, four or more resident per SM, so that the
  // TMA loads of some blocks overlap the transforms of others (measured: -14% at 128^3
  // against 192-thread blocks)
  return Split<NZ>::P == 3 ? 8 : (Split<NZ>::P == 6 ? 4 : 96 / (3 * Split<NZ>::P));
}
template <int NZ>
__host__ __device__ constexpr int z_threads() { return 3 * z_lines<NZ>() * Split<NZ>::P; }
template <int NZ>
__host__ __device__ constexpr int z_min_blocks() {
  return z_threads<NZ>() > 192 ? 1 : (384 / z_threads<NZ>() > 2 ? 384 / z_threads<NZ>() : 2);
}
// Line pitch of the transform buffer: room for the padded transposed layout
// k1 * (P + 1) + p (conflict-free column reads), and = 8 (mod 16) so that the two lines
// of a half-warp fall in disjoint banks.
template <int NZ>
__host__ __device__ constexpr int z_ld() {
  return ((Split<NZ>::E * (Split<NZ>::P + 1) > NZ ? Split<NZ>::E * (Split<NZ>::P + 1) : NZ) + 7) / 16 * 16 + 8;
}

struct ZLayout {  // byte offsets inside the z pass's dynamic shared memory
  size_t zbuf, rst, est, lst, total;
};
// Modes 1 and 3 (compiled per mode) read their strain rows (and, mode 1, lambda and mu)
// only after the inverse z transform: those rows are staged late, into the region of the
// spectrum rows once they have been expanded into the transform buffer, so that the copies
// overlap the transform and the block needs less shared memory (at 128: 27 KB and eight
// resident blocks for mode 3 instead of 39 KB and five; 31 KB and seven for mode 1).
template <int MODE>
__host__ __device__ constexpr bool z_late() { return MODE == 1 || MODE == 3; }
// MODE < 0: the mode is a run-time argument (every staging region); otherwise only the
// regions that mode stages (spectrum rows for 1 and 3, strain rows for 1-3, lambda and mu
// rows for 0-2), so that the other modes keep more blocks resident.
template <int NZ, int MODE = -1>
__host__ __device__ constexpr ZLayout z_layout() {
  constexpr int L = z_lines<NZ>(), NZH = NZ / 2 + 1;
  constexpr bool r = MODE < 0 || MODE == 1 || MODE == 3;
  constexpr bool e = MODE != 0;
  constexpr bool l = MODE != 3;
  constexpr size_t zb = (size_t)3 * L * z_ld<NZ>() * 8;
  constexpr size_t rs = r ? (size_t)6 * L * NZH * 8 : 0;
  constexpr size_t es = e ? (size_t)6 * L * NZ * 4 : 0;
  constexpr size_t ls = l ? (size_t)2 * L * NZ * 4 : 0;
  if constexpr (z_late<MODE>())
    return ZLayout{0, zb, zb, zb + es, zb + (rs > es + ls ? rs : es + ls)};
  return ZLayout{0, zb, zb + rs, zb + rs + es, zb + rs + es + ls};
}

// In-place four-step FFT of the 3L lines of zbuf (natural order in and out).
template <int NZ>
__device__ __forceinline__ void zline_fft(float2* zbuf, int q, int p, const float2* __restrict__ tw) {
  constexpr int E = Split<NZ>::E, P = Split<NZ>::P, LD = z_ld<NZ>(), NJ = rounds<NZ>();
  float2* line = zbuf + (size_t)q * LD;
  float2 v[E];
  float2 o[NJ * P];
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = line[p + P * e];
  step_a<NZ>(v, p, tw);
  __syncthreads();
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) line[k1 * (P + 1) + p] = v[k1];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    const int k1 = p + P * j;
    if (k1 >= E) break;
    float2 w[P];
#pragma unroll
    for (int qq = 0; qq < P; ++qq) w[qq] = line[k1 * (P + 1) + qq];
    Bfly<P>::run(w);
#pragma unroll
    for (int k2 = 0; k2 < P; ++k2) o[j * P + k2] = w[k2];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NJ; ++j)
    if (p + P * j < E) {
#pragma unroll
      for (int k2 = 0; k2 < P; ++k2) line[(p + P * j) + E * k2] = o[j * P + k2];
    }
  __syncthreads();
}

// Resident blocks the kernel of a mode is compiled for: the plain update (mode 1, whose
// late staging leaves room for seven blocks at 128) as many as its shared memory allows,
// at most eight; the other modes z_min_blocks.
template <int NZ, int MODE>
__host__ __device__ constexpr int z_min_blocks_mode() {
  constexpr int smem = (int)((228u * 1024) / (z_layout<NZ, MODE>().total + 1024 + 128));
  constexpr int want = smem > 8 ? 8 : smem;
  return MODE == 1 && want > z_min_blocks<NZ>() ? want : z_min_blocks<NZ>();
}

// Modes as the generic z pass: 0 init from eps_bar/eps0, 1 plain update, 2 keep eps
// (not rewritten), 3 Anderson residual into the rings.
// bulk: the block's global chunks are 16-byte aligned (TMA bulk copies); otherwise the
// staging buffers are filled by ordinary loads.
// LAW: 0 isotropic (lambda, mu staged), 1 damage extension, 2 anisotropic stiffness (21
// entries read per voxel from global memory; lambda and mu not staged).
// MODE >= 0 fixes the mode at compile time (mode_arg is then ignored).
template <int NZ, int LAW, int MODE>
__global__ void __launch_bounds__(z_threads<NZ>(), z_min_blocks_mode<NZ, MODE>()) zpass_fast(
    GridDesc g, int mode_arg, int bulk, const float* __restrict__ lambda, const float* __restrict__ mu,
    float* __restrict__ eps, float2* __restrict__ spec, const double* __restrict__ eps_bar,
    const float* __restrict__ eps0, InstanceState* __restrict__ st, const Medium* __restrict__ med,
    AndersonArgs<float> aa) {
  constexpr int P = Split<NZ>::P, L = z_lines<NZ>(), LD = z_ld<NZ>(), NZH = NZ / 2 + 1;
  constexpr ZLayout LY = z_layout<NZ, MODE>();
  const int mode = MODE >= 0 ? MODE : mode_arg;
  extern __shared__ __align__(128) unsigned char zfraw[];
  float2* zbuf = reinterpret_cast<float2*>(zfraw + LY.zbuf);  // 3L lines of LD values
  float2* rst = reinterpret_cast<float2*>(zfraw + LY.rst);    // [6][L][NZH] spectrum rows
  float* est = reinterpret_cast<float*>(zfraw + LY.est);      // [6][L][NZ] strain rows
  float* lst = reinterpret_cast<float*>(zfraw + LY.lst);      // [2][L][NZ] lambda, mu rows
  __shared__ __align__(8) unsigned long long mbar_word[2];  // early and late staging
  constexpr bool late = z_late<MODE>();
  const int b = blockIdx.y;
  if (!active32(st[b])) return;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int p = tid % P, q = tid / P;
  const long long nlines = (long long)g.nx * g.ny;
  const long long l0 = (long long)blockIdx.x * L;
  float* eb = eps + (size_t)b * 6 * g.nv;
  float2* sb = spec + (size_t)b * 6 * g.nm;
  const float2* tw = g.pz.tw;
  lambda += (size_t)(b / g.lame_group) * g.nv;
  mu += (size_t)(b / g.lame_group) * g.nv;
  med += b / g.lame_group;
  const bool need_r = (mode == 1 || mode == 3);
  const bool need_e = (mode == 1 || mode == 2 || mode == 3);
  const bool need_l = (mode != 3) && LAW != 2;

  // ---- stage this block's inputs in shared memory (modes 1 and 3: the spectrum rows now,
  // the strain (and lambda, mu) rows after the spectrum rows are consumed)
  const unsigned ebytes = L * NZ * 4;
  auto stage_late_bulk = [&](unsigned mbar2) {
    // (the block's reads of the spectrum rows are ordered before these async-proxy writes
    // by the preceding barrier and the proxy fence)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    const unsigned total = 6 * ebytes + (need_l ? 2 * ebytes : 0);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(mbar2), "r"(total) : "memory");
    for (int c = 0; c < 6; ++c)
      bulk_g2s(est + (size_t)c * L * NZ, eb + (size_t)c * g.nv + l0 * NZ, ebytes, mbar2);
    if (need_l) {
      bulk_g2s(lst, lambda + l0 * NZ, ebytes, mbar2);
      bulk_g2s(lst + L * NZ, mu + l0 * NZ, ebytes, mbar2);
    }
  };
  if (bulk) {
    const unsigned mbar = smem_u32(&mbar_word[0]);
    if (tid == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(mbar) : "memory");
      if (late) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar_word[1])) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
      const unsigned rbytes = L * NZH * 8;
      const bool e_now = need_e && !late, l_now = need_l && !late;
      const unsigned total = (need_r ? 6 * rbytes : 0) + (e_now ? 6 * ebytes : 0) + (l_now ? 2 * ebytes : 0);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(mbar), "r"(total) : "memory");
      for (int c = 0; c < 6; ++c) {
        if (need_r) bulk_g2s(rst + (size_t)c * L * NZH, sb + ((size_t)c * nlines + l0) * NZH, rbytes, mbar);
        if (e_now) bulk_g2s(est + (size_t)c * L * NZ, eb + (size_t)c * g.nv + l0 * NZ, ebytes, mbar);
      }
      if (l_now) {
        bulk_g2s(lst, lambda + l0 * NZ, ebytes, mbar);
        bulk_g2s(lst + L * NZ, mu + l0 * NZ, ebytes, mbar);
      }
    }
    if (!mbar_wait(mbar)) {
      // the copies did not land in time: report and leave this instance stopped; wait once
      // more (bounded) for them before the block's shared memory is released, and record
      // when even that wait ran out (the instance's buffers are then suspect)
      if (tid == 0) {
        st[b].status = kTimeout;
        st[b].done = 1;
      }
      if (!mbar_wait(mbar) && tid == 0) st[b].copies_lost = 1;
      return;
    }
  } else {
    for (int c = 0; c < 6; ++c) {
      if (need_r)
        for (int i = tid; i < L * NZH; i += nt) rst[c * L * NZH + i] = sb[((size_t)c * nlines + l0) * NZH + i];
      if (need_e && !late)
        for (int i = tid; i < L * NZ; i += nt) est[c * L * NZ + i] = eb[(size_t)c * g.nv + l0 * NZ + i];
    }
    if (need_l && !late)
      for (int i = tid; i < L * NZ; i += nt) {
        lst[i] = lambda[l0 * NZ + i];
        lst[L * NZ + i] = mu[l0 * NZ + i];
      }
    __syncthreads();
  }

  if (need_r) {
    // conj(Z) with Z[k] = A[k] + i B[k] (Hermitian extension; DC and Nyquist taken real)
    for (int idx = tid; idx < 3 * L * NZH; idx += nt) {
      const int pr = idx / (L * NZH);
      const int rem = idx - pr * (L * NZH);
      const int l = rem / NZH, k = rem - l * NZH;
      float2 A = rst[(2 * pr) * L * NZH + rem];
      float2 B = rst[(2 * pr + 1) * L * NZH + rem];
      const bool selfconj = (k == 0) || (2 * k == NZ);
      if (selfconj) { A.y = 0.f; B.y = 0.f; }
      float2* Z = zbuf + (size_t)(pr * L + l) * LD;
      Z[k] = make_float2(A.x - B.y, -(A.y + B.x));
      if (!selfconj) Z[NZ - k] = make_float2(A.x + B.y, A.y - B.x);
    }
    __syncthreads();
    if constexpr (late) {
      // the strain (and lambda, mu) rows into the spectrum rows' region, during the transform
      if (bulk) {
        if (tid == 0) stage_late_bulk(smem_u32(&mbar_word[1]));
      } else {
        for (int c = 0; c < 6; ++c)
          for (int i = tid; i < L * NZ; i += nt) est[c * L * NZ + i] = eb[(size_t)c * g.nv + l0 * NZ + i];
        if (need_l)
          for (int i = tid; i < L * NZ; i += nt) {
            lst[i] = lambda[l0 * NZ + i];
            lst[L * NZ + i] = mu[l0 * NZ + i];
          }
      }
    }
    zline_fft<NZ>(zbuf, q, p, tw);  // (ends with a barrier: the plain late loads are visible)
    if constexpr (late) {
      if (bulk && !mbar_wait(smem_u32(&mbar_word[1]))) {
        // as for the early copies: report, stop the instance, wait once more (bounded)
        if (tid == 0) {
          st[b].status = kTimeout;
          st[b].done = 1;
        }
        if (!mbar_wait(smem_u32(&mbar_word[1])) && tid == 0) st[b].copies_lost = 1;
        return;
      }
    }
  }

  if (mode == 3) {
    const int M1 = aa.depth + 1;
    const size_t ring = (size_t)6 * g.nv;
    const int slot = (st[b].iter - 1 - st[b].aa_base) % M1;
    __half* rb = aa.r + (size_t)b * M1 * ring;
    float* gb = aa.g + (size_t)b * M1 * ring;
    const float inv_nv = (float)(1.0 / (double)g.nv);
    const int kexp = ring_exponent(st[b].ring_max, eps_bar + 6 * b);
    const float rscale = ldexpf(1.f, kexp);
    if (blockIdx.x == 0 && tid == 0) st[b].ring_exp[slot] = kexp;
    for (int idx = tid; idx < L * NZ; idx += nt) {
      const int l = idx / NZ, n = idx % NZ;
      const size_t vx = (size_t)(l0 + l) * NZ + n;
      float r[6];
#pragma unroll
      for (int pr = 0; pr < 3; ++pr) {
        float2 w = zbuf[(size_t)(pr * L + l) * LD + n];
        r[2 * pr] = w.x * inv_nv;
        r[2 * pr + 1] = -w.y * inv_nv;
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        const size_t o = (size_t)c * g.nv + vx;
        rb[slot * ring + o] = ring_store(r[c], rscale);
        gb[slot * ring + o] = est[c * L * NZ + idx] + r[c];
      }
    }
    return;
  }

  float shift[6];
  if (mode != 0) {
#pragma unroll
    for (int c = 0; c < 6; ++c) shift[c] = (float)st[b].shift[c];
  } else {
    const double* e = eps_bar + 6 * b;
    const double tr = e[0] + e[1] + e[2];
#pragma unroll
    for (int c = 0; c < 6; ++c)
      shift[c] = (float)((c < 3 ? med->lmean * tr : 0.0) + 2.0 * med->mmean * e[c]);
    if constexpr (LAW == 2) {  // anisotropic: C^0 eps_bar
      const double* c0 = g.c0 + (size_t)(b / g.lame_group) * 21;
      double sh[6];
      aniso_stress<double>([&](int k) { return c0[k]; }, e, sh);
#pragma unroll
      for (int c = 0; c < 6; ++c) shift[c] = (float)sh[c];
    }
    if (blockIdx.x == 0 && tid == 0) {
#pragma unroll
      for (int c = 0; c < 6; ++c) st[b].shift[c] = (double)shift[c];
    }
  }

  {
    const float inv_nv = (float)(1.0 / (double)g.nv);
    for (int idx = tid; idx < L * NZ; idx += nt) {
      const int l = idx / NZ, n = idx % NZ;
      const size_t vx = (size_t)(l0 + l) * NZ + n;
      float e[6];
      if (mode == 1) {
#pragma unroll
        for (int pr = 0; pr < 3; ++pr) {
          float2 w = zbuf[(size_t)(pr * L + l) * LD + n];
          e[2 * pr] = est[(2 * pr) * L * NZ + idx] + w.x * inv_nv;
          e[2 * pr + 1] = est[(2 * pr + 1) * L * NZ + idx] - w.y * inv_nv;
        }
      } else if (mode == 2) {
#pragma unroll
        for (int c = 0; c < 6; ++c) e[c] = est[c * L * NZ + idx];
      } else if (eps0 != nullptr) {
#pragma unroll
        for (int c = 0; c < 6; ++c) e[c] = eps0[((size_t)b * 6 + c) * g.nv + vx];
      } else {
#pragma unroll
        for (int c = 0; c < 6; ++c) e[c] = (float)eps_bar[b * 6 + c];
      }
      if (mode != 2) {
#pragma unroll
        for (int c = 0; c < 6; ++c) eb[(size_t)c * g.nv + vx] = e[c];
      }
      float s[6];
      if constexpr (LAW == 2) {
        const float* cfb = g.cf32 + (size_t)(b / g.lame_group) * 21 * g.nv + vx;
        aniso_stress<float>([&](int k) { return cfb[(size_t)k * g.nv]; }, e, s);
      } else if constexpr (LAW == 1) {
        // the damage extension's law (damage field read per voxel, not staged)
        const float om = 1.f - g.dmg32[(size_t)(b / g.lame_group) * g.nv + vx];
        damaged_stress<float>(e, lst[idx], lst[L * NZ + idx], om * om + (float)g.dmg_k, s);
      } else {
        const float lam = lst[idx], tmu = 2.f * lst[L * NZ + idx];
        const float ltr = lam * (e[0] + e[1] + e[2]);
#pragma unroll
        for (int c = 0; c < 3; ++c) s[c] = tmu * e[c] + ltr;
#pragma unroll
        for (int c = 3; c < 6; ++c) s[c] = tmu * e[c];
      }
#pragma unroll
      for (int pr = 0; pr < 3; ++pr)
        zbuf[(size_t)(pr * L + l) * LD + n] =
            make_float2(s[2 * pr] - shift[2 * pr], s[2 * pr + 1] - shift[2 * pr + 1]);
    }
  }
  __syncthreads();
  zline_fft<NZ>(zbuf, q, p, tw);

  for (int idx = tid; idx < 3 * L * NZH; idx += nt) {
    const int pr = idx / (L * NZH);
    const int rem = idx - pr * (L * NZH);
    const int l = rem / NZH, k = rem - l * NZH;
    const long long line = l0 + l;
    const float2* Z = zbuf + (size_t)(pr * L + l) * LD;
    const float2 zk = Z[k];
    const float2 zm = Z[k == 0 ? 0 : NZ - k];
    sb[((size_t)(2 * pr) * nlines + line) * NZH + k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    sb[((size_t)(2 * pr + 1) * nlines + line) * NZH + k] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
  }
}

// ----------------------------------------------------------------------------- slab pass
// The inverse y pass, the z pass and the forward y pass of one x-plane of one instance in
// one kernel: a thread-block cluster of CS = nz / 16 blocks holds the plane's half
// spectrum, 6 x ny x (nz/2+1) complex values, in distributed shared memory, rank r owning
// the kz columns of tile r (8 columns, read from and written to the tiled layout as one
// 64-byte row per (component, ky)) and, on the last rank, the z Nyquist column; and the
// ny / CS rows y in [r ny / CS, (r+1) ny / CS) for the z transforms.
//   phase A  inverse y DFT of the rank's columns (in place in shared memory)
//   phase B  per batch of R rows: gather the rows' half spectra from the ranks' columns,
//            inverse z transform (two components per complex line), the pointwise stage
//            of the mode, forward z transform, scatter the half spectra back
//   phase C  forward y DFT of the rank's columns, store
// Modes as the z pass: 0 init (eps from eps_bar or eps0), 1 plain update, 2 stress of the
// eps in memory (after the Anderson combine), 3 Anderson residual into the rings (phases A
// and B, no forward transforms). The arithmetic is that of ypass_fast and zpass_fast
// (same splits, same order), so the fields equal theirs bit for bit; the spectrum never
// leaves the plane between the y and z transforms, which saves their two HBM round trips.
namespace cg = cooperative_groups;

constexpr int kSlabKW = kTW + 1;  // local columns per rank: one tile and the Nyquist slot
constexpr int kSlabR = 8;         // rows per batch of phase B

template <int NZ>
__host__ __device__ constexpr int slab_ranks() { return NZ / 2 / kTW; }
template <int NZ>
__host__ __device__ constexpr int slab_threads() { return 3 * kSlabR * Split<NZ>::P; }

struct SlabLayout {  // byte offsets inside the slab kernel's dynamic shared memory
  size_t cols, zbuf, total;
};
template <int NY, int NZ>
__host__ __device__ constexpr SlabLayout slab_layout() {
  constexpr size_t cols = (size_t)6 * NY * kSlabKW * 8;
  constexpr size_t zb = (size_t)3 * kSlabR * z_ld<NZ>() * 8;
  return SlabLayout{0, cols, cols + zb};
}

// In-place y DFT of the ncols columns of `cols` ([6][NY][kSlabKW], column q = (c, kk) with
// kk < kw) by groups of P threads; forward, or inverse through the conjugates. Same
// arithmetic as ypass_fast.
template <int NY>
__device__ __forceinline__ void slab_ydft(float2* cols, int kw, bool inverse, const float2* __restrict__ tw) {
  constexpr int E = YSplit<NY>::E, P = YSplit<NY>::P, NJ = (E + P - 1) / P;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int per_round = nt / P;
  const int ncols = 6 * kw;
  // columns across the lanes, as in ypass_fast: the lanes of a warp touch neighbouring
  // columns of one slot, so neither step has bank conflicts (p across the lanes put every
  // step-B read of a warp in one bank)
  const int qq = tid % per_round, p = tid / per_round;
  for (int base = 0; base < ncols; base += per_round) {
    const int q = base + qq;
    const bool on = p < P && q < ncols;
    float2* col = cols + (on ? ((size_t)(q / kw) * NY * kSlabKW + (q % kw)) : 0);
    float2 v[E];
    if (on) {
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const float2 a = col[(size_t)(p + P * e) * kSlabKW];
        v[e] = inverse ? conj2(a) : a;
      }
    }
    __syncthreads();
    if (on) {
      step_a<NY, E>(v, p, tw);
#pragma unroll
      for (int k1 = 0; k1 < E; ++k1) col[(size_t)(k1 * P + p) * kSlabKW] = v[k1];
    }
    __syncthreads();
    float2 o[NJ * P];
    if (on) {
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int k1 = p + P * j;
        if (k1 >= E) break;
        float2 w[P];
#pragma unroll
        for (int q2 = 0; q2 < P; ++q2) w[q2] = col[(size_t)(k1 * P + q2) * kSlabKW];
        Bfly<P>::run(w);
#pragma unroll
        for (int k2 = 0; k2 < P; ++k2) o[j * P + k2] = inverse ? conj2(w[k2]) : w[k2];
      }
    }
    __syncthreads();
    if (on) {
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int k1 = p + P * j;
        if (k1 >= E) break;
#pragma unroll
        for (int k2 = 0; k2 < P; ++k2) col[(size_t)(k1 + E * k2) * kSlabKW] = o[j * P + k2];
      }
    }
    __syncthreads();
  }
}

template <int NY, int NZ, int MODE>
__global__ void __launch_bounds__(slab_threads<NZ>(), 1) slab_fast(
    GridDesc g, const float* __restrict__ lambda, const float* __restrict__ mu,
    float* __restrict__ eps, float2* __restrict__ tspec, const double* __restrict__ eps_bar,
    const float* __restrict__ eps0, InstanceState* __restrict__ st, const Medium* __restrict__ med,
    AndersonArgs<float> aa) {
  constexpr int CS = slab_ranks<NZ>(), NZH = NZ / 2 + 1, LD = z_ld<NZ>(), R = kSlabR;
  constexpr int P = Split<NZ>::P, ROWS = NY / CS, NF = NZ / 2 / kTW;
  constexpr SlabLayout LY = slab_layout<NY, NZ>();
  static_assert(ROWS % R == 0, "rows per rank must be whole batches");
  extern __shared__ __align__(128) unsigned char slraw[];
  float2* cols = reinterpret_cast<float2*>(slraw + LY.cols);  // [6][NY][kSlabKW]
  float2* zbuf = reinterpret_cast<float2*>(slraw + LY.zbuf);  // 3R lines of LD values
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int x = blockIdx.y, b = blockIdx.z;
  // uniform over the cluster (all ranks read the same state): no rank reaches a cluster
  // barrier that the others skip
  if (!active32(st[b])) return;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int nx = g.nx;
  const long long nv = g.nv;
  const int kw = rank == CS - 1 ? kTW + 1 : kTW;  // used local columns
  float2* tb = tspec + (size_t)b * 6 * g.nm;
  float* eb = eps + (size_t)b * 6 * nv;
  const size_t tail0 = (size_t)NY * NF * nx * kTW;
  constexpr bool kInverse = MODE == 1 || MODE == 3;
  constexpr bool kForward = MODE != 3;
  // phase B reads this rank's rows of the strain (and lambda, mu): contiguous ROWS x NZ
  // chunks, prefetched into L2 now so that those loads do not wait on DRAM after phase A
  // (bulk prefetches need 16-byte aligned addresses: skipped for unaligned caller buffers)
  const bool aligned = ((reinterpret_cast<uintptr_t>(eb) | reinterpret_cast<uintptr_t>(lambda) |
                         reinterpret_cast<uintptr_t>(mu)) & 15) == 0;
  if (tid == 0 && aligned && (MODE == 1 || MODE == 2 || MODE == 3)) {
    const size_t row0 = ((size_t)x * NY + (size_t)rank * ROWS) * NZ;
    const unsigned bytes = ROWS * NZ * 4;
#pragma unroll
    for (int c = 0; c < 6; ++c)
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(eb + (size_t)c * nv + row0), "r"(bytes) : "memory");
    if (MODE != 3) {
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(lambda + (size_t)(b / g.lame_group) * nv + row0), "r"(bytes) : "memory");
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(mu + (size_t)(b / g.lame_group) * nv + row0), "r"(bytes) : "memory");
    }
  }

  // ---- phase A: the rank's columns (tile `rank`, and the Nyquist column on the last rank)
  if constexpr (kInverse) {
    for (int i = tid; i < 6 * NY * (kTW / 2); i += nt) {
      const int c = i / (NY * (kTW / 2)), rem = i % (NY * (kTW / 2));
      const int ky = rem / (kTW / 2), h = rem % (kTW / 2);
      const float4 v = *reinterpret_cast<const float4*>(
          tb + (size_t)c * g.nm + ((size_t)(rank * NY + ky) * nx + x) * kTW + 2 * h);
      float2* d = cols + ((size_t)c * NY + ky) * kSlabKW + 2 * h;
      d[0] = make_float2(v.x, v.y);
      d[1] = make_float2(v.z, v.w);
    }
    if (rank == CS - 1) {
      for (int i = tid; i < 6 * NY; i += nt) {
        const int c = i / NY, ky = i % NY;
        cols[((size_t)c * NY + ky) * kSlabKW + kTW] =
            tb[(size_t)c * g.nm + tail0 + ((size_t)(ky / kTW) * nx + x) * kTW + (ky % kTW)];
      }
    }
    __syncthreads();
    slab_ydft<NY>(cols, kw, true, g.py.tw);
  }
  cluster.sync();

  // ---- phase B: rows of this rank, R at a time
  const int q = tid / P, p = tid % P;
  const float inv_nv = (float)(1.0 / (double)nv);
  float shift[6];
  if constexpr (MODE == 0) {
    const double* e = eps_bar + 6 * b;
    const double tr = e[0] + e[1] + e[2];
    const Medium& md = med[b / g.lame_group];
#pragma unroll
    for (int c = 0; c < 6; ++c) shift[c] = (float)((c < 3 ? md.lmean * tr : 0.0) + 2.0 * md.mmean * e[c]);
    if (x == 0 && rank == 0 && tid == 0) {
#pragma unroll
      for (int c = 0; c < 6; ++c) st[b].shift[c] = (double)shift[c];
    }
  } else {
#pragma unroll
    for (int c = 0; c < 6; ++c) shift[c] = (float)st[b].shift[c];
  }
  const float* lam = lambda + (size_t)(b / g.lame_group) * nv;
  const float* muf = mu + (size_t)(b / g.lame_group) * nv;
  int slot = 0;
  __half* rb = nullptr;
  float* gb = nullptr;
  float rscale = 1.f;
  if constexpr (MODE == 3) {
    const int M1 = aa.depth + 1;
    slot = (st[b].iter - 1 - st[b].aa_base) % M1;
    rb = aa.r + (size_t)b * M1 * 6 * nv + (size_t)slot * 6 * nv;
    gb = aa.g + (size_t)b * M1 * 6 * nv + (size_t)slot * 6 * nv;
    const int kexp = ring_exponent(st[b].ring_max, eps_bar + 6 * b);
    rscale = ldexpf(1.f, kexp);
    if (rank == 0 && x == 0 && tid == 0) st[b].ring_exp[slot] = kexp;
  }
  // owner rank and local column of half-spectrum column k
  auto owner = [&](int k) { return k < NF * kTW ? k / kTW : CS - 1; };
  auto local = [&](int k) { return k < NF * kTW ? k % kTW : kTW; };
  for (int y0 = rank * ROWS; y0 < (rank + 1) * ROWS; y0 += R) {
    if constexpr (kInverse) {
      // gather (conj of the Hermitian extension of A + i B, as the z pass)
      for (int idx = tid; idx < 3 * R * NZH; idx += nt) {
        const int pr = idx / (R * NZH), rem = idx % (R * NZH);
        const int l = rem / NZH, k = rem % NZH;
        const float2* src = cluster.map_shared_rank(cols, (unsigned)owner(k));
        float2 A = src[((size_t)(2 * pr) * NY + y0 + l) * kSlabKW + local(k)];
        float2 B = src[((size_t)(2 * pr + 1) * NY + y0 + l) * kSlabKW + local(k)];
        const bool selfconj = (k == 0) || (2 * k == NZ);
        if (selfconj) { A.y = 0.f; B.y = 0.f; }
        float2* Z = zbuf + (size_t)(pr * R + l) * LD;
        Z[k] = make_float2(A.x - B.y, -(A.y + B.x));
        if (!selfconj) Z[NZ - k] = make_float2(A.x + B.y, A.y - B.x);
      }
      __syncthreads();
      zline_fft<NZ>(zbuf, q, p, g.pz.tw);
    }
    // pointwise stage of the mode
    for (int idx = tid; idx < R * NZ; idx += nt) {
      const int l = idx / NZ, n = idx % NZ;
      const size_t vx = ((size_t)x * NY + y0 + l) * NZ + n;
      float e[6];
      if constexpr (MODE == 3) {
#pragma unroll
        for (int pr = 0; pr < 3; ++pr) {
          const float2 w = zbuf[(size_t)(pr * R + l) * LD + n];
          const float r0 = w.x * inv_nv, r1 = -w.y * inv_nv;
          const size_t o0 = (size_t)(2 * pr) * nv + vx, o1 = (size_t)(2 * pr + 1) * nv + vx;
          rb[o0] = ring_store(r0, rscale);
          rb[o1] = ring_store(r1, rscale);
          gb[o0] = eb[o0] + r0;
          gb[o1] = eb[o1] + r1;
        }
        continue;
      } else {
        if constexpr (MODE == 1) {
#pragma unroll
          for (int pr = 0; pr < 3; ++pr) {
            const float2 w = zbuf[(size_t)(pr * R + l) * LD + n];
            e[2 * pr] = eb[(size_t)(2 * pr) * nv + vx] + w.x * inv_nv;
            e[2 * pr + 1] = eb[(size_t)(2 * pr + 1) * nv + vx] - w.y * inv_nv;
          }
        } else if constexpr (MODE == 2) {
#pragma unroll
          for (int c = 0; c < 6; ++c) e[c] = eb[(size_t)c * nv + vx];
        } else {
          if (eps0 != nullptr) {
#pragma unroll
            for (int c = 0; c < 6; ++c) e[c] = eps0[((size_t)b * 6 + c) * nv + vx];
          } else {
#pragma unroll
            for (int c = 0; c < 6; ++c) e[c] = (float)eps_bar[b * 6 + c];
          }
        }
        if constexpr (MODE != 2) {
#pragma unroll
          for (int c = 0; c < 6; ++c) eb[(size_t)c * nv + vx] = e[c];
        }
        const float lmv = lam[vx], tmu = 2.f * muf[vx];
        const float ltr = lmv * (e[0] + e[1] + e[2]);
        float sg[6];
#pragma unroll
        for (int c = 0; c < 3; ++c) sg[c] = tmu * e[c] + ltr;
#pragma unroll
        for (int c = 3; c < 6; ++c) sg[c] = tmu * e[c];
        // (the inverse transform's line is fully read above by this same thread before
        // being overwritten: both index the line by (pr, l, n) of this idx)
#pragma unroll
        for (int pr = 0; pr < 3; ++pr)
          zbuf[(size_t)(pr * R + l) * LD + n] =
              make_float2(sg[2 * pr] - shift[2 * pr], sg[2 * pr + 1] - shift[2 * pr + 1]);
      }
    }
    __syncthreads();
    if constexpr (kForward) {
      zline_fft<NZ>(zbuf, q, p, g.pz.tw);
      // scatter the two half spectra of every line back to the owners' columns
      for (int idx = tid; idx < 3 * R * NZH; idx += nt) {
        const int pr = idx / (R * NZH), rem = idx % (R * NZH);
        const int l = rem / NZH, k = rem % NZH;
        const float2* Z = zbuf + (size_t)(pr * R + l) * LD;
        const float2 zk = Z[k];
        const float2 zm = Z[k == 0 ? 0 : NZ - k];
        float2* dst = cluster.map_shared_rank(cols, (unsigned)owner(k));
        dst[((size_t)(2 * pr) * NY + y0 + l) * kSlabKW + local(k)] =
            make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        dst[((size_t)(2 * pr + 1) * NY + y0 + l) * kSlabKW + local(k)] =
            make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
      }
      __syncthreads();
    }
  }
  cluster.sync();
  if constexpr (!kForward) return;  // (after the barrier: no rank still reads this one's columns)

  // ---- phase C: forward y DFT of the rank's columns, store
  slab_ydft<NY>(cols, kw, false, g.py.tw);
  for (int i = tid; i < 6 * NY * (kTW / 2); i += nt) {
    const int c = i / (NY * (kTW / 2)), rem = i % (NY * (kTW / 2));
    const int ky = rem / (kTW / 2), h = rem % (kTW / 2);
    const float2* sv = cols + ((size_t)c * NY + ky) * kSlabKW + 2 * h;
    *reinterpret_cast<float4*>(tb + (size_t)c * g.nm + ((size_t)(rank * NY + ky) * nx + x) * kTW + 2 * h) =
        make_float4(sv[0].x, sv[0].y, sv[1].x, sv[1].y);
  }
  if (rank == CS - 1) {
    for (int i = tid; i < 6 * NY; i += nt) {
      const int c = i / NY, ky = i % NY;
      tb[(size_t)c * g.nm + tail0 + ((size_t)(ky / kTW) * nx + x) * kTW + (ky % kTW)] =
          cols[((size_t)c * NY + ky) * kSlabKW + kTW];
    }
  }
}

// ----------------------------------------------------------------------------- host side
static bool pow2_supported(int n) {
  return n == 16 || n == 32 || n == 48 || n == 64 || n == 96 || n == 128 || n == 256;
}

bool supported(const GridDesc& g) {
  return pow2_supported(g.nx) && pow2_supported(g.ny) && pow2_supported(g.nz);
}

template <int N>
static int x_blocks(const GridDesc& g, int v) {
  const int t = v ? x_cols_v<N, 1>() : x_cols_v<N, 0>();
  return (g.nzh + t - 1) / t;
}

int x_tiles(const GridDesc& g, int variant) {
  switch (g.nx) {
    case 16: return x_blocks<16>(g, variant);
    case 32: return x_blocks<32>(g, variant);
    case 48: return x_blocks<48>(g, variant);
    case 96: return x_blocks<96>(g, variant);
    case 64: return x_blocks<64>(g, variant);
    case 128: return x_blocks<128>(g, variant);
    default: return x_blocks<256>(g, variant);
  }
}

// (power-of-two ny only: at ny = 48 and 96 the tiled y pass measured 2-4x slower than the
// in-place one, 0.50 against 0.11 ms at 48^3 x 96 instances)
bool tiled_supported(const GridDesc& g) {
  const bool ypow2 = (g.ny & (g.ny - 1)) == 0;
  return supported(g) && g.nx <= 128 && ypow2 && g.ny % kTW == 0 && (g.nzh - 1) % kTW == 0;
}

int x_tiles_tiled(const GridDesc& g) { return g.ny * ((g.nzh - 1) / kTW) + g.ny / kTW; }

bool slab_supported(const GridDesc& g) {
  const int n = g.nz;
  return tiled_supported(g) && g.ny == n && n <= 128;
}

template <int N>
static size_t slab_smem() { return slab_layout<N, N>().total; }

template <int N, int MODE>
static cudaError_t slab_launch_n(const GridDesc& g, int batch, const float* lambda, const float* mu,
                                 float* eps, float2* tspec, const double* eps_bar, const float* eps0,
                                 InstanceState* st, const Medium* med, const AndersonArgs<float>& aa,
                                 cudaStream_t s) {
  constexpr int CS = slab_ranks<N>();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(CS, g.nx, batch);
  cfg.blockDim = dim3(slab_threads<N>());
  cfg.dynamicSmemBytes = slab_smem<N>();
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CS;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, slab_fast<N, N, MODE>, g, lambda, mu, eps, tspec, eps_bar, eps0, st,
                            med, aa);
}

template <int N>
static cudaError_t slab_launch_m(const GridDesc& g, int mode, int batch, const float* lambda,
                                 const float* mu, float* eps, float2* tspec, const double* eps_bar,
                                 const float* eps0, InstanceState* st, const Medium* med,
                                 const AndersonArgs<float>& aa, cudaStream_t s) {
  switch (mode) {
    case 0: return slab_launch_n<N, 0>(g, batch, lambda, mu, eps, tspec, eps_bar, eps0, st, med, aa, s);
    case 1: return slab_launch_n<N, 1>(g, batch, lambda, mu, eps, tspec, eps_bar, eps0, st, med, aa, s);
    case 2: return slab_launch_n<N, 2>(g, batch, lambda, mu, eps, tspec, eps_bar, eps0, st, med, aa, s);
    default: return slab_launch_n<N, 3>(g, batch, lambda, mu, eps, tspec, eps_bar, eps0, st, med, aa, s);
  }
}

cudaError_t launch_slab(const GridDesc& g, int mode, int batch, const float* lambda, const float* mu,
                        float* eps, float2* tspec, const double* eps_bar, const float* eps0,
                        InstanceState* st, const Medium* med, const AndersonArgs<float>& aa,
                        cudaStream_t s) {
  switch (g.nz) {
    case 16: return slab_launch_m<16>(g, mode, batch, lambda, mu, eps, tspec, eps_bar, eps0, st, med, aa, s);
    case 32: return slab_launch_m<32>(g, mode, batch, lambda, mu, eps, tspec, eps_bar, eps0, st, med, aa, s);
    case 48: return slab_launch_m<48>(g, mode, batch, lambda, mu, eps, tspec, eps_bar, eps0, st, med, aa, s);
    case 64: return slab_launch_m<64>(g, mode, batch, lambda, mu, eps, tspec, eps_bar, eps0, st, med, aa, s);
    case 96: return slab_launch_m<96>(g, mode, batch, lambda, mu, eps, tspec, eps_bar, eps0, st, med, aa, s);
    default: return slab_launch_m<128>(g, mode, batch, lambda, mu, eps, tspec, eps_bar, eps0, st, med, aa, s);
  }
}

size_t tile_index(const GridDesc& g, int x, int ky, int kz) {
  return tile_offset(g.nx, g.ny, (g.nzh - 1) / kTW, x, ky, kz);
}

template <int N>
static size_t xtsmem() { return (size_t)6 * x_region<N, kTW, XTSplit<N>>() * sizeof(float2); }

template <int N, int MODE = -1>
static size_t zsmem() { return z_layout<N, MODE>().total; }
template <int N>
static int z_blocks_for(const GridDesc& g) {
  return (int)(((long long)g.nx * g.ny + z_lines<N>() - 1) / z_lines<N>());
}
template <int N, int V>
static size_t xsmem() {
  return (size_t)6 * x_region<N, x_cols_v<N, V>()>() * sizeof(float2);
}

template <int N>
static cudaError_t configure_n() {
  const int zs = (int)zsmem<N>();
  cudaError_t e = cudaFuncSetAttribute(zpass_fast<N, 1, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, zs);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(zpass_fast<N, 2, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, zs);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(zpass_fast<N, 0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem<N, 0>());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(zpass_fast<N, 0, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem<N, 1>());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(zpass_fast<N, 0, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem<N, 2>());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(zpass_fast<N, 0, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem<N, 3>());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(xpass_fast<N, 0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xsmem<N, 0>());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(xpass_fast<N, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xsmem<N, 1>());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(xpass_fast<N, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xsmem<N, 0>());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(xpass_fast<N, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xsmem<N, 1>());
  if constexpr (N <= 128) {
    const int ss = (int)slab_smem<N>();
    if (e == cudaSuccess) e = cudaFuncSetAttribute(slab_fast<N, N, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(slab_fast<N, N, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(slab_fast<N, N, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(slab_fast<N, N, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(xpass_tiled<N, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xtsmem<N>());
    if (e == cudaSuccess) e = cudaFuncSetAttribute(xpass_tiled<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)xtsmem<N>());
  }
  return e;
}

cudaError_t configure() {
  cudaError_t e;
  if ((e = configure_n<16>()) != cudaSuccess) return e;
  if ((e = configure_n<32>()) != cudaSuccess) return e;
  if ((e = configure_n<48>()) != cudaSuccess) return e;
  if ((e = configure_n<64>()) != cudaSuccess) return e;
  if ((e = configure_n<96>()) != cudaSuccess) return e;
  if ((e = configure_n<128>()) != cudaSuccess) return e;
  return configure_n<256>();
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

template <int N>
static void zlaunch(const GridDesc& g, int mode, int batch, const float* lambda, const float* mu,
                    float* eps, float2* spec, const double* eps_bar, const float* eps0,
                    InstanceState* st, const Medium* med, const AndersonArgs<float>& aa, cudaStream_t s) {
  dim3 grid((unsigned)z_blocks_for<N>(g), batch);
  // every chunk offset is a multiple of 16 bytes when the base pointers are
  const int bulk = aligned16(lambda) && aligned16(mu) && aligned16(eps) && aligned16(spec) ? 1 : 0;
  if (g.cf32) {
    zpass_fast<N, 2, -1><<<grid, z_threads<N>(), zsmem<N>(), s>>>(g, mode, bulk, lambda, mu, eps, spec,
                                                                 eps_bar, eps0, st, med, aa);
    return;
  }
  if (g.dmg32) {
    zpass_fast<N, 1, -1><<<grid, z_threads<N>(), zsmem<N>(), s>>>(g, mode, bulk, lambda, mu, eps, spec,
                                                                 eps_bar, eps0, st, med, aa);
    return;
  }
  switch (mode) {
    case 0:
      zpass_fast<N, 0, 0><<<grid, z_threads<N>(), zsmem<N, 0>(), s>>>(g, mode, bulk, lambda, mu, eps, spec,
                                                                     eps_bar, eps0, st, med, aa);
      break;
    case 1:
      zpass_fast<N, 0, 1><<<grid, z_threads<N>(), zsmem<N, 1>(), s>>>(g, mode, bulk, lambda, mu, eps, spec,
                                                                     eps_bar, eps0, st, med, aa);
      break;
    case 2:
      zpass_fast<N, 0, 2><<<grid, z_threads<N>(), zsmem<N, 2>(), s>>>(g, mode, bulk, lambda, mu, eps, spec,
                                                                     eps_bar, eps0, st, med, aa);
      break;
    default:
      zpass_fast<N, 0, 3><<<grid, z_threads<N>(), zsmem<N, 3>(), s>>>(g, mode, bulk, lambda, mu, eps, spec,
                                                                     eps_bar, eps0, st, med, aa);
      break;
  }
}

void launch_zpass(const GridDesc& g, int mode, int batch, const float* lambda, const float* mu,
                  float* eps, float2* spec, const double* eps_bar, const float* eps0,
                  InstanceState* st, const Medium* med, const AndersonArgs<float>& aa, cudaStream_t s) {
  switch (g.nz) {
    case 16: zlaunch<16>(g, mode, batch, lambda, mu, eps, spec, eps_bar, eps0, st, med, aa, s); break;
    case 32: zlaunch<32>(g, mode, batch, lambda, mu, eps, spec, eps_bar, eps0, st, med, aa, s); break;
    case 48: zlaunch<48>(g, mode, batch, lambda, mu, eps, spec, eps_bar, eps0, st, med, aa, s); break;
    case 96: zlaunch<96>(g, mode, batch, lambda, mu, eps, spec, eps_bar, eps0, st, med, aa, s); break;
    case 64: zlaunch<64>(g, mode, batch, lambda, mu, eps, spec, eps_bar, eps0, st, med, aa, s); break;
    case 128: zlaunch<128>(g, mode, batch, lambda, mu, eps, spec, eps_bar, eps0, st, med, aa, s); break;
    default: zlaunch<256>(g, mode, batch, lambda, mu, eps, spec, eps_bar, eps0, st, med, aa, s); break;
  }
}

template <int N>
static int z_blocks_n(const GridDesc& g) { return z_blocks_for<N>(g); }

int z_blocks(const GridDesc& g) {
  switch (g.nz) {
    case 16: return z_blocks_n<16>(g);
    case 32: return z_blocks_n<32>(g);
    case 48: return z_blocks_n<48>(g);
    case 96: return z_blocks_n<96>(g);
    case 64: return z_blocks_n<64>(g);
    case 128: return z_blocks_n<128>(g);
    default: return z_blocks_n<256>(g);
  }
}

template <int N, int YV>
static void ylaunch_v(const GridDesc& g, bool inverse, int batch, float2* spec, float2* tspec,
                      const InstanceState* st, cudaStream_t s) {
  // with a one-column tail, full tiles + one tail tile (see ypass_fast)
  constexpr int YT = y_cols<N, YV>();
  dim3 grid(g.nzh % YT == 1 ? g.nzh / YT + 1 : (g.nzh + YT - 1) / YT, g.nx, 6 * batch);
  if (tspec)
    ypass_fast<N, true, YV><<<dim3(grid.y, grid.x, grid.z), y_threads<N, YV>(), 0, s>>>(
        g, inverse ? 1 : 0, spec, tspec, st);
  else
    ypass_fast<N, false, YV><<<grid, y_threads<N, YV>(), 0, s>>>(g, inverse ? 1 : 0, spec, spec, st);
}

template <int N>
static void ylaunch(int variant, const GridDesc& g, bool inverse, int batch, float2* spec, float2* tspec,
                    const InstanceState* st, cudaStream_t s) {
  if (variant) ylaunch_v<N, 1>(g, inverse, batch, spec, tspec, st, s);
  else ylaunch_v<N, 0>(g, inverse, batch, spec, tspec, st, s);
}

void launch_ypass(const GridDesc& g, int variant, bool inverse, int batch, float2* spec, float2* tspec,
                  const InstanceState* st, cudaStream_t s) {
  switch (g.ny) {
    case 16: ylaunch<16>(variant, g, inverse, batch, spec, tspec, st, s); break;
    case 32: ylaunch<32>(variant, g, inverse, batch, spec, tspec, st, s); break;
    case 48: ylaunch<48>(variant, g, inverse, batch, spec, tspec, st, s); break;
    case 96: ylaunch<96>(variant, g, inverse, batch, spec, tspec, st, s); break;
    case 64: ylaunch<64>(variant, g, inverse, batch, spec, tspec, st, s); break;
    case 128: ylaunch<128>(variant, g, inverse, batch, spec, tspec, st, s); break;
    default: ylaunch<256>(variant, g, inverse, batch, spec, tspec, st, s); break;
  }
}

template <int N, int V>
static void xlaunch(const GridDesc& g, int batch, float2* spec, const Medium* med, InstanceState* st,
                    double* partials, cudaStream_t s) {
  dim3 grid(x_blocks<N>(g, V), g.ny, batch);
  const int threads = 6 * XSplit<N>::P * x_cols_v<N, V>();
  if (g.c0)
    xpass_fast<N, V, true><<<grid, threads, xsmem<N, V>(), s>>>(g, spec, med, st, partials);
  else
    xpass_fast<N, V, false><<<grid, threads, xsmem<N, V>(), s>>>(g, spec, med, st, partials);
}

template <int N>
static void xlaunch_v(int variant, const GridDesc& g, int batch, float2* spec, const Medium* med,
                      InstanceState* st, double* partials, cudaStream_t s) {
  if (variant) xlaunch<N, 1>(g, batch, spec, med, st, partials, s);
  else xlaunch<N, 0>(g, batch, spec, med, st, partials, s);
}

template <int N>
static void xtlaunch(const GridDesc& g, int batch, float2* tspec, const Medium* med, InstanceState* st,
                     double* partials, cudaStream_t s) {
  if constexpr (N <= 128) {
    dim3 grid((unsigned)x_tiles_tiled(g), batch);
    if (g.c0)
      xpass_tiled<N, true><<<grid, xt_threads<N>(), xtsmem<N>(), s>>>(g, tspec, med, st, partials);
    else
      xpass_tiled<N, false><<<grid, xt_threads<N>(), xtsmem<N>(), s>>>(g, tspec, med, st, partials);
  }
}

void launch_xpass_tiled(const GridDesc& g, int batch, float2* tspec, const Medium* med,
                        InstanceState* st, double* partials, cudaStream_t s) {
  switch (g.nx) {
    case 16: xtlaunch<16>(g, batch, tspec, med, st, partials, s); break;
    case 32: xtlaunch<32>(g, batch, tspec, med, st, partials, s); break;
    case 48: xtlaunch<48>(g, batch, tspec, med, st, partials, s); break;
    case 96: xtlaunch<96>(g, batch, tspec, med, st, partials, s); break;
    case 64: xtlaunch<64>(g, batch, tspec, med, st, partials, s); break;
    default: xtlaunch<128>(g, batch, tspec, med, st, partials, s); break;
  }
}

void launch_xpass(const GridDesc& g, int variant, int batch, float2* spec, const Medium* med,
                  InstanceState* st, double* partials, cudaStream_t s) {
  switch (g.nx) {
    case 16: xlaunch_v<16>(variant, g, batch, spec, med, st, partials, s); break;
    case 32: xlaunch_v<32>(variant, g, batch, spec, med, st, partials, s); break;
    case 48: xlaunch_v<48>(variant, g, batch, spec, med, st, partials, s); break;
    case 96: xlaunch_v<96>(variant, g, batch, spec, med, st, partials, s); break;
    case 64: xlaunch_v<64>(variant, g, batch, spec, med, st, partials, s); break;
    case 128: xlaunch_v<128>(variant, g, batch, spec, med, st, partials, s); break;
    default: xlaunch_v<256>(variant, g, batch, spec, med, st, partials, s); break;
  }
}

}  // namespace fast
}  // namespace lsb
