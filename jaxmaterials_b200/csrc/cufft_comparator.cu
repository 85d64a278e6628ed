// The plain Moulinec-Suquet iteration with its three-dimensional transforms on cuFFT, as a
// comparator for the hand-written passes of liblippmannschwinger.so.
//
// Per iteration, as the reference's CUDA loop (cuda/src/lippmann_schwinger.cu:192-216):
//   stress kernel          sigma = lambda tr(eps) I + 2 mu eps           (eps, lambda, mu -> sigma)
//   cufftExecR2C           batch 6 per instance, [nx][ny][nz] -> [nx][ny][nz/2+1]
//   gamma kernel           FP64 criterion partials, r_hat = -Gamma^0 sigma_hat in place
//   cufftExecC2R           batch 6 per instance, back to [nx][ny][nz]
//   update kernel          eps += r / N
// The pointwise kernels are this file's own (coalesced, one thread per voxel or mode);
// only the transforms are the library's. The criterion, Gamma^0 and the modified wave
// vectors are the solver's (FP64 wave vectors with the 1e-12 guard of
// src/jaxmaterials/solver/fourier.py:84). No mean-stress shift and no stop decision: the
// comparator runs a fixed number of iterations, which is what it times.
//
// Not part of the solver: bench.py loads it to time the library transforms beside the
// hand-written ones on the same workload.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include <cufft.h>

#include "ls_types.cuh"

namespace {

thread_local std::string g_err;

int fail(int code, const char* msg) {
  g_err = msg;
  return code;
}

struct Handle {
  int nx, ny, nz, nzh, batch;
  long long nv, nm;
  double Lx, Ly, Lz;
  cufftHandle fwd = 0, inv = 0;
  float* sigma = nullptr;   // [batch][6][nv] stress, then the residual field r
  float2* spec = nullptr;   // [batch][6][nm]
  double* tab = nullptr;    // sin/cos(pi k / n) per axis: sx cx sy cy sz cz
  double* num = nullptr;    // [batch] criterion numerator of the last iteration
  double* zero = nullptr;   // [batch][12] zero mode of sigma_hat of the last iteration
  cudaStream_t stream = nullptr;
  ~Handle() {
    if (fwd) cufftDestroy(fwd);
    if (inv) cufftDestroy(inv);
    cudaFree(sigma);
    cudaFree(spec);
    cudaFree(tab);
    cudaFree(num);
    cudaFree(zero);
    if (stream) cudaStreamDestroy(stream);
  }
};

__global__ void stress_kernel(long long nv, int lame_group, const float* __restrict__ lam,
                              const float* __restrict__ mu, const float* __restrict__ eps,
                              float* __restrict__ sig) {
  const int b = blockIdx.y;
  const long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const float* e = eps + (size_t)b * 6 * nv + v;
  float* s = sig + (size_t)b * 6 * nv + v;
  const float l = lam[(size_t)(b / lame_group) * nv + v], tm = 2.f * mu[(size_t)(b / lame_group) * nv + v];
  float ev[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) ev[c] = e[(size_t)c * nv];
  const float ltr = l * (ev[0] + ev[1] + ev[2]);
#pragma unroll
  for (int c = 0; c < 6; ++c) s[(size_t)c * nv] = tm * ev[c] + (c < 3 ? ltr : 0.f);
}

// One thread per half-spectrum mode of one instance: the weighted |xi~ . sigma_hat|^2
// (block sums into num[b] by one FP64 atomic per block) and r_hat = -Gamma^0 sigma_hat.
__global__ void gamma_kernel(int nx, int ny, int nz, int nzh, long long nm, double fx, double fy,
                             double fz, const double* __restrict__ tab, float c_a, float c_b,
                             float2* __restrict__ spec, double* __restrict__ num,
                             double* __restrict__ zero) {
  __shared__ double red[32];
  const int b = blockIdx.y;
  const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double acc = 0.0;
  if (m < nm) {
    const int kz = (int)(m % nzh);
    const long long rest = m / nzh;
    const int ky = (int)(rest % ny), kx = (int)(rest / ny);
    const double* sx = tab;
    const double* cx = sx + nx;
    const double* sy = cx + nx;
    const double* cy = sy + ny;
    const double* sz = cy + ny;
    const double* cz = sz + nzh;
    const double x0 = fx * sx[kx] * cy[ky] * cz[kz];
    const double x1 = fy * cx[kx] * sy[ky] * cz[kz];
    const double x2 = fz * cx[kx] * cy[ky] * sz[kz];
    float2* sp = spec + (size_t)b * 6 * nm + m;
    float2 s[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) s[c] = sp[(size_t)c * nm];
    if (m == 0) {
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        zero[b * 12 + 2 * c] = s[c].x;
        zero[b * 12 + 2 * c + 1] = s[c].y;
      }
    }
    const float f0 = (float)x0, f1 = (float)x1, f2 = (float)x2;
    const float2 d0 = make_float2(f0 * s[0].x + f1 * s[3].x + f2 * s[4].x, f0 * s[0].y + f1 * s[3].y + f2 * s[4].y);
    const float2 d1 = make_float2(f0 * s[3].x + f1 * s[1].x + f2 * s[5].x, f0 * s[3].y + f1 * s[1].y + f2 * s[5].y);
    const float2 d2 = make_float2(f0 * s[4].x + f1 * s[5].x + f2 * s[2].x, f0 * s[4].y + f1 * s[5].y + f2 * s[2].y);
    const double m2 = (double)d0.x * d0.x + (double)d0.y * d0.y + (double)d1.x * d1.x +
                      (double)d1.y * d1.y + (double)d2.x * d2.x + (double)d2.y * d2.y;
    acc = ((kz == 0 || 2 * kz == nz) ? 1.0 : 2.0) * m2;
    const double n2 = x0 * x0 + x1 * x1 + x2 * x2;
    const double inv = n2 < 1.0e-24 ? 1.0 : rsqrt(n2);
    const float z0 = (float)(x0 * inv), z1 = (float)(x1 * inv), z2 = (float)(x2 * inv);
    const float z00 = z0 * z0, z11 = z1 * z1, z22 = z2 * z2;
    const float z01 = z0 * z1, z02 = z0 * z2, z12 = z1 * z2;
    float r[2][6];
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      const float t0 = part ? s[0].y : s[0].x, t1 = part ? s[1].y : s[1].x, t2 = part ? s[2].y : s[2].x;
      const float t3 = part ? s[3].y : s[3].x, t4 = part ? s[4].y : s[4].x, t5 = part ? s[5].y : s[5].x;
      const float rho = z00 * t0 + z11 * t1 + z22 * t2 + 2.f * (z01 * t3 + z02 * t4 + z12 * t5);
      const float a0 = z0 * (z0 * t0 + z2 * t4 + z1 * t3);
      const float a1 = z1 * (z1 * t1 + z2 * t5 + z0 * t3);
      const float a2 = z2 * (z2 * t2 + z1 * t5 + z0 * t4);
      const float a3 = 0.5f * (z01 * (t0 + t1) + (z00 + z11) * t3 + z2 * (z0 * t5 + z1 * t4));
      const float a4 = 0.5f * (z02 * (t0 + t2) + (z00 + z22) * t4 + z1 * (z0 * t5 + z2 * t3));
      const float a5 = 0.5f * (z12 * (t1 + t2) + (z11 + z22) * t5 + z0 * (z1 * t4 + z2 * t3));
      r[part][0] = c_a * a0 + c_b * rho * z00;
      r[part][1] = c_a * a1 + c_b * rho * z11;
      r[part][2] = c_a * a2 + c_b * rho * z22;
      r[part][3] = c_a * a3 + c_b * rho * z01;
      r[part][4] = c_a * a4 + c_b * rho * z02;
      r[part][5] = c_a * a5 + c_b * rho * z12;
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) sp[(size_t)c * nm] = make_float2(r[0][c], r[1][c]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) t += red[w];
    atomicAdd(num + b, t);
  }
}

__global__ void update_kernel(long long n6, float inv_nv, const float* __restrict__ r,
                              float* __restrict__ eps) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n6) eps[i] += r[i] * inv_nv;
}

__global__ void fill_kernel(long long nv, const double* __restrict__ eps_bar, float* __restrict__ eps) {
  const int b = blockIdx.y;
  const long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (v >= nv) return;
#pragma unroll
  for (int c = 0; c < 6; ++c) eps[((size_t)b * 6 + c) * nv + v] = (float)eps_bar[b * 6 + c];
}

}  // namespace

extern "C" {

const char* cmp_cufft_last_error(void) { return g_err.c_str(); }

// Plans the batch-6-per-instance R2C / C2R transforms of `batch` instances on an n^3 grid
// and allocates the comparator's work buffers.
int cmp_cufft_create(void** out, const int voxels[3], const double extents[3], int batch) {
  if (!out || !voxels || !extents || batch < 1) return fail(-1, "bad argument");
  auto* h = new Handle();
  h->nx = voxels[0];
  h->ny = voxels[1];
  h->nz = voxels[2];
  h->nzh = h->nz / 2 + 1;
  h->batch = batch;
  h->nv = (long long)h->nx * h->ny * h->nz;
  h->nm = (long long)h->nx * h->ny * h->nzh;
  h->Lx = extents[0];
  h->Ly = extents[1];
  h->Lz = extents[2];
  int n[3] = {h->nx, h->ny, h->nz};
  int nc[3] = {h->nx, h->ny, h->nzh};
  bool ok = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&h->sigma, sizeof(float) * 6 * batch * h->nv) == cudaSuccess &&
            cudaMalloc(&h->spec, sizeof(float2) * 6 * batch * h->nm) == cudaSuccess &&
            cudaMalloc(&h->tab, sizeof(double) * 2 * (h->nx + h->ny + h->nzh)) == cudaSuccess &&
            cudaMalloc(&h->num, sizeof(double) * batch) == cudaSuccess &&
            cudaMalloc(&h->zero, sizeof(double) * 12 * batch) == cudaSuccess;
  ok = ok && cufftPlanMany(&h->fwd, 3, n, n, 1, (int)h->nv, nc, 1, (int)h->nm, CUFFT_R2C, 6 * batch) == CUFFT_SUCCESS &&
       cufftPlanMany(&h->inv, 3, n, nc, 1, (int)h->nm, n, 1, (int)h->nv, CUFFT_C2R, 6 * batch) == CUFFT_SUCCESS &&
       cufftSetStream(h->fwd, h->stream) == CUFFT_SUCCESS && cufftSetStream(h->inv, h->stream) == CUFFT_SUCCESS;
  if (!ok) {
    delete h;
    return fail(-2, "allocation or cuFFT plan failed");
  }
  std::vector<double> tab;
  auto add = [&](int nn, int count) {
    for (int k = 0; k < count; ++k) tab.push_back(std::sin(M_PI * k / nn));
    for (int k = 0; k < count; ++k) tab.push_back(std::cos(M_PI * k / nn));
  };
  add(h->nx, h->nx);
  add(h->ny, h->ny);
  add(h->nz, h->nzh);
  if (cudaMemcpy(h->tab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    delete h;
    return fail(-2, "table upload failed");
  }
  *out = h;
  return 0;
}

void cmp_cufft_destroy(void* handle) { delete static_cast<Handle*>(handle); }

// Runs `iters` plain iterations from eps = eps_bar for every instance (instance b uses the
// Lame fields of structure b / lame_group, device [structures][nv]; eps_bar host
// double[batch*6]; lambda0, mu0 the reference medium). Writes device d_eps
// [batch][6][nv], the mean time per iteration (CUDA events on the comparator's stream),
// the last iteration's relative criterion per instance and its mean stress (host
// double[batch], double[batch*6]).
int cmp_cufft_run(void* handle, const float* d_lambda, const float* d_mu, int lame_group,
                  const double* eps_bar, double lambda0, double mu0, float* d_eps, int iters,
                  float* ms_per_iter, double* criterion, double* mean_sigma) {
  auto* h = static_cast<Handle*>(handle);
  if (!h || !d_lambda || !d_mu || !eps_bar || !d_eps || iters < 1 || lame_group < 1 ||
      h->batch % lame_group != 0)
    return fail(-1, "bad argument");
  const int B = h->batch;
  double* d_eb = nullptr;
  if (cudaMalloc(&d_eb, sizeof(double) * 6 * B) != cudaSuccess) return fail(-2, "allocation failed");
  cudaMemcpy(d_eb, eps_bar, sizeof(double) * 6 * B, cudaMemcpyHostToDevice);
  const dim3 gv((unsigned)((h->nv + 255) / 256), B), gm((unsigned)((h->nm + 255) / 256), B);
  const long long n6 = 6LL * B * h->nv;
  const float c_a = (float)(-1.0 / mu0), c_b = (float)((lambda0 + mu0) / (mu0 * (lambda0 + 2.0 * mu0)));
  const float inv_nv = (float)(1.0 / (double)h->nv);
  cudaStream_t st = h->stream;
  fill_kernel<<<gv, 256, 0, st>>>(h->nv, d_eb, d_eps);
  auto iteration = [&]() -> bool {
    cudaMemsetAsync(h->num, 0, sizeof(double) * B, st);
    stress_kernel<<<gv, 256, 0, st>>>(h->nv, lame_group, d_lambda, d_mu, d_eps, h->sigma);
    if (cufftExecR2C(h->fwd, h->sigma, reinterpret_cast<cufftComplex*>(h->spec)) != CUFFT_SUCCESS) return false;
    gamma_kernel<<<gm, 256, 0, st>>>(h->nx, h->ny, h->nz, h->nzh, h->nm, 2.0 * h->nx / h->Lx,
                                     2.0 * h->ny / h->Ly, 2.0 * h->nz / h->Lz, h->tab, c_a, c_b,
                                     h->spec, h->num, h->zero);
    if (cufftExecC2R(h->inv, reinterpret_cast<cufftComplex*>(h->spec), h->sigma) != CUFFT_SUCCESS) return false;
    update_kernel<<<(unsigned)((n6 + 255) / 256), 256, 0, st>>>(n6, inv_nv, h->sigma, d_eps);
    return true;
  };
  // first iteration: e0 (criterion of eps_bar) for the relative criterion
  if (!iteration()) {
    cudaFree(d_eb);
    return fail(-2, "cuFFT execution failed");
  }
  std::vector<double> num0(B), zero0(12 * B);
  cudaMemcpyAsync(num0.data(), h->num, sizeof(double) * B, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(zero0.data(), h->zero, sizeof(double) * 12 * B, cudaMemcpyDeviceToHost, st);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  bool ok = true;
  for (int i = 1; i < iters && ok; ++i) ok = iteration();
  cudaEventRecord(e1, st);
  std::vector<double> num(B), zero(12 * B);
  cudaMemcpyAsync(num.data(), h->num, sizeof(double) * B, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(zero.data(), h->zero, sizeof(double) * 12 * B, cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  float ms = 0.f;
  if (e == cudaSuccess && iters > 1) e = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_eb);
  if (!ok) return fail(-2, "cuFFT execution failed");
  if (e != cudaSuccess) return fail(-2, cudaGetErrorString(e));
  if (ms_per_iter) *ms_per_iter = iters > 1 ? ms / (float)(iters - 1) : 0.f;
  auto crit = [&](const std::vector<double>& nu, const std::vector<double>& z, int b) {
    double den = 0.0;
    for (int c = 0; c < 6; ++c)
      den += (c < 3 ? 1.0 : 2.0) * (z[12 * b + 2 * c] * z[12 * b + 2 * c] + z[12 * b + 2 * c + 1] * z[12 * b + 2 * c + 1]);
    return den > 0.0 ? std::sqrt(nu[b]) / std::sqrt(den) : 0.0;
  };
  for (int b = 0; b < B; ++b) {
    if (criterion) {
      const double c0 = crit(num0, zero0, b);
      criterion[b] = c0 > 0.0 ? crit(num, zero, b) / c0 : 0.0;
    }
    if (mean_sigma)
      for (int c = 0; c < 6; ++c) mean_sigma[6 * b + c] = zero[12 * b + 2 * c] / (double)h->nv;
  }
  return 0;
}

}  // extern "C"
