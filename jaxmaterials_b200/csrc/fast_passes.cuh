// FP32 passes with compile-time power-of-two lengths (implemented in fast_passes.cu).
#pragma once

#include "ls_types.cuh"

namespace lsb {
namespace fast {

// True when every extent is one of 16, 32, 48, 64, 96, 128, 256.
bool supported(const GridDesc& g);
// x-pass blocks per (ky) row for tile variant 0 or 1: the number of kz tiles.
int x_tiles(const GridDesc& g, int variant);
cudaError_t configure();
// z-pass blocks per instance (number of Gram-row partials in the Anderson residual mode).
int z_blocks(const GridDesc& g);
void launch_zpass(const GridDesc& g, int mode, int batch, const float* lambda, const float* mu,
                  float* eps, float2* spec, const double* eps_bar, const float* eps0,
                  InstanceState* st, const Medium* med, const AndersonArgs<float>& aa, cudaStream_t s);
// tspec != nullptr: the x-pass side is the tiled layout in tspec (the forward pass writes
// it, the inverse pass reads it); otherwise the transform runs in place on spec. variant:
// kz columns per block (0: 8 at 128, 16 elsewhere; 1: the other of 8 and 16).
void launch_ypass(const GridDesc& g, int variant, bool inverse, int batch, float2* spec, float2* tspec,
                  const InstanceState* st, cudaStream_t s);
// The tiled spectrum layout between the y and x passes applies (nx <= 128, ny and nz/2 a
// multiple of 8, every extent supported).
bool tiled_supported(const GridDesc& g);
// x-pass blocks per instance over the tiled layout (every tile one block).
int x_tiles_tiled(const GridDesc& g);
// Offset of mode (x, ky, kz) of one component in the tiled layout.
size_t tile_index(const GridDesc& g, int x, int ky, int kz);
void launch_xpass_tiled(const GridDesc& g, int batch, float2* tspec, const Medium* med,
                        InstanceState* st, double* partials, cudaStream_t s);
// The fused slab pass applies (tiled layout, ny == nz <= 128).
bool slab_supported(const GridDesc& g);
// Inverse y, z pass of `mode` (0 init, 1 plain update, 2 stress of eps, 3 Anderson residual
// rings) and forward y (modes 0-2) of every x-plane, over the tiled layout in tspec; one
// thread-block cluster per plane and instance. Isotropic law only.
cudaError_t launch_slab(const GridDesc& g, int mode, int batch, const float* lambda, const float* mu,
                        float* eps, float2* tspec, const double* eps_bar, const float* eps0,
                        InstanceState* st, const Medium* med, const AndersonArgs<float>& aa,
                        cudaStream_t s);
void launch_xpass(const GridDesc& g, int variant, int batch, float2* spec, const Medium* med,
                  InstanceState* st, double* partials, cudaStream_t s);

}  // namespace fast
}  // namespace lsb
