// Stand-alone CIC paint / readout / neighbour kernels (the operators of
// flowpm/utils.py:32-91 cic_paint and :163-210 cic_readout) and their C ABI.
#include "fpm_internal.cuh"

namespace fpm {

// mesh[b] += sum_c w_c * weight at the 8 neighbours of each particle.
// One thread per particle, FP32 reductions to global memory.
__global__ void __launch_bounds__(kThreads)
k_cic_paint(float* __restrict__ mesh, int nx, int ny, int nz,
            const float* __restrict__ part, int64_t npart, int64_t total,
            const float* __restrict__ weight) {
  const int64_t ncell = (int64_t)nx * ny * nz;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = g / npart;
    const float x = part[3 * g + 0], y = part[3 * g + 1], z = part[3 * g + 2];
    const float wt = weight ? weight[g] : 1.0f;
    Axis ax = cic_axis(x, nx), ay = cic_axis(y, ny), az = cic_axis(z, nz);
    float* m = mesh + b * ncell;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int cx = conn_x(c), cy = conn_y(c), cz = conn_z(c);
      float w = cic_w(ax, ay, az, cx, cy, cz);
      if (weight) w = __fmul_rn(wt, w);
      const int ix = cx ? ax.i1 : ax.i0, iy = cy ? ay.i1 : ay.i0,
                iz = cz ? az.i1 : az.i0;
      red_add(m + ((int64_t)ix * ny + iy) * nz + iz, w);
    }
  }
}

__global__ void __launch_bounds__(kThreads)
k_cic_readout(const float* __restrict__ mesh, int nx, int ny, int nz,
              const float* __restrict__ part, int64_t npart, int64_t total,
              float* __restrict__ out) {
  const int64_t ncell = (int64_t)nx * ny * nz;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = g / npart;
    const float x = part[3 * g + 0], y = part[3 * g + 1], z = part[3 * g + 2];
    Axis ax = cic_axis(x, nx), ay = cic_axis(y, ny), az = cic_axis(z, nz);
    const float* m = mesh + b * ncell;
    float acc = 0.0f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int cx = conn_x(c), cy = conn_y(c), cz = conn_z(c);
      const float w = cic_w(ax, ay, az, cx, cy, cz);
      const int ix = cx ? ax.i1 : ax.i0, iy = cy ? ay.i1 : ay.i0,
                iz = cz ? az.i1 : az.i0;
      acc = __fadd_rn(acc,
                      __fmul_rn(__ldg(m + ((int64_t)ix * ny + iy) * nz + iz),
                                w));
    }
    out[g] = acc;
  }
}

__global__ void __launch_bounds__(kThreads)
k_cic_neighbours(int nx, int ny, int nz, const float* __restrict__ part,
                 int64_t n, int32_t* __restrict__ idx, float* __restrict__ w) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n;
       g += (int64_t)gridDim.x * blockDim.x) {
    const float x = part[3 * g + 0], y = part[3 * g + 1], z = part[3 * g + 2];
    Axis ax = cic_axis(x, nx), ay = cic_axis(y, ny), az = cic_axis(z, nz);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int cx = conn_x(c), cy = conn_y(c), cz = conn_z(c);
      const int ix = cx ? ax.i1 : ax.i0, iy = cy ? ay.i1 : ay.i0,
                iz = cz ? az.i1 : az.i0;
      idx[8 * g + c] = (ix * ny + iy) * nz + iz;
      w[8 * g + c] = cic_w(ax, ay, az, cx, cy, cz);
    }
  }
}

static unsigned grid_elems(int64_t n) {
  int64_t blocks = (n + kThreads - 1) / kThreads;
  const int64_t cap = (int64_t)kNumSMs * 32;
  if (blocks < 1) blocks = 1;
  return (unsigned)(blocks < cap ? blocks : cap);
}

static bool bad_dims(int batch, int nx, int ny, int nz) {
  return batch < 1 || nx < 1 || ny < 1 || nz < 1 ||
         (int64_t)nx * ny * nz > (int64_t)1 << 31;
}

}  // namespace fpm

using namespace fpm;

extern "C" int fpm_cic_paint(float* mesh, int batch, int nx, int ny, int nz,
                             const float* part, int64_t npart,
                             const float* weight, void* stream) {
  if (!mesh || (!part && npart > 0) || npart < 0 || bad_dims(batch, nx, ny, nz))
    return FPM_ERR_ARG;
  const int64_t total = (int64_t)batch * npart;
  if (total == 0) return FPM_OK;
  k_cic_paint<<<grid_elems(total), kThreads, 0, (cudaStream_t)stream>>>(
      mesh, nx, ny, nz, part, npart, total, weight);
  return cudaGetLastError() == cudaSuccess ? FPM_OK : FPM_ERR_CUDA;
}

extern "C" int fpm_cic_readout(const float* mesh, int batch, int nx, int ny,
                               int nz, const float* part, int64_t npart,
                               float* out, void* stream) {
  if (!mesh || ((!part || !out) && npart > 0) || npart < 0 ||
      bad_dims(batch, nx, ny, nz))
    return FPM_ERR_ARG;
  const int64_t total = (int64_t)batch * npart;
  if (total == 0) return FPM_OK;
  k_cic_readout<<<grid_elems(total), kThreads, 0, (cudaStream_t)stream>>>(
      mesh, nx, ny, nz, part, npart, total, out);
  return cudaGetLastError() == cudaSuccess ? FPM_OK : FPM_ERR_CUDA;
}

extern "C" int fpm_cic_neighbours(int nx, int ny, int nz, const float* part,
                                  int64_t npart, int32_t* idx, float* w,
                                  void* stream) {
  if (npart < 0 || bad_dims(1, nx, ny, nz) ||
      (npart > 0 && (!part || !idx || !w)))
    return FPM_ERR_ARG;
  if (npart == 0) return FPM_OK;
  k_cic_neighbours<<<grid_elems(npart), kThreads, 0, (cudaStream_t)stream>>>(
      nx, ny, nz, part, npart, idx, w);
  return cudaGetLastError() == cudaSuccess ? FPM_OK : FPM_ERR_CUDA;
}

namespace fpm {

__global__ void __launch_bounds__(kThreads)
k_lattice_shift(const float* __restrict__ in, float* __restrict__ out,
                int64_t np, int64_t total, int ny, int nz, float sign) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t local = g % np;
    const int64_t t = local / nz;
    const int k = (int)(local - t * nz);
    const int i = (int)(t / ny);
    const int j = (int)(t - (int64_t)i * ny);
    out[3 * g + 0] = __fadd_rn(in[3 * g + 0], sign * (float)i);
    out[3 * g + 1] = __fadd_rn(in[3 * g + 1], sign * (float)j);
    out[3 * g + 2] = __fadd_rn(in[3 * g + 2], sign * (float)k);
  }
}

__global__ void __launch_bounds__(kThreads)
k_saxpy(float* __restrict__ y, const float* __restrict__ x, float a,
        int64_t n) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n;
       g += (int64_t)gridDim.x * blockDim.x)
    y[g] = __fadd_rn(y[g], __fmul_rn(a, x[g]));
}

}  // namespace fpm

extern "C" int fpm_lattice_shift(const float* in, float* out, int batch,
                                 int nx, int ny, int nz, int sign,
                                 void* stream) {
  if (!in || !out || bad_dims(batch, nx, ny, nz) || (sign != 1 && sign != -1))
    return FPM_ERR_ARG;
  const int64_t np = (int64_t)nx * ny * nz;
  const int64_t total = (int64_t)batch * np;
  k_lattice_shift<<<grid_elems(total), kThreads, 0, (cudaStream_t)stream>>>(
      in, out, np, total, ny, nz, (float)sign);
  return cudaGetLastError() == cudaSuccess ? FPM_OK : FPM_ERR_CUDA;
}

extern "C" int fpm_saxpy(float* y, const float* x, float a, int64_t n,
                         void* stream) {
  if (n < 0 || (n > 0 && (!x || !y))) return FPM_ERR_ARG;
  if (n == 0) return FPM_OK;
  k_saxpy<<<grid_elems(n), kThreads, 0, (cudaStream_t)stream>>>(y, x, a, n);
  return cudaGetLastError() == cudaSuccess ? FPM_OK : FPM_ERR_CUDA;
}
