// 2-D CIC paint and lensing density planes (flowpm/utils.py:94-160
// cic_paint_2d, flowpm/raytracing.py:49-109 density_plane) and their
// adjoints, as single passes over the particles.
//
// cic_paint_2d: neighbours floor + {0,1}^2, weight (1 - |x - n|)(1 - |y - n|)
// times the particle weight, indices cast to int and taken modulo ny on
// both axes (the reference's nc = ny).  When nx < ny an x index can land at
// nx or beyond; such a deposit is dropped (the reference's scatter would
// fail there) and counted in the status word.
//
// density_plane: positions rotated (R x), shifted (+ nc * shift), xy taken
// modulo nx (both components, as the reference), rescaled by res / nx;
// particles with lo < z <= hi painted into the plane; each plane is then
// divided by (nx / res) (ny / res) width.  One launch serves up to
// kMaxPlanes planes (a particle may fall into several).
#include <atomic>

#include "fpm_kernels.cuh"

namespace fpm {

namespace {

#define FPM_PLANES_TRY(x) \
  do {                    \
    const int rc_ = (x);  \
    if (rc_) return rc_;  \
  } while (0)

constexpr int kMaxPlanes = 64;

struct PlaneParams {
  float rot[9];  // row-major, applied as R x
  float shift[3];  // already times (nx, ny, nz)
  int use_rot, use_shift;
  int nplanes, res;
  float lo[kMaxPlanes], hi[kMaxPlanes];
  float norm[kMaxPlanes];  // (nx / res) (ny / res) width
  float scale;  // res / nx
  float fnx;    // nx as float (modulus of xy)
};

// Floor-mod of the reference (tf.math.mod on floats): the sign of y.
__device__ __forceinline__ float floor_mod(float x, float y) {
  float r = fmodf(x, y);
  if (r != 0.f && ((r < 0.f) != (y < 0.f))) r += y;
  return r;
}

struct Cic2 {
  int ix[2], iy[2];
  float wx[2], wy[2];
  float gx[2], gy[2];  // d w / d x per neighbour (-sign, sign(0) = 0)
};

__device__ __forceinline__ Cic2 cic2(float x, float y, int ny) {
  Cic2 c;
  const float fx = floorf(x), fy = floorf(y);
  const float nx1 = __fadd_rn(fx, 1.f), ny1 = __fadd_rn(fy, 1.f);
  c.wx[0] = __fsub_rn(1.f, fabsf(__fsub_rn(x, fx)));
  c.wx[1] = __fsub_rn(1.f, fabsf(__fsub_rn(x, nx1)));
  c.wy[0] = __fsub_rn(1.f, fabsf(__fsub_rn(y, fy)));
  c.wy[1] = __fsub_rn(1.f, fabsf(__fsub_rn(y, ny1)));
  c.gx[0] = (x - fx > 0.f) ? -1.f : 0.f;
  c.gx[1] = 1.f;
  c.gy[0] = (y - fy > 0.f) ? -1.f : 0.f;
  c.gy[1] = 1.f;
  const int ax = __float2int_rz(fx), ay = __float2int_rz(fy);
  c.ix[0] = wrap_index(ax, ny);
  c.ix[1] = wrap_index(ax + 1, ny);
  c.iy[0] = wrap_index(ay, ny);
  c.iy[1] = wrap_index(ay + 1, ny);
  return c;
}

// Neighbour order of flowpm/utils.py:133: (0,0) (1,0) (0,1) (1,1).
__device__ __forceinline__ int c2x(int c) { return c & 1; }
__device__ __forceinline__ int c2y(int c) { return c >> 1; }

__global__ void __launch_bounds__(kThreads)
k_cic_paint_2d(float* __restrict__ mesh, int B, int nx, int ny,
               const float* __restrict__ part, int64_t np,
               const float* __restrict__ weight,
               const uint8_t* __restrict__ mask, int32_t* dropped) {
  const int64_t n = (int64_t)B * np;
  for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * kThreads) {
    if (mask && !mask[e]) continue;
    const int64_t b = e / np;
    const Cic2 c = cic2(part[2 * e], part[2 * e + 1], ny);
    const float pw = weight ? weight[e] : 1.f;
    float* m = mesh + b * nx * ny;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int ix = c.ix[c2x(q)], iy = c.iy[c2y(q)];
      float w = __fmul_rn(c.wx[c2x(q)], c.wy[c2y(q)]);
      if (weight) w = __fmul_rn(pw, w);
      if (ix >= nx) {
        atomicAdd(dropped, 1);
        continue;
      }
      red_add(m + (int64_t)ix * ny + iy, w);
    }
  }
}

// Adjoint of k_cic_paint_2d for the cotangent g of the mesh: d part and
// d weight (either may be null).
__global__ void __launch_bounds__(kThreads)
k_cic_paint_2d_adjoint(const float* __restrict__ g, int B, int nx, int ny,
                       const float* __restrict__ part, int64_t np,
                       const float* __restrict__ weight,
                       const uint8_t* __restrict__ mask,
                       float* __restrict__ gpart, float* __restrict__ gweight) {
  const int64_t n = (int64_t)B * np;
  for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * kThreads) {
    float dx = 0.f, dy = 0.f, dw = 0.f;
    if (!mask || mask[e]) {
      const int64_t b = e / np;
      const Cic2 c = cic2(part[2 * e], part[2 * e + 1], ny);
      const float pw = weight ? weight[e] : 1.f;
      const float* m = g + b * nx * ny;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int ix = c.ix[c2x(q)], iy = c.iy[c2y(q)];
        if (ix >= nx) continue;
        const float v = m[(int64_t)ix * ny + iy];
        const float wx = c.wx[c2x(q)], wy = c.wy[c2y(q)];
        dw += v * (wx * wy);
        dx += v * pw * (c.gx[c2x(q)] * wy);
        dy += v * pw * (wx * c.gy[c2y(q)]);
      }
    }
    if (gpart) {
      gpart[2 * e] = dx;
      gpart[2 * e + 1] = dy;
    }
    if (gweight) gweight[e] = dw;
  }
}

// Transformed position of particle e: plane coordinates (u, v) and depth d.
__device__ __forceinline__ void plane_coords(const PlaneParams& P,
                                             const float* X, int64_t e,
                                             float& u, float& v, float& d) {
  float x = X[3 * e], y = X[3 * e + 1], z = X[3 * e + 2];
  if (P.use_rot) {
    const float rx = P.rot[0] * x + P.rot[1] * y + P.rot[2] * z;
    const float ry = P.rot[3] * x + P.rot[4] * y + P.rot[5] * z;
    const float rz = P.rot[6] * x + P.rot[7] * y + P.rot[8] * z;
    x = rx;
    y = ry;
    z = rz;
  }
  if (P.use_shift) {
    x = __fadd_rn(x, P.shift[0]);
    y = __fadd_rn(y, P.shift[1]);
    z = __fadd_rn(z, P.shift[2]);
  }
  // xy = mod(xy, nx); xy = xy / nx * res
  u = __fmul_rn(__fdiv_rn(floor_mod(x, P.fnx), P.fnx), (float)P.res);
  v = __fmul_rn(__fdiv_rn(floor_mod(y, P.fnx), P.fnx), (float)P.res);
  d = z;
}

__global__ void __launch_bounds__(kThreads)
k_density_planes(const float* __restrict__ X, int B, int64_t np,
                 PlaneParams P, float* __restrict__ planes,
                 int32_t* dropped) {
  const int64_t n = (int64_t)B * np;
  const int64_t psz = (int64_t)P.res * P.res;
  for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * kThreads) {
    float u, v, d;
    plane_coords(P, X, e, u, v, d);
    const int64_t b = e / np;
    bool any = false;
    for (int p = 0; p < P.nplanes; ++p) any |= (d > P.lo[p] && d <= P.hi[p]);
    if (!any) continue;
    const Cic2 c = cic2(u, v, P.res);
    for (int p = 0; p < P.nplanes; ++p) {
      if (!(d > P.lo[p] && d <= P.hi[p])) continue;
      float* m = planes + (b * P.nplanes + p) * psz;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int ix = c.ix[c2x(q)], iy = c.iy[c2y(q)];
        if (ix >= P.res) {
          atomicAdd(dropped, 1);
          continue;
        }
        red_add(m + (int64_t)ix * P.res + iy,
                __fmul_rn(c.wx[c2x(q)], c.wy[c2y(q)]));
      }
    }
  }
}

// planes[b, p] /= norm[p]
__global__ void __launch_bounds__(kThreads)
k_scale_planes(float* __restrict__ planes, int B, int64_t psz,
               PlaneParams P) {
  const int64_t n = (int64_t)B * P.nplanes * psz;
  for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * kThreads) {
    const int p = (int)((e / psz) % P.nplanes);
    planes[e] = __fdiv_rn(planes[e], P.norm[p]);
  }
}

// dX of the density planes for their cotangent g: dX = R^T (res / nx)
// (du, dv, 0) for the particles inside a slab (the mod and the slab test
// have unit or zero derivative), du, dv the paint adjoint of g / norm.
__global__ void __launch_bounds__(kThreads)
k_density_planes_adjoint(const float* __restrict__ X, int B, int64_t np,
                         PlaneParams P, const float* __restrict__ g,
                         float* __restrict__ gX) {
  const int64_t n = (int64_t)B * np;
  const int64_t psz = (int64_t)P.res * P.res;
  for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * kThreads) {
    float u, v, d;
    plane_coords(P, X, e, u, v, d);
    const int64_t b = e / np;
    float du = 0.f, dv = 0.f;
    const Cic2 c = cic2(u, v, P.res);
    for (int p = 0; p < P.nplanes; ++p) {
      if (!(d > P.lo[p] && d <= P.hi[p])) continue;
      const float* m = g + (b * P.nplanes + p) * psz;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int ix = c.ix[c2x(q)], iy = c.iy[c2y(q)];
        if (ix >= P.res) continue;
        const float val = __fdiv_rn(m[(int64_t)ix * P.res + iy], P.norm[p]);
        du += val * (c.gx[c2x(q)] * c.wy[c2y(q)]);
        dv += val * (c.wx[c2x(q)] * c.gy[c2y(q)]);
      }
    }
    du *= P.scale;
    dv *= P.scale;
    float gx = du, gy = dv, gz = 0.f;
    if (P.use_rot) {  // R^T (du, dv, 0)
      gx = P.rot[0] * du + P.rot[3] * dv;
      gy = P.rot[1] * du + P.rot[4] * dv;
      gz = P.rot[2] * du + P.rot[5] * dv;
    }
    gX[3 * e] = gx;
    gX[3 * e + 1] = gy;
    gX[3 * e + 2] = gz;
  }
}

unsigned grid_elems(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  const int64_t cap = (int64_t)kNumSMs * 32;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

int make_params(int nx, int ny, int nz, const double* rotation,
                const double* shift, int nplanes, const double* centers,
                const double* widths, int res, PlaneParams& P) {
  if (nx < 1 || ny < 1 || nz < 1 || res < 1 || nplanes < 1 ||
      nplanes > kMaxPlanes || !centers || !widths)
    return FPM_ERR_ARG;
  P.use_rot = rotation ? 1 : 0;
  P.use_shift = shift ? 1 : 0;
  for (int i = 0; i < 9; ++i) P.rot[i] = rotation ? (float)rotation[i] : 0.f;
  const double n3[3] = {(double)nx, (double)ny, (double)nz};
  // [nx, ny, nz] * shift is a double product in the reference (NumPy),
  // added to the float32 positions after rounding
  for (int i = 0; i < 3; ++i)
    P.shift[i] = shift ? (float)(n3[i] * shift[i]) : 0.f;
  P.nplanes = nplanes;
  P.res = res;
  for (int p = 0; p < nplanes; ++p) {
    P.lo[p] = (float)(centers[p] - widths[p] / 2);
    P.hi[p] = (float)(centers[p] + widths[p] / 2);
    P.norm[p] = (float)((double)nx / res * ((double)ny / res) * widths[p]);
  }
  P.scale = (float)res / (float)nx;
  P.fnx = (float)nx;
  return FPM_OK;
}

// Device counter of dropped deposits (stream-ordered allocation).
int dropped_alloc(int32_t** d, cudaStream_t st) {
  void* p = nullptr;
  if (cudaMallocAsync(&p, sizeof(int32_t), st) != cudaSuccess) {
    cudaGetLastError();
    return FPM_ERR_OOM;
  }
  *d = (int32_t*)p;
  if (cudaMemsetAsync(p, 0, sizeof(int32_t), st) != cudaSuccess) {
    cudaGetLastError();
    cudaFreeAsync(p, st);
    return FPM_ERR_CUDA;
  }
  return FPM_OK;
}

int finish(int32_t* dropped, cudaStream_t st) {
  int32_t h = 0;
  if (cudaMemcpyAsync(&h, dropped, sizeof(h), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    cudaGetLastError();
    cudaFreeAsync(dropped, st);
    return FPM_ERR_CUDA;
  }
  cudaFreeAsync(dropped, st);
  return h ? FPM_ERR_RANGE : FPM_OK;
}

}  // namespace

}  // namespace fpm

using namespace fpm;

extern "C" int fpm_cic_paint_2d(float* mesh, int batch, int nx, int ny,
                                const float* part, int64_t npart,
                                const float* weight, const uint8_t* mask,
                                void* stream) {
  if (!mesh || batch < 1 || nx < 1 || ny < 1 || npart < 0 ||
      (npart > 0 && !part))
    return FPM_ERR_ARG;
  if (npart == 0) return FPM_OK;
  cudaStream_t st = (cudaStream_t)stream;
  int32_t* dropped = nullptr;
  FPM_PLANES_TRY(dropped_alloc(&dropped, st));
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_cic_paint_2d<<<grid_elems((int64_t)batch * npart), kThreads, 0, st>>>(
      mesh, batch, nx, ny, part, npart, weight, mask, dropped);
  if (cudaGetLastError() != cudaSuccess) return FPM_ERR_CUDA;
  return finish(dropped, st);
}

extern "C" int fpm_cic_paint_2d_adjoint(const float* grad_mesh, int batch,
                                        int nx, int ny, const float* part,
                                        int64_t npart, const float* weight,
                                        const uint8_t* mask, float* grad_part,
                                        float* grad_weight, void* stream) {
  if (!grad_mesh || batch < 1 || nx < 1 || ny < 1 || npart < 0 ||
      (npart > 0 && !part))
    return FPM_ERR_ARG;
  if (npart == 0 || (!grad_part && !grad_weight)) return FPM_OK;
  cudaStream_t st = (cudaStream_t)stream;
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_cic_paint_2d_adjoint<<<grid_elems((int64_t)batch * npart), kThreads, 0,
                           st>>>(grad_mesh, batch, nx, ny, part, npart, weight,
                                 mask, grad_part, grad_weight);
  return cudaGetLastError() == cudaSuccess ? FPM_OK : FPM_ERR_CUDA;
}

extern "C" int fpm_density_planes(const float* X, int batch, int64_t npart,
                                  int nx, int ny, int nz,
                                  const double* rotation, const double* shift,
                                  int nplanes, const double* centers,
                                  const double* widths, int res,
                                  float* planes, void* stream) {
  if (!X || !planes || batch < 1 || npart < 0) return FPM_ERR_ARG;
  PlaneParams P;
  FPM_PLANES_TRY(make_params(nx, ny, nz, rotation, shift, nplanes, centers, widths,
                      res, P));
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t psz = (int64_t)res * res;
  if (cudaMemsetAsync(planes, 0, sizeof(float) * batch * nplanes * psz, st) !=
      cudaSuccess) {
    cudaGetLastError();
    return FPM_ERR_CUDA;
  }
  int32_t* dropped = nullptr;
  FPM_PLANES_TRY(dropped_alloc(&dropped, st));
  g_launches.fetch_add(2, std::memory_order_relaxed);
  if (npart > 0)
    k_density_planes<<<grid_elems((int64_t)batch * npart), kThreads, 0, st>>>(
        X, batch, npart, P, planes, dropped);
  k_scale_planes<<<grid_elems((int64_t)batch * nplanes * psz), kThreads, 0,
                   st>>>(planes, batch, psz, P);
  if (cudaGetLastError() != cudaSuccess) return FPM_ERR_CUDA;
  return finish(dropped, st);
}

extern "C" int fpm_density_planes_adjoint(
    const float* X, int batch, int64_t npart, int nx, int ny, int nz,
    const double* rotation, const double* shift, int nplanes,
    const double* centers, const double* widths, int res,
    const float* grad_planes, float* grad_X, void* stream) {
  if (!X || !grad_planes || !grad_X || batch < 1 || npart < 0)
    return FPM_ERR_ARG;
  PlaneParams P;
  FPM_PLANES_TRY(make_params(nx, ny, nz, rotation, shift, nplanes, centers, widths,
                      res, P));
  if (npart == 0) return FPM_OK;
  cudaStream_t st = (cudaStream_t)stream;
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_density_planes_adjoint<<<grid_elems((int64_t)batch * npart), kThreads, 0,
                             st>>>(X, batch, npart, P, grad_planes, grad_X);
  return cudaGetLastError() == cudaSuccess ? FPM_OK : FPM_ERR_CUDA;
}
