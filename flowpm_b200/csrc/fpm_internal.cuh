// Internal definitions shared by the flowpm_b200 CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/flowpm_b200.h"

namespace fpm {

constexpr int kThreads = 256;    // threads per block of the streaming kernels
constexpr int kItems = 4;        // particles (or cells) per thread per chunk
constexpr int kChunk = kThreads * kItems;
constexpr int kNumSMs = 148;     // B200

// One simulation of a plan, as the device kernels see it.
struct SimDev {
  int nx, ny, nz;        // particle lattice (= linear-field mesh)
  int bf;                // force mesh factor
  int mx, my, mz, mzh;   // force mesh and its half-spectrum z extent
  int lzh;               // lattice half-spectrum z extent
  int tab;               // offset of this sim's force-mesh axis tables
  int ltab;              // offset of this sim's lattice axis tables
  int pad_;
  int64_t np;            // particles
  int64_t p_off;         // first particle
  int64_t m_off;         // first force-mesh cell
  int64_t s_off;         // first force-mesh half-spectrum mode
  int64_t l_off;         // first lattice cell
  int64_t ls_off;        // first lattice half-spectrum mode
  int64_t ch_p;          // first particle chunk
  int64_t ch_s;          // first force-spectrum chunk
  int64_t ch_m;          // first force-mesh chunk
  int64_t ch_l;          // first lattice-cell chunk
  int64_t ch_ls;         // first lattice-spectrum chunk
};

// Per-axis Fourier tables.  For an axis of n cells and index i,
// k = 2*pi*fftfreq(i, n) (flowpm/kernels.py:10-25):
//   kk  = k^2 (double), grad = (8 sin k - sin 2k)/6 (kernels.py:72-76) or
//   k with the Nyquist entry zeroed (order 0, kernels.py:66-70),
//   win = sinc(k / 2pi)^-2 (kernels.py:137-152).
struct AxisTabs {
  const double* kk;
  const float* grad;
  const float* win;
};

enum ChunkKind { kPart = 0, kSpec = 1, kMesh = 2, kLat = 3, kLatSpec = 4 };

__device__ __forceinline__ int64_t chunk_first(const SimDev& s, int kind) {
  switch (kind) {
    case kPart: return s.ch_p;
    case kSpec: return s.ch_s;
    case kMesh: return s.ch_m;
    case kLat: return s.ch_l;
    default: return s.ch_ls;
  }
}

// Simulation owning chunk c (binary search over the sims' first chunks).
__device__ __forceinline__ int find_sim(const SimDev* sims, int nsims,
                                        int64_t c, int kind) {
  int lo = 0, hi = nsims - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (chunk_first(sims[mid], kind) <= c) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int wrap_index(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

// CIC neighbours along one axis with the reference arithmetic
// (flowpm/utils.py:63-81): floor, neighbour = floor + {0, 1} (float),
// weight = 1 - |x - neighbour|, cell = int(neighbour) mod n.  A NaN or
// infinite x still yields in-range cells (cvt saturates, NaN -> 0).
struct Axis {
  int i0, i1;
  float w0, w1;
};

__device__ __forceinline__ Axis cic_axis(float x, int n) {
  Axis a;
  float f = floorf(x);
  float f1 = __fadd_rn(f, 1.0f);
  a.w0 = __fsub_rn(1.0f, fabsf(__fsub_rn(x, f)));
  a.w1 = __fsub_rn(1.0f, fabsf(__fsub_rn(x, f1)));
  int c = __float2int_rz(f);
  a.i0 = wrap_index(c, n);
  a.i1 = (a.i0 + 1 == n) ? 0 : a.i0 + 1;
  return a;
}

// Weight of neighbour (cx, cy, cz): (wx * wy) * wz, as the reference's
// kernel[..., 0] * kernel[..., 1] * kernel[..., 2].
__device__ __forceinline__ float cic_w(const Axis& ax, const Axis& ay,
                                       const Axis& az, int cx, int cy,
                                       int cz) {
  float wx = cx ? ax.w1 : ax.w0;
  float wy = cy ? ay.w1 : ay.w0;
  float wz = cz ? az.w1 : az.w0;
  return __fmul_rn(__fmul_rn(wx, wy), wz);
}

// Neighbour order of flowpm/utils.py:66-67:
// (0,0,0) (1,0,0) (0,1,0) (0,0,1) (1,1,0) (1,0,1) (0,1,1) (1,1,1).
__host__ __device__ __forceinline__ int conn_x(int c) {
  return (c == 1 || c == 4 || c == 5 || c == 7) ? 1 : 0;
}
__host__ __device__ __forceinline__ int conn_y(int c) {
  return (c == 2 || c == 4 || c == 6 || c == 7) ? 1 : 0;
}
__host__ __device__ __forceinline__ int conn_z(int c) {
  return (c == 3 || c == 5 || c == 6 || c == 7) ? 1 : 0;
}

__device__ __forceinline__ void red_add(float* p, float v) {
  asm volatile("red.global.add.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

__device__ __forceinline__ bool finite3(float a, float b, float c) {
  return isfinite(a) && isfinite(b) && isfinite(c);
}

inline unsigned grid_for(int64_t chunks) {
  int64_t g = chunks < 1 ? 1 : chunks;
  const int64_t cap = (int64_t)kNumSMs * 16;
  return (unsigned)(g < cap ? g : cap);
}

}  // namespace fpm
