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

// Lattice blocks of the particle kernels: (kPlanes wi) x kBJ x kBK
// particles, z fastest, wi (SimDev::wi) particles per thread, chosen per
// simulation; one pass of the block's threads covers kPlanes x planes.
// Measured on B200 with kBJ = 4 / 8 / 16 at equal particles per block:
// k_step at 2 x 512^3 8.92 / 8.70 / 8.68 ms, at 128^3 88.1 / 84.7 / 84.0
// us; k_adj_position 15.4 / 15.8 / 16.7 ms.
#ifndef FPM_BJ
#define FPM_BJ 8
#endif
constexpr int kBJ = FPM_BJ, kBK = 16;
constexpr int kPlanes = kThreads / (kBJ * kBK);
static_assert(kPlanes * kBJ * kBK == kThreads, "whole x planes per pass");

// One simulation of a plan, as the device kernels see it.

struct SimDev {
  int nx, ny, nz;        // particle lattice (= linear-field mesh)
  int bf;                // force mesh factor
  int mx, my, mz, mzh;   // force mesh and its half-spectrum z extent
  int lzh;               // lattice half-spectrum z extent
  int tab;               // offset of this sim's force-mesh axis tables
  int ltab;              // offset of this sim's lattice axis tables
  int fused;             // force meshes by the fused Fourier solve
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
  int64_t ch_b;          // first lattice-block chunk
  int nbi, nbj, nbk;     // lattice blocks per axis
  int wi;                // particles per thread of a lattice block, whose
                         // x extent is kPlanes wi
  int xpass;             // cuFFT plane transforms + the x-pass kernel
  // Eulerian cell tiles of the binned step (fpm_plan_set_binning): tiles of
  // T^3 force-mesh cells, ntx x nty x ntz of them, the first one at ch_t in
  // the plan's tile enumeration
  int ntx, nty, ntz;
  int64_t ch_t;
  // bit widths of the lattice site (i, j, k) packed into the carried
  // index of the binned order: k in the low qkb bits, j in the next qjb
  int qkb, qjb;
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

// Transfer function of the potential, common to the three force
// components (evaluated per mode; s = the mode's simulation):
// * force (pgd null): the Green's function 1/k^2 rounded to float (0 at
//   k = 0, where the gradient vanishes anyway), times the optional
//   Gaussian long-range split exp(-k^2 r2) and CIC deconvolution
//   (flowpm/tfpm.py:199-215, kernels.py:28-48, :81-102, :137-152);
// * PGD (pgd set): the same 1/k^2 times the PGD kernel
//   exp(-kl^2 / k^2) exp(-k^4 / ks^4) in float32 (flowpm/tfpm.py:222-270,
//   kernels.py:105-134), (kl, ks) = pgd[(s * pgd_stride + pos) * 3 + 1, 2].
struct Green {
  double r2;
  int deconv;
  int pgd_stride;
  const float* pgd;
  int pos;
};

__host__ __device__ inline Green force_green(double r2, int deconv) {
  Green g;
  g.r2 = r2;
  g.deconv = deconv;
  g.pgd_stride = 0;
  g.pgd = nullptr;
  g.pos = 0;
  return g;
}

__device__ __forceinline__ float green_w(const Green& G, int s, double kk,
                                         float wx, float wy, float wz) {
  if (kk == 0.0) return 0.f;
  float w = (float)(1.0 / kk);
  if (G.pgd) {
    const float* q = G.pgd + ((int64_t)s * G.pgd_stride + G.pos) * 3;
    const float kkf = (float)kk, kl = q[1], ks = q[2];
    const float kl2 = kl * kl, ks4 = (ks * ks) * (ks * ks);
    const float v = expf(-kl2 / kkf) * expf(-(kkf * kkf) / ks4);
    return __fmul_rn(w, v);
  }
  if (G.r2 != 0.0) w = __fmul_rn(w, (float)exp(-kk * G.r2));
  if (G.deconv) w = __fmul_rn(w, __fmul_rn(__fmul_rn(wx, wy), wz));
  return w;
}

enum ChunkKind {
  kPart = 0, kSpec = 1, kMesh = 2, kLat = 3, kLatSpec = 4, kBlock = 5,
  kTile = 6
};

__device__ __forceinline__ int64_t chunk_first(const SimDev& s, int kind) {
  switch (kind) {
    case kPart: return s.ch_p;
    case kSpec: return s.ch_s;
    case kMesh: return s.ch_m;
    case kLat: return s.ch_l;
    case kBlock: return s.ch_b;
    case kTile: return s.ch_t;
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

// The particle kernels are bound by the SM's conversion / special-function
// pipe when floor, float <-> int conversion and integer modulo go through
// it, so the common cases below stay on the FP32 and integer pipes.
//
// floor(x) as a float and as an int for |x| < 2^22: adding 1.5 * 2^23
// rounds x to the nearest integer, held exactly in the low mantissa bits
// (the sum lies in [2^23, 2^24), where the float spacing is 1); the
// difference back is exact, and one compare turns round-to-nearest into
// floor.  Returns false (NaN, |x| >= 2^22) when the caller must take the
// general path.
constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;

__device__ __forceinline__ bool floor_small(float x, float& f, int& c) {
  if (!(fabsf(x) < 4194304.0f)) return false;
  const float r = __fadd_rn(x, kMagic);
  int ci = __float_as_int(r) - kMagicBits;
  float rf = __fsub_rn(r, kMagic);
  if (rf > x) {
    rf = __fsub_rn(rf, 1.0f);
    ci -= 1;
  }
  f = rf;
  c = ci;
  return true;
}

// (float)i, exact, for 0 <= i < 2^22 (lattice and mesh indices).
__device__ __forceinline__ float index_float(int i) {
  return __fsub_rn(__int_as_float(kMagicBits + i), kMagic);
}

// c mod n in [0, n): one conditional add or subtract for |c| < 2n (every
// particle within one box length of the mesh), the full modulo otherwise.
__device__ __forceinline__ int wrap_near(int c, int n) {
  if (c < 0) c += n;
  else if (c >= n) c -= n;
  if ((unsigned)c >= (unsigned)n) c = wrap_index(c, n);
  return c;
}

__device__ __forceinline__ Axis cic_axis(float x, int n) {
  Axis a;
  float f;
  int c;
  if (!floor_small(x, f, c)) {
    f = floorf(x);
    c = __float2int_rz(f);
  }
  float f1 = __fadd_rn(f, 1.0f);
  a.w0 = __fsub_rn(1.0f, fabsf(__fsub_rn(x, f)));
  a.w1 = __fsub_rn(1.0f, fabsf(__fsub_rn(x, f1)));
  a.i0 = wrap_near(c, n);
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

// p[0..3] += v as one 16-byte vector reduction (p 16-byte aligned).
__device__ __forceinline__ void red_add_f4(float* p, float4 v) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p),
               "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
               : "memory");
}

// p[0..2] += (a, b, c) as one 16-byte vector reduction (p 16-byte aligned;
// p[3] += 0).
__device__ __forceinline__ void red_add_v4(float* p, float a, float b,
                                           float c) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p),
               "f"(a), "f"(b), "f"(c), "f"(0.f)
               : "memory");
}

// Tuning knobs of the particle kernels (compile-time).
#ifndef FPM_STEP_BLOCKED
#define FPM_STEP_BLOCKED 1  // the particle kernels walk lattice blocks
#endif
// Measured on B200, k_step per leapfrog step at 128^3 / 256^3: 3 blocks
// (80 registers) 87.4 / 621 us, 4 blocks (64) 84.6 / 594, 5 blocks (48)
// 85.4 / 583, 6 blocks (40, spills) 96.1 / 657.  The v4 pair reduction is
// slower than two scalar reductions (33 vs 49 us for 2^21 particles).  Painting
// after the readout phase of the whole block, directly or through a
// shared-memory tile of the block's cells, was slower (103 and 144 vs 87 us
// per step): the paint's reductions overlap the readout's gathers best when
// each warp issues both, particle by particle.  Neither more memory-level
// parallelism (items unrolled by 2, at 64 or 80 registers; the next
// particle's state prefetched into L1; reductions without a compiler memory
// barrier) nor an interleaved force mesh (one float4 (f_x, f_y, f_z, 0) per
// cell, 8 gathers per readout instead of 24) moved k_step by more than 1-3 %
// at 128^3 and 256^3: it is not latency-bound and not bound by its gathers.
// A z-adjacent pair as one 8-byte red.global.add.v2.f32 where aligned (half
// the pairs) was 1-2 % slower than two scalar reductions.
#ifndef FPM_STEP_MINBLOCKS
#define FPM_STEP_MINBLOCKS 4   // resident blocks of 256 threads per SM
#endif
// Resident blocks of the reverse-sweep kernels that gather forces and
// scatter their VJP (k_adj_position, k_adj_vjp, k_adj_pgd), which carry
// more state per particle, for plans whose particles mostly walk long
// lattice blocks (the others take FPM_STEP_MINBLOCKS: at 2 x 192^3, 8x8x16
// blocks, k_adj_position took 838 us with 3 blocks against 784 us with 4,
// cold and serialised).  Measured on B200 at 2 x 512^3: k_adj_position
// 15.9 ms with 3 blocks (78 registers), 17.3 ms with 4 (64 registers),
// 21.6 ms with 5 (48, spills); k_adj_vjp 14.3 against 14.9 ms with 4.
// k_adj_drift_paint, a drift and paint like k_step, keeps 4 (10.8 against
// 11.1 ms with 3).
#ifndef FPM_ADJ_MINBLOCKS
#define FPM_ADJ_MINBLOCKS 3
#endif
// k_adj_position over the binned order sums the scatter of lanes that start
// from the same base cell before depositing (1), or deposits lane by lane
// (0).  Measured on B200 (C4, 128^3 forward + adjoint with the potential
// tape, re-sorted every 4 positions): 5.14 G particle-updates/s with the
// sums against 5.43 G without -- the 24 values a lane deposits make the
// shuffles cost more than the vector reductions they save.
#ifndef FPM_ADJ_SORTED_SEGSUM
#define FPM_ADJ_SORTED_SEGSUM 0
#endif
// Resident blocks of k_adj_position over the binned particle order.
#ifndef FPM_ADJ_SORTED_MINBLOCKS
#define FPM_ADJ_SORTED_MINBLOCKS 3
#endif
// Programmatic dependent launch (sm_90 and later).  A kernel launched by
// launch_pdl may be scheduled as soon as its predecessor in the stream
// completes, without the launch gap; pdl_wait() (first statement of such
// kernels, before any global memory access) blocks until the predecessor's
// writes are visible, and is a no-op after an ordinary launch.  The kernels
// do not trigger their dependents early: measured on B200 at 128^3, letting
// the next kernel's blocks in before completion (launch_dependents at the
// top of every kernel) took 5.66 ms per simulation, against 5.07 without
// PDL and 5.03 with PDL and the implicit trigger at completion.
__device__ __forceinline__ void pdl_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

#ifndef FPM_PDL
#define FPM_PDL 1  // launch the leapfrog's kernels with launch_pdl
#endif
template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block,
                       size_t smem, cudaStream_t st, Args... args) {
#if FPM_PDL
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k, args...);  // errors surface in launch_ok()
#else
  k<<<grid, block, smem, st>>>(args...);
#endif
}

__device__ __forceinline__ bool finite3(float a, float b, float c) {
  return isfinite(a) && isfinite(b) && isfinite(c);
}

// ---------------------------------------------------------------------------
// Particle / mode helpers shared by the step and adjoint kernels
// ---------------------------------------------------------------------------
// Lattice coordinates of particle `local` of a sim (index (i*ny + j)*nz + k,
// the order of np.indices(nc).reshape(3, -1).T at flowpm/tfpm.py:162).
__device__ __forceinline__ void lattice_ijk(const SimDev& S, int64_t local,
                                            int& i, int& j, int& k) {
  // per-simulation indices are < 2^31: 32-bit unsigned division
  const unsigned l = (unsigned)local;
  const unsigned t = l / (unsigned)S.nz;
  k = (int)(l - t * (unsigned)S.nz);
  i = (int)(t / (unsigned)S.ny);
  j = (int)(t - (unsigned)i * (unsigned)S.ny);
}

// The carried index of the binned order: lattice site (i, j, k) packed as
// (i << (kb + jb)) | (j << kb) | k, so that q comes back with shifts and
// masks instead of two integer divisions.
__device__ __forceinline__ void unpack_site(uint32_t l, int kb, int jb,
                                            int& i, int& j, int& k) {
  k = (int)(l & ((1u << kb) - 1u));
  j = (int)((l >> kb) & ((1u << jb) - 1u));
  i = (int)(l >> (kb + jb));
}
__device__ __forceinline__ uint32_t pack_site(int i, int j, int k, int kb,
                                              int jb) {
  return ((uint32_t)i << (kb + jb)) | ((uint32_t)j << kb) | (uint32_t)k;
}
// Lagrangian index (i*ny + j)*nz + k of a site inside its simulation.
__device__ __forceinline__ int64_t site_local(const SimDev& S, int i, int j,
                                              int k) {
  return (int64_t)(((unsigned)i * (unsigned)S.ny + (unsigned)j) *
                       (unsigned)S.nz + (unsigned)k);
}

// Lanes of a warp with equal keys in a row form a run (particles sorted by
// cell make the particles of a cell contiguous); the run's first lane (its
// head) adds, claims or deposits for the whole run.  Returns the mask of
// heads; lanes past the end of the input must carry keys of their own.
__device__ __forceinline__ unsigned run_heads(uint32_t key, int lane) {
  const uint32_t up = __shfl_up_sync(0xffffffffu, key, 1);
  return __ballot_sync(0xffffffffu, lane == 0 || up != key);
}
// Lanes from this head to the next head.
__device__ __forceinline__ int run_length(unsigned heads, int lane) {
  const unsigned above = heads & ~((2u << lane) - 1u);
  return (above ? __ffs(above) - 1 : 32) - lane;
}
// The head of this lane's run.
__device__ __forceinline__ int run_head(unsigned heads, int lane) {
  return 31 - __clz(heads & ((2u << lane) - 1u));
}

// Position in force-mesh units: (q + d) * bf, as the reference's
// state[0] * pm_nc_factor with state[0] = q + d.
__device__ __forceinline__ float3 mesh_pos(const SimDev& S, int i, int j,
                                           int k, float3 d) {
  const float b = (float)S.bf;
  float3 x;
  x.x = __fmul_rn(__fadd_rn(index_float(i), d.x), b);
  x.y = __fmul_rn(__fadd_rn(index_float(j), d.y), b);
  x.z = __fmul_rn(__fadd_rn(index_float(k), d.z), b);
  return x;
}

// The 8 CIC neighbours of one position as 4 (x, y) rows of 2 z cells, with
// 32-bit offsets inside one simulation's mesh (meshes hold < 2^31 cells):
// neighbour (cx, cy, cz) is m[row[cx + 2 cy] + (cz ? z1 : z0)] with weight
// (wx * wy) * wz, the reference's product order.
struct Cic8 {
  unsigned row[4];
  unsigned z0, z1;
  float wxy[4];
  float wz0, wz1;
};

__device__ __forceinline__ Cic8 cic8(const Axis& ax, const Axis& ay,
                                     const Axis& az, int my, int mz) {
  Cic8 c;
  const unsigned x0 = (unsigned)ax.i0 * (unsigned)my;
  const unsigned x1 = (unsigned)ax.i1 * (unsigned)my;
  c.row[0] = (x0 + (unsigned)ay.i0) * (unsigned)mz;
  c.row[1] = (x1 + (unsigned)ay.i0) * (unsigned)mz;
  c.row[2] = (x0 + (unsigned)ay.i1) * (unsigned)mz;
  c.row[3] = (x1 + (unsigned)ay.i1) * (unsigned)mz;
  c.z0 = (unsigned)az.i0;
  c.z1 = (unsigned)az.i1;
  c.wxy[0] = __fmul_rn(ax.w0, ay.w0);
  c.wxy[1] = __fmul_rn(ax.w1, ay.w0);
  c.wxy[2] = __fmul_rn(ax.w0, ay.w1);
  c.wxy[3] = __fmul_rn(ax.w1, ay.w1);
  c.wz0 = az.w0;
  c.wz1 = az.w1;
  return c;
}

// Deposit s * W at the 8 neighbours (s = 1: plain paint).
__device__ __forceinline__ void paint_cic8(float* __restrict__ m,
                                           const Cic8& c, float s) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float w0 = __fmul_rn(c.wxy[q], c.wz0), w1 = __fmul_rn(c.wxy[q], c.wz1);
    if (s != 1.f) {
      w0 = __fmul_rn(s, w0);
      w1 = __fmul_rn(s, w1);
    }
    red_add(m + c.row[q] + c.z0, w0);
    red_add(m + c.row[q] + c.z1, w1);
  }
}

__device__ __forceinline__ void paint8(float* __restrict__ m, int mx, int my,
                                       int mz, const Axis& ax, const Axis& ay,
                                       const Axis& az) {
  paint_cic8(m, cic8(ax, ay, az, my, mz), 1.f);
}

// Deposit s * W at the 8 neighbours.
__device__ __forceinline__ void paint_scaled(float* __restrict__ m, int mx,
                                             int my, int mz, const Axis& ax,
                                             const Axis& ay, const Axis& az,
                                             float s) {
  paint_cic8(m, cic8(ax, ay, az, my, mz), s);
}

// Readout of the three force components (planes f0, f0 + mcells,
// f0 + 2 mcells) at the same 8 neighbours.
__device__ __forceinline__ float3 readout_cic8(const float* __restrict__ f0,
                                               int64_t mcells,
                                               const Cic8& c) {
  const float* f1 = f0 + mcells;
  const float* f2 = f1 + mcells;
  float r0 = 0.f, r1 = 0.f, r2 = 0.f;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const unsigned o0 = c.row[q] + c.z0, o1 = c.row[q] + c.z1;
    const float w0 = __fmul_rn(c.wxy[q], c.wz0);
    const float w1 = __fmul_rn(c.wxy[q], c.wz1);
    r0 = __fadd_rn(r0, __fmul_rn(__ldg(f0 + o0), w0));
    r1 = __fadd_rn(r1, __fmul_rn(__ldg(f1 + o0), w0));
    r2 = __fadd_rn(r2, __fmul_rn(__ldg(f2 + o0), w0));
    r0 = __fadd_rn(r0, __fmul_rn(__ldg(f0 + o1), w1));
    r1 = __fadd_rn(r1, __fmul_rn(__ldg(f1 + o1), w1));
    r2 = __fadd_rn(r2, __fmul_rn(__ldg(f2 + o1), w1));
  }
  return make_float3(r0, r1, r2);
}

__device__ __forceinline__ float3 ld3(const float* p, int64_t g) {
  return make_float3(p[3 * g], p[3 * g + 1], p[3 * g + 2]);
}
__device__ __forceinline__ void st3(float* p, int64_t g, float3 v) {
  p[3 * g] = v.x;
  p[3 * g + 1] = v.y;
  p[3 * g + 2] = v.z;
}
// a + s * b with the two roundings of the reference (update = fac * F,
// state = state + update).
__device__ __forceinline__ float3 axpy(float3 a, float s, float3 b) {
  return make_float3(__fadd_rn(a.x, __fmul_rn(s, b.x)),
                     __fadd_rn(a.y, __fmul_rn(s, b.y)),
                     __fadd_rn(a.z, __fmul_rn(s, b.z)));
}

__device__ __forceinline__ void mode_ijl(int64_t local, int ny, int nzh,
                                         int& i, int& j, int& l) {
  const unsigned m = (unsigned)local;
  const unsigned t = m / (unsigned)nzh;
  l = (int)(m - t * (unsigned)nzh);
  i = (int)(t / (unsigned)ny);
  j = (int)(t - (unsigned)i * (unsigned)ny);
}

// Chunk kind and particle enumeration of the particle kernels that gather
// from or scatter to the meshes (lattice blocks when FPM_STEP_BLOCKED, else
// kChunk consecutive particles).
constexpr int kTraverse = FPM_STEP_BLOCKED ? kBlock : kPart;

__device__ __forceinline__ int64_t traverse_first(const SimDev& S) {
  return FPM_STEP_BLOCKED ? S.ch_b : S.ch_p;
}

// One chunk of the traversal: the lattice origin of its block (blocked
// traversal) or its first flat particle.  Built once per chunk, so the
// divisions by the block counts are not repeated per particle.
struct Walk {
  int i0, j0, k0;
  int64_t base;
};

// Chunk `rel` (relative to the sim's first chunk).
__device__ __forceinline__ Walk walk_chunk(const SimDev& S, int64_t rel) {
  Walk w;
#if FPM_STEP_BLOCKED
  const unsigned b = (unsigned)rel;
  const unsigned r = b / (unsigned)S.nbk;
  const unsigned bi = r / (unsigned)S.nbj;
  w.i0 = (int)bi * kPlanes * S.wi;
  w.j0 = (int)(r - bi * (unsigned)S.nbj) * kBJ;
  w.k0 = (int)(b - r * (unsigned)S.nbk) * kBK;
  w.base = 0;
#else
  w.i0 = w.j0 = w.k0 = 0;
  w.base = rel * kChunk;
#endif
  return w;
}

// Item `item` (0 <= item < kItems) of this thread in the chunk: lattice
// coordinates and flat particle index; false when the particle does not
// exist (edge blocks, last chunk).  Particle t = threadIdx.x + item *
// kThreads of a block sits at (t / (kBJ kBK), (t / kBK) % kBJ, t % kBK)
// from the origin, z fastest, so consecutive lanes are consecutive z.
__device__ __forceinline__ bool walk_particle(const SimDev& S, const Walk& w,
                                              int item, int& i, int& j,
                                              int& k, int64_t& local) {
  const int t = threadIdx.x + item * kThreads;
#if FPM_STEP_BLOCKED
  i = w.i0 + t / (kBJ * kBK);
  j = w.j0 + (t / kBK) % kBJ;
  k = w.k0 + t % kBK;
  local = (int64_t)(((unsigned)i * (unsigned)S.ny + (unsigned)j) *
                        (unsigned)S.nz + (unsigned)k);
  return i < S.nx && j < S.ny && k < S.nz;
#else
  local = w.base + t;
  if (local >= S.np) return false;
  lattice_ijk(S, local, i, j, k);
  return true;
#endif
}

inline unsigned grid_for(int64_t chunks) {
  int64_t g = chunks < 1 ? 1 : chunks;
  const int64_t cap = (int64_t)kNumSMs * 16;
  return (unsigned)(g < cap ? g : cap);
}

}  // namespace fpm
