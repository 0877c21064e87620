// Fused Fourier solve of the force meshes for power-of-two meshes of 16 to
// 128 cells per axis: density -> three force meshes in three kernels,
// without cuFFT and without intermediate passes over HBM.
//
//   k_fft_plane_fwd  (one CTA per x plane)  rho(x, y, z) -> S(x, ky, kz)
//       real-to-complex DFT along z, complex DFT along y, the plane held in
//       shared memory; also zeroes rho for the next paint.
//   k_fft_columns    (one CTA per group of (ky, kz) columns)
//       DFT along x, then per component d the force spectrum
//       F_d = S * pre * w(k) * i g_d (the transfer function of
//       flowpm/tfpm.py:199-215 apply_longrange, the same arithmetic as
//       k_fourier_force), inverse DFT along x -> F_d(x, ky, kz).
//   k_fft_plane_inv  (one CTA per x plane and component)
//       inverse DFT along y, complex-to-real along z -> force mesh d.
//
// The transforms are unnormalised in both directions, as cuFFT's, so the
// spectra have cuFFT's R2C layout (x, y, z/2 + 1) and the results match
// the cuFFT path to rounding.  Every length-N DFT runs as N = N1 * N2 (the
// "four-step" split): a group of N2 threads, each holding N1 values in
// registers, does N1-point DFTs, a twiddle, one exchange through shared
// memory and N2-point DFTs.  Twiddles come from a table of
// exp(-2 pi i m / 128) computed in double on the host.
#include <cmath>
#include <mutex>

#include "fpm_kernels.cuh"

namespace fpm {

namespace {

constexpr int kFftThreads = 256;

__constant__ float2 c_w128[128];  // exp(-2 pi i m / 128), m = 0..127
__device__ float2 g_w128[128];    // the same, for lane-dependent indices
__device__ float2 g_w512[512];    // exp(-2 pi i m / 512), m = 0..511

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

template <int N>
struct Split;
template <>
struct Split<8> {
  static constexpr int N1 = 4, N2 = 2;
};
template <>
struct Split<16> {
  static constexpr int N1 = 4, N2 = 4;
};
template <>
struct Split<32> {
  static constexpr int N1 = 8, N2 = 4;
};
template <>
struct Split<64> {
  static constexpr int N1 = 8, N2 = 8;
};
template <>
struct Split<128> {
  static constexpr int N1 = 16, N2 = 8;
};

// In-register radix-2 DFT of N (<= 16) values, decimation in time:
// forward X[k] = sum_j x[j] exp(-2 pi i jk / N), inverse with +i.
// In-register DFT of N (2 to 16) values by even/odd (radix-2, decimation
// in time) recursion, every index a compile-time constant: forward
// X[k] = sum_j x[j] exp(-2 pi i jk / N), inverse with +i.
template <int N, bool INV>
struct Dft {
  static __device__ __forceinline__ void run(float2 (&a)[N]) {
    constexpr int H = N / 2;
    float2 e[H], o[H];
#pragma unroll
    for (int j = 0; j < H; ++j) {
      e[j] = a[2 * j];
      o[j] = a[2 * j + 1];
    }
    Dft<H, INV>::run(e);
    Dft<H, INV>::run(o);
#pragma unroll
    for (int k = 0; k < H; ++k) {
      float2 v = o[k];
      if (k != 0) {
        if (4 * k == N) {  // exp(-+ i pi / 2) = -+ i
          v = INV ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
        } else {
          const float2 w = c_w128[k * (128 / N)];
          v = INV ? cmulc(v, w) : cmul(v, w);
        }
      }
      a[k] = make_float2(e[k].x + v.x, e[k].y + v.y);
      a[k + H] = make_float2(e[k].x - v.x, e[k].y - v.y);
    }
  }
};
template <bool INV>
struct Dft<1, INV> {
  static __device__ __forceinline__ void run(float2 (&)[1]) {}
};

template <int N, bool INV>
__device__ __forceinline__ void dft(float2 (&a)[N]) {
  Dft<N, INV>::run(a);
}

// Forward DFT of one line of N values by the N2 threads g of its group;
// `line` (element e at line[e * es]) is the exchange buffer.  Every thread
// of the block calls it; invalid threads (valid = false) get an in-bounds
// line to read and write nothing.
// On entry a[j1] = x[N2 j1 + g]; on exit a[u N2 + k2] = X[g + N2 u + N1 k2].
// The caller syncs before writing the results back into `line`.
template <int N>
__device__ __forceinline__ void fwd_line(float2 (&a)[Split<N>::N1],
                                         float2* line, int es, int g,
                                         bool valid) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  dft<N1, false>(a);
#pragma unroll
  for (int k1 = 1; k1 < N1; ++k1)
    a[k1] = cmul(a[k1], c_w128[((g * k1) & (N - 1)) * (128 / N)]);
  __syncthreads();  // every line has been loaded
  if (valid) {
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) line[(k1 * N2 + g) * es] = a[k1];
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < N1 / N2; ++u) {
    const int k1 = g + N2 * u;
    float2 b[N2];
#pragma unroll
    for (int j = 0; j < N2; ++j)
      b[j] = line[(k1 * N2 + j) * es];
    dft<N2, false>(b);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) a[u * N2 + k2] = b[k2];
  }
}

// Inverse (unnormalised) DFT of one line, the converse of fwd_line:
// on entry a[u N2 + k2] = X[g + N2 u + N1 k2]; on exit a[j1] = x[N2 j1 + g].
template <int N>
__device__ __forceinline__ void inv_line(float2 (&a)[Split<N>::N1],
                                         float2* line, int es, int g,
                                         bool valid) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  __syncthreads();  // every line has been loaded
#pragma unroll
  for (int u = 0; u < N1 / N2; ++u) {
    const int k1 = g + N2 * u;
    float2 b[N2];
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) b[k2] = a[u * N2 + k2];
    dft<N2, true>(b);
#pragma unroll
    for (int j2 = 0; j2 < N2; ++j2) {
      if (j2 != 0 && k1 != 0)
        b[j2] = cmulc(b[j2], c_w128[((j2 * k1) & (N - 1)) * (128 / N)]);
      if (valid) line[(k1 * N2 + j2) * es] = b[j2];
    }
  }
  __syncthreads();
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1)
    a[k1] = line[(k1 * N2 + g) * es];
  dft<N1, true>(a);
}

// Forward DFT along the rows (stride 1, length N, row stride rs) of
// `nrows` rows of the shared plane P, in place, natural order out.
template <int N, int T>
__device__ __forceinline__ void rows_fwd(float2* P, int nrows, int rs) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  constexpr int RP = T / N2;  // rows per pass (>= 32: warp-uniform g)
  const int rl = threadIdx.x % RP, g = threadIdx.x / RP;
#pragma unroll 1
  for (int r0 = 0; r0 < nrows; r0 += RP) {
    const int r = r0 + rl;
    const bool valid = r < nrows;
    float2* line = P + (valid ? r : 0) * rs;  // idle threads read row 0
    float2 a[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; ++j1)
      a[j1] = valid ? line[N2 * j1 + g] : make_float2(0.f, 0.f);
    fwd_line<N>(a, line, 1, g, valid);
    __syncthreads();
    if (valid) {
#pragma unroll
      for (int u = 0; u < N1 / N2; ++u)
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2)
          line[g + N2 * u + N1 * k2] = a[u * N2 + k2];
    }
    __syncthreads();
  }
}

// Inverse DFT along the rows, in place, natural order in and out.
template <int N, int T>
__device__ __forceinline__ void rows_inv(float2* P, int nrows, int rs) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  constexpr int RP = T / N2;
  const int rl = threadIdx.x % RP, g = threadIdx.x / RP;
#pragma unroll 1
  for (int r0 = 0; r0 < nrows; r0 += RP) {
    const int r = r0 + rl;
    const bool valid = r < nrows;
    float2* line = P + (valid ? r : 0) * rs;  // idle threads read row 0
    float2 a[N1];
#pragma unroll
    for (int u = 0; u < N1 / N2; ++u)
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2)
        a[u * N2 + k2] =
            valid ? line[g + N2 * u + N1 * k2] : make_float2(0.f, 0.f);
    inv_line<N>(a, line, 1, g, valid);
    __syncthreads();
    if (valid) {
#pragma unroll
      for (int j1 = 0; j1 < N1; ++j1) line[N2 * j1 + g] = a[j1];
    }
    __syncthreads();
  }
}

// Forward / inverse DFT along the first NCOLS columns (length N, stride CS)
// of P, in place, in one pass: T / N2 >= NCOLS.
template <int N, bool INV, int T, int NCOLS, int CS>
__device__ __forceinline__ void cols_dft(float2* P) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  constexpr int CP = T / N2;
  static_assert(CP >= NCOLS, "one pass over the columns");
  const int c = threadIdx.x % CP, g = threadIdx.x / CP;
  const bool valid = c < NCOLS;
  float2* line = P + (valid ? c : 0);  // idle threads read column 0
  float2 a[N1];
  if constexpr (!INV) {
#pragma unroll
    for (int j1 = 0; j1 < N1; ++j1)
      a[j1] = line[(N2 * j1 + g) * CS];
    fwd_line<N>(a, line, CS, g, valid);
    __syncthreads();
    if (valid) {
#pragma unroll
      for (int u = 0; u < N1 / N2; ++u)
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2)
          line[(g + N2 * u + N1 * k2) * CS] = a[u * N2 + k2];
    }
  } else {
#pragma unroll
    for (int u = 0; u < N1 / N2; ++u)
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2)
        a[u * N2 + k2] = line[(g + N2 * u + N1 * k2) * CS];
    inv_line<N>(a, line, CS, g, valid);
    __syncthreads();
    if (valid) {
#pragma unroll
      for (int j1 = 0; j1 < N1; ++j1) line[(N2 * j1 + g) * CS] = a[j1];
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// One x plane of one simulation of the run: rho -> S.  The real rows of
// 2M cells are read as M complex values z[m] = x[2m] + i x[2m+1]; after the
// M-point DFT Z, X[k] = E[k] + W^k O[k] (W = exp(-2 pi i / 2M)) with
// E[k] = (Z[k] + conj Z[M-k]) / 2 and O[k] = (Z[k] - conj Z[M-k]) / 2i.
// The columns kz = 0 and kz = M are real: they go through the y DFT
// together as column 0 = X[.][0] + i X[.][M] and are separated on the way
// out (Y0 = (C[ky] + conj C[-ky]) / 2, YM = (C[ky] - conj C[-ky]) / 2i), so
// the y pass covers M columns.
// Measured on B200 at 128^3 (Fourier solve per step): 512 threads 51 us,
// 1024 threads 52 us; splitting each plane over a cluster of two CTAs
// (the y pass through distributed shared memory) 63 us.
#ifndef FPM_PLANE_THREADS
#define FPM_PLANE_THREADS 512
#endif
constexpr int kPlaneThreads = FPM_PLANE_THREADS;  // threads of the plane kernels

template <int NY, int M>
__global__ void __launch_bounds__(kPlaneThreads)
k_fft_plane_fwd(const SimDev* __restrict__ sims, int first, int nx,
                float* __restrict__ rho, float2* __restrict__ dk,
                int zero_rho) {
  pdl_wait();  // the density painted before
  extern __shared__ float2 P[];  // NY rows of M + 1
  constexpr int T = kPlaneThreads;
  constexpr int NZH = M + 1;
  const int s = first + blockIdx.x / nx;
  const int x = blockIdx.x % nx;
  const SimDev& S = sims[s];
  float4* src = reinterpret_cast<float4*>(rho + S.m_off + (int64_t)x * NY * 2 * M);
  float2* dst = dk + S.s_off + (int64_t)x * NY * NZH;
  constexpr int NV = NY * M / 2;  // float4 (two complex) per plane
#pragma unroll 8
  for (int e = threadIdx.x; e < NV; e += T) {
    const float4 v = src[e];
    const int r = (2 * e) / M, m = (2 * e) % M;
    P[r * NZH + m] = make_float2(v.x, v.y);
    P[r * NZH + m + 1] = make_float2(v.z, v.w);
  }
  if (zero_rho) {
    for (int e = threadIdx.x; e < NV; e += T)
      src[e] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  rows_fwd<M, T>(P, NY, NZH);
  // real-to-complex unpacking, one (k, M - k) pair per work item
  constexpr int KP = M / 2 + 1;
  for (int e = threadIdx.x; e < NY * KP; e += T) {
    const int r = e / KP, k = e % KP;
    float2* line = P + r * NZH;
    if (k == 0) {
      const float2 z = line[0];
      line[0] = make_float2(z.x + z.y, z.x - z.y);  // X[0] + i X[M]
    } else if (2 * k == M) {
      const float2 z = line[k];
      line[k] = make_float2(z.x, -z.y);
    } else {
      const float2 zk = line[k], zm = line[M - k];
      const float2 E = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
      const float2 O = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
      const float2 W = cmul(__ldg(&g_w128[k * (64 / M)]), O);
      line[k] = make_float2(E.x + W.x, E.y + W.y);
      line[M - k] = make_float2(E.x - W.x, -(E.y - W.y));
    }
  }
  __syncthreads();
  cols_dft<NY, false, T, M, NZH>(P);
  for (int e = threadIdx.x; e < NY * NZH; e += T) {
    const int ky = e / NZH, kz = e - ky * NZH;
    float2 v;
    if (kz == 0 || kz == M) {
      const float2 c = P[ky * NZH];
      const float2 cm = P[((NY - ky) & (NY - 1)) * NZH];
      v = kz == 0 ? make_float2(0.5f * (c.x + cm.x), 0.5f * (c.y - cm.y))
                  : make_float2(0.5f * (c.y + cm.y), -0.5f * (c.x - cm.x));
    } else {
      v = P[e];
    }
    dst[e] = v;
  }
}

// Columns (ky, kz) of the spectra of one simulation: DFT along x, the three
// force spectra, inverse DFT along x.  C = 256 / N2 columns per CTA, lanes
// on consecutive columns (coalesced; warp-uniform group index g).
template <int NX, bool GRAD3>
__global__ void __launch_bounds__(kFftThreads)
k_fft_columns(const SimDev* __restrict__ sims, int first, int nblk,
              float2* dk, float2* __restrict__ fk, AxisTabs tabs, Green G) {
  pdl_wait();
  constexpr int N1 = Split<NX>::N1, N2 = Split<NX>::N2;
  constexpr int C = kFftThreads / N2;
  __shared__ float2 ex[C * NX];
  const int s = first + blockIdx.x / nblk;
  const SimDev& S = sims[s];
  const int ny = S.my, nzh = S.mzh;
  const int ncols = ny * nzh;
  const int cl = threadIdx.x % C, g = threadIdx.x / C;
  const int c = (blockIdx.x % nblk) * C + cl;
  const bool valid = c < ncols;
  const int64_t nmodes = (int64_t)NX * ncols;
  const float2* src = dk + S.s_off + c;
  float2* line = ex + cl;
  float2 a[N1];
#pragma unroll
  for (int j1 = 0; j1 < N1; ++j1)
    a[j1] = valid ? src[(int64_t)(N2 * j1 + g) * ncols] : make_float2(0.f, 0.f);
  fwd_line<NX>(a, line, C, g, valid);
  // potential spectrum delta * pre * w(k), w the transfer function G
  const int ky = valid ? c / nzh : 0;
  const int kz = valid ? c - ky * nzh : 0;
  const float pre = (float)((double)S.bf * S.bf * S.bf /
                            ((double)S.mx * S.my * S.mz));
  const double* kkx = tabs.kk + S.tab;
  const double* kky = kkx + S.mx;
  const double* kkz = kky + S.my;
  const float* wx = tabs.win + S.tab;
  const float* wy = wx + S.mx;
  const float* wz = wy + S.my;
  const float* gx = tabs.grad + S.tab;
  const float* gy = gx + S.mx;
  const float* gz = gy + S.my;
  const double kyz = kky[ky] + kkz[kz];
  const float wyv = wy[ky], wzv = wz[kz];
#pragma unroll
  for (int u = 0; u < N1 / N2; ++u)
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
      const int kx = g + N2 * u + N1 * k2;
      const float w = green_w(G, s, kkx[kx] + kyz, wx[kx], wyv, wzv);
      float2 v = a[u * N2 + k2];
      v.x = __fmul_rn(__fmul_rn(v.x, pre), w);
      v.y = __fmul_rn(__fmul_rn(v.y, pre), w);
      a[u * N2 + k2] = v;
    }
  if (!GRAD3) {  // potential only, in place
    inv_line<NX>(a, line, C, g, valid);
    if (valid) {
      float2* o = dk + S.s_off + c;
#pragma unroll
      for (int j1 = 0; j1 < N1; ++j1)
        o[(int64_t)(N2 * j1 + g) * ncols] = a[j1];
    }
    return;
  }
  const float gyv = gy[ky], gzv = gz[kz];
#pragma unroll 1
  for (int d = 0; d < 3; ++d) {
    float2 b[N1];
#pragma unroll
    for (int u = 0; u < N1 / N2; ++u)
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) {
        const int kx = g + N2 * u + N1 * k2;
        const float gd = d == 0 ? gx[kx] : (d == 1 ? gyv : gzv);
        const float2 v = a[u * N2 + k2];
        b[u * N2 + k2] = make_float2(-__fmul_rn(v.y, gd), __fmul_rn(v.x, gd));
      }
    inv_line<NX>(b, line, C, g, valid);
    if (valid) {
      float2* o = fk + 3 * S.s_off + d * nmodes + c;
#pragma unroll
      for (int j1 = 0; j1 < N1; ++j1)
        o[(int64_t)(N2 * j1 + g) * ncols] = b[j1];
    }
  }
}

// x pass of the Fourier solve of meshes with 256 or 512 cells along x,
// between batched two-dimensional (y, z) transforms of cuFFT (the
// spectrum in cuFFT's R2C layout (x, y, z/2 + 1), unnormalised):
// out = inverse-DFT_x(pre * w(k) * DFT_x(in)) for the kXCols consecutive
// (ky, kz) columns of one simulation held by the block (the potential of
// k_fourier_potential, the same arithmetic per mode).  The x DFT of
// length NX = R * 64 runs on the stride-R sub-lines x = R b + a as 64-point
// DFTs (cols_dft), a twiddle W_NX^(a kb) and R-point DFTs in registers,
// where the transfer function is applied and the inverse starts; the
// column block moves through shared memory as rows of kXCols modes.  With
// rho_zero, the block also zeroes its share of that buffer: zmul floats per
// cell of the sim (1: the density mesh; 4: the interleaved adjoint force
// mesh).
// Columns per x-pass block.  Measured on B200 at 2 x 512^3: 8 columns
// (64-byte rows, 32 KB) 1.19 ms per pass, 16 (128-byte rows, 64 KB) 1.01
// ms; a persistent variant with cp.async double buffering of 8-column
// blocks took 1.53 ms.
#ifndef FPM_XPASS_COLS
#define FPM_XPASS_COLS 16
#endif
constexpr int kXThreads = 512, kXCols = FPM_XPASS_COLS;

template <int NX>
__global__ void __launch_bounds__(kXThreads)
k_fft_xcols(const SimDev* __restrict__ sims, int first, int nblk,
            const float2* in, float2* out, float* __restrict__ rho_zero,
            int zmul, AxisTabs tabs, Green G,
            const int32_t* __restrict__ nsteps, int pos) {
  constexpr int R = NX / 64, C = kXCols, T = kXThreads;
  constexpr int NP = 64 * C / T;                  // (kb, column) pairs
  constexpr int NS = R * C, NS1 = NS < 64 ? NS : 64;  // sub-lines per pass
  static_assert(64 * C % T == 0 && NS % NS1 == 0, "block shape");
  extern __shared__ __align__(16) float2 buf[];   // x of column c at x C + c
  pdl_wait();  // the spectrum written before
  const int s = first + blockIdx.x / nblk;
  if (nsteps && pos > nsteps[s]) return;  // finished simulation
  const int blk = blockIdx.x % nblk;
  const SimDev& S = sims[s];
  const int ncols = S.my * S.mzh;
  const int c0 = blk * C;
  const float4* src = reinterpret_cast<const float4*>(in + S.s_off + c0);
  float4* dst = reinterpret_cast<float4*>(out + S.s_off + c0);
  const int64_t rstride = ncols / 2;  // float4 per x plane
  float4* b4 = reinterpret_cast<float4*>(buf);
#pragma unroll
  for (int i = 0; i < NX * C / 2 / T; ++i) {
    const int e = threadIdx.x + i * T;
    b4[e] = src[(int64_t)(e / (C / 2)) * rstride + e % (C / 2)];
  }
  if (rho_zero) {  // this block's share, in float4
    const int64_t q4 = (int64_t)zmul * S.mx * S.my * S.mz / 4;
    const int64_t per = (q4 + nblk - 1) / nblk;
    float4* r4 = reinterpret_cast<float4*>(rho_zero + zmul * S.m_off);
    const int64_t e1 = min(q4, (blk + 1) * per);
    for (int64_t e = blk * per + threadIdx.x; e < e1; e += T)
      r4[e] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
#pragma unroll
  for (int h = 0; h < NS / NS1; ++h)  // each ends with a barrier
    cols_dft<64, false, T, NS1, NS>(buf + h * NS1);
  const float pre = (float)((double)S.bf * S.bf * S.bf /
                            ((double)S.mx * S.my * S.mz));
#pragma unroll 1
  for (int pr = 0; pr < NP; ++pr) {
  const int kb = (threadIdx.x + pr * T) / C, c = threadIdx.x % C;
  float2 v[R];
#pragma unroll
  for (int a = 0; a < R; ++a) {
    v[a] = buf[(R * kb + a) * C + c];
    if (a != 0 && kb != 0)
      v[a] = cmul(v[a], g_w512[(a * kb * (512 / NX)) & 511]);
  }
  dft<R, false>(v);  // v[ka] = X[kb + 64 ka]
  const int j = c0 + c;
  const int ky = j / S.mzh, kz = j - ky * S.mzh;
  const double* kkx = tabs.kk + S.tab;
  const double kyv = kkx[S.mx + ky], kzv = kkx[S.mx + S.my + kz];
  const float* wx = tabs.win + S.tab;
  // the CIC windows only enter with deconvolution
  const float wyv = G.deconv ? wx[S.mx + ky] : 1.f;
  const float wzv = G.deconv ? wx[S.mx + S.my + kz] : 1.f;
#pragma unroll
  for (int ka = 0; ka < R; ++ka) {
    const int kx = kb + 64 * ka;
    const float w = green_w(G, s, (kkx[kx] + kyv) + kzv,
                            G.deconv ? wx[kx] : 1.f, wyv, wzv);
    float2 d = v[ka];
    d.x = __fmul_rn(d.x, pre);
    d.y = __fmul_rn(d.y, pre);
    v[ka] = make_float2(__fmul_rn(d.x, w), __fmul_rn(d.y, w));
  }
  dft<R, true>(v);  // v[a] = sum_ka X W_R^(-a ka)
#pragma unroll
  for (int a = 0; a < R; ++a) {
    if (a != 0 && kb != 0)
      v[a] = cmulc(v[a], g_w512[(a * kb * (512 / NX)) & 511]);
    buf[(R * kb + a) * C + c] = v[a];  // the positions this thread read
  }
  }
  __syncthreads();
#pragma unroll
  for (int h = 0; h < NS / NS1; ++h)
    cols_dft<64, true, T, NS1, NS>(buf + h * NS1);
#pragma unroll
  for (int i = 0; i < NX * C / 2 / T; ++i) {
    const int e = threadIdx.x + i * T;
    dst[(int64_t)(e / (C / 2)) * rstride + e % (C / 2)] = b4[e];
  }
}

// 4-point central difference with periodic wrap, the arithmetic of
// k_stencil_grad: (8 (f[+1] - f[-1]) - (f[+2] - f[-2])) / 12.
__device__ __forceinline__ float stencil4f(float m2, float m1, float p1,
                                           float p2) {
  return __fmul_rn(__fsub_rn(__fmul_rn(8.f, __fsub_rn(p1, m1)),
                             __fsub_rn(p2, m2)),
                   1.0f / 12.0f);
}

// One x plane of one force component: inverse DFT along y, then
// complex-to-real along z: Zc[k] = A + i conj(W^k) B with A = X[k] +
// conj X[M-k], B = X[k] - conj X[M-k], and the inverse M-point DFT of Zc
// gives x[2m] + i x[2m+1].  The columns kz = 0 and kz = M, real after the y
// inverse, share one complex column (X[.][0] + i X[.][M]).
// Output modes of k_fft_plane_inv.
enum PlaneOut {
  kOutStencil = 0,  // potential -> phi, force y and z by the 4-point stencil
  kOutGrad3 = 1,    // three force spectra -> the three force meshes
  kOutReal = 2      // one spectrum -> one real mesh (phi)
};

template <int NY, int M, int MODE>
__global__ void __launch_bounds__(kPlaneThreads)
k_fft_plane_inv(const SimDev* __restrict__ sims, int first, int nx,
                const float2* __restrict__ spec, float* __restrict__ fmesh,
                float* __restrict__ phi) {
  pdl_wait();
  constexpr bool GRAD3 = MODE == kOutGrad3;
  extern __shared__ float2 P[];
  constexpr int T = kPlaneThreads;
  constexpr int NZH = M + 1;
  const int d = GRAD3 ? blockIdx.x % 3 : 0;
  const int rest = GRAD3 ? blockIdx.x / 3 : blockIdx.x;
  const int x = rest % nx;
  const int s = first + rest / nx;
  const SimDev& S = sims[s];
  const int64_t nmodes = (int64_t)nx * NY * NZH;
  const int64_t mcells = (int64_t)nx * NY * 2 * M;
  const int64_t plane = (int64_t)x * NY * 2 * M;
  const float2* src = spec + (GRAD3 ? 3 * S.s_off + d * nmodes : S.s_off) +
                      (int64_t)x * NY * NZH;
  // M columns per row after packing kz = 0 and kz = M into column 0
  constexpr int NL = NY * M;
#pragma unroll
  for (int i = 0; i < (NL + T - 1) / T; ++i) {
    const int e = threadIdx.x + i * T;
    if (NL % T == 0 || e < NL) {
      const int ky = e / M, kz = e % M;
      const float2* row = src + ky * NZH;
      float2 v = row[kz];
      if (kz == 0) {
        const float2 xm = row[M];
        v = make_float2(v.x - xm.y, v.y + xm.x);
      }
      P[ky * NZH + kz] = v;
    }
  }
  __syncthreads();
  cols_dft<NY, true, T, M, NZH>(P);
  constexpr int KP = M / 2 + 1;
  for (int e = threadIdx.x; e < NY * KP; e += T) {
    const int r = e / KP, k = e % KP;
    float2* line = P + r * NZH;
    if (k == 0) {
      const float2 c = line[0];  // X[0] + i X[M], both real
      line[0] = make_float2(c.x + c.y, c.x - c.y);
    } else if (2 * k == M) {
      const float2 v = line[k];
      line[k] = make_float2(2.f * v.x, -2.f * v.y);
    } else {
      const float2 xk = line[k], xm = line[M - k];
      const float2 A = make_float2(xk.x + xm.x, xk.y - xm.y);
      const float2 B = make_float2(xk.x - xm.x, xk.y + xm.y);
      const float2 cb = cmulc(B, __ldg(&g_w128[k * (64 / M)]));
      const float2 Tw = make_float2(-cb.y, cb.x);  // i conj(W^k) B
      line[k] = make_float2(A.x + Tw.x, A.y + Tw.y);
      line[M - k] = make_float2(A.x - Tw.x, -(A.y - Tw.y));
    }
  }
  __syncthreads();
  rows_inv<M, T>(P, NY, NZH);
  constexpr int NV = NY * M / 2;  // float4 per plane
  if (MODE != kOutStencil) {
    float4* dst = reinterpret_cast<float4*>(
        GRAD3 ? fmesh + 3 * S.m_off + d * mcells + plane
              : phi + S.m_off + plane);
    for (int e = threadIdx.x; e < NV; e += T) {
      const int r = (2 * e) / M, m = (2 * e) % M;
      const float2 a = P[r * NZH + m], b = P[r * NZH + m + 1];
      dst[e] = make_float4(a.x, a.y, b.x, b.y);
    }
    return;
  }
  // potential plane: store it (the x stencil reads it) and take the y and
  // z components of the force here, from shared memory
  constexpr int RS = 2 * NZH;  // floats per row
  constexpr int NZ = 2 * M;
  const float* f = reinterpret_cast<const float*>(P);
  float* gphi = phi + S.m_off + plane;
  float* gy = fmesh + 3 * S.m_off + mcells + plane;
  float* gz = fmesh + 3 * S.m_off + 2 * mcells + plane;
  // consecutive lanes on consecutive z: conflict-free shared reads,
  // coalesced stores
  for (int e = threadIdx.x; e < NY * NZ; e += T) {
    const int y = e / NZ, z = e % NZ;
    const float* r0 = f + y * RS;
    const float v = r0[z];
    const float fy = stencil4f(f[((y - 2) & (NY - 1)) * RS + z],
                               f[((y - 1) & (NY - 1)) * RS + z],
                               f[((y + 1) & (NY - 1)) * RS + z],
                               f[((y + 2) & (NY - 1)) * RS + z]);
    const float fz = stencil4f(r0[(z - 2) & (NZ - 1)], r0[(z - 1) & (NZ - 1)],
                               r0[(z + 1) & (NZ - 1)], r0[(z + 2) & (NZ - 1)]);
    gphi[e] = v;
    gy[e] = fy;
    gz[e] = fz;
  }
}

// x component of the force from the potential planes x - 2 .. x + 2
// (periodic), four z cells per thread.
template <int NY, int NZ>
__global__ void __launch_bounds__(kFftThreads)
k_fft_stencil_x(const SimDev* __restrict__ sims, int first, int nx,
                const float* __restrict__ phi, float* __restrict__ fmesh) {
  pdl_wait();
  constexpr int PL = NY * NZ / 4;  // float4 per plane
  const int64_t total = (int64_t)nx * PL;
  const int s = first + blockIdx.y;
  const SimDev& S = sims[s];
  const float4* p = reinterpret_cast<const float4*>(phi + S.m_off);
  float4* o = reinterpret_cast<float4*>(fmesh + 3 * S.m_off);
  for (int64_t e = (int64_t)blockIdx.x * kFftThreads + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * kFftThreads) {
    const int x = (int)(e / PL);
    const int r = (int)(e - (int64_t)x * PL);
    const float4 m2 = p[(int64_t)((x - 2 + nx) % nx) * PL + r];
    const float4 m1 = p[(int64_t)((x - 1 + nx) % nx) * PL + r];
    const float4 p1 = p[(int64_t)((x + 1) % nx) * PL + r];
    const float4 p2 = p[(int64_t)((x + 2) % nx) * PL + r];
    o[e] = make_float4(stencil4f(m2.x, m1.x, p1.x, p2.x),
                       stencil4f(m2.y, m1.y, p1.y, p2.y),
                       stencil4f(m2.z, m1.z, p1.z, p2.z),
                       stencil4f(m2.w, m1.w, p1.w, p2.w));
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

std::mutex g_tw_mu;
bool g_tw_ready[64] = {};

template <int NY, int M>
int set_plane_smem() {
  const int bytes = NY * (M + 1) * (int)sizeof(float2);
  if (cudaFuncSetAttribute(k_fft_plane_fwd<NY, M>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           bytes) != cudaSuccess ||
      cudaFuncSetAttribute(k_fft_plane_inv<NY, M, kOutStencil>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           bytes) != cudaSuccess ||
      cudaFuncSetAttribute(k_fft_plane_inv<NY, M, kOutGrad3>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           bytes) != cudaSuccess ||
      cudaFuncSetAttribute(k_fft_plane_inv<NY, M, kOutReal>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           bytes) != cudaSuccess) {
    cudaGetLastError();
    return FPM_ERR_CUDA;
  }
  return FPM_OK;
}

#define FPM_FFT_SIZES(X) X(16) X(32) X(64) X(128)
#define FPM_FFT_HALF(X) X(8) X(16) X(32) X(64)

bool pow2_in_range(int n) { return n >= 16 && n <= 128 && (n & (n - 1)) == 0; }

template <int NY>
int prepare_ny(int M) {
  switch (M) {
#define FPM_PREP_M(MM) \
  case MM: return set_plane_smem<NY, MM>();
    FPM_FFT_HALF(FPM_PREP_M)
#undef FPM_PREP_M
  }
  return FPM_ERR_UNSUPPORTED;
}

// The kernels of one mesh shape (NY, M = nz / 2).
template <int NY, int M>
void launch_shape(const SimDev* sims, int first, int n, int nx, float* rho,
                  int zero_rho, float2* dk, float2* fk, float* fmesh,
                  float* phi, AxisTabs tabs, const Green& G, bool grad3,
                  bool real_out, cudaStream_t st) {
  const size_t smem = (size_t)NY * (M + 1) * sizeof(float2);
  launch_pdl(k_fft_plane_fwd<NY, M>, dim3(n * nx), dim3(kPlaneThreads), smem,
             st, sims, first, nx, rho, dk, zero_rho);
  const int ncols = NY * (M + 1);
  if (!grad3 && nx == 128) {
    // x DFT, potential, inverse x DFT by the x-pass kernel (R = 2): four
    // values per thread instead of sixteen, so more loads in flight
    // (measured at 128^3: 47.7 against 48.7 us per Fourier solve)
    const int nblk = ncols / kXCols;  // NY is a multiple of 16
    launch_pdl(k_fft_xcols<128>, dim3(n * nblk), dim3(kXThreads),
               (size_t)128 * kXCols * sizeof(float2), st, sims, first, nblk,
               (const float2*)dk, dk, (float*)nullptr, 1, tabs, G,
               (const int32_t*)nullptr, 0);
  } else switch (nx) {
#define FPM_COL_CASE(NN)                                                   \
  case NN: {                                                               \
    constexpr int C = kFftThreads / Split<NN>::N2;                         \
    const int nblk = (ncols + C - 1) / C;                                  \
    if (grad3)                                                             \
      launch_pdl(k_fft_columns<NN, true>, dim3(n * nblk), dim3(kFftThreads), \
                 0, st, sims, first, nblk, dk, fk, tabs, G);               \
    else                                                                   \
      launch_pdl(k_fft_columns<NN, false>, dim3(n * nblk),                 \
                 dim3(kFftThreads), 0, st, sims, first, nblk, dk, fk, tabs, \
                 G);                                                       \
    break;                                                                 \
  }
    FPM_FFT_SIZES(FPM_COL_CASE)
#undef FPM_COL_CASE
  }
  if (grad3) {
    k_fft_plane_inv<NY, M, kOutGrad3><<<n * nx * 3, kPlaneThreads, smem, st>>>(
        sims, first, nx, fk, fmesh, phi);
    return;
  }
  if (real_out) {  // potential of `rho` -> phi
    k_fft_plane_inv<NY, M, kOutReal><<<n * nx, kPlaneThreads, smem, st>>>(
        sims, first, nx, dk, nullptr, phi);
    return;
  }
  launch_pdl(k_fft_plane_inv<NY, M, kOutStencil>, dim3(n * nx),
             dim3(kPlaneThreads), smem, st, sims, first, nx,
             (const float2*)dk, fmesh, phi);
  const int64_t quads = (int64_t)nx * NY * 2 * M / 4;
  int64_t bx = (quads + kFftThreads - 1) / kFftThreads;
  const int64_t cap = (int64_t)kNumSMs * 8 / (n < 1 ? 1 : n) + 1;
  if (bx > cap) bx = cap;
  launch_pdl(k_fft_stencil_x<NY, 2 * M>, dim3((unsigned)bx, (unsigned)n),
             dim3(kFftThreads), 0, st, sims, first, nx, (const float*)phi,
             fmesh);
}

template <int NY>
void launch_ny(int M, const SimDev* sims, int first, int n, int nx,
               float* rho, int zero_rho, float2* dk, float2* fk, float* fmesh,
               float* phi, AxisTabs tabs, const Green& G, bool grad3,
               bool real_out, cudaStream_t st) {
  switch (M) {
#define FPM_SHAPE_CASE(MM)                                                  \
  case MM:                                                                  \
    launch_shape<NY, MM>(sims, first, n, nx, rho, zero_rho, dk, fk, fmesh,  \
                         phi, tabs, G, grad3, real_out, st);                \
    break;
    FPM_FFT_HALF(FPM_SHAPE_CASE)
#undef FPM_SHAPE_CASE
  }
}

}  // namespace

bool fft_fused_supported(int nx, int ny, int nz) {
  return pow2_in_range(nx) && pow2_in_range(ny) && pow2_in_range(nz);
}

int fft_fused_prepare(int nx, int ny, int nz) {
  if (!fft_fused_supported(nx, ny, nz)) return FPM_ERR_UNSUPPORTED;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return FPM_ERR_CUDA;
  }
  {
    std::lock_guard<std::mutex> lock(g_tw_mu);
    if (!g_tw_ready[dev]) {
      float2 w[128];
      for (int m = 0; m < 128; ++m) {
        const double t = -2.0 * 3.14159265358979323846 * m / 128.0;
        w[m] = make_float2((float)std::cos(t), (float)std::sin(t));
      }
      if (cudaMemcpyToSymbol(c_w128, w, sizeof(w)) != cudaSuccess ||
          cudaMemcpyToSymbol(g_w128, w, sizeof(w)) != cudaSuccess) {
        cudaGetLastError();
        return FPM_ERR_CUDA;
      }
      g_tw_ready[dev] = true;
    }
  }
  if (nx == 128 && fft_xpass_prepare() != FPM_OK) return FPM_ERR_CUDA;
  const int M = nz / 2;
  switch (ny) {
#define FPM_PREP_CASE(NN) \
  case NN: return prepare_ny<NN>(M);
    FPM_FFT_SIZES(FPM_PREP_CASE)
#undef FPM_PREP_CASE
  }
  return FPM_ERR_UNSUPPORTED;
}

void launch_fft_force(const SimDev* sims, int first, int n, int nx, int ny,
                      int nz, float* rho, int zero_rho, float2* dk,
                      float2* fk, float* fmesh, float* phi, AxisTabs tabs,
                      const Green& G, bool grad3, cudaStream_t st) {
  if (n <= 0) return;
  g_launches.fetch_add(grad3 ? 3 : 4, std::memory_order_relaxed);
  switch (ny) {
#define FPM_NY_CASE(NN)                                                      \
  case NN:                                                                   \
    launch_ny<NN>(nz / 2, sims, first, n, nx, rho, zero_rho, dk, fk, fmesh,  \
                  phi, tabs, G, grad3, false, st);                           \
    break;
    FPM_FFT_SIZES(FPM_NY_CASE)
#undef FPM_NY_CASE
  }
}

void launch_fft_potential(const SimDev* sims, int first, int n, int nx,
                          int ny, int nz, const float* in, float2* dk,
                          float* out, AxisTabs tabs, const Green& G,
                          cudaStream_t st) {
  if (n <= 0) return;
  g_launches.fetch_add(3, std::memory_order_relaxed);
  float* src = const_cast<float*>(in);  // read only (zero_rho = 0)
  switch (ny) {
#define FPM_NY_CASE(NN)                                                   \
  case NN:                                                                \
    launch_ny<NN>(nz / 2, sims, first, n, nx, src, 0, dk, nullptr,        \
                  nullptr, out, tabs, G, false, true, st);                \
    break;
    FPM_FFT_SIZES(FPM_NY_CASE)
#undef FPM_NY_CASE
  }
}

size_t xpass_smem(int nx) { return (size_t)nx * kXCols * sizeof(float2); }

bool fft_xpass_supported(int nx, int ny, int nz) {
  return (nx == 256 || nx == 512) && ny % kXCols == 0 && nz % 2 == 0;
}

int fft_xpass_prepare() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return FPM_ERR_CUDA;
  }
  static bool ready[64] = {};
  std::lock_guard<std::mutex> lock(g_tw_mu);
  if (ready[dev]) return FPM_OK;
  float2 w[512];
  for (int m = 0; m < 512; ++m) {
    const double t = -2.0 * 3.14159265358979323846 * m / 512.0;
    w[m] = make_float2((float)std::cos(t), (float)std::sin(t));
  }
  float2 w128[128];
  for (int m = 0; m < 128; ++m) w128[m] = w[4 * m];
  if (cudaMemcpyToSymbol(g_w512, w, sizeof(w)) != cudaSuccess ||
      cudaMemcpyToSymbol(c_w128, w128, sizeof(w128)) != cudaSuccess ||
      cudaMemcpyToSymbol(g_w128, w128, sizeof(w128)) != cudaSuccess ||
      cudaFuncSetAttribute(k_fft_xcols<512>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)xpass_smem(512)) != cudaSuccess ||
      cudaFuncSetAttribute(k_fft_xcols<256>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)xpass_smem(256)) != cudaSuccess) {
    cudaGetLastError();
    return FPM_ERR_CUDA;
  }
  ready[dev] = true;
  return FPM_OK;
}

void launch_fft_xpass(const SimDev* sims, int first, int n, int nx, int ny,
                      int nzh, const float2* in, float2* out, float* rho_zero,
                      int zmul, AxisTabs tabs, const Green& G,
                      const int32_t* nsteps, int pos, cudaStream_t st) {
  if (n <= 0) return;
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const int nblk = ny * nzh / kXCols;
  const unsigned grid = (unsigned)(n * nblk);
  if (nx == 512)
    k_fft_xcols<512><<<grid, kXThreads, xpass_smem(512), st>>>(
        sims, first, nblk, in, out, rho_zero, zmul, tabs, G, nsteps, pos);
  else
    k_fft_xcols<256><<<grid, kXThreads, xpass_smem(256), st>>>(
        sims, first, nblk, in, out, rho_zero, zmul, tabs, G, nsteps, pos);
}

}  // namespace fpm
