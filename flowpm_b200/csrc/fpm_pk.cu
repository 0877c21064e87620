// Binned power spectrum on the device, the estimator of flowpm/pk.py:7-103
// (_initialize_pk / power_spectrum):
//   P[b] = (sum_{modes in bin b} W |F(k)|^2) / (sum_{modes in bin b} W)
//          * prod(boxsize) / (nx ny nz)^2,     b = 1 .. nedges - 1
// where F is the unnormalised FFT of the field, the bin of a mode is
// numpy.digitize(|k|, edges) with edges = kmin + n dk (n < nedges) and
// |k| = sqrt(sum_d (2 pi i_d / L_d)^2), and W is the reference's weight on
// the full spectrum: 1 on the z planes 0 and nz - 1, 2 elsewhere.  The sums
// run over the half spectrum of an R2C transform, each mode standing for
// itself and its Hermitian mirror (full-spectrum z index nz - l).
#include <cufft.h>

#include <atomic>
#include <map>
#include <mutex>
#include <tuple>

#include "fpm_kernels.cuh"

namespace fpm {

struct PkGeom {
  int nx, ny, nz, nzh;
  double vx, vy, vz;  // 2 pi / L_d: k_d = i_d * v_d
  double kmin, dk;
  int nedges;
};

__device__ __forceinline__ double pk_edge(const PkGeom& g, int n) {
  return g.kmin + (double)n * g.dk;  // numpy.arange(kmin, kmax, dk)[n]
}

// numpy.digitize(x, edges): number of edges <= x.
__device__ __forceinline__ int pk_bin(const PkGeom& g, double x) {
  int b = (int)floor((x - g.kmin) / g.dk) + 1;
  b = b < 0 ? 0 : (b > g.nedges ? g.nedges : b);
  while (b > 0 && x < pk_edge(g, b - 1)) --b;
  while (b < g.nedges && x >= pk_edge(g, b)) ++b;
  return b;
}

__device__ __forceinline__ int signed_freq(int i, int n) {
  return i < (n - 1) / 2 + 1 ? i : i - n;
}

// Full-spectrum weight W of z index l (flowpm/pk.py:12-15).
__device__ __forceinline__ double pk_w(int l, int nz) {
  return (l == 0 || l == nz - 1) ? 1.0 : 2.0;
}

// Accumulates, for every batch entry b, psum[b][bin] += w |F|^2 and
// nsum[b][bin] += w into scratch (2 * batch * (nedges + 1) doubles,
// zeroed by the caller).  With shared, per-block shared-memory histograms
// first (2 (nedges + 1) doubles of dynamic shared memory); without (bin
// counts whose histogram does not fit), straight into scratch.
__global__ void __launch_bounds__(256)
k_pk_accumulate(const float2* __restrict__ dk, int batch, PkGeom g,
                double* __restrict__ scratch, int shared) {
  extern __shared__ double sh_[];
  const int nb = g.nedges + 1;
  const int64_t nmodes = (int64_t)g.nx * g.ny * g.nzh;
  for (int b = 0; b < batch; ++b) {
    double* out = scratch + (int64_t)b * 2 * nb;
    double* sh = shared ? sh_ : out;
    if (shared) {
      for (int t = threadIdx.x; t < 2 * nb; t += blockDim.x) sh[t] = 0.0;
      __syncthreads();
    }
    const float2* f = dk + (int64_t)b * nmodes;
    for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
         m < nmodes; m += (int64_t)gridDim.x * blockDim.x) {
      int i, j, l;
      mode_ijl(m, g.ny, g.nzh, i, j, l);
      const double kx = signed_freq(i, g.nx) * g.vx;
      const double ky = signed_freq(j, g.ny) * g.vy;
      const double kz = signed_freq(l, g.nz) * g.vz;
      const double kmag = sqrt(kx * kx + ky * ky + kz * kz);
      double w = pk_w(l, g.nz);
      if (l != 0 && 2 * l != g.nz) w += pk_w(g.nz - l, g.nz);
      const float2 v = f[m];
      const double p2 = (double)v.x * v.x + (double)v.y * v.y;
      const int bin = pk_bin(g, kmag);
      atomicAdd(&sh[bin], w * p2);
      atomicAdd(&sh[nb + bin], w);
    }
    if (shared) {
      __syncthreads();
      for (int t = threadIdx.x; t < 2 * nb; t += blockDim.x)
        if (sh[t] != 0.0) atomicAdd(&out[t], sh[t]);
      __syncthreads();
    }
  }
}

// power[b][i] = psum[b][i+1] / nsum[b][i+1] * vol / ncell^2, i < nedges - 1.
__global__ void k_pk_finalize(const double* __restrict__ scratch, int batch,
                              int nedges, double scale,
                              float* __restrict__ power) {
  const int nb = nedges + 1, nout = nedges - 1;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < batch * nout;
       t += gridDim.x * blockDim.x) {
    const int b = t / nout, i = t - b * nout;
    const double* s = scratch + (int64_t)b * 2 * nb;
    power[t] = (float)(s[i + 1] / s[nb + i + 1] * scale);
  }
}

int pk_check(const void* dk, int batch, int nx, int ny, int nz,
             const double* boxsize, double dkw, int nedges, const float* power) {
  if (!dk || !power || !boxsize || batch < 1 || nx < 1 || ny < 1 || nz < 1 ||
      nedges < 2 || !(dkw > 0) || !(boxsize[0] > 0) || !(boxsize[1] > 0) ||
      !(boxsize[2] > 0))
    return FPM_ERR_ARG;
  return FPM_OK;
}

PkGeom pk_geom(int nx, int ny, int nz, const double* boxsize, double kmin,
               double dkw, int nedges) {
  PkGeom g;
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.nzh = nz / 2 + 1;
  // numpy.fft.fftfreq(N, 1 / (N 2 pi / L)) = i * (1 / (N d))
  const double dx = 1. / (nx * 2 * M_PI / boxsize[0]);
  const double dy = 1. / (ny * 2 * M_PI / boxsize[1]);
  const double dz = 1. / (nz * 2 * M_PI / boxsize[2]);
  g.vx = 1.0 / (nx * dx);
  g.vy = 1.0 / (ny * dy);
  g.vz = 1.0 / (nz * dz);
  g.kmin = kmin;
  g.dk = dkw;
  g.nedges = nedges;
  return g;
}

// Launch the accumulate + finalize pair on zeroed scratch.
int pk_launch(const float2* dk, int batch, const PkGeom& g, double* scratch,
              double vol, float* power, cudaStream_t st) {
  const int nb = g.nedges + 1;
  // Shared-memory histograms up to the default 48 KiB of dynamic shared
  // memory (3071 edges); larger bin counts accumulate in global memory.
  const size_t hist = 2 * sizeof(double) * (size_t)nb;
  const int shared = hist <= 48 * 1024 ? 1 : 0;
  const int64_t nmodes = (int64_t)g.nx * g.ny * g.nzh;
  int64_t blocks = (nmodes + 255) / 256;
  if (blocks > kNumSMs * 8) blocks = kNumSMs * 8;
  if (blocks < 1) blocks = 1;
  g_launches.fetch_add(2, std::memory_order_relaxed);
  k_pk_accumulate<<<(unsigned)blocks, 256, shared ? hist : 0, st>>>(
      dk, batch, g, scratch, shared);
  const double ncell = (double)g.nx * g.ny * g.nz;
  const int nout = batch * (g.nedges - 1);
  k_pk_finalize<<<(nout + 255) / 256, 256, 0, st>>>(
      scratch, batch, g.nedges, vol / (ncell * ncell), power);
  return cudaGetLastError() == cudaSuccess ? FPM_OK : FPM_ERR_CUDA;
}

}  // namespace fpm

using namespace fpm;

extern "C" int fpm_pk_bin(const void* delta_k, int batch, int nx, int ny,
                          int nz, const double* boxsize, double kmin,
                          double dk, int nedges, float* power, void* stream) {
  int rc = pk_check(delta_k, batch, nx, ny, nz, boxsize, dk, nedges, power);
  if (rc != FPM_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const PkGeom g = pk_geom(nx, ny, nz, boxsize, kmin, dk, nedges);
  const size_t n = 2 * (size_t)batch * (nedges + 1);
  double* scratch = nullptr;
  if (cudaMallocAsync((void**)&scratch, n * sizeof(double), st) != cudaSuccess) {
    cudaGetLastError();
    return FPM_ERR_OOM;
  }
  rc = cudaMemsetAsync(scratch, 0, n * sizeof(double), st) == cudaSuccess
           ? FPM_OK
           : FPM_ERR_CUDA;
  if (rc == FPM_OK)
    rc = pk_launch((const float2*)delta_k, batch, g, scratch,
                   boxsize[0] * boxsize[1] * boxsize[2], power, st);
  cudaFreeAsync(scratch, st);
  return rc;
}

namespace {
// R2C plans of fpm_power_spectrum per (device, batch, nx, ny, nz), at most
// kMaxPkPlans of them: past that the least recently used one is destroyed
// (cufftDestroy frees its work area with cudaFree, which waits for the work
// already queued on the device).  The lock is held while a plan is bound to
// the caller's stream and its transform is queued.
constexpr size_t kMaxPkPlans = 8;
struct PkPlan {
  cufftHandle h;
  uint64_t used;
};
std::mutex g_pk_mu;
std::map<std::tuple<int, int, int, int, int>, PkPlan> g_pk_plans;
uint64_t g_pk_tick = 0;
}  // namespace

extern "C" int fpm_power_spectrum(const float* field, int batch, int nx,
                                  int ny, int nz, const double* boxsize,
                                  double kmin, double dk, int nedges,
                                  float* power, void* stream) {
  if (!field) return FPM_ERR_ARG;
  int rc = pk_check(field, batch, nx, ny, nz, boxsize, dk, nedges, power);
  if (rc != FPM_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FPM_ERR_CUDA;
  const size_t nmodes = (size_t)batch * nx * ny * (nz / 2 + 1);
  float2* spec = nullptr;
  if (cudaMallocAsync((void**)&spec, nmodes * sizeof(float2), st) !=
      cudaSuccess) {
    cudaGetLastError();
    return FPM_ERR_OOM;
  }
  {
    std::lock_guard<std::mutex> lk(g_pk_mu);
    const auto key = std::make_tuple(dev, batch, nx, ny, nz);
    auto it = g_pk_plans.find(key);
    if (it == g_pk_plans.end()) {
      if (g_pk_plans.size() >= kMaxPkPlans) {
        auto old = g_pk_plans.begin();
        for (auto j = g_pk_plans.begin(); j != g_pk_plans.end(); ++j)
          if (j->second.used < old->second.used) old = j;
        cufftDestroy(old->second.h);
        g_pk_plans.erase(old);
      }
      int n[3] = {nx, ny, nz};
      cufftHandle h;
      if (cufftPlanMany(&h, 3, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C,
                        batch) != CUFFT_SUCCESS) {
        cudaFreeAsync(spec, st);
        return FPM_ERR_CUFFT;
      }
      it = g_pk_plans.emplace(key, PkPlan{h, 0}).first;
    }
    it->second.used = ++g_pk_tick;
    if (cufftSetStream(it->second.h, st) != CUFFT_SUCCESS ||
        cufftExecR2C(it->second.h, (cufftReal*)field, (cufftComplex*)spec) !=
            CUFFT_SUCCESS)
      rc = FPM_ERR_CUFFT;
  }
  if (rc == FPM_OK)
    rc = fpm_pk_bin(spec, batch, nx, ny, nz, boxsize, kmin, dk, nedges,
                    power, stream);
  cudaFreeAsync(spec, st);
  return rc;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of fpm_pk_bin.
//
// Some callers cannot let a library allocate device memory: applications
// that hand all of a GPU's memory to their own pool or arena (where a
// cudaMalloc / cudaMallocAsync from a library fails or fragments it), and
// latency-critical loops that forbid allocation after start-up because an
// allocation can synchronise the device.  For them the bin accumulators of
// the power spectrum live in a fixed file-scope device array instead of
// stream-ordered scratch.  The array is part of this library's module, so
// every GPU that loads the library holds it (128 KiB) until the process
// exits.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double
    g_pk_static_scratch[FPM_PK_NOALLOC_MAX_DOUBLES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
double* g_static_ptr[kMaxDevices] = {};

// Device address of g_pk_static_scratch on the current device.  On host,
// the name g_pk_static_scratch is only a stand-in for the device symbol,
// so its device address is looked up once per device (with that device
// current) and cached for the life of the process: a cudaDeviceReset,
// which unloads the module, is not supported in between.
int static_scratch(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FPM_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return FPM_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_pk_static_scratch) != cudaSuccess ||
        !p) {
      cudaGetLastError();
      return FPM_ERR_CUDA;
    }
    g_static_ptr[dev] = (double*)p;
  }
  *out = g_static_ptr[dev];
  return FPM_OK;
}

}  // namespace

extern "C" int fpm_pk_bin_noalloc(const void* delta_k, int batch, int nx,
                                  int ny, int nz, const double* boxsize,
                                  double kmin, double dk, int nedges,
                                  float* power, void* stream) {
  int rc = pk_check(delta_k, batch, nx, ny, nz, boxsize, dk, nedges, power);
  if (rc != FPM_OK) return rc;
  const int64_t n = 2 * (int64_t)batch * (nedges + 1);
  if (n > FPM_PK_NOALLOC_MAX_DOUBLES) return FPM_ERR_LIMIT;
  double* scratch = nullptr;
  rc = static_scratch(&scratch);
  if (rc != FPM_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // The array keeps the previous call's sums: clear the part this call uses.
  if (cudaMemsetAsync(scratch, 0, n * sizeof(double), st) != cudaSuccess)
    return FPM_ERR_CUDA;
  const PkGeom g = pk_geom(nx, ny, nz, boxsize, kmin, dk, nedges);
  return pk_launch((const float2*)delta_k, batch, g, scratch,
                   boxsize[0] * boxsize[1] * boxsize[2], power, st);
}
