// Plans, cuFFT orchestration and the C ABI of the particle-mesh step.
//
// A plan holds a set of simulations advanced together, their device
// descriptors, the per-axis Fourier tables, the mesh work buffers and the
// batched cuFFT plans (one set per run of consecutive simulations with equal
// dimensions).  Everything a call needs is allocated at creation, so the
// step entry points are stream-ordered launches only and can be captured in
// a CUDA graph.
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <tuple>
#include <vector>

#include "fpm_adjoint.cuh"
#include "fpm_bin.cuh"

using namespace fpm;

namespace {

// Kernels timed by fpm_plan_profile.
// 0 step, 1 Fourier solve, 2 initial paint, and on the cuFFT path of the
// solve 3 the Green's-function kernel, 4 the stencil gradient kernel;
// reverse sweep: 5 reverse drift + paint, 6 force VJP, 7 divergence
// stencil, 8 adjoint potential solve, 9 the whole reverse step; 10 the
// particle sort of the binned step (fpm_plan_set_binning)
constexpr int kProfKinds = 11;

// Particles per thread of the lattice blocks of lattices of 2^26 particles
// or more (x extent twice that).
#ifndef FPM_WALK_LARGE
#define FPM_WALK_LARGE 32
#endif

struct Run {
  int first, count;        // simulations [first, first + count)
  bool fused = false;      // force meshes by the fused Fourier solve
  bool xpass = false;      // r2c / c2r1 are batched (y, z) plane transforms
                           // around the x-pass kernel
  int div_xc = 0;          // x chunk of the tiled divergence stencil
  // Simulations of the run still active at leapfrog position it (a prefix
  // when the run is ordered by non-increasing step count), and the batched
  // cuFFT plans of each smaller active count.
  std::vector<int> active;
  int64_t bsum_off = 0;    // this run's chunk sums in fpm_plan::bsums
  int min_steps = 0;       // fewest leapfrog steps of the run's simulations
  int max_steps = 0;       // most leapfrog steps of the run's simulations
  std::map<int, cufftHandle> r2c_n, c2r3_n, r2c3_n, c2r1_n;
  cufftHandle r2c = 0, c2r3 = 0;     // force mesh
  cufftHandle r2c3 = 0, c2r1 = 0;    // force mesh, adjoint
  cufftHandle lr2c = 0, lc2r9 = 0, lc2r3 = 0, lc2r1 = 0;  // lattice
  cufftHandle lr2c3 = 0, lr2c9 = 0;  // lattice, adjoint
};

template <typename T>
T* dalloc(size_t n, size_t& total, bool& ok) {
  if (!ok || n == 0) return nullptr;
  void* p = nullptr;
  if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) {
    ok = false;
    return nullptr;
  }
  total += n * sizeof(T);
  return (T*)p;
}

}  // namespace

struct fpm_plan {
  int nsims = 0;
  unsigned flags = 0;
  double r_split = 0;
  std::vector<SimDev> sims;
  std::vector<Run> runs;
  SimDev* d_sims = nullptr;
  int64_t total_np = 0, total_m = 0, total_s = 0, total_l = 0, total_ls = 0;
  int64_t ch_p = 0, ch_s = 0, ch_m = 0, ch_l = 0, ch_ls = 0, ch_b = 0;
  // tables
  double* d_kk = nullptr;
  float* d_grad = nullptr;
  float* d_win = nullptr;
  // force-mesh buffers
  float* rho = nullptr;
  float2* dk = nullptr;
  float2* fk = nullptr;
  float* fmesh = nullptr;
  float* phi = nullptr;     // potential mesh (stencil force path)
  float* tape = nullptr;    // caller's potential tape: position it at
                            // tape + it * total_m (fpm_nbody_set_tape)
  int64_t tape_floats = 0;
  bool quads = false;       // every mesh: mz % 4 == 0 and m_off % 4 == 0
  bool div_tiled = false;   // every run takes the tiled divergence stencil
  // side streams for the fused-solve runs after the first (created with
  // the plan), and the events that fork them off and join them back
  std::vector<cudaStream_t> side;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
  bool all_xpass = false;   // every run on the x-pass path: its x pass in
                            // the reverse sweep zeroes the adjoint force
                            // mesh after the divergence has read it
  // lattice buffers (FPM_PLAN_LPT)
  float* lreal1 = nullptr;
  float2* lspec1 = nullptr;
  float2* lspec9 = nullptr;
  float* lreal9 = nullptr;
  float* lreal3 = nullptr;
  // adjoint buffers (FPM_PLAN_ADJOINT)
  float* lmesh = nullptr;   // adjoint force meshes (float4 per cell on the
                            // stencil path, else 3 planes)
  float* lrho = nullptr;    // adjoint density mesh
  float* fpart = nullptr;   // per-particle force of the reverse sweep
  // parameters
  float* d_coefs = nullptr;
  int coef_cap = 0;     // steps capacity of d_coefs
  int max_steps = 0;
  int32_t* d_nsteps = nullptr;
  float* d_ffac = nullptr;
  float* d_lcoef = nullptr;
  // PGD correction: (alpha, kl, ks) per sim and step (stride coef_cap), and
  // per sim for one fpm_pgd call
  float* d_pgd = nullptr;
  int pgd_cap = 0;
  bool pgd_on = false;
  float* d_pgd1 = nullptr;
  int32_t* d_status = nullptr;
  void* work = nullptr;
  size_t device_bytes = 0;
  bool steps_set = false;
  int64_t coef_gen = 0;   // bumped whenever d_coefs is reallocated
  int64_t sched_gen = 0;  // bumped whenever the active-prefix schedule moves
  size_t work_bytes = 0;  // size of the shared cuFFT work area
  // Eulerian binning of the forward step (fpm_plan_set_binning): tile size
  // (0: the lattice walk), sort period, the sorted state in two buffers,
  // the carried Lagrangian indices, per-cell counts / end slots and the
  // scan's chunk sums
  int bin_tile = 0;
  int bin_every = 1;
  int bin_mode = FPM_BIN_TILES;
  int64_t total_tiles = 0;
  float* bd[2] = {nullptr, nullptr};
  float* bp[2] = {nullptr, nullptr};
  uint32_t* blag[2] = {nullptr, nullptr};
  int32_t* bcell = nullptr;
  int32_t* bcount = nullptr;  // per-cell counts, zero between sorts
  int32_t* bsums = nullptr;
  size_t bin_bytes = 0;
  // the reverse sweep in the binned order (fpm_plan_set_adjoint_binning):
  // sort period in positions (0: the lattice walk) and the sorted
  // cotangents (lam_x, lam_p) in two buffers; the state uses bd / bp
  int adj_every = 0;
  int adj_req = 0;  // the period asked for, kept across tile changes
  float* blx[2] = {nullptr, nullptr};
  float* blp[2] = {nullptr, nullptr};
  size_t adj_bin_bytes = 0;
  // optional per-kernel timing (fpm_plan_profile)
  bool profile = false;
  std::vector<cudaEvent_t> ev[kProfKinds];
  size_t ev_used[kProfKinds] = {};
};

namespace {

AxisTabs tabs_of(const fpm_plan* p) { return AxisTabs{p->d_kk, p->d_grad, p->d_win}; }

Green plan_green(const fpm_plan* p) {
  return force_green(p->r_split * p->r_split,
                     (p->flags & FPM_PLAN_CIC_DECONV) ? 1 : 0);
}

// PGD transfer function of step `pos` (table d_pgd) or of one fpm_pgd call.
Green pgd_green(const fpm_plan* p, int pos, bool single) {
  Green g = force_green(0.0, 0);
  g.pgd = single ? p->d_pgd1 : p->d_pgd;
  g.pgd_stride = single ? 1 : p->pgd_cap;
  g.pos = single ? 0 : pos;
  return g;
}

// Chunks of the mesh-touching particle kernels (see kTraverse).
int64_t traverse_chunks(const fpm_plan* p) {
  return FPM_STEP_BLOCKED ? p->ch_b : p->ch_p;
}

// Record the next timing event of `kind` on st (no-op unless profiling).
void prof_mark(fpm_plan* p, int kind, cudaStream_t st) {
  if (!p->profile) return;
  auto& v = p->ev[kind];
  if (p->ev_used[kind] == v.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    v.push_back(e);
  }
  cudaEventRecord(v[p->ev_used[kind]++], st);
}

void destroy_handles(fpm_plan* p) {
  for (auto& r : p->runs) {
    for (auto* m : {&r.r2c_n, &r.c2r3_n, &r.r2c3_n, &r.c2r1_n}) {
      for (auto& kv : *m) cufftDestroy(kv.second);
      m->clear();
    }
    cufftHandle* hs[] = {&r.r2c,   &r.c2r3,  &r.r2c3,  &r.c2r1, &r.lr2c,
                         &r.lc2r9, &r.lc2r3, &r.lc2r1, &r.lr2c3, &r.lr2c9};
    for (cufftHandle* h : hs)
      if (*h) {
        cufftDestroy(*h);
        *h = 0;
      }
  }
}

void free_all(fpm_plan* p) {
  destroy_handles(p);
  for (cudaStream_t s : p->side) cudaStreamDestroy(s);
  for (cudaEvent_t e : p->ev_join) cudaEventDestroy(e);
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  for (int k = 0; k < kProfKinds; ++k)
    for (cudaEvent_t e : p->ev[k]) cudaEventDestroy(e);
  void* bufs[] = {p->d_sims, p->d_kk,   p->d_grad,  p->d_win,   p->rho,
                  p->dk,     p->fk,     p->fmesh,   p->lreal1,  p->lspec1,
                  p->lspec9, p->lreal9, p->lreal3,  p->d_coefs, p->d_nsteps,
                  p->d_ffac, p->d_lcoef, p->d_status, p->work, p->d_pgd,
                  p->d_pgd1,
                  p->lmesh,  p->lrho,   p->fpart,   p->phi};
  for (void* b : bufs)
    if (b) cudaFree(b);
  void* bins[] = {p->bd[0],   p->bd[1],  p->bp[0],  p->bp[1],
                  p->blag[0], p->blag[1], p->bcell,  p->bsums, p->bcount,
                  p->blx[0],  p->blx[1], p->blp[0], p->blp[1]};
  for (void* b : bins)
    if (b) cudaFree(b);
}

// k = 2 pi fftfreq(i, n) exactly as numpy: (i * (1/n)) * (2 pi), with
// i -> i - n for i >= (n + 1) / 2 (flowpm/kernels.py:16-17).
double kfreq(int i, int n) {
  const int half = (n - 1) / 2 + 1;
  const double v = 1.0 / (double)n;
  const double f = (double)(i < half ? i : i - n) * v;
  return f * (2.0 * M_PI);
}

void axis_tables(int n, bool order0, std::vector<double>& kk,
                 std::vector<float>& grad, std::vector<float>& win) {
  for (int i = 0; i < n; ++i) {
    const double k = kfreq(i, n);
    kk.push_back(k * k);
    double g;
    if (order0) {
      g = (i == n / 2) ? 0.0 : k;  // kernels.py:66-70 zeroes entry len//2
    } else {
      g = 1 / 6.0 * (8 * std::sin(k) - std::sin(2 * k));  // kernels.py:75
    }
    grad.push_back((float)g);
    const double x = k / (2 * M_PI);
    const double sc = x == 0.0 ? 1.0 : std::sin(M_PI * x) / (M_PI * x);
    win.push_back((float)(1.0 / (sc * sc)));
  }
}

int make_plan(cufftHandle* h, int nx, int ny, int nz, cufftType type,
              int batch, size_t* ws) {
  if (cufftCreate(h) != CUFFT_SUCCESS) return FPM_ERR_CUFFT;
  if (cufftSetAutoAllocation(*h, 0) != CUFFT_SUCCESS) return FPM_ERR_CUFFT;
  long long n[3] = {nx, ny, nz};
  size_t w = 0;
  cufftResult r = cufftMakePlanMany64(*h, 3, n, nullptr, 1, 0, nullptr, 1, 0,
                                      type, batch, &w);
  if (r == CUFFT_ALLOC_FAILED) return FPM_ERR_OOM;
  if (r != CUFFT_SUCCESS) return FPM_ERR_CUFFT;
  if (w > *ws) *ws = w;
  return FPM_OK;
}

int exec_r2c(cufftHandle h, float* in, float2* out, cudaStream_t st) {
  if (cufftSetStream(h, st) != CUFFT_SUCCESS) return FPM_ERR_CUFFT;
  return cufftExecR2C(h, in, (cufftComplex*)out) == CUFFT_SUCCESS
             ? FPM_OK
             : FPM_ERR_CUFFT;
}

int exec_c2r(cufftHandle h, float2* in, float* out, cudaStream_t st) {
  if (cufftSetStream(h, st) != CUFFT_SUCCESS) return FPM_ERR_CUFFT;
  return cufftExecC2R(h, (cufftComplex*)in, out) == CUFFT_SUCCESS
             ? FPM_OK
             : FPM_ERR_CUFFT;
}

int launch_ok() {
  return cudaGetLastError() == cudaSuccess ? FPM_OK : FPM_ERR_CUDA;
}

#define FPM_TRY(x)            \
  do {                        \
    int rc_ = (x);            \
    if (rc_ != FPM_OK) return rc_; \
  } while (0)

#define FPM_CUDA(x) \
  do {              \
    if ((x) != cudaSuccess) return FPM_ERR_CUDA; \
  } while (0)

// Simulations of run r active at position it (all when it < 0).
int run_active(const Run& r, int it) {
  if (it < 0 || it >= (int)r.active.size()) return r.count;
  return r.active[it];
}

// Batched two-dimensional (y, z) transforms of `planes` consecutive x
// planes, in cuFFT's default layout: the spectrum of plane x at
// x * ny * (nz/2 + 1), the layout of the three-dimensional R2C.
int make_plane_plan(cufftHandle* h, int ny, int nz, cufftType type,
                    int planes, size_t* ws) {
  if (cufftCreate(h) != CUFFT_SUCCESS) return FPM_ERR_CUFFT;
  if (cufftSetAutoAllocation(*h, 0) != CUFFT_SUCCESS) return FPM_ERR_CUFFT;
  long long n[2] = {ny, nz};
  size_t w = 0;
  cufftResult r = cufftMakePlanMany64(*h, 2, n, nullptr, 1, 0, nullptr, 1, 0,
                                      type, planes, &w);
  if (r == CUFFT_ALLOC_FAILED) return FPM_ERR_OOM;
  if (r != CUFFT_SUCCESS) return FPM_ERR_CUFFT;
  if (w > *ws) *ws = w;
  return FPM_OK;
}

// The force-mesh R2C (or C2R) of n sims of run r: three-dimensional, or
// the plane transforms of the x-pass path.
int make_mesh_plan(cufftHandle* h, const Run& r, const SimDev& S,
                   cufftType type, int n, size_t* ws) {
  if (r.xpass) return make_plane_plan(h, S.my, S.mz, type, S.mx * n, ws);
  return make_plan(h, S.mx, S.my, S.mz, type, n, ws);
}

// Plan for `n` of the run's simulations: the full-run plan or the one of
// the smaller active prefix.
cufftHandle pick(const Run& r, int n, cufftHandle full,
                 const std::map<int, cufftHandle>& m) {
  if (n == r.count) return full;
  auto it = m.find(n);
  return it == m.end() ? full : it->second;
}

// True for the default force path: potential spectrum, one C2R, and the
// 4-point gradient as a real-space stencil.  The order-0 gradient i k has
// no finite stencil and keeps three spectra and a batched C2R.
bool stencil_path(const fpm_plan* p) {
  return (p->flags & FPM_PLAN_GRAD_ORDER0) == 0;
}

// The potential spectrum out = pre w(k) in of the sims on the cuFFT path
// (k_fourier_potential), or, for runs on the x-pass path, the x pass that
// wraps it (both skip the sims with nsteps < pos when act is given); with
// rho_zero, their density meshes are zeroed.
void potential_modes(fpm_plan* p, const float2* in, float2* out,
                     float* rho_zero, const Green& G, const int32_t* act,
                     int pos, cudaStream_t st, int zmul = 1) {
  bool other = false;
  for (auto& r : p->runs) {
    if (r.fused) continue;
    if (!r.xpass) {
      other = true;
      continue;
    }
    const int n = run_active(r, pos);
    const SimDev& S = p->sims[r.first];
    launch_fft_xpass(p->d_sims, r.first, n, S.mx, S.my, S.mzh, in, out,
                     rho_zero, zmul, tabs_of(p), G, act, pos, st);
  }
  if (other)
    launch_fourier_potential(p->d_sims, p->nsims, p->ch_s, in, out, rho_zero,
                             tabs_of(p), G, act, pos, 1, st);
}

// The three force meshes D_d phi of the sims (with act, those with nsteps
// >= pos; with skip_fused, not the fused-solve runs, which make their own):
// the tiled stencil when every run takes the tiled stencils, else the
// per-chunk one.
void stencil_grad(fpm_plan* p, const float* phi, const int32_t* act, int pos,
                  int skip_fused, cudaStream_t st) {
  if (!p->div_tiled) {
    launch_stencil_grad(p->d_sims, p->nsims, p->ch_m, phi, p->fmesh, act, pos,
                        skip_fused, p->quads, st);
    return;
  }
  for (auto& r : p->runs) {
    if (skip_fused && r.fused) continue;
    const int n = run_active(r, pos);
    if (n == 0) continue;
    const SimDev& S = p->sims[r.first];
    launch_stencil_grad_tiled(p->d_sims, r.first, n, S.mx, S.my, S.mz,
                              r.div_xc, phi, p->fmesh, act, pos, st);
  }
}

// Density of the current positions -> force meshes (paint must be done).
// At leapfrog position it (>= 0) only the active prefix of each run is
// transformed.
int force_meshes(fpm_plan* p, cudaStream_t st, bool zero_rho, int it = -1,
                 float* phi = nullptr) {
  if (!phi) phi = p->phi;  // potential mesh of the stencil path
  const int32_t* act = it >= 0 ? p->d_nsteps : nullptr;
  const double r2 = p->r_split * p->r_split;
  const int deconv = (p->flags & FPM_PLAN_CIC_DECONV) ? 1 : 0;
  const Green G = plan_green(p);
  // profile kind 1 brackets the whole solve, density -> force meshes
  bool any_cufft = false;
  prof_mark(p, 1, st);
  // runs on the fused solve: a few launches each, straight to fmesh.  With
  // several, the second and later go to the plan's side streams, so that
  // the latency-bound kernels of the small runs overlap the large run's
  // (the runs touch disjoint parts of every buffer)
  int forked = 0;
  for (auto& r : p->runs) {
    if (!r.fused) {
      any_cufft = true;
      continue;
    }
    const SimDev& S = p->sims[r.first];
    const int n = run_active(r, it);
    if (n == 0) continue;
    cudaStream_t rs = st;
    if (forked > 0 || !p->side.empty()) {
      if (forked == 0) {
        rs = st;  // the first active run stays on the call's stream
        FPM_CUDA(cudaEventRecord(p->ev_fork, st));
      } else {
        rs = p->side[(forked - 1) % p->side.size()];
        if (forked - 1 < (int)p->side.size())
          FPM_CUDA(cudaStreamWaitEvent(rs, p->ev_fork, 0));
      }
    }
    launch_fft_force(p->d_sims, r.first, n, S.mx, S.my, S.mz, p->rho,
                     zero_rho ? 1 : 0, p->dk, p->fk, p->fmesh, phi,
                     tabs_of(p), G, !stencil_path(p), rs);
    ++forked;
  }
  for (int k = 0; k + 1 < forked && k < (int)p->side.size(); ++k) {
    FPM_CUDA(cudaEventRecord(p->ev_join[k], p->side[k]));
    FPM_CUDA(cudaStreamWaitEvent(st, p->ev_join[k], 0));
  }
  FPM_TRY(launch_ok());
  if (!any_cufft) {
    prof_mark(p, 1, st);
    return FPM_OK;
  }
  for (auto& r : p->runs) {
    if (r.fused) continue;
    const SimDev& S = p->sims[r.first];
    const int n = run_active(r, it);
    if (n == 0) continue;
    FPM_TRY(exec_r2c(pick(r, n, r.r2c, r.r2c_n), p->rho + S.m_off,
                     p->dk + S.s_off, st));
  }
  prof_mark(p, 3, st);
  if (stencil_path(p)) {
    potential_modes(p, p->dk, p->fk, zero_rho ? p->rho : nullptr, G, act, it,
                    st);
  } else {
    launch_fourier_force(p->d_sims, p->nsims, p->ch_s, p->dk, p->fk,
                         zero_rho ? p->rho : nullptr, tabs_of(p), r2, deconv,
                         act, it, 1, st);
  }
  prof_mark(p, 3, st);
  FPM_TRY(launch_ok());
  for (auto& r : p->runs) {
    if (r.fused) continue;
    const SimDev& S = p->sims[r.first];
    const int n = run_active(r, it);
    if (n == 0) continue;
    if (stencil_path(p))
      FPM_TRY(exec_c2r(pick(r, n, r.c2r1, r.c2r1_n), p->fk + S.s_off,
                       phi + S.m_off, st));
    else
      FPM_TRY(exec_c2r(pick(r, n, r.c2r3, r.c2r3_n), p->fk + 3 * S.s_off,
                       p->fmesh + 3 * S.m_off, st));
  }
  if (stencil_path(p)) {
    prof_mark(p, 4, st);
    stencil_grad(p, phi, act, it, 1, st);
    prof_mark(p, 4, st);
    FPM_TRY(launch_ok());
  }
  prof_mark(p, 1, st);
  return FPM_OK;
}

// PGD displacement meshes (into fmesh) of the density in rho, which is
// zeroed: the force solve's path with the PGD transfer function and the
// 4-point stencil gradient (flowpm/tfpm.py:222-270 uses order 1 whatever
// the force's gradient).  pos >= 0: the sims still moving at step pos
// (nsteps > pos) with the parameters of step pos; pos < 0: every sim with
// the parameters of one fpm_pgd call.
int pgd_meshes(fpm_plan* p, cudaStream_t st, int pos, float* phi = nullptr) {
  if (!phi) phi = p->phi;
  const bool single = pos < 0;
  const Green G = pgd_green(p, pos, single);
  const int32_t* act = single ? nullptr : p->d_nsteps;
  const int apos = single ? -1 : pos + 1;  // sims with nsteps >= pos + 1
  bool any_cufft = false;
  for (auto& r : p->runs) {
    if (!r.fused) {
      any_cufft = true;
      continue;
    }
    const SimDev& S = p->sims[r.first];
    const int n = run_active(r, apos);
    if (n == 0) continue;
    launch_fft_force(p->d_sims, r.first, n, S.mx, S.my, S.mz, p->rho, 1,
                     p->dk, p->fk, p->fmesh, phi, tabs_of(p), G, false, st);
  }
  FPM_TRY(launch_ok());
  if (!any_cufft) return FPM_OK;
  for (auto& r : p->runs) {
    if (r.fused) continue;
    const SimDev& S = p->sims[r.first];
    const int n = run_active(r, apos);
    if (n == 0) continue;
    FPM_TRY(exec_r2c(pick(r, n, r.r2c, r.r2c_n), p->rho + S.m_off,
                     p->dk + S.s_off, st));
  }
  potential_modes(p, p->dk, p->fk, p->rho, G, act, apos, st);
  FPM_TRY(launch_ok());
  for (auto& r : p->runs) {
    if (r.fused) continue;
    const SimDev& S = p->sims[r.first];
    const int n = run_active(r, apos);
    if (n == 0) continue;
    FPM_TRY(exec_c2r(pick(r, n, r.c2r1, r.c2r1_n), p->fk + S.s_off,
                     phi + S.m_off, st));
  }
  stencil_grad(p, phi, act, apos, 1, st);
  return launch_ok();
}

// Potential tape layout: the force potential of position it (0..T) at
// it * Nc; with PGD, the PGD potential of step it (0..T-1) at
// (T + 1 + it) * Nc and the displacement before the PGD move of step it at
// (2T + 1) * Nc + 3 it Np (Nc, Np: the plan's mesh cells and particles).
int64_t tape_needed(const fpm_plan* p) {
  int64_t n = (int64_t)(p->max_steps + 1) * p->total_m;
  if (p->pgd_on)
    n += (int64_t)p->max_steps * (p->total_m + 3 * p->total_np);
  return n;
}
float* tape_phi(const fpm_plan* p, int it) {
  return p->tape + (size_t)it * p->total_m;
}
float* tape_pgd_phi(const fpm_plan* p, int it) {
  return p->tape + (size_t)(p->max_steps + 1 + it) * p->total_m;
}
float* tape_pgd_disp(const fpm_plan* p, int it) {
  return p->tape + (size_t)(2 * p->max_steps + 1) * p->total_m +
         (size_t)it * 3 * p->total_np;
}

// Per run and position, the active prefix of the run; batched cuFFT plans
// for every prefix length used, sharing the plan's work area.
int update_schedule(fpm_plan* p, int max_steps, const int32_t* nsteps,
                    cudaStream_t st) {
  bool changed = false;
  const bool adj = (p->flags & FPM_PLAN_ADJOINT) != 0;
  for (auto& r : p->runs) {
    bool prefix = true;
    for (int s = r.first + 1; s < r.first + r.count; ++s)
      if (nsteps[s] > nsteps[s - 1]) prefix = false;
    r.min_steps = r.max_steps = nsteps[r.first];
    for (int s = r.first + 1; s < r.first + r.count; ++s) {
      r.min_steps = std::min(r.min_steps, (int)nsteps[s]);
      r.max_steps = std::max(r.max_steps, (int)nsteps[s]);
    }
    std::vector<int> act(max_steps + 1, r.count);
    if (prefix)
      for (int it = 0; it <= max_steps; ++it) {
        int n = 0;
        while (n < r.count && nsteps[r.first + n] >= it) ++n;
        act[it] = n;
      }
    if (act != r.active) changed = true;
    r.active = act;
    const SimDev& S = p->sims[r.first];
    for (int n : act) {
      if (n == 0 || n == r.count || r.r2c_n.count(n)) continue;
      size_t ws = 0;
      cufftHandle a = 0, b = 0, c = 0, d = 0;
      int rc = make_mesh_plan(&a, r, S, CUFFT_R2C, n, &ws);
      if (rc == FPM_OK)
        rc = make_plan(&b, S.mx, S.my, S.mz, CUFFT_C2R, 3 * n, &ws);
      if (adj && rc == FPM_OK)
        rc = make_plan(&c, S.mx, S.my, S.mz, CUFFT_R2C, 3 * n, &ws);
      if (rc == FPM_OK) rc = make_mesh_plan(&d, r, S, CUFFT_C2R, n, &ws);
      if (rc == FPM_OK && ws > p->work_bytes) rc = FPM_ERR_UNSUPPORTED;
      for (cufftHandle h : {a, b, c, d})
        if (rc == FPM_OK && h && cufftSetWorkArea(h, p->work) != CUFFT_SUCCESS)
          rc = FPM_ERR_CUFFT;
      if (rc != FPM_OK) {
        for (cufftHandle h : {a, b, c, d})
          if (h) cufftDestroy(h);
        // fall back to full-run transforms for this run
        std::fill(r.active.begin(), r.active.end(), r.count);
        changed = true;
        break;
      }
      r.r2c_n[n] = a;
      r.c2r3_n[n] = b;
      r.c2r1_n[n] = d;
      if (adj) r.r2c3_n[n] = c;
    }
  }
  (void)st;
  if (changed) p->sched_gen++;
  return FPM_OK;
}

int upload_ffac(fpm_plan* p, const double* force_fac, cudaStream_t st) {
  std::vector<float> f(p->nsims);
  for (int s = 0; s < p->nsims; ++s) f[s] = (float)force_fac[s];
  FPM_CUDA(cudaMemcpyAsync(p->d_ffac, f.data(), sizeof(float) * p->nsims,
                           cudaMemcpyHostToDevice, st));
  return FPM_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" int fpm_version(void) { return 100; }

extern "C" const char* fpm_error_string(int code) {
  switch (code) {
    case FPM_OK: return "ok";
    case FPM_ERR_ARG: return "invalid argument";
    case FPM_ERR_ALIGN: return "misaligned pointer";
    case FPM_ERR_OOM: return "out of device memory";
    case FPM_ERR_CUDA: return "CUDA runtime error";
    case FPM_ERR_CUFFT: return "cuFFT error";
    case FPM_ERR_NONFINITE: return "non-finite particle state";
    case FPM_ERR_STATE: return "call out of order";
    case FPM_ERR_UNSUPPORTED: return "unsupported request";
    case FPM_ERR_LIMIT:
      return "request exceeds the fixed scratch of an allocation-free entry";
    case FPM_ERR_RANGE: return "deposit outside the mesh";
    default: return "unknown error";
  }
}

extern "C" int fpm_plan_create(fpm_plan** out, int nsims, const int32_t* dims,
                               double r_split, unsigned flags) {
  if (!out || nsims < 1 || !dims || r_split < 0) return FPM_ERR_ARG;
  *out = nullptr;
  fpm_plan* p = new (std::nothrow) fpm_plan();
  if (!p) return FPM_ERR_OOM;
  p->nsims = nsims;
  p->flags = flags;
  p->r_split = r_split;
  std::vector<double> kk;
  std::vector<float> grad, win;
  const bool order0 = (flags & FPM_PLAN_GRAD_ORDER0) != 0;
  const int64_t kMaxCells = (int64_t)1 << 31;
  for (int s = 0; s < nsims; ++s) {
    SimDev S;
    std::memset(&S, 0, sizeof(S));
    S.nx = dims[4 * s];
    S.ny = dims[4 * s + 1];
    S.nz = dims[4 * s + 2];
    S.bf = dims[4 * s + 3];
    if (S.nx < 2 || S.ny < 2 || S.nz < 2 || S.bf < 1 || S.bf > 8) {
      delete p;
      return FPM_ERR_ARG;
    }
    S.mx = S.nx * S.bf;
    S.my = S.ny * S.bf;
    S.mz = S.nz * S.bf;
    if ((int64_t)S.mx * S.my * S.mz >= kMaxCells) {
      delete p;
      return FPM_ERR_UNSUPPORTED;
    }
    S.mzh = S.mz / 2 + 1;
    S.lzh = S.nz / 2 + 1;
    S.np = (int64_t)S.nx * S.ny * S.nz;
    S.p_off = p->total_np;
    S.m_off = p->total_m;
    S.s_off = p->total_s;
    S.l_off = p->total_l;
    S.ls_off = p->total_ls;
    const int64_t nm = (int64_t)S.mx * S.my * S.mz;
    const int64_t ns = (int64_t)S.mx * S.my * S.mzh;
    const int64_t nls = (int64_t)S.nx * S.ny * S.lzh;
    S.ch_p = p->ch_p;
    S.ch_s = p->ch_s;
    S.ch_m = p->ch_m;
    S.ch_l = p->ch_l;
    S.ch_ls = p->ch_ls;
    // larger lattice blocks for large lattices: the items of a thread walk
    // along x, each reusing in L1 the cells of the previous one.  Measured
    // at 2 x 512^3: k_step 9.14 / 8.90 / 8.73 / 8.70 ms and the reverse
    // position 18.1 / 17.5 / 17.3 / 17.1 ms at wi = 4 / 8 / 16 / 32; at
    // 128^3 wi = 4 is best (k_step 85 / 87 / 97 us at 4 / 8 / 16), larger
    // blocks leaving too few of them for the SMs
    S.wi = !FPM_STEP_BLOCKED ? kItems
           : (flags & FPM_PLAN_SMALL_BLOCKS) ? 4
           : S.np >= ((int64_t)1 << 26) ? FPM_WALK_LARGE
           : S.np >= ((int64_t)1 << 23) ? 8 : 4;
    S.nbi = (S.nx + kPlanes * S.wi - 1) / (kPlanes * S.wi);
    S.nbj = (S.ny + kBJ - 1) / kBJ;
    S.nbk = (S.nz + kBK - 1) / kBK;
    S.ch_b = p->ch_b;
    p->ch_b += (int64_t)S.nbi * S.nbj * S.nbk;
    p->ch_p += (S.np + kChunk - 1) / kChunk;
    p->ch_s += (ns + kChunk - 1) / kChunk;
    p->ch_m += (nm + kChunk - 1) / kChunk;
    p->ch_l += (S.np + kChunk - 1) / kChunk;
    p->ch_ls += (nls + kChunk - 1) / kChunk;
    p->total_np += S.np;
    p->total_m += nm;
    p->total_s += ns;
    p->total_l += S.np;
    p->total_ls += nls;
    S.tab = (int)kk.size();
    axis_tables(S.mx, order0, kk, grad, win);
    axis_tables(S.my, order0, kk, grad, win);
    axis_tables(S.mz, order0, kk, grad, win);
    S.ltab = (int)kk.size();
    axis_tables(S.nx, order0, kk, grad, win);
    axis_tables(S.ny, order0, kk, grad, win);
    axis_tables(S.nz, order0, kk, grad, win);
    p->sims.push_back(S);
    if (s > 0 && dims[4 * s] == dims[4 * s - 4] &&
        dims[4 * s + 1] == dims[4 * s - 3] &&
        dims[4 * s + 2] == dims[4 * s - 2] &&
        dims[4 * s + 3] == dims[4 * s - 1]) {
      p->runs.back().count++;
    } else {
      Run r;
      r.first = s;
      r.count = 1;
      p->runs.push_back(r);
    }
  }

  p->quads = true;
  for (const SimDev& S : p->sims)
    if (S.mz % 4 != 0 || S.m_off % 4 != 0) p->quads = false;
  p->div_tiled = true;
  for (auto& r : p->runs) {
    const SimDev& S0 = p->sims[r.first];
    r.div_xc = stencil_div_chunk(S0.mx, S0.my, S0.mz, S0.m_off, r.count);
    for (int s = r.first; s < r.first + r.count; ++s)
      if (p->sims[s].m_off % 4 != 0) r.div_xc = 0;
    if (r.div_xc == 0) p->div_tiled = false;
  }
  int rc = FPM_OK;
  size_t ws = 0;
  const bool lpt = (flags & FPM_PLAN_LPT) != 0;
  const bool adj = (flags & FPM_PLAN_ADJOINT) != 0;
  for (auto& r : p->runs) {
    const SimDev& S0 = p->sims[r.first];
    // the fused kernels move density and force planes as float4
    bool aligned = true;
    for (int s = r.first; s < r.first + r.count; ++s)
      if (p->sims[s].m_off % 4 != 0) aligned = false;
    if (!(flags & FPM_PLAN_CUFFT) && aligned &&
        fft_fused_supported(S0.mx, S0.my, S0.mz) &&
        fft_fused_prepare(S0.mx, S0.my, S0.mz) == FPM_OK) {
      r.fused = true;
      for (int s = r.first; s < r.first + r.count; ++s) p->sims[s].fused = 1;
    }
  }
  for (auto& r : p->runs) {
    if (r.fused || (flags & FPM_PLAN_CUFFT) || (flags & FPM_PLAN_GRAD_ORDER0))
      continue;
    const SimDev& S0 = p->sims[r.first];
    bool aligned = true;  // float4 spectrum rows and density zeroing
    for (int s = r.first; s < r.first + r.count; ++s)
      if (p->sims[s].s_off % 2 != 0 || p->sims[s].m_off % 4 != 0)
        aligned = false;
    if (aligned && fft_xpass_supported(S0.mx, S0.my, S0.mz) &&
        fft_xpass_prepare() == FPM_OK) {
      r.xpass = true;
      for (int s = r.first; s < r.first + r.count; ++s) p->sims[s].xpass = 1;
    }
  }
  p->all_xpass = !p->runs.empty();
  for (auto& r : p->runs)
    if (!r.xpass) p->all_xpass = false;
  {  // side streams for the fused runs after the first (at most three)
    int nf = 0;
    for (auto& r : p->runs) nf += r.fused ? 1 : 0;
    const int ns = nf > 4 ? 3 : nf - 1;
    bool sok = true;
    if (ns > 0) sok = cudaEventCreateWithFlags(&p->ev_fork,
                                               cudaEventDisableTiming) ==
                      cudaSuccess;
    for (int k = 0; sok && k < ns; ++k) {
      cudaStream_t sk = nullptr;
      cudaEvent_t ek = nullptr;
      if (cudaStreamCreateWithFlags(&sk, cudaStreamNonBlocking) !=
          cudaSuccess) {
        sok = false;
        break;
      }
      p->side.push_back(sk);
      if (cudaEventCreateWithFlags(&ek, cudaEventDisableTiming) !=
          cudaSuccess) {
        sok = false;
        break;
      }
      p->ev_join.push_back(ek);
    }
    if (!sok) {
      cudaGetLastError();
      free_all(p);
      delete p;
      return FPM_ERR_CUDA;
    }
  }
  for (auto& r : p->runs) {
    const SimDev& S = p->sims[r.first];
    if (rc == FPM_OK)
      rc = make_mesh_plan(&r.r2c, r, S, CUFFT_R2C, r.count, &ws);
    if (rc == FPM_OK)
      rc = make_plan(&r.c2r3, S.mx, S.my, S.mz, CUFFT_C2R, 3 * r.count, &ws);
    if (rc == FPM_OK)
      rc = make_mesh_plan(&r.c2r1, r, S, CUFFT_C2R, r.count, &ws);
    if (adj && rc == FPM_OK)
      rc = make_plan(&r.r2c3, S.mx, S.my, S.mz, CUFFT_R2C, 3 * r.count, &ws);
    if (lpt) {
      if (rc == FPM_OK)
        rc = make_plan(&r.lr2c3, S.nx, S.ny, S.nz, CUFFT_R2C, 3 * r.count, &ws);
      if (rc == FPM_OK)
        rc = make_plan(&r.lr2c9, S.nx, S.ny, S.nz, CUFFT_R2C, 9 * r.count, &ws);
      if (rc == FPM_OK)
        rc = make_plan(&r.lr2c, S.nx, S.ny, S.nz, CUFFT_R2C, r.count, &ws);
      if (rc == FPM_OK)
        rc = make_plan(&r.lc2r9, S.nx, S.ny, S.nz, CUFFT_C2R, 9 * r.count, &ws);
      if (rc == FPM_OK)
        rc = make_plan(&r.lc2r3, S.nx, S.ny, S.nz, CUFFT_C2R, 3 * r.count, &ws);
      if (rc == FPM_OK)
        rc = make_plan(&r.lc2r1, S.nx, S.ny, S.nz, CUFFT_C2R, r.count, &ws);
    }
  }
  if (rc != FPM_OK) {
    free_all(p);
    delete p;
    return rc;
  }

  bool ok = true;
  size_t& tot = p->device_bytes;
  p->d_sims = dalloc<SimDev>(nsims, tot, ok);
  p->d_kk = dalloc<double>(kk.size(), tot, ok);
  p->d_grad = dalloc<float>(grad.size(), tot, ok);
  p->d_win = dalloc<float>(win.size(), tot, ok);
  p->rho = dalloc<float>(p->total_m, tot, ok);
  p->dk = dalloc<float2>(p->total_s, tot, ok);
  p->fk = dalloc<float2>(3 * p->total_s, tot, ok);
  p->fmesh = dalloc<float>(3 * p->total_m, tot, ok);
  p->phi = dalloc<float>(p->total_m, tot, ok);
  if (lpt) {
    p->lreal1 = dalloc<float>(p->total_l, tot, ok);
    p->lspec1 = dalloc<float2>(p->total_ls, tot, ok);
    p->lspec9 = dalloc<float2>(9 * p->total_ls, tot, ok);
    p->lreal9 = dalloc<float>(9 * p->total_l, tot, ok);
    p->lreal3 = dalloc<float>(3 * p->total_l, tot, ok);
  }
  if (adj) {
    p->lmesh = dalloc<float>((stencil_path(p) ? 4 : 3) * p->total_m, tot, ok);
    p->lrho = dalloc<float>(p->total_m, tot, ok);
    p->fpart = dalloc<float>(3 * p->total_np, tot, ok);
  }
  p->d_nsteps = dalloc<int32_t>(nsims, tot, ok);
  p->d_ffac = dalloc<float>(nsims, tot, ok);
  p->d_lcoef = dalloc<float>(6 * (size_t)nsims, tot, ok);
  p->d_status = dalloc<int32_t>(1, tot, ok);
  if (ws > 0) {
    if (ok && cudaMalloc(&p->work, ws) != cudaSuccess) ok = false;
    if (ok) tot += ws;
    if (ok) p->work_bytes = ws;
  }
  if (!ok) {
    cudaGetLastError();
    free_all(p);
    delete p;
    return FPM_ERR_OOM;
  }
  for (auto& r : p->runs) {
    cufftHandle hs[] = {r.r2c,   r.c2r3,  r.r2c3,  r.c2r1, r.lr2c,
                        r.lc2r9, r.lc2r3, r.lc2r1, r.lr2c3, r.lr2c9};
    for (cufftHandle h : hs)
      if (h && cufftSetWorkArea(h, p->work) != CUFFT_SUCCESS) rc = FPM_ERR_CUFFT;
  }
  if (rc == FPM_OK &&
      (cudaMemcpy(p->d_sims, p->sims.data(), sizeof(SimDev) * nsims,
                  cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(p->d_kk, kk.data(), sizeof(double) * kk.size(),
                  cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(p->d_grad, grad.data(), sizeof(float) * grad.size(),
                  cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(p->d_win, win.data(), sizeof(float) * win.size(),
                  cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemset(p->d_status, 0, sizeof(int32_t)) != cudaSuccess))
    rc = FPM_ERR_CUDA;
  if (rc != FPM_OK) {
    free_all(p);
    delete p;
    return rc;
  }
  *out = p;
  return FPM_OK;
}

extern "C" int fpm_plan_destroy(fpm_plan* p) {
  if (!p) return FPM_ERR_ARG;
  free_all(p);
  delete p;
  return FPM_OK;
}

extern "C" int fpm_plan_info(const fpm_plan* p, int64_t* total_particles,
                             int64_t* device_bytes) {
  if (!p) return FPM_ERR_ARG;
  if (total_particles) *total_particles = p->total_np;
  if (device_bytes) *device_bytes = (int64_t)p->device_bytes;
  return FPM_OK;
}

extern "C" int fpm_plan_status(fpm_plan* p, int32_t* status, void* stream) {
  if (!p || !status) return FPM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  int32_t v = 0;
  FPM_CUDA(cudaMemcpyAsync(&v, p->d_status, sizeof(int32_t),
                           cudaMemcpyDeviceToHost, st));
  FPM_CUDA(cudaMemsetAsync(p->d_status, 0, sizeof(int32_t), st));
  FPM_CUDA(cudaStreamSynchronize(st));
  *status = v;
  return FPM_OK;
}

extern "C" int fpm_force(fpm_plan* p, const float* disp,
                         const double* force_fac, float* force, void* stream) {
  if (!p || !disp || !force_fac || !force) return FPM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  FPM_TRY(upload_ffac(p, force_fac, st));
  FPM_CUDA(cudaMemsetAsync(p->rho, 0, sizeof(float) * p->total_m, st));
  launch_paint_lattice(p->d_sims, p->nsims, traverse_chunks(p), disp, p->rho,
                       p->d_status, st);
  FPM_TRY(launch_ok());
  FPM_TRY(force_meshes(p, st, false));
  launch_force_readout(p->d_sims, p->nsims, traverse_chunks(p), disp, p->fmesh,
                       p->d_ffac, force, st);
  return launch_ok();
}

extern "C" int fpm_nbody_set_steps(fpm_plan* p, int max_steps,
                                   const int32_t* nsteps, const double* coefs,
                                   const double* force_fac, void* stream) {
  if (!p || max_steps < 0 || !nsteps || !force_fac ||
      (max_steps > 0 && !coefs))
    return FPM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  for (int s = 0; s < p->nsims; ++s)
    if (nsteps[s] < 0 || nsteps[s] > max_steps) return FPM_ERR_ARG;
  if (max_steps > p->coef_cap) {
    if (p->d_coefs) {
      FPM_CUDA(cudaStreamSynchronize(st));
      cudaFree(p->d_coefs);
      p->device_bytes -= sizeof(float) * 3 * (size_t)p->nsims * p->coef_cap;
      p->d_coefs = nullptr;
      p->coef_cap = 0;
    }
    if (cudaMalloc(&p->d_coefs, sizeof(float) * 3 * (size_t)p->nsims *
                                    max_steps) != cudaSuccess) {
      cudaGetLastError();
      return FPM_ERR_OOM;
    }
    p->coef_cap = max_steps;
    p->coef_gen++;
    p->device_bytes += sizeof(float) * 3 * (size_t)p->nsims * max_steps;
    if (p->pgd_on) {  // its table has the old stride: set it again
      p->pgd_on = false;
      p->sched_gen++;
    }
  }
  if (max_steps > 0) {
    std::vector<float> c(3 * (size_t)p->nsims * max_steps);
    for (size_t i = 0; i < c.size(); ++i) c[i] = (float)coefs[i];
    FPM_CUDA(cudaMemcpyAsync(p->d_coefs, c.data(), sizeof(float) * c.size(),
                             cudaMemcpyHostToDevice, st));
  }
  FPM_CUDA(cudaMemcpyAsync(p->d_nsteps, nsteps, sizeof(int32_t) * p->nsims,
                           cudaMemcpyHostToDevice, st));
  FPM_TRY(upload_ffac(p, force_fac, st));
  // The uploads read pageable host vectors that die with this call.
  FPM_CUDA(cudaStreamSynchronize(st));
  FPM_TRY(update_schedule(p, max_steps, nsteps, st));
  p->max_steps = max_steps;
  p->steps_set = true;
  return FPM_OK;
}

// Several runs, all on the fused solve, no PGD, no profiling: the runs'
// simulations are independent, so each run integrates as its own chain
// (solve, step, solve, ...) on its own stream -- the call's stream for the
// first run, the side streams for the others, forked and joined by events
// (parallel branches when captured).  The small runs' latency-bound
// kernels then overlap the large run's throughout the leapfrog.
bool chains_ok(const fpm_plan* p) {
  if (p->runs.size() < 2 || p->pgd_on || p->profile ||
      p->side.size() + 1 < p->runs.size())
    return false;
  for (const auto& r : p->runs)
    if (!r.fused) return false;
  return true;
}

int64_t run_chunk(const fpm_plan* p, size_t k) {
  if (k >= p->runs.size()) return traverse_chunks(p);
  const SimDev& S = p->sims[p->runs[k].first];
  return FPM_STEP_BLOCKED ? S.ch_b : S.ch_p;
}

int nbody_chains(fpm_plan* p, StepArgs a, cudaStream_t st) {
  const Green G = plan_green(p);
  FPM_CUDA(cudaEventRecord(p->ev_fork, st));
  for (size_t k = 0; k < p->runs.size(); ++k) {
    Run& r = p->runs[k];
    const SimDev& S = p->sims[r.first];
    cudaStream_t rs = k == 0 ? st : p->side[k - 1];
    if (k > 0) FPM_CUDA(cudaStreamWaitEvent(rs, p->ev_fork, 0));
    const int64_t c0 = run_chunk(p, k), c1 = run_chunk(p, k + 1);
    for (int it = 0; it <= p->max_steps; ++it) {
      const int n = run_active(r, it);
      if (n == 0) continue;  // every simulation of the run has finished
      launch_fft_force(p->d_sims, r.first, n, S.mx, S.my, S.mz, p->rho,
                       it < p->max_steps ? 1 : 0, p->dk, p->fk, p->fmesh,
                       p->tape ? tape_phi(p, it) : p->phi, tabs_of(p), G,
                       !stencil_path(p), rs);
      a.it = it;
      launch_step(p->d_sims, p->nsims, c0, c1, a, rs);
    }
    if (k > 0) {
      FPM_CUDA(cudaEventRecord(p->ev_join[k - 1], rs));
      FPM_CUDA(cudaStreamWaitEvent(st, p->ev_join[k - 1], 0));
    }
  }
  return launch_ok();
}

// ---------------------------------------------------------------------------
// Binned forward step (fpm_plan_set_binning)
// ---------------------------------------------------------------------------
BinRun bin_run(const fpm_plan* p, const Run& r) {
  const SimDev& S = p->sims[r.first];
  BinRun R;
  R.nx = S.nx;
  R.ny = S.ny;
  R.nz = S.nz;
  R.bf = S.bf;
  R.mx = S.mx;
  R.my = S.my;
  R.mz = S.mz;
  R.ntx = S.ntx;
  R.nty = S.nty;
  R.ntz = S.ntz;
  R.count = r.count;
  R.qkb = S.qkb;
  R.qjb = S.qjb;
  R.np = S.np;
  R.ncell = (int64_t)S.mx * S.my * S.mz;
  R.p0 = S.p_off;
  R.m0 = S.m_off;
  return R;
}

// Counting sort of run k's particles from (d, pm, lag) -- lag NULL: the
// caller's Lagrangian order -- into the plan's sorted buffer dst.
int bin_sort_run(fpm_plan* p, size_t k, const float* d, const float* pm,
                 const uint32_t* lag, int dst, bool counted, cudaStream_t st) {
  const Run& r = p->runs[k];
  return launch_bin_sort(p->bin_tile, bin_run(p, r), d, pm, lag, p->bcount,
                         p->bcell, p->bsums + r.bsum_off, p->bd[dst],
                         p->bp[dst], p->blag[dst], counted, st);
}

// Whether the step kernel of step it counts the cells for the sort that
// follows it (k_step_sorted, every simulation of run k still drifting).
bool fused_count(const fpm_plan* p, const Run& r, int it) {
  return p->bin_mode != FPM_BIN_TILES && it < r.min_steps;
}

int64_t run_part_chunk(const fpm_plan* p, size_t k) {
  if (k >= p->runs.size()) return p->ch_p;
  return p->sims[p->runs[k].first].ch_p;
}

int64_t run_tile_chunk(const fpm_plan* p, size_t k) {
  if (k >= p->runs.size()) return p->total_tiles;
  return p->sims[p->runs[k].first].ch_t;
}

BinStepArgs bin_args(const fpm_plan* p, const StepArgs& a, int cur,
                     bool count = false) {
  BinStepArgs b;
  b.a = a;
  b.bd = p->bd[cur];
  b.bp = p->bp[cur];
  b.blag = p->blag[cur];
  b.cell_end = p->bcell;
  b.count = count ? p->bcount : nullptr;
  b.tile_log2 = p->bin_tile == 16 ? 4 : 3;
  b.claim = nullptr;  // in place unless nbody_flow sets the claims
  b.od = b.op = nullptr;
  b.olag = nullptr;
  return b;
}

// Whether every run's simulations take the same number of steps (the
// particles re-sorted as they move keep a simulation's slots only when
// every one of them moves at every step).
bool runs_uniform(const fpm_plan* p) {
  for (const Run& r : p->runs)
    if (r.min_steps != r.max_steps) return false;
  return true;
}

// The leapfrog with the particles re-sorted as they move (FPM_BIN_FLOW):
// the cells of the caller's Lagrangian state are counted and scanned into
// first slots; then at every step each particle claims the next slot of
// its cell at the start of the step and k_step_sorted writes it there in
// the other buffer, counting the cells of the drifted particles for the
// next step's scan.  The order a step sees is its previous step's, with no
// sort pass; the last step writes the final d, p and F in Lagrangian order.
int nbody_flow(fpm_plan* p, StepArgs a, cudaStream_t st) {
  FPM_CUDA(cudaMemsetAsync(p->bcount, 0, sizeof(int32_t) * p->total_m, st));
  auto args = [&](int cur, int it, const Run* r) {
    // cur < 0: the caller's Lagrangian arrays
    BinStepArgs b = bin_args(p, a, cur < 0 ? 0 : cur);
    const int nxt = cur < 0 ? 0 : 1 - cur;
    if (cur < 0) {
      b.bd = a.disp;
      b.bp = a.mom;
      b.blag = nullptr;
    }
    const int T = r ? r->min_steps : p->max_steps;
    if (it < T) {
      b.claim = p->bcell;
      b.count = p->bcount;
      b.od = p->bd[nxt];
      b.op = p->bp[nxt];
      b.olag = p->blag[nxt];
    }
    b.a.it = it;
    return b;
  };
  for (size_t k = 0; k < p->runs.size(); ++k) {
    const Run& r = p->runs[k];
    FPM_TRY(launch_bin_count_scan(p->bin_tile, bin_run(p, r), a.disp, nullptr,
                                  p->bcount, p->bcell,
                                  p->bsums + r.bsum_off, st));
  }
  if (chains_ok(p)) {
    const Green G = plan_green(p);
    FPM_CUDA(cudaEventRecord(p->ev_fork, st));
    for (size_t k = 0; k < p->runs.size(); ++k) {
      Run& r = p->runs[k];
      const SimDev& S = p->sims[r.first];
      cudaStream_t rs = k == 0 ? st : p->side[k - 1];
      if (k > 0) FPM_CUDA(cudaStreamWaitEvent(rs, p->ev_fork, 0));
      int cur = -1;
      for (int it = 0; it <= r.min_steps; ++it) {
        launch_fft_force(p->d_sims, r.first, r.count, S.mx, S.my, S.mz,
                         p->rho, it < p->max_steps ? 1 : 0, p->dk, p->fk,
                         p->fmesh, p->tape ? tape_phi(p, it) : p->phi,
                         tabs_of(p), G, !stencil_path(p), rs);
        launch_step_sorted(p->d_sims, p->nsims, run_part_chunk(p, k),
                           run_part_chunk(p, k + 1), args(cur, it, &r), rs);
        if (it < r.min_steps) {
          FPM_TRY(launch_bin_scan(bin_run(p, r), p->bcount, p->bcell,
                                  p->bsums + r.bsum_off, rs));
          cur = cur < 0 ? 0 : 1 - cur;
        }
      }
      if (k > 0) {
        FPM_CUDA(cudaEventRecord(p->ev_join[k - 1], rs));
        FPM_CUDA(cudaStreamWaitEvent(st, p->ev_join[k - 1], 0));
      }
    }
    return launch_ok();
  }
  int cur = -1;
  for (int it = 0; it <= p->max_steps; ++it) {
    FPM_TRY(force_meshes(p, st, it < p->max_steps, it,
                         p->tape ? tape_phi(p, it) : nullptr));
    prof_mark(p, 0, st);
    launch_step_sorted(p->d_sims, p->nsims, 0, p->ch_p,
                       args(cur, it, nullptr), st);
    prof_mark(p, 0, st);
    FPM_TRY(launch_ok());
    if (it < p->max_steps) {
      prof_mark(p, 10, st);
      for (size_t k = 0; k < p->runs.size(); ++k) {
        const Run& r = p->runs[k];
        FPM_TRY(launch_bin_scan(bin_run(p, r), p->bcount, p->bcell,
                                p->bsums + r.bsum_off, st));
      }
      prof_mark(p, 10, st);
      cur = cur < 0 ? 0 : 1 - cur;
    }
  }
  return FPM_OK;
}

// The leapfrog on the binned step: the caller's Lagrangian state is sorted
// into buffer 0, then every step runs the solve and the binned step, and
// every bin_every steps the particles are sorted into the other buffer.
// The last step writes the final d, p and F back in Lagrangian order.
int nbody_binned(fpm_plan* p, StepArgs a, cudaStream_t st) {
  if (p->bin_mode == FPM_BIN_FLOW && runs_uniform(p)) return nbody_flow(p, a, st);
  // the counts are zero between sorts; a run interrupted by an error may
  // have left some behind
  FPM_CUDA(cudaMemsetAsync(p->bcount, 0, sizeof(int32_t) * p->total_m, st));
  for (size_t k = 0; k < p->runs.size(); ++k)
    FPM_TRY(bin_sort_run(p, k, a.disp, a.mom, nullptr, 0, false, st));
  if (chains_ok(p)) {
    const Green G = plan_green(p);
    FPM_CUDA(cudaEventRecord(p->ev_fork, st));
    for (size_t k = 0; k < p->runs.size(); ++k) {
      Run& r = p->runs[k];
      const SimDev& S = p->sims[r.first];
      cudaStream_t rs = k == 0 ? st : p->side[k - 1];
      if (k > 0) FPM_CUDA(cudaStreamWaitEvent(rs, p->ev_fork, 0));
      const int64_t c0 = run_tile_chunk(p, k), c1 = run_tile_chunk(p, k + 1);
      int cur = 0;
      for (int it = 0; it <= p->max_steps; ++it) {
        const int n = run_active(r, it);
        if (n == 0) continue;  // every simulation of the run has finished
        launch_fft_force(p->d_sims, r.first, n, S.mx, S.my, S.mz, p->rho,
                         it < p->max_steps ? 1 : 0, p->dk, p->fk, p->fmesh,
                         p->tape ? tape_phi(p, it) : p->phi, tabs_of(p), G,
                         !stencil_path(p), rs);
        a.it = it;
        const bool sort = it < p->max_steps && (it + 1) % p->bin_every == 0;
        const bool counted = sort && fused_count(p, r, it);
        if (p->bin_mode != FPM_BIN_TILES)
          launch_step_sorted(p->d_sims, p->nsims, run_part_chunk(p, k),
                             run_part_chunk(p, k + 1),
                             bin_args(p, a, cur, counted), rs);
        else
          launch_step_binned(p->bin_tile, p->d_sims, p->nsims, c0, c1,
                             bin_args(p, a, cur), rs);
        if (sort) {
          FPM_TRY(bin_sort_run(p, k, p->bd[cur], p->bp[cur], p->blag[cur],
                               1 - cur, counted, rs));
          cur = 1 - cur;
        }
      }
      if (k > 0) {
        FPM_CUDA(cudaEventRecord(p->ev_join[k - 1], rs));
        FPM_CUDA(cudaStreamWaitEvent(st, p->ev_join[k - 1], 0));
      }
    }
    return launch_ok();
  }
  int cur = 0;
  for (int it = 0; it <= p->max_steps; ++it) {
    FPM_TRY(force_meshes(p, st, it < p->max_steps, it,
                         p->tape ? tape_phi(p, it) : nullptr));
    a.it = it;
    const bool sort = it < p->max_steps && (it + 1) % p->bin_every == 0;
    // one launch steps every run: it counts only when every run may
    bool counted = sort;
    for (const Run& r : p->runs) counted = counted && fused_count(p, r, it);
    prof_mark(p, 0, st);
    if (p->bin_mode != FPM_BIN_TILES)
      launch_step_sorted(p->d_sims, p->nsims, 0, p->ch_p,
                         bin_args(p, a, cur, counted), st);
    else
      launch_step_binned(p->bin_tile, p->d_sims, p->nsims, 0, p->total_tiles,
                         bin_args(p, a, cur), st);
    prof_mark(p, 0, st);
    FPM_TRY(launch_ok());
    if (sort) {
      prof_mark(p, 10, st);
      for (size_t k = 0; k < p->runs.size(); ++k)
        FPM_TRY(bin_sort_run(p, k, p->bd[cur], p->bp[cur], p->blag[cur],
                             1 - cur, counted, st));
      prof_mark(p, 10, st);
      cur = 1 - cur;
    }
  }
  return FPM_OK;
}

extern "C" int fpm_nbody_run(fpm_plan* p, float* disp, float* mom,
                             float* force, float* inter, unsigned flags,
                             float* ckpt, int ckpt_every, void* stream) {
  if (!p || !disp || !mom || !force || (ckpt && ckpt_every < 1))
    return FPM_ERR_ARG;
  if (!p->steps_set) return FPM_ERR_STATE;
  if ((flags & FPM_NBODY_INTERMEDIATE) && !inter) return FPM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  StepArgs a;
  a.disp = disp;
  a.mom = mom;
  a.force_out = force;
  a.inter = (flags & FPM_NBODY_INTERMEDIATE) ? inter : nullptr;
  a.fmesh = p->fmesh;
  a.rho = p->rho;
  a.coefs = p->d_coefs;
  a.ffac = p->d_ffac;
  a.nsteps = p->d_nsteps;
  a.status = p->d_status;
  a.ckpt = ckpt;
  a.ckpt_every = ckpt ? ckpt_every : 1;
  a.total_np = p->total_np;
  a.max_steps = p->max_steps;
  FPM_CUDA(cudaMemsetAsync(p->rho, 0, sizeof(float) * p->total_m, st));
  prof_mark(p, 2, st);
  launch_paint_lattice(p->d_sims, p->nsims, traverse_chunks(p), disp, p->rho,
                       p->d_status, st);
  prof_mark(p, 2, st);
  FPM_TRY(launch_ok());
  if (p->tape && p->tape_floats < tape_needed(p)) return FPM_ERR_ARG;
  if (p->bin_tile && p->bin_mode != FPM_BIN_WALK && !p->pgd_on)
    return nbody_binned(p, a, st);
  if (chains_ok(p)) return nbody_chains(p, a, st);
  for (int it = 0; it <= p->max_steps; ++it) {
    FPM_TRY(force_meshes(p, st, it < p->max_steps, it,
                         p->tape ? tape_phi(p, it) : nullptr));
    a.it = it;
    prof_mark(p, 0, st);
    launch_step(p->d_sims, p->nsims, 0, traverse_chunks(p), a, st);
    prof_mark(p, 0, st);
    FPM_TRY(launch_ok());
    if (p->pgd_on && it < p->max_steps) {  // after the drift of step it
      FPM_TRY(pgd_meshes(p, st, it,
                         p->tape ? tape_pgd_phi(p, it) : nullptr));
      if (p->tape)  // the displacement before the move, for the adjoint
        FPM_CUDA(cudaMemcpyAsync(tape_pgd_disp(p, it), disp,
                                 sizeof(float) * 3 * p->total_np,
                                 cudaMemcpyDeviceToDevice, st));
      launch_pgd(p->d_sims, p->nsims, traverse_chunks(p), disp, p->fmesh,
                 p->rho, p->d_pgd, p->pgd_cap, it, p->d_nsteps, p->d_status,
                 st);
      FPM_TRY(launch_ok());
    }
  }
  return FPM_OK;
}

extern "C" int fpm_nbody_set_pgd(fpm_plan* p, int enable, const double* params,
                                 void* stream) {
  if (!p || (enable && !params)) return FPM_ERR_ARG;
  if (!enable) {
    if (p->pgd_on) {
      p->pgd_on = false;
      p->sched_gen++;
    }
    return FPM_OK;
  }
  if (!p->steps_set) return FPM_ERR_STATE;
  cudaStream_t st = (cudaStream_t)stream;
  const int cap = p->coef_cap > 0 ? p->coef_cap : 1;
  if (!p->d_pgd || p->pgd_cap != cap) {
    if (p->d_pgd) {
      FPM_CUDA(cudaStreamSynchronize(st));
      cudaFree(p->d_pgd);
      p->device_bytes -= sizeof(float) * 3 * (size_t)p->nsims * p->pgd_cap;
      p->d_pgd = nullptr;
    }
    if (cudaMalloc(&p->d_pgd, sizeof(float) * 3 * (size_t)p->nsims * cap) !=
        cudaSuccess) {
      cudaGetLastError();
      p->pgd_cap = 0;
      return FPM_ERR_OOM;
    }
    p->pgd_cap = cap;
    p->coef_gen++;  // captured graphs hold the old table
    p->device_bytes += sizeof(float) * 3 * (size_t)p->nsims * cap;
  }
  std::vector<float> h(3 * (size_t)p->nsims * cap, 0.f);
  for (int s = 0; s < p->nsims; ++s)
    for (int t = 0; t < p->max_steps; ++t)
      for (int q = 0; q < 3; ++q)
        h[((size_t)s * cap + t) * 3 + q] =
            (float)params[((size_t)s * p->max_steps + t) * 3 + q];
  FPM_CUDA(cudaMemcpyAsync(p->d_pgd, h.data(), sizeof(float) * h.size(),
                           cudaMemcpyHostToDevice, st));
  FPM_CUDA(cudaStreamSynchronize(st));  // h is pageable and dies here
  if (!p->pgd_on) {
    p->pgd_on = true;
    p->sched_gen++;
  }
  return FPM_OK;
}

namespace {

void free_adj_bins(fpm_plan* p) {
  void* bins[] = {p->blx[0], p->blx[1], p->blp[0], p->blp[1]};
  for (void* b : bins)
    if (b) cudaFree(b);
  p->blx[0] = p->blx[1] = p->blp[0] = p->blp[1] = nullptr;
  p->device_bytes -= p->adj_bin_bytes;
  p->adj_bin_bytes = 0;
  p->adj_every = 0;
}

int alloc_adj_bins(fpm_plan* p) {
  bool ok = true;
  size_t tot = 0;
  for (int b = 0; b < 2; ++b) {
    p->blx[b] = dalloc<float>(3 * p->total_np, tot, ok);
    p->blp[b] = dalloc<float>(3 * p->total_np, tot, ok);
  }
  p->adj_bin_bytes = tot;
  p->device_bytes += tot;
  if (!ok) {
    cudaGetLastError();
    free_adj_bins(p);
    return FPM_ERR_OOM;
  }
  return FPM_OK;
}

void free_bins(fpm_plan* p) {
  free_adj_bins(p);
  void* bins[] = {p->bd[0],   p->bd[1], p->bp[0],  p->bp[1],    p->blag[0],
                  p->blag[1], p->bcell, p->bsums, p->bcount};
  for (void* b : bins)
    if (b) cudaFree(b);
  p->bd[0] = p->bd[1] = p->bp[0] = p->bp[1] = nullptr;
  p->blag[0] = p->blag[1] = nullptr;
  p->bcell = p->bsums = p->bcount = nullptr;
  p->device_bytes -= p->bin_bytes;
  p->bin_bytes = 0;
}

}  // namespace

extern "C" int fpm_plan_set_binning(fpm_plan* p, int tile, int sort_every,
                                    int mode) {
  if (!p || tile < 0 || sort_every < 1 ||
      (mode != FPM_BIN_TILES && mode != FPM_BIN_CHUNKS &&
       mode != FPM_BIN_WALK && mode != FPM_BIN_FLOW))
    return FPM_ERR_ARG;
  if (tile == 0) {
    if (p->bin_tile) {
      if (cudaDeviceSynchronize() != cudaSuccess) return FPM_ERR_CUDA;
      free_bins(p);
      p->bin_tile = 0;
      p->sched_gen++;
    }
    return FPM_OK;
  }
  if (p->total_np >= ((int64_t)1 << 31) - 1) return FPM_ERR_UNSUPPORTED;
  for (const SimDev& S : p->sims)
    if (!bin_tile_supported(tile, S.mx, S.my, S.mz) || S.m_off % 4 != 0)
      return FPM_ERR_UNSUPPORTED;
  for (const Run& r : p->runs) {
    const SimDev& S = p->sims[r.first];
    int kb, jb;
    if (!bin_run_supported(S.nx, S.ny, S.nz, (int64_t)S.mx * S.my * S.mz,
                           r.count, &kb, &jb))
      return FPM_ERR_UNSUPPORTED;
  }
  if (tile == p->bin_tile) {
    if (sort_every != p->bin_every || mode != p->bin_mode) {
      p->bin_every = sort_every;
      p->bin_mode = mode;
      p->sched_gen++;  // captured graphs hold the old schedule and kernel
    }
    return FPM_OK;
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return FPM_ERR_CUDA;
  // the old tile's buffers go first; until the new ones exist the plan
  // takes the lattice walk (also when their allocation fails below)
  free_bins(p);
  p->bin_tile = 0;
  p->sched_gen++;
  std::vector<SimDev> sims = p->sims;
  int64_t tiles = 0;
  for (SimDev& S : sims) {
    S.ntx = S.mx / tile;
    S.nty = S.my / tile;
    S.ntz = S.mz / tile;
    S.ch_t = tiles;
    tiles += (int64_t)S.ntx * S.nty * S.ntz;
    bin_run_supported(S.nx, S.ny, S.nz, (int64_t)S.mx * S.my * S.mz, 1,
                      &S.qkb, &S.qjb);
  }
  int64_t nsum = 0;
  for (auto& r : p->runs) {
    r.bsum_off = nsum;
    const SimDev& S = sims[r.first];
    nsum += (int64_t)bin_scan_blocks((int64_t)r.count * S.mx * S.my * S.mz);
  }
  bool ok = true;
  size_t tot = 0;
  for (int b = 0; b < 2; ++b) {
    p->bd[b] = dalloc<float>(3 * p->total_np, tot, ok);
    p->bp[b] = dalloc<float>(3 * p->total_np, tot, ok);
    p->blag[b] = dalloc<uint32_t>(p->total_np, tot, ok);
  }
  p->bcell = dalloc<int32_t>(p->total_m, tot, ok);
  p->bcount = dalloc<int32_t>(p->total_m, tot, ok);
  p->bsums = dalloc<int32_t>(nsum, tot, ok);
  p->bin_bytes = tot;
  p->device_bytes += tot;
  if (!ok) {
    cudaGetLastError();
    free_bins(p);
    return FPM_ERR_OOM;
  }
  if (cudaMemcpy(p->d_sims, sims.data(), sizeof(SimDev) * sims.size(),
                 cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(p->bcount, 0, sizeof(int32_t) * p->total_m) != cudaSuccess) {
    free_bins(p);
    return FPM_ERR_CUDA;
  }
  p->sims = sims;
  p->total_tiles = tiles;
  p->bin_tile = tile;
  p->bin_every = sort_every;
  p->bin_mode = mode;
  p->sched_gen++;
  // a reverse sweep in the binned order asked for before keeps it, if its
  // buffers fit (else it takes the lattice walk)
  if (p->adj_req > 0 && alloc_adj_bins(p) == FPM_OK) p->adj_every = p->adj_req;
  return FPM_OK;
}

extern "C" int fpm_plan_set_adjoint_binning(fpm_plan* p, int sort_every) {
  if (!p || sort_every < 0) return FPM_ERR_ARG;
  if (!(p->flags & FPM_PLAN_ADJOINT)) return FPM_ERR_STATE;
  if (sort_every == 0) {
    p->adj_req = 0;
    if (p->adj_bin_bytes) {
      if (cudaDeviceSynchronize() != cudaSuccess) return FPM_ERR_CUDA;
      free_adj_bins(p);
      p->sched_gen++;
    }
    return FPM_OK;
  }
  if (!p->bin_tile) return FPM_ERR_STATE;  // the order comes from the tiles
  if (!p->adj_bin_bytes) {
    if (cudaDeviceSynchronize() != cudaSuccess) return FPM_ERR_CUDA;
    FPM_TRY(alloc_adj_bins(p));
  }
  p->adj_req = sort_every;
  if (p->adj_every != sort_every) p->sched_gen++;
  p->adj_every = sort_every;
  return FPM_OK;
}

extern "C" int fpm_pgd(fpm_plan* p, float* disp, const double* params,
                       void* stream) {
  if (!p || !disp || !params) return FPM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (!p->d_pgd1) {
    if (cudaMalloc(&p->d_pgd1, sizeof(float) * 3 * (size_t)p->nsims) !=
        cudaSuccess) {
      cudaGetLastError();
      return FPM_ERR_OOM;
    }
    p->device_bytes += sizeof(float) * 3 * (size_t)p->nsims;
  }
  std::vector<float> h(3 * (size_t)p->nsims);
  for (size_t i = 0; i < h.size(); ++i) h[i] = (float)params[i];
  FPM_CUDA(cudaMemcpyAsync(p->d_pgd1, h.data(), sizeof(float) * h.size(),
                           cudaMemcpyHostToDevice, st));
  FPM_CUDA(cudaMemsetAsync(p->rho, 0, sizeof(float) * p->total_m, st));
  launch_paint_lattice(p->d_sims, p->nsims, traverse_chunks(p), disp, p->rho,
                       p->d_status, st);
  FPM_TRY(launch_ok());
  FPM_TRY(pgd_meshes(p, st, -1));
  launch_pgd(p->d_sims, p->nsims, traverse_chunks(p), disp, p->fmesh, p->rho,
             p->d_pgd1, 1, 0, nullptr, p->d_status, st);
  FPM_TRY(launch_ok());
  FPM_CUDA(cudaStreamSynchronize(st));  // h is pageable and dies here
  return FPM_OK;
}

extern "C" int fpm_nbody(fpm_plan* p, float* disp, float* mom, float* force,
                         int max_steps, const int32_t* nsteps,
                         const double* coefs, const double* force_fac,
                         float* inter, unsigned flags, void* stream) {
  FPM_TRY(fpm_nbody_set_steps(p, max_steps, nsteps, coefs, force_fac, stream));
  return fpm_nbody_run(p, disp, mom, force, inter, flags, nullptr, 0, stream);
}

// Stencil path: the adjoint density lrho of the adjoint force meshes in
// lmesh, for the sims with nsteps >= pos: lphi = -sum_d D_d lf_d, then
// lrho = pre C2R(w R2C(lphi)) with the transfer function G (real, so its
// own transpose).
static int adjoint_density(fpm_plan* p, int pos, const Green& G,
                           cudaStream_t st) {
  const int32_t* act = p->d_nsteps;
  prof_mark(p, 7, st);
  if (p->div_tiled) {
    for (auto& r : p->runs) {
      const int n = run_active(r, pos);
      if (n == 0) continue;
      const SimDev& S = p->sims[r.first];
      launch_stencil_div_tiled(p->d_sims, r.first, n, S.mx, S.my, S.mz,
                               r.div_xc, p->lmesh, p->phi, act, pos, st);
    }
  } else {
    launch_stencil_div(p->d_sims, p->nsims, p->ch_m, p->lmesh, p->phi, act,
                       pos, st);
  }
  prof_mark(p, 7, st);
  FPM_TRY(launch_ok());
  prof_mark(p, 8, st);
  bool any_cufft = false;
  for (auto& r : p->runs) {
    const SimDev& S = p->sims[r.first];
    const int n = run_active(r, pos);
    if (n == 0) continue;
    if (r.fused) {  // lrho straight from lphi
      launch_fft_potential(p->d_sims, r.first, n, S.mx, S.my, S.mz, p->phi,
                           p->dk, p->lrho, tabs_of(p), G, st);
      continue;
    }
    any_cufft = true;
    FPM_TRY(exec_r2c(pick(r, n, r.r2c, r.r2c_n), p->phi + S.m_off,
                     p->dk + S.s_off, st));
  }
  FPM_TRY(launch_ok());
  if (any_cufft) {
    // on the x-pass path the x pass also clears the adjoint force mesh,
    // which the divergence above has consumed, for the next scatter
    potential_modes(p, p->dk, p->dk, p->all_xpass ? p->lmesh : nullptr, G,
                    act, pos, st, 4);
    FPM_TRY(launch_ok());
    for (auto& r : p->runs) {
      const SimDev& S = p->sims[r.first];
      const int n = run_active(r, pos);
      if (n == 0 || r.fused) continue;
      FPM_TRY(exec_c2r(pick(r, n, r.c2r1, r.c2r1_n), p->dk + S.s_off,
                       p->lrho + S.m_off, st));
    }
  }
  prof_mark(p, 8, st);
  return FPM_OK;
}

// One position of the reverse sweep (flowpm's nbody adjoint, see
// fpm_nbody_adjoint): reverse drift and paint of x_it, its force meshes,
// the force VJP into the adjoint force meshes, and their adjoint density
// lrho for the next (earlier) position.
static int adjoint_step(fpm_plan* p, AdjArgs& a, int it, cudaStream_t st) {
  const double r2 = p->r_split * p->r_split;
  const int deconv = (p->flags & FPM_PLAN_CIC_DECONV) ? 1 : 0;
  const bool tape = p->tape != nullptr;
  const size_t lbytes = sizeof(float) * (a.lvec4 ? 4 : 3) * p->total_m;
  if (tape && p->pgd_on && it < p->max_steps) {
    // the PGD move of step it (x' -> x_{it+1}) in reverse, for the sims
    // with nsteps > it: its displacement meshes at x' from the stored PGD
    // potential, the paint adjoint of the force at x_{it+1} and the PGD
    // VJP at the stored x' (k_adj_pgd), then the adjoint density of the
    // PGD meshes, which the reverse drift below gathers at x'
    stencil_grad(p, tape_pgd_phi(p, it), p->d_nsteps, it + 1, 0, st);
    FPM_TRY(launch_ok());
    if (!p->all_xpass) FPM_CUDA(cudaMemsetAsync(p->lmesh, 0, lbytes, st));
    a.pgd = p->d_pgd;
    a.pgd_stride = p->pgd_cap;
    a.pgd_disp = tape_pgd_disp(p, it);
    launch_adj_pgd(p->d_sims, p->nsims, traverse_chunks(p), a, st);
    FPM_TRY(launch_ok());
    FPM_TRY(adjoint_density(p, it + 1, pgd_green(p, it, false), st));
  }
  if (tape) {
    // the force meshes of x_it from the stored potential, then the reverse
    // drift and the force VJP of position it in one particle pass
    prof_mark(p, 1, st);
    stencil_grad(p, tape_phi(p, it), p->d_nsteps, it, 0, st);
    prof_mark(p, 1, st);
    FPM_TRY(launch_ok());
    if (!p->all_xpass) FPM_CUDA(cudaMemsetAsync(p->lmesh, 0, lbytes, st));
    prof_mark(p, 6, st);
    launch_adj_position(p->d_sims, p->nsims, traverse_chunks(p), a, st);
    prof_mark(p, 6, st);
    FPM_TRY(launch_ok());
  } else {
    FPM_CUDA(cudaMemsetAsync(p->rho, 0, sizeof(float) * p->total_m, st));
    prof_mark(p, 5, st);
    launch_adj_drift_paint(p->d_sims, p->nsims, traverse_chunks(p), a, st);
    prof_mark(p, 5, st);
    FPM_TRY(launch_ok());
    FPM_TRY(force_meshes(p, st, false, it));
    if (!p->all_xpass) FPM_CUDA(cudaMemsetAsync(p->lmesh, 0, lbytes, st));
    prof_mark(p, 6, st);
    launch_adj_vjp(p->d_sims, p->nsims, traverse_chunks(p), a, st);
    prof_mark(p, 6, st);
    FPM_TRY(launch_ok());
  }
  if (stencil_path(p)) return adjoint_density(p, it, plan_green(p), st);
  prof_mark(p, 8, st);
  for (auto& r : p->runs) {
    const SimDev& S = p->sims[r.first];
    const int n = run_active(r, it);
    if (n == 0) continue;
    FPM_TRY(exec_r2c(pick(r, n, r.r2c3, r.r2c3_n), p->lmesh + 3 * S.m_off,
                     p->fk + 3 * S.s_off, st));
  }
  launch_adj_fourier(p->d_sims, p->nsims, p->ch_s, p->fk, p->dk, tabs_of(p),
                     r2, deconv, st);
  FPM_TRY(launch_ok());
  for (auto& r : p->runs) {
    const SimDev& S = p->sims[r.first];
    const int n = run_active(r, it);
    if (n == 0) continue;
    FPM_TRY(exec_c2r(pick(r, n, r.c2r1, r.c2r1_n), p->dk + S.s_off,
                     p->lrho + S.m_off, st));
  }
  prof_mark(p, 8, st);
  return FPM_OK;
}

// Sort of the reverse sweep's particle arrays of run k from src (lag NULL:
// the caller's Lagrangian order) into the plan's buffer set dst.
static int adj_sort_run(fpm_plan* p, size_t k, float* const src[4],
                        const uint32_t* lag, int dst, cudaStream_t st) {
  const Run& r = p->runs[k];
  BinPayload pay;
  pay.n = 4;
  for (int q = 0; q < 4; ++q) pay.src[q] = src[q];
  pay.dst[0] = p->bd[dst];
  pay.dst[1] = p->bp[dst];
  pay.dst[2] = p->blx[dst];
  pay.dst[3] = p->blp[dst];
  return launch_bin_sort(p->bin_tile, bin_run(p, r), pay, lag, p->bcount,
                         p->bcell, p->bsums + r.bsum_off, p->blag[dst], st);
}

// The reverse sweep of a potential-tape plan in the binned order: the
// caller's Lagrangian (d, p, lam_x, lam_p) are sorted by the cell of the
// final position, every position runs k_adj_position over the sorted
// slots, the particles are re-sorted by their current cell every
// adj_every positions, and after position 0 they go back to the caller's
// arrays in Lagrangian order for the last gather (a.it = -1).
static int adjoint_binned(fpm_plan* p, AdjArgs a, cudaStream_t st) {
  float* user[4] = {a.disp, a.mom, a.lam_x, a.lam_p};
  FPM_CUDA(cudaMemsetAsync(p->bcount, 0, sizeof(int32_t) * p->total_m, st));
  for (size_t k = 0; k < p->runs.size(); ++k)
    FPM_TRY(adj_sort_run(p, k, user, nullptr, 0, st));
  int cur = 0;
  const size_t lbytes = sizeof(float) * 4 * p->total_m;
  for (int it = p->max_steps; it >= 0; --it) {
    a.it = it;
    a.disp = p->bd[cur];
    a.mom = p->bp[cur];
    a.lam_x = p->blx[cur];
    a.lam_p = p->blp[cur];
    a.lag = p->blag[cur];
    prof_mark(p, 9, st);
    prof_mark(p, 1, st);
    stencil_grad(p, tape_phi(p, it), p->d_nsteps, it, 0, st);
    prof_mark(p, 1, st);
    FPM_TRY(launch_ok());
    if (!p->all_xpass) FPM_CUDA(cudaMemsetAsync(p->lmesh, 0, lbytes, st));
    prof_mark(p, 6, st);
    launch_adj_position_sorted(p->d_sims, p->nsims, p->ch_p, a, st);
    prof_mark(p, 6, st);
    FPM_TRY(launch_ok());
    FPM_TRY(adjoint_density(p, it, plan_green(p), st));
    prof_mark(p, 9, st);
    if (it > 0 && (p->max_steps - it + 1) % p->adj_every == 0) {
      prof_mark(p, 10, st);
      float* src[4] = {p->bd[cur], p->bp[cur], p->blx[cur], p->blp[cur]};
      for (size_t k = 0; k < p->runs.size(); ++k)
        FPM_TRY(adj_sort_run(p, k, src, p->blag[cur], 1 - cur, st));
      prof_mark(p, 10, st);
      cur = 1 - cur;
    }
  }
  BinPayload pay;
  pay.n = 4;
  pay.src[0] = p->bd[cur];
  pay.src[1] = p->bp[cur];
  pay.src[2] = p->blx[cur];
  pay.src[3] = p->blp[cur];
  for (int q = 0; q < 4; ++q) pay.dst[q] = user[q];
  for (size_t k = 0; k < p->runs.size(); ++k)
    FPM_TRY(launch_bin_unsort(bin_run(p, p->runs[k]), pay, p->blag[cur], st));
  a.disp = user[0];
  a.mom = user[1];
  a.lam_x = user[2];
  a.lam_p = user[3];
  a.lag = nullptr;
  a.it = -1;
  launch_adj_drift_paint(p->d_sims, p->nsims, traverse_chunks(p), a, st);
  return launch_ok();
}

extern "C" int fpm_nbody_adjoint(fpm_plan* p, float* disp, float* mom,
                                 const float* force, float* lam_x,
                                 float* lam_p, const float* lam_f,
                                 const float* ckpt, int ckpt_every,
                                 void* stream) {
  if (!p || !disp || !mom || !force || !lam_x || !lam_p ||
      (ckpt && ckpt_every < 1))
    return FPM_ERR_ARG;
  if (!(p->flags & FPM_PLAN_ADJOINT) || !p->steps_set) return FPM_ERR_STATE;
  // the PGD move cannot be undone in place: its adjoint needs the tape
  if (p->pgd_on && !p->tape) return FPM_ERR_UNSUPPORTED;
  if (p->tape && p->tape_floats < tape_needed(p)) return FPM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  FPM_CUDA(cudaMemcpyAsync(p->fpart, force, sizeof(float) * 3 * p->total_np,
                           cudaMemcpyDeviceToDevice, st));
  AdjArgs a;
  a.disp = disp;
  a.mom = mom;
  a.lam_x = lam_x;
  a.lam_p = lam_p;
  a.fpart = p->fpart;
  a.lam_f = lam_f;
  a.fmesh = p->fmesh;
  a.lrho = p->lrho;
  a.lmesh = p->lmesh;
  a.lvec4 = stencil_path(p) ? 1 : 0;
  a.pgd = nullptr;
  a.pgd_stride = 0;
  a.pgd_disp = nullptr;
  if (p->all_xpass)  // later positions find it cleared by the x pass
    FPM_CUDA(cudaMemsetAsync(p->lmesh, 0, sizeof(float) * 4 * p->total_m,
                             st));
  a.rho = p->rho;
  a.coefs = p->d_coefs;
  a.ffac = p->d_ffac;
  a.nsteps = p->d_nsteps;
  a.ckpt = ckpt;
  a.ckpt_every = ckpt ? ckpt_every : 1;
  a.status = p->d_status;
  a.lag = nullptr;
  a.total_np = p->total_np;
  a.max_steps = p->max_steps;
  {
    int64_t long_np = 0;
    for (const SimDev& S : p->sims)
      if (S.wi >= 16) long_np += S.np;
    a.long_walk = 2 * long_np > p->total_np ? 1 : 0;
  }
  if (p->tape && p->adj_every > 0 && p->bin_tile && !p->pgd_on)
    return adjoint_binned(p, a, st);
  for (int it = p->max_steps; it >= 0; --it) {
    a.it = it;
    prof_mark(p, 9, st);
    FPM_TRY(adjoint_step(p, a, it, st));
    prof_mark(p, 9, st);
  }
  a.it = -1;
  launch_adj_drift_paint(p->d_sims, p->nsims, traverse_chunks(p), a, st);
  return launch_ok();
}

extern "C" int fpm_nbody_set_tape(fpm_plan* p, float* tape, int64_t floats) {
  if (!p || (tape && floats < 0)) return FPM_ERR_ARG;
  if (tape && (!stencil_path(p) || p->total_m % 4 != 0))
    return FPM_ERR_UNSUPPORTED;
  if (tape != p->tape) p->sched_gen++;  // captured graphs hold the pointer
  p->tape = tape;
  p->tape_floats = tape ? floats : 0;
  return FPM_OK;
}

extern "C" int fpm_lpt_init(fpm_plan* p, const float* linear,
                            const double* coef, int order, float* disp,
                            float* mom, float* force, void* stream) {
  if (!p || !linear || !coef || !disp || !mom || !force ||
      (order != 1 && order != 2))
    return FPM_ERR_ARG;
  if (!(p->flags & FPM_PLAN_LPT)) return FPM_ERR_STATE;
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<float> c(6 * (size_t)p->nsims);
  for (size_t i = 0; i < c.size(); ++i) c[i] = (float)coef[i];
  FPM_CUDA(cudaMemcpyAsync(p->d_lcoef, c.data(), sizeof(float) * c.size(),
                           cudaMemcpyHostToDevice, st));
  // cuFFT R2C may use its input as scratch for some sizes: transform a copy.
  FPM_CUDA(cudaMemcpyAsync(p->lreal1, linear, sizeof(float) * p->total_l,
                           cudaMemcpyDeviceToDevice, st));
  for (auto& r : p->runs) {
    const SimDev& S = p->sims[r.first];
    FPM_TRY(exec_r2c(r.lr2c, p->lreal1 + S.l_off, p->lspec1 + S.ls_off, st));
  }
  launch_lpt_fourier(p->d_sims, p->nsims, p->ch_ls, p->lspec1, p->lspec9, 0,
                     tabs_of(p), st);
  FPM_TRY(launch_ok());
  for (auto& r : p->runs) {
    const SimDev& S = p->sims[r.first];
    FPM_TRY(exec_c2r(r.lc2r9, p->lspec9 + 9 * S.ls_off,
                     p->lreal9 + 9 * S.l_off, st));
  }
  const float* psi2 = nullptr;
  if (order == 2) {
    launch_lpt2_source(p->d_sims, p->nsims, p->ch_l, p->lreal9, p->lreal1, st);
    FPM_TRY(launch_ok());
    for (auto& r : p->runs) {
      const SimDev& S = p->sims[r.first];
      FPM_TRY(exec_r2c(r.lr2c, p->lreal1 + S.l_off, p->lspec1 + S.ls_off, st));
    }
    launch_lpt_fourier(p->d_sims, p->nsims, p->ch_ls, p->lspec1, p->lspec9, 1,
                       tabs_of(p), st);
    FPM_TRY(launch_ok());
    for (auto& r : p->runs) {
      const SimDev& S = p->sims[r.first];
      FPM_TRY(exec_c2r(r.lc2r3, p->lspec9 + 3 * S.ls_off,
                       p->lreal3 + 3 * S.l_off, st));
    }
    psi2 = p->lreal3;
  }
  launch_lpt_particles(p->d_sims, p->nsims, p->ch_p, p->lreal9, 9, psi2, 3,
                       p->d_lcoef, disp, mom, force, st);
  FPM_TRY(launch_ok());
  // The coefficient upload reads a host vector that dies with this call.
  FPM_CUDA(cudaStreamSynchronize(st));
  return FPM_OK;
}

extern "C" int fpm_lpt1(fpm_plan* p, const void* dlin_kv, const float* pos,
                        int64_t npart, float* disp, void* stream) {
  const float2* dlin_k = (const float2*)dlin_kv;
  if (!p || !dlin_k || !pos || !disp || npart < 0) return FPM_ERR_ARG;
  if (!(p->flags & FPM_PLAN_LPT)) return FPM_ERR_STATE;
  if (npart == 0) return FPM_OK;
  cudaStream_t st = (cudaStream_t)stream;
  launch_lat_spectrum(p->d_sims, p->nsims, p->ch_ls, dlin_k, p->lspec1, 0, 0,
                      st);
  launch_lpt_fourier(p->d_sims, p->nsims, p->ch_ls, p->lspec1, p->lspec9, 1,
                     tabs_of(p), st, 1);
  FPM_TRY(launch_ok());
  for (auto& r : p->runs) {
    const SimDev& S = p->sims[r.first];
    FPM_TRY(exec_c2r(r.lc2r3, p->lspec9 + 3 * S.ls_off,
                     p->lreal3 + 3 * S.l_off, st));
  }
  launch_lpt_readout(p->d_sims, p->nsims, p->lreal3, pos, npart, disp, st);
  return launch_ok();
}

extern "C" int fpm_lpt2_source(fpm_plan* p, const void* dlin_kv,
                               void* source_kv, void* stream) {
  const float2* dlin_k = (const float2*)dlin_kv;
  float2* source_k = (float2*)source_kv;
  if (!p || !dlin_k || !source_k) return FPM_ERR_ARG;
  if (!(p->flags & FPM_PLAN_LPT)) return FPM_ERR_STATE;
  cudaStream_t st = (cudaStream_t)stream;
  launch_lat_spectrum(p->d_sims, p->nsims, p->ch_ls, dlin_k, p->lspec1, 0, 0,
                      st);
  launch_lpt_fourier(p->d_sims, p->nsims, p->ch_ls, p->lspec1, p->lspec9, 0,
                     tabs_of(p), st, 1);
  FPM_TRY(launch_ok());
  for (auto& r : p->runs) {
    const SimDev& S = p->sims[r.first];
    FPM_TRY(exec_c2r(r.lc2r9, p->lspec9 + 9 * S.ls_off,
                     p->lreal9 + 9 * S.l_off, st));
  }
  launch_lpt2_source(p->d_sims, p->nsims, p->ch_l, p->lreal9, p->lreal1, st);
  FPM_TRY(launch_ok());
  for (auto& r : p->runs) {
    const SimDev& S = p->sims[r.first];
    FPM_TRY(exec_r2c(r.lr2c, p->lreal1 + S.l_off, p->lspec1 + S.ls_off, st));
  }
  launch_lat_spectrum(p->d_sims, p->nsims, p->ch_l, p->lspec1, source_k, 1, 1,
                      st);
  return launch_ok();
}

extern "C" int fpm_lpt_adjoint(fpm_plan* p, const float* linear,
                               const double* coef, int order,
                               const float* lam_disp, const float* lam_mom,
                               const float* lam_force, float* lam_linear,
                               void* stream) {
  if (!p || !linear || !coef || !lam_disp || !lam_linear ||
      (order != 1 && order != 2))
    return FPM_ERR_ARG;
  if (!(p->flags & FPM_PLAN_LPT)) return FPM_ERR_STATE;
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<float> c(6 * (size_t)p->nsims);
  for (size_t i = 0; i < c.size(); ++i) c[i] = (float)coef[i];
  FPM_CUDA(cudaMemcpyAsync(p->d_lcoef, c.data(), sizeof(float) * c.size(),
                           cudaMemcpyHostToDevice, st));
  if (order == 2) {
    // recompute the second-derivative meshes phi_ij of the forward
    FPM_CUDA(cudaMemcpyAsync(p->lreal1, linear, sizeof(float) * p->total_l,
                             cudaMemcpyDeviceToDevice, st));
    for (auto& r : p->runs) {
      const SimDev& S = p->sims[r.first];
      FPM_TRY(exec_r2c(r.lr2c, p->lreal1 + S.l_off, p->lspec1 + S.ls_off, st));
    }
    launch_lpt_fourier(p->d_sims, p->nsims, p->ch_ls, p->lspec1, p->lspec9, 0,
                       tabs_of(p), st);
    FPM_TRY(launch_ok());
    for (auto& r : p->runs) {
      const SimDev& S = p->sims[r.first];
      FPM_TRY(exec_c2r(r.lc2r9, p->lspec9 + 9 * S.ls_off,
                       p->lreal9 + 9 * S.l_off, st));
    }
  } else {
    for (const SimDev& S : p->sims)
      FPM_CUDA(cudaMemsetAsync(p->lreal9 + 9 * S.l_off + 3 * S.np, 0,
                               sizeof(float) * 6 * S.np, st));
  }
  launch_lpt_adj_particles(p->d_sims, p->nsims, p->ch_p, lam_disp, lam_mom,
                           lam_force, p->d_lcoef, p->lreal9, 9,
                           order == 2 ? p->lreal3 : nullptr, 3, st);
  FPM_TRY(launch_ok());
  if (order == 2) {
    for (auto& r : p->runs) {
      const SimDev& S = p->sims[r.first];
      FPM_TRY(exec_r2c(r.lr2c3, p->lreal3 + 3 * S.l_off,
                       p->lspec9 + 3 * S.ls_off, st));
    }
    launch_lpt_adj_fourier(p->d_sims, p->nsims, p->ch_ls, p->lspec9, 3,
                           p->lspec1, tabs_of(p), st);
    FPM_TRY(launch_ok());
    for (auto& r : p->runs) {
      const SimDev& S = p->sims[r.first];
      FPM_TRY(exec_c2r(r.lc2r1, p->lspec1 + S.ls_off, p->lreal1 + S.l_off, st));
    }
    launch_lpt_adj_phi(p->d_sims, p->nsims, p->ch_l, p->lreal1, p->lreal9, st);
    FPM_TRY(launch_ok());
  }
  for (auto& r : p->runs) {
    const SimDev& S = p->sims[r.first];
    FPM_TRY(exec_r2c(r.lr2c9, p->lreal9 + 9 * S.l_off,
                     p->lspec9 + 9 * S.ls_off, st));
  }
  launch_lpt_adj_fourier(p->d_sims, p->nsims, p->ch_ls, p->lspec9, 9,
                         p->lspec1, tabs_of(p), st);
  FPM_TRY(launch_ok());
  for (auto& r : p->runs) {
    const SimDev& S = p->sims[r.first];
    FPM_TRY(exec_c2r(r.lc2r1, p->lspec1 + S.ls_off, lam_linear + S.l_off, st));
  }
  FPM_CUDA(cudaStreamSynchronize(st));
  return FPM_OK;
}

extern "C" int fpm_linear_field(fpm_plan* p, const float* amp, uint64_t seed,
                                int generate, float* white, float* linear,
                                void* stream) {
  if (!p || !amp || !linear || (!generate && !white)) return FPM_ERR_ARG;
  if (!(p->flags & FPM_PLAN_LPT)) return FPM_ERR_STATE;
  cudaStream_t st = (cudaStream_t)stream;
  if (generate) {
    float* w = white ? white : p->lreal1;
    for (int s = 0; s < p->nsims; ++s) {
      const SimDev& S = p->sims[s];
      launch_white_noise(w + S.l_off, S.l_off, S.np, seed,
                         std::sqrt((double)S.np), st);
    }
    FPM_TRY(launch_ok());
    if (w != p->lreal1)
      FPM_CUDA(cudaMemcpyAsync(p->lreal1, w, sizeof(float) * p->total_l,
                               cudaMemcpyDeviceToDevice, st));
  } else {
    FPM_CUDA(cudaMemcpyAsync(p->lreal1, white, sizeof(float) * p->total_l,
                             cudaMemcpyDeviceToDevice, st));
  }
  for (auto& r : p->runs) {
    const SimDev& S = p->sims[r.first];
    FPM_TRY(exec_r2c(r.lr2c, p->lreal1 + S.l_off, p->lspec1 + S.ls_off, st));
  }
  launch_linear_mul(p->d_sims, p->nsims, p->ch_ls, p->lspec1, amp, st);
  FPM_TRY(launch_ok());
  for (auto& r : p->runs) {
    const SimDev& S = p->sims[r.first];
    FPM_TRY(exec_c2r(r.lc2r1, p->lspec1 + S.ls_off, linear + S.l_off, st));
  }
  return FPM_OK;
}

extern "C" int fpm_white_noise(float* out, int64_t n, uint64_t seed,
                               double stddev, void* stream) {
  if (n < 0 || (n > 0 && !out)) return FPM_ERR_ARG;
  if (n == 0) return FPM_OK;
  launch_white_noise(out, 0, n, seed, stddev, (cudaStream_t)stream);
  return launch_ok();
}

extern "C" int fpm_plan_profile(fpm_plan* p, int enable) {
  if (!p) return FPM_ERR_ARG;
  p->profile = enable != 0;
  for (int k = 0; k < kProfKinds; ++k) p->ev_used[k] = 0;
  return FPM_OK;
}

extern "C" int fpm_plan_profile_read(fpm_plan* p, int kind, double* total_ms,
                                     int64_t* launches) {
  if (!p || kind < 0 || kind >= kProfKinds || !total_ms || !launches)
    return FPM_ERR_ARG;
  double t = 0;
  const size_t n = p->ev_used[kind] / 2;
  for (size_t i = 0; i < n; ++i) {
    float ms = 0;
    if (cudaEventSynchronize(p->ev[kind][2 * i + 1]) != cudaSuccess ||
        cudaEventElapsedTime(&ms, p->ev[kind][2 * i],
                             p->ev[kind][2 * i + 1]) != cudaSuccess)
      return FPM_ERR_CUDA;
    t += ms;
  }
  *total_ms = t;
  *launches = (int64_t)n;
  p->ev_used[kind] = 0;
  return FPM_OK;
}

// ---------------------------------------------------------------------------
// CUDA graphs of the leapfrog and of its adjoint
// ---------------------------------------------------------------------------
struct fpm_graph {
  fpm_plan* plan = nullptr;
  cudaGraphExec_t exec = nullptr;
  int max_steps = 0;
  int64_t coef_gen = 0;
  int64_t sched_gen = 0;
};

namespace {

template <typename F>
int capture(fpm_plan* p, fpm_graph** out, F&& body) {
  if (!p || !out) return FPM_ERR_ARG;
  if (!p->steps_set) return FPM_ERR_STATE;
  *out = nullptr;
  cudaStream_t cs;
  FPM_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  const bool prof = p->profile;
  p->profile = false;
  cudaGraph_t g = nullptr;
  int rc = FPM_OK;
  if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) !=
      cudaSuccess) {
    rc = FPM_ERR_CUDA;
  } else {
    rc = body(cs);
    if (cudaStreamEndCapture(cs, &g) != cudaSuccess && rc == FPM_OK)
      rc = FPM_ERR_CUDA;
  }
  p->profile = prof;
  cudaGraphExec_t exec = nullptr;
  if (rc == FPM_OK && cudaGraphInstantiate(&exec, g, 0) != cudaSuccess)
    rc = FPM_ERR_CUDA;
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cs);
  if (rc != FPM_OK) {
    cudaGetLastError();
    return rc;
  }
  fpm_graph* gr = new (std::nothrow) fpm_graph();
  if (!gr) {
    cudaGraphExecDestroy(exec);
    return FPM_ERR_OOM;
  }
  gr->plan = p;
  gr->exec = exec;
  gr->max_steps = p->max_steps;
  gr->coef_gen = p->coef_gen;
  gr->sched_gen = p->sched_gen;
  *out = gr;
  return FPM_OK;
}

}  // namespace

extern "C" int fpm_graph_capture_nbody(fpm_plan* p, float* disp, float* mom,
                                       float* force, float* inter,
                                       unsigned flags, float* ckpt,
                                       int ckpt_every, fpm_graph** out) {
  return capture(p, out, [&](cudaStream_t cs) {
    return fpm_nbody_run(p, disp, mom, force, inter, flags, ckpt, ckpt_every,
                         cs);
  });
}

extern "C" int fpm_graph_capture_adjoint(fpm_plan* p, float* disp, float* mom,
                                         const float* force, float* lam_x,
                                         float* lam_p, const float* lam_f,
                                         const float* ckpt, int ckpt_every,
                                         fpm_graph** out) {
  return capture(p, out, [&](cudaStream_t cs) {
    return fpm_nbody_adjoint(p, disp, mom, force, lam_x, lam_p, lam_f, ckpt,
                             ckpt_every, cs);
  });
}

extern "C" int fpm_graph_launch(fpm_graph* g, void* stream) {
  if (!g || !g->exec) return FPM_ERR_ARG;
  if (g->plan->max_steps != g->max_steps ||
      g->plan->coef_gen != g->coef_gen || g->plan->sched_gen != g->sched_gen)
    return FPM_ERR_STATE;
  FPM_CUDA(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
  return FPM_OK;
}

extern "C" int fpm_graph_destroy(fpm_graph* g) {
  if (!g) return FPM_ERR_ARG;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  delete g;
  return FPM_OK;
}

// ---------------------------------------------------------------------------
// Full-spectrum normalised FFTs (flowpm/utils.py:213 r2c3d, :244 c2r3d).
// ---------------------------------------------------------------------------
namespace {

std::mutex g_fft_mu;
std::map<std::tuple<int, int, int, int, int, int>, cufftHandle> g_fft_plans;

int c2c_plan(int batch, int nx, int ny, int nz, int dbl, cufftHandle* h) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FPM_ERR_CUDA;
  auto key = std::make_tuple(dev, batch, nx, ny, nz, dbl);
  std::lock_guard<std::mutex> lk(g_fft_mu);
  auto it = g_fft_plans.find(key);
  if (it != g_fft_plans.end()) {
    *h = it->second;
    return FPM_OK;
  }
  int n[3] = {nx, ny, nz};
  cufftHandle hh;
  if (cufftPlanMany(&hh, 3, n, nullptr, 1, 0, nullptr, 1, 0,
                    dbl ? CUFFT_Z2Z : CUFFT_C2C, batch) != CUFFT_SUCCESS)
    return FPM_ERR_CUFFT;
  g_fft_plans[key] = hh;
  *h = hh;
  return FPM_OK;
}

template <typename R, typename C>
__global__ void k_real_to_complex(const R* in, C* out, int64_t n, R scale) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    C v;
    v.x = in[i] * scale;
    v.y = 0;
    out[i] = v;
  }
}

template <typename C, typename R>
__global__ void k_scale_complex(C* data, int64_t n, R scale) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    C v = data[i];
    v.x *= scale;
    v.y *= scale;
    data[i] = v;
  }
}

template <typename C, typename R>
__global__ void k_complex_real(const C* in, R* out, int64_t n, R scale) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[i].x * scale;
}

unsigned grid_n(int64_t n) {
  int64_t b = (n + 255) / 256;
  if (b > (int64_t)kNumSMs * 32) b = (int64_t)kNumSMs * 32;
  return (unsigned)(b < 1 ? 1 : b);
}

}  // namespace

extern "C" int fpm_r2c3d(const void* rfield, void* cfield, int batch, int nx,
                         int ny, int nz, double scale, int double_precision,
                         void* stream) {
  if (!rfield || !cfield || batch < 1 || nx < 1 || ny < 1 || nz < 1)
    return FPM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n = (int64_t)batch * nx * ny * nz;
  cufftHandle h;
  FPM_TRY(c2c_plan(batch, nx, ny, nz, double_precision, &h));
  if (cufftSetStream(h, st) != CUFFT_SUCCESS) return FPM_ERR_CUFFT;
  if (double_precision) {
    k_real_to_complex<<<grid_n(n), 256, 0, st>>>(
        (const double*)rfield, (double2*)cfield, n, 1.0);
    if (cufftExecZ2Z(h, (cufftDoubleComplex*)cfield,
                     (cufftDoubleComplex*)cfield,
                     CUFFT_FORWARD) != CUFFT_SUCCESS)
      return FPM_ERR_CUFFT;
    k_scale_complex<<<grid_n(n), 256, 0, st>>>((double2*)cfield, n, scale);
  } else {
    k_real_to_complex<<<grid_n(n), 256, 0, st>>>(
        (const float*)rfield, (float2*)cfield, n, 1.0f);
    if (cufftExecC2C(h, (cufftComplex*)cfield, (cufftComplex*)cfield,
                     CUFFT_FORWARD) != CUFFT_SUCCESS)
      return FPM_ERR_CUFFT;
    k_scale_complex<<<grid_n(n), 256, 0, st>>>((float2*)cfield, n,
                                                (float)scale);
  }
  return launch_ok();
}

extern "C" int fpm_c2r3d(const void* cfield, void* rfield, int batch, int nx,
                         int ny, int nz, double scale, int double_precision,
                         void* stream) {
  if (!rfield || !cfield || batch < 1 || nx < 1 || ny < 1 || nz < 1)
    return FPM_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t n = (int64_t)batch * nx * ny * nz;
  cufftHandle h;
  FPM_TRY(c2c_plan(batch, nx, ny, nz, double_precision, &h));
  if (cufftSetStream(h, st) != CUFFT_SUCCESS) return FPM_ERR_CUFFT;
  const size_t bytes = (size_t)n * (double_precision ? 16 : 8);
  void* tmp = nullptr;
  FPM_CUDA(cudaMallocAsync(&tmp, bytes, st));
  int rc = FPM_OK;
  if (double_precision) {
    if (cufftExecZ2Z(h, (cufftDoubleComplex*)cfield, (cufftDoubleComplex*)tmp,
                     CUFFT_INVERSE) != CUFFT_SUCCESS)
      rc = FPM_ERR_CUFFT;
    else
      k_complex_real<<<grid_n(n), 256, 0, st>>>((const double2*)tmp,
                                                 (double*)rfield, n, scale);
  } else {
    if (cufftExecC2C(h, (cufftComplex*)cfield, (cufftComplex*)tmp,
                     CUFFT_INVERSE) != CUFFT_SUCCESS)
      rc = FPM_ERR_CUFFT;
    else
      k_complex_real<<<grid_n(n), 256, 0, st>>>(
          (const float2*)tmp, (float*)rfield, n, (float)scale);
  }
  cudaFreeAsync(tmp, st);
  if (rc != FPM_OK) return rc;
  return launch_ok();
}

// ---------------------------------------------------------------------------
// Autotuner of the forward step's particle traversal
// ---------------------------------------------------------------------------
namespace {

// (tile, sort period, mode) of each configuration fpm_plan_autotune times:
// the lattice walk; the sorted particles in equal chunks (keys tile-major
// in tiles of 16 cells) re-sorted every 4, 6, 10 or 16 leapfrog steps, or
// sorted once at the start; re-sorted as they move, in tiles of 16; the
// shared-memory tiles of 16 cells re-sorted every 4 steps.
constexpr int kTune[FPM_TUNE_CONFIGS][3] = {
    {0, 1, FPM_BIN_CHUNKS},  {16, 4, FPM_BIN_CHUNKS}, {16, 6, FPM_BIN_CHUNKS},
    {16, 10, FPM_BIN_CHUNKS}, {16, 16, FPM_BIN_CHUNKS},
    {16, 1 << 20, FPM_BIN_CHUNKS},
    {16, 1, FPM_BIN_FLOW},   {16, 4, FPM_BIN_TILES}};

std::mutex g_tune_mu;
// choice per (device, plan flags, step count, PGD, tape, dims...)
std::map<std::vector<int64_t>, int> g_tune_cache;

std::vector<int64_t> tune_key(const fpm_plan* p) {
  int dev = -1;
  cudaGetDevice(&dev);
  std::vector<int64_t> k = {dev, (int64_t)p->flags, p->max_steps,
                            p->pgd_on ? 1 : 0, p->tape ? 1 : 0, p->nsims};
  for (const SimDev& S : p->sims) {
    k.push_back(S.nx);
    k.push_back(S.ny);
    k.push_back(S.nz);
    k.push_back(S.bf);
  }
  return k;
}

}  // namespace

extern "C" int fpm_plan_autotune(fpm_plan* p, const float* disp,
                                 const float* mom, int reps, int retune,
                                 int32_t* choice, float* ms, void* stream) {
  if (!p || !choice || reps < 1 || (!retune && !disp) != (!retune && !mom) ||
      (retune && (!disp || !mom)))
    return FPM_ERR_ARG;
  if (!p->steps_set) return FPM_ERR_STATE;
  cudaStream_t st = (cudaStream_t)stream;
  const std::vector<int64_t> key = tune_key(p);
  if (!retune) {
    int c = -1;
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tune_cache.find(key);
      if (it != g_tune_cache.end()) c = it->second;
    }
    if (c >= 0) {
      FPM_TRY(fpm_plan_set_binning(p, kTune[c][0], kTune[c][1], kTune[c][2]));
      choice[0] = kTune[c][0];
      choice[1] = kTune[c][1];
      choice[2] = kTune[c][2];
      if (ms)
        for (int k = 0; k < FPM_TUNE_CONFIGS; ++k) ms[k] = -1.f;
      return FPM_OK;
    }
    if (!disp) return FPM_ERR_STATE;  // nothing cached, nothing to time on
  }
  // candidates run on scratch copies of the state, each as one graph replay
  const size_t nb = sizeof(float) * 3 * (size_t)p->total_np;
  float *sd = nullptr, *sp = nullptr, *sf = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = FPM_OK;
  if (cudaMalloc(&sd, nb) != cudaSuccess || cudaMalloc(&sp, nb) != cudaSuccess ||
      cudaMalloc(&sf, nb) != cudaSuccess)
    rc = FPM_ERR_OOM;
  if (rc == FPM_OK && (cudaEventCreate(&e0) != cudaSuccess ||
                       cudaEventCreate(&e1) != cudaSuccess))
    rc = FPM_ERR_CUDA;
  int best = -1;
  float best_ms = 0.f;
  for (int c = 0; rc == FPM_OK && c < FPM_TUNE_CONFIGS; ++c) {
    if (ms) ms[c] = -1.f;
    const int src =
        fpm_plan_set_binning(p, kTune[c][0], kTune[c][1], kTune[c][2]);
    if (src == FPM_ERR_UNSUPPORTED) continue;
    if (src == FPM_ERR_OOM) {  // larger configurations will not fit either
      cudaGetLastError();
      continue;
    }
    if (src != FPM_OK) {
      rc = src;
      break;
    }
    fpm_graph* g = nullptr;
    rc = fpm_graph_capture_nbody(p, sd, sp, sf, nullptr, 0, nullptr, 0, &g);
    float tmin = 0.f;
    for (int r = 0; rc == FPM_OK && r <= reps; ++r) {
      if (cudaMemcpyAsync(sd, disp, nb, cudaMemcpyDeviceToDevice, st) !=
              cudaSuccess ||
          cudaMemcpyAsync(sp, mom, nb, cudaMemcpyDeviceToDevice, st) !=
              cudaSuccess ||
          cudaEventRecord(e0, st) != cudaSuccess) {
        rc = FPM_ERR_CUDA;
        break;
      }
      rc = fpm_graph_launch(g, st);
      if (rc != FPM_OK) break;
      float t = 0.f;
      if (cudaEventRecord(e1, st) != cudaSuccess ||
          cudaEventSynchronize(e1) != cudaSuccess ||
          cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) {
        rc = FPM_ERR_CUDA;
        break;
      }
      if (r > 0 && (r == 1 || t < tmin)) tmin = t;  // r = 0 warms up
    }
    if (g) fpm_graph_destroy(g);
    if (rc != FPM_OK) break;
    if (ms) ms[c] = tmin;
    if (best < 0 || tmin < best_ms) {
      best = c;
      best_ms = tmin;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(sd);
  cudaFree(sp);
  cudaFree(sf);
  if (rc == FPM_OK && best < 0) rc = FPM_ERR_UNSUPPORTED;
  if (rc != FPM_OK) {
    cudaGetLastError();
    fpm_plan_set_binning(p, 0, 1, FPM_BIN_CHUNKS);
    return rc;
  }
  FPM_TRY(fpm_plan_set_binning(p, kTune[best][0], kTune[best][1],
                               kTune[best][2]));
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = best;
  }
  choice[0] = kTune[best][0];
  choice[1] = kTune[best][1];
  choice[2] = kTune[best][2];
  return FPM_OK;
}
