// Launch wrappers of the particle-mesh step kernels (fpm_kernels.cu), used by
// the plan orchestration in fpm_plan.cu.
#pragma once

#include "fpm_internal.cuh"

#include <atomic>

namespace fpm {

// Kernels launched by the library since it was loaded (fpm_launch_count).
extern std::atomic<int64_t> g_launches;

struct StepArgs {
  float* disp;             // (total_np, 3) displacement from the lattice
  float* mom;              // (total_np, 3)
  float* force_out;        // (total_np, 3), written when a sim finishes
  float* inter;            // (max_steps, 3, total_np, 3) or null
  const float* fmesh;      // force meshes: sim s, component c at
                           //   fmesh + 3*m_off + c*mcells
  float* rho;              // density target of the next paint
  const float* coefs;      // (nsims, max_steps, 3) {kick_start, drift, kick_end}
  const float* ffac;       // (nsims) force prefactor (1.5 Omega_m)
  const int32_t* nsteps;   // (nsims)
  int32_t* status;         // device status word
  float* ckpt;             // checkpoint slots (d, p) or null
  int ckpt_every;          // position j is saved in slot j / ckpt_every
  int64_t total_np;
  int max_steps;
  int it;                  // global iteration 0..max_steps
};

// Paint every particle at (q + disp) * bf into rho (which must be zeroed).
void launch_paint_lattice(const SimDev* sims, int nsims, int64_t nchunks,
                          const float* disp, float* rho, int32_t* status,
                          cudaStream_t st);

// R2C output -> three force spectra (Green's function * gradient, optional
// CIC deconvolution and Gaussian long-range window); also zeroes rho.  With
// nsteps, simulations with nsteps[s] < pos (finished) are skipped, and with
// skip_fused those whose force meshes come from the fused solve.
void launch_fourier_force(const SimDev* sims, int nsims, int64_t nchunks,
                          const float2* dk, float2* fk, float* rho_zero,
                          AxisTabs tabs, double r_split2, int deconv,
                          const int32_t* nsteps, int pos, int skip_fused,
                          cudaStream_t st);

// Potential spectrum delta_k * pre * w(k) with w the transfer function G
// (one output per sim, layout of dk); also zeroes rho_zero when given.  The
// adjoint reuses it as is; the PGD correction passes its own G.
void launch_fourier_potential(const SimDev* sims, int nsims, int64_t nchunks,
                              const float2* dk, float2* out, float* rho_zero,
                              AxisTabs tabs, const Green& G,
                              const int32_t* nsteps, int pos, int skip_fused,
                              cudaStream_t st);

// f_d = D_d phi with the 4-point stencil (nchunks = mesh chunks; quads:
// four cells per thread, every mesh with mz % 4 == 0 and m_off % 4 == 0),
// and its
// adjoint lphi = -sum_d D_d lf_d (lf interleaved: float4 per cell).
void launch_stencil_grad(const SimDev* sims, int nsims, int64_t nchunks,
                         const float* phi, float* fmesh, const int32_t* nsteps,
                         int pos, int skip_fused, bool quads, cudaStream_t st);
void launch_stencil_div(const SimDev* sims, int nsims, int64_t nchunks,
                        const float* lf, float* lphi, const int32_t* nsteps,
                        int pos, cudaStream_t st);
// Tiled k_stencil_div over the sims [first, first + count) of one mesh
// shape; stencil_div_chunk gives its x chunk (0: shape not supported, use
// launch_stencil_div).
int stencil_div_chunk(int mx, int my, int mz, int64_t m_off, int count);
// Tiled k_stencil_grad (the same tiles and x chunk as the tiled
// divergence) over the sims [first, first + count) of one mesh shape.
void launch_stencil_grad_tiled(const SimDev* sims, int first, int count,
                               int mx, int my, int mz, int xc,
                               const float* phi, float* fmesh,
                               const int32_t* nsteps, int pos,
                               cudaStream_t st);
void launch_stencil_div_tiled(const SimDev* sims, int first, int count,
                              int mx, int my, int mz, int xc, const float* lf,
                              float* lphi, const int32_t* nsteps, int pos,
                              cudaStream_t st);

// Fused Fourier solve (fpm_fft.cu) for meshes with every axis a power of
// two in [16, 128]: density -> three force meshes (the transfer function of
// launch_fourier_force) in three kernels over the sims [first, first + n)
// of one run (equal shapes); also zeroes rho when zero_rho.  dk and fk are
// the spectrum scratch (R2C layout, fk three spectra per sim).
bool fft_fused_supported(int nx, int ny, int nz);
// Once per shape and device before the first launch (twiddle table, shared
// memory limits).
int fft_fused_prepare(int nx, int ny, int nz);
// With the 4-point gradient (grad3 false) the solve produces the potential
// and takes the gradient with the real-space stencil (phi: potential mesh
// scratch); with grad3 (order-0 gradient) it transforms three force spectra
// (fk scratch).
void launch_fft_force(const SimDev* sims, int first, int n, int nx, int ny,
                      int nz, float* rho, int zero_rho, float2* dk,
                      float2* fk, float* fmesh, float* phi, AxisTabs tabs,
                      const Green& G, bool grad3, cudaStream_t st);
// out = C2R(pre * w(k) * R2C(in)) for the sims [first, first + n) of one
// run (the adjoint's density cotangent from the potential cotangent); in is
// only read.
void launch_fft_potential(const SimDev* sims, int first, int n, int nx,
                          int ny, int nz, const float* in, float2* dk,
                          float* out, AxisTabs tabs, const Green& G,
                          cudaStream_t st);
// Meshes of 256 or 512 cells along x on the cuFFT path: the x pass between
// batched (y, z) plane transforms, potential spectrum out = x-pass(in) of
// the sims [first, first + n) of one run (in == out allowed; with nsteps,
// the sims with nsteps < pos skip); with rho_zero it also zeroes their
// part of that buffer, zmul floats per cell (1: density mesh, 4: the
// interleaved adjoint force mesh).  fft_xpass_prepare uploads its twiddles (once per
// device).
bool fft_xpass_supported(int nx, int ny, int nz);
int fft_xpass_prepare();
void launch_fft_xpass(const SimDev* sims, int first, int n, int nx, int ny,
                      int nzh, const float2* in, float2* out, float* rho_zero,
                      int zmul, AxisTabs tabs, const Green& G,
                      const int32_t* nsteps, int pos, cudaStream_t st);

// Fused readout + kick(end) + kick(start) + drift + paint of one iteration,
// over the traversal chunks [ch0, ch1) (whole simulations).
void launch_step(const SimDev* sims, int nsims, int64_t ch0, int64_t ch1,
                 const StepArgs& a, cudaStream_t st);

// PGD correction of one step: d += alpha * readout(PGD meshes) / bf, then
// the paint of the moved particles into rho (see k_pgd).
void launch_pgd(const SimDev* sims, int nsims, int64_t nchunks, float* disp,
                const float* fmesh, float* rho, const float* pgd,
                int pgd_stride, int pos, const int32_t* nsteps,
                int32_t* status, cudaStream_t st);

// Readout of the three force meshes at (q + disp) * bf, times ffac / bf.
void launch_force_readout(const SimDev* sims, int nsims, int64_t nchunks,
                          const float* disp, const float* fmesh,
                          const float* ffac, float* force, cudaStream_t st);

// Lattice spectra for LPT.  mode 0: from delta_L write 9 spectra
// {psi1_x, psi1_y, psi1_z, phi_00, phi_11, phi_22, phi_12, phi_20, phi_01};
// mode 1: write the 3 spectra psi_d.  Input is the unnormalised R2C output,
// scaled by 1 / (nx ny nz), or, with normalised, already scaled.
void launch_lpt_fourier(const SimDev* sims, int nsims, int64_t nchunks,
                        const float2* dk, float2* out, int mode, AxisTabs tabs,
                        cudaStream_t st, int normalised = 0);

// Lattice spectra, full (nx, ny, nz) <-> half (nx, ny, nz/2 + 1):
// to_full = 0 keeps l <= nz/2 (nchunks = lattice-spectrum chunks),
// to_full = 1 fills l > nz/2 by Hermitian symmetry (nchunks = lattice
// chunks); both scaled by 1 / (nx ny nz) when inv_n.
void launch_lat_spectrum(const SimDev* sims, int nsims, int64_t nchunks,
                         const float2* in, float2* out, int to_full,
                         int inv_n, cudaStream_t st);

// out[s, p] = CIC readout of the three lattice meshes psi + 3 l_off + d Nc
// at pos[s, p] (npart particles per simulation).
void launch_lpt_readout(const SimDev* sims, int nsims, const float* psi,
                        const float* pos, int64_t npart, float* out,
                        cudaStream_t st);

// 2LPT source 3/7 * sum(phi_ii phi_jj - phi_ij^2) on the lattice meshes.
void launch_lpt2_source(const SimDev* sims, int nsims, int64_t nchunks,
                        const float* phi9, float* source, cudaStream_t st);

// LPT particle initialisation from the psi meshes (order 1 or 2).
// psi1 / psi2 of sim s start at psi + m * l_off (m = meshes per sim).
void launch_lpt_particles(const SimDev* sims, int nsims, int64_t nchunks,
                          const float* psi1, int m1, const float* psi2, int m2,
                          const float* coef, float* disp, float* mom,
                          float* force, cudaStream_t st);

// lineark = R2C(white) / N^3 * amp, in place on the lattice spectra.
void launch_linear_mul(const SimDev* sims, int nsims, int64_t nchunks,
                       float2* wk, const float* amp, cudaStream_t st);

// Philox4x32-10 + Box-Muller white noise: out[e - off] = stddev * N(0, 1)
// for the global element indices e in [off, off + n).
void launch_white_noise(float* out, int64_t off, int64_t n, uint64_t seed,
                        double stddev, cudaStream_t st);

}  // namespace fpm
