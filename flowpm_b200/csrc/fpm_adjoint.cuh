// Launch wrappers of the adjoint kernels (fpm_adjoint.cu).
#pragma once

#include "fpm_kernels.cuh"

namespace fpm {

struct AdjArgs {
  float* disp;            // (total_np, 3) displacement, reconstructed in place
                          // (the per-particle arrays disp, mom, lam_x,
                          // lam_p are in Lagrangian order, or with lag set
                          // in the binned order of launch_adj_position_sorted)
  float* mom;             // (total_np, 3) momentum, reconstructed in place
  float* lam_x;           // (total_np, 3) dL/dX
  float* lam_p;           // (total_np, 3) dL/dp
  float* fpart;           // (total_np, 3) force at the current position
  const float* lam_f;     // (total_np, 3) dL/dF at the final position or null
  const float* fmesh;     // forward force meshes at the current position
  const float* lrho;      // adjoint density mesh of the previous position
  float* lmesh;           // adjoint force meshes (scatter target): with
                          // lvec4 one float4 (x, y, z, 0) per cell (sim s
                          // at lmesh + 4 m_off), else three planes
                          // (lmesh + 3 m_off + d mcells)
  int lvec4;
  float* rho;             // density target of the paint
  const float* pgd;       // PGD rows (alpha, kl, ks), stride pgd_stride per
  int pgd_stride;         //   sim (k_adj_pgd)
  const float* pgd_disp;  // (total_np, 3) displacement before the PGD move
  const float* coefs;     // (nsims, max_steps, 3) {kick_start, drift, kick_end}
  const float* ffac;      // (nsims)
  const int32_t* nsteps;  // (nsims)
  const float* ckpt;      // checkpoint slots (d, p) or null
  int ckpt_every;
  int32_t* status;
  const uint32_t* lag;    // binned order: packed lattice site of each slot
  int64_t total_np;
  int max_steps;
  int it;
  int long_walk;  // most particles walk long lattice blocks (wi >= 16): the
                  // launchers take the FPM_ADJ_MINBLOCKS instances
};

void launch_adj_drift_paint(const SimDev* sims, int nsims, int64_t nchunks,
                            const AdjArgs& a, cudaStream_t st);
void launch_adj_vjp(const SimDev* sims, int nsims, int64_t nchunks,
                    const AdjArgs& a, cudaStream_t st);
// k_adj_drift_paint without the paint followed by k_adj_vjp at the same
// position (a.it >= 0), in one pass; the force meshes of x_it must be ready.
void launch_adj_position(const SimDev* sims, int nsims, int64_t nchunks,
                         const AdjArgs& a, cudaStream_t st);
// launch_adj_position over particles kept sorted by cell (the binned order
// of fpm_bin.cu): the particle chunks [0, nchunks) of the plan, slot i of
// disp, mom, lam_x and lam_p holding the particle of packed lattice site
// a.lag[i] (pack_site) of its simulation; checkpoints and lam_f are read in
// Lagrangian order.
void launch_adj_position_sorted(const SimDev* sims, int nsims,
                                int64_t nchunks, const AdjArgs& a,
                                cudaStream_t st);
// The PGD move of step a.it (x' -> x_{it+1}) in reverse, sims with
// nsteps > a.it: lam_x += B sum_c lam_rho[c] grad W at x_{it+1} (the force
// paint adjoint), then at x' = q + pgd_disp with the PGD displacement
// meshes in fmesh: lam_x += alpha sum_c grad W (lam_x . g[c]) and
// lmesh[c] += (alpha / B) lam_x W; disp = pgd_disp.
void launch_adj_pgd(const SimDev* sims, int nsims, int64_t nchunks,
                    const AdjArgs& a, cudaStream_t st);
void launch_adj_fourier(const SimDev* sims, int nsims, int64_t nchunks,
                        const float2* lk, float2* out, AxisTabs tabs,
                        double r_split2, int deconv, cudaStream_t st);
void launch_lpt_adj_particles(const SimDev* sims, int nsims, int64_t nchunks,
                              const float* ld, const float* lp,
                              const float* lf, const float* coef, float* psi1,
                              int m1, float* psi2, int m2, cudaStream_t st);
void launch_lpt_adj_fourier(const SimDev* sims, int nsims, int64_t nchunks,
                            const float2* in, int nin, float2* out,
                            AxisTabs tabs, cudaStream_t st);
void launch_lpt_adj_phi(const SimDev* sims, int nsims, int64_t nchunks,
                        const float* ls, float* phi9, cudaStream_t st);

}  // namespace fpm
