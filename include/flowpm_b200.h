/*
 * flowpm_b200 -- C ABI of the B200 particle-mesh library (libflowpm_b200.so).
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream
 * (passed as void*), is stream-ordered, performs no host synchronisation
 * unless stated, and returns FPM_OK (0) or one of the FPM_ERR_* codes; it
 * never exits, aborts or traps.  The caller owns every buffer it passes; the
 * library owns only what fpm_plan_create allocates (cuFFT plans, the mesh
 * work buffers and a device status word), released by fpm_plan_destroy.
 *
 * Conventions (those of the reference, flowpm/utils.py and flowpm/tfpm.py):
 *   meshes            float32, (batch, nx, ny, nz), z fastest;
 *   particle arrays   float32, (batch, npart, 3) in mesh units;
 *   nbody state       kept as displacement d from the Lagrangian lattice
 *                     q = (i, j, k) of particle index (i*ny + j)*nz + k
 *                     (absolute position X = q + d), momentum p, force f,
 *                     each (total_particles, 3).
 */
#ifndef FLOWPM_B200_H
#define FLOWPM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  FPM_OK = 0,
  FPM_ERR_ARG = 1,        /* bad shape, size or null pointer            */
  FPM_ERR_ALIGN = 2,      /* pointer not aligned as required            */
  FPM_ERR_OOM = 3,        /* device allocation failed                   */
  FPM_ERR_CUDA = 4,       /* a CUDA runtime call failed                 */
  FPM_ERR_CUFFT = 5,      /* a cuFFT call failed                        */
  FPM_ERR_NONFINITE = 6,  /* device status: non-finite particle state   */
  FPM_ERR_STATE = 7,      /* call out of order (e.g. missing workspace) */
  FPM_ERR_UNSUPPORTED = 8, /* valid request this build does not handle  */
  FPM_ERR_LIMIT = 9,       /* request larger than the fixed scratch of an
                              allocation-free entry point                  */
  FPM_ERR_RANGE = 10       /* a deposit fell outside the mesh (2-D paint
                              with nx < ny, where the reference's indices
                              wrap by ny); the others were made           */
};

/* Device status bits accumulated by the kernels of a plan. */
enum {
  FPM_STATUS_NONFINITE_POS = 1, /* a particle position was NaN or inf */
  FPM_STATUS_NONFINITE_MOM = 2  /* a momentum or force was NaN or inf */
};

/* Plan option flags (fpm_plan_create). */
enum {
  FPM_PLAN_CIC_DECONV = 1u << 0, /* divide the force by the CIC window
                                    prod_d sinc^2(k_d / 2pi)
                                    (flowpm/kernels.py:137 cic_compensation);
                                    off in the reference force              */
  FPM_PLAN_LPT = 1u << 1,        /* also allocate the LPT / linear-field
                                    buffers on the particle lattice         */
  FPM_PLAN_GRAD_ORDER0 = 1u << 2, /* gradient i*k (order 0) instead of the
                                    4-point finite difference (order 1)   */
  FPM_PLAN_ADJOINT = 1u << 3,    /* also allocate the adjoint buffers and
                                    cuFFT plans (fpm_nbody_adjoint)         */
  FPM_PLAN_CUFFT = 1u << 4,      /* force meshes through cuFFT for every
                                    mesh shape; by default meshes of 16 to
                                    128 cells (powers of two) per axis use
                                    the library's fused Fourier solve       */
  FPM_PLAN_SMALL_BLOCKS = 1u << 5 /* the particle kernels walk every lattice
                                    in blocks of 8x8x16 particles; by
                                    default lattices of 2^23 particles or
                                    more take 16x8x16 blocks, and of 2^26 or
                                    more 64x8x16 (faster there)             */
};

/* nbody flags (fpm_nbody). */
enum {
  FPM_NBODY_INTERMEDIATE = 1u << 0 /* write the state after every step */
};

typedef struct fpm_plan fpm_plan;
typedef struct fpm_graph fpm_graph;

/* Library version (major*10000 + minor*100 + patch) and error text. */
int fpm_version(void);
const char* fpm_error_string(int code);

/* Number of CUDA kernels this library has launched since it was loaded
 * (its own kernels; cuFFT's are not counted). */
int64_t fpm_launch_count(void);

/* ---------------------------------------------------------------------
 * Stand-alone CIC operators.
 * ------------------------------------------------------------------ */

/* mesh[b] += CIC deposit of part[b] with weights weight[b] (or 1 when
 * weight is NULL).  Replaces flowpm/utils.py:32-91 cic_paint
 * (tf.scatter_nd over 8 neighbours, mod-N periodic wrap). */
int fpm_cic_paint(float* mesh, int batch, int nx, int ny, int nz,
                  const float* part, int64_t npart, const float* weight,
                  void* stream);

/* out[b, p] = sum over the 8 CIC neighbours of mesh[b] * weight.
 * Replaces flowpm/utils.py:163-210 cic_readout (tf.gather_nd). */
int fpm_cic_readout(const float* mesh, int batch, int nx, int ny, int nz,
                    const float* part, int64_t npart, float* out,
                    void* stream);

/* Adjoint of fpm_cic_paint: lam_part = weight * sum_c lam_mesh[c] grad W,
 * lam_weight = sum_c lam_mesh[c] W (either output may be NULL).  The CIC
 * weight derivative follows d|x|/dx = sign(x), sign(0) = 0. */
int fpm_cic_paint_adjoint(const float* lam_mesh, int batch, int nx, int ny,
                          int nz, const float* part, int64_t npart,
                          const float* weight, float* lam_part,
                          float* lam_weight, void* stream);

/* Adjoint of fpm_cic_readout: lam_mesh += scatter of lam_out with the CIC
 * weights; lam_part = lam_out * sum_c mesh[c] grad W (either may be NULL). */
int fpm_cic_readout_adjoint(const float* mesh, int batch, int nx, int ny,
                            int nz, const float* part, int64_t npart,
                            const float* lam_out, float* lam_mesh,
                            float* lam_part, void* stream);

/* Neighbour cells and weights of each particle, in the reference's
 * neighbour order (flowpm/utils.py:66-67): idx[p*8 + c] is the flat cell
 * (ix*ny + iy)*nz + iz, w[p*8 + c] the CIC weight.  Exposed so that cell
 * indices and neighbour sets can be compared bit for bit. */
int fpm_cic_neighbours(int nx, int ny, int nz, const float* part,
                       int64_t npart, int32_t* idx, float* w, void* stream);

/* ---------------------------------------------------------------------
 * Full-spectrum FFTs behind flowpm/utils.py:213 r2c3d and :244 c2r3d:
 *   fpm_r2c3d: out = FFT3(complex(in)) * scale            (r2c3d: 1/norm)
 *   fpm_c2r3d: out = Re(sum_k in_k e^{+ikx}) * scale      (c2r3d: norm/N^3)
 * over the three innermost axes of (batch, nx, ny, nz) arrays.
 * double_precision selects float64 / complex128 buffers.  Plans are cached
 * inside the library per device and shape (created on first use);
 * fpm_c2r3d takes a temporary buffer from the stream-ordered allocator.
 * ------------------------------------------------------------------ */
int fpm_r2c3d(const void* rfield, void* cfield, int batch, int nx, int ny,
              int nz, double scale, int double_precision, void* stream);
int fpm_c2r3d(const void* cfield, void* rfield, int batch, int nx, int ny,
              int nz, double scale, int double_precision, void* stream);

/* ---------------------------------------------------------------------
 * Plans: one set of simulations advanced together.  dims holds, for each
 * simulation, {nx, ny, nz, pm_nc_factor}: the particle lattice (= the
 * linear-field mesh, flowpm/tfpm.py:148) and the force-mesh factor
 * (flowpm/tfpm.py:317 pm_nc_factor).  Consecutive simulations with equal
 * dims share batched cuFFT plans.  Particle arrays of the plan are the
 * simulations' arrays concatenated in order.
 * ------------------------------------------------------------------ */
int fpm_plan_create(fpm_plan** plan, int nsims, const int32_t* dims,
                    double r_split, unsigned flags);
int fpm_plan_destroy(fpm_plan* plan);
/* Total particles of the plan and bytes of device memory it holds. */
int fpm_plan_info(const fpm_plan* plan, int64_t* total_particles,
                  int64_t* device_bytes);
/* Copy the device status word to *status and clear it (synchronises the
 * stream). */
int fpm_plan_status(fpm_plan* plan, int32_t* status, void* stream);

/* Per-kernel timing: while enabled, fpm_nbody_run records a CUDA event
 * pair around every launch of the fused step kernel (kind 0), every
 * Fourier solve -- density to the three force meshes, all of its
 * transforms and kernels (kind 1) -- and the initial paint (kind 2) on the
 * call's stream; for meshes on the cuFFT path also around the
 * Green's-function kernel (kind 3) and the stencil gradient (kind 4).
 * fpm_nbody_adjoint records, per position of the reverse sweep, the
 * reverse drift + paint kernel (kind 5), the force VJP kernel (kind 6; with
 * a potential tape, the one kernel that does the reverse drift and the
 * VJP, and no kind 5),
 * the divergence stencil (kind 7, stencil path), the adjoint potential
 * solve -- adjoint force meshes to the adjoint density, all of its
 * transforms and kernels (kind 8) -- and the whole position (kind 9); its
 * force solves add to kinds 1, 3 and 4 (with a potential tape, kind 1 is
 * the stencil of the stored potential).  fpm_plan_profile_read waits for
 * the last event, returns the summed device time and the number of timed
 * launches of `kind`, and resets that kind.  Not for use under CUDA graph
 * capture. */
int fpm_plan_profile(fpm_plan* plan, int enable);
int fpm_plan_profile_read(fpm_plan* plan, int kind, double* total_ms,
                          int64_t* launches);

/* Force on every particle at positions q + disp:
 * flowpm/tfpm.py:317-366 force() = paint at X*B, /nbar, r2c, Green's
 * function * 4-point gradient * force_fac[s] (1.5 Omega_m in the
 * reference), c2r, readout at X*B, /B.  force has the layout of disp. */
int fpm_force(fpm_plan* plan, const float* disp, const double* force_fac,
              float* force, void* stream);

/* KDK leapfrog of flowpm/tfpm.py:425-503 for every simulation of the
 * plan.  coefs holds, per simulation s and step i < nsteps[s], the three
 * FP64 prefactors {kick_start, drift, kick_end} at
 * coefs[(s*max_steps + i)*3 + 0..2]:
 *   kick_start_i = kick(a_i, a_i, ah_i), drift_i = drift(a_i, ah_i, a_i+1),
 *   kick_end_i   = kick(ah_i, a_i+1, a_i+1)   (flowpm/tfpm.py:273-314).
 * disp and mom are updated in place; force receives the force at the
 * final positions.  With FPM_NBODY_INTERMEDIATE, inter (max_steps x 3 x
 * total_particles x 3 floats) receives (X = q + d, p, f) after each step. */
int fpm_nbody(fpm_plan* plan, float* disp, float* mom, float* force,
              int max_steps, const int32_t* nsteps, const double* coefs,
              const double* force_fac, float* inter, unsigned flags,
              void* stream);

/* fpm_nbody in two parts: fpm_nbody_set_steps uploads the step tables
 * (host arrays; synchronises the stream once), fpm_nbody_run launches the
 * whole leapfrog with kernels and cuFFT executions only, so that it can be
 * captured into a CUDA graph and replayed. */
int fpm_nbody_set_steps(fpm_plan* plan, int max_steps, const int32_t* nsteps,
                        const double* coefs, const double* force_fac,
                        void* stream);
int fpm_nbody_run(fpm_plan* plan, float* disp, float* mom, float* force,
                  float* inter, unsigned flags, float* ckpt, int ckpt_every,
                  void* stream);

/* PGD correction (flowpm/tfpm.py:369-422, applied by nbody after each drift
 * at :487-488): with enable, every later fpm_nbody_run moves the particles
 * of step t after its drift by alpha * readout(c2r(delta_k * lap(k) *
 * exp(-kl^2/k^2) exp(-k^4/ks^4) * i D_d(k))) / pm_nc_factor (4-point
 * gradient), then paints them for the force.  params: (alpha, kl, ks) per
 * simulation and step, nsims x max_steps x 3 doubles, kl and ks in the
 * units of the force mesh's k = 2 pi fftfreq.  Call after
 * fpm_nbody_set_steps (a set_steps that grows the tables switches PGD off
 * again).  enable = 0 switches it off.  With PGD on, fpm_nbody_adjoint
 * needs a potential tape (fpm_nbody_set_tape; else FPM_ERR_UNSUPPORTED).
 * Synchronises the stream once. */
int fpm_nbody_set_pgd(fpm_plan* plan, int enable, const double* params,
                      void* stream);

/* One PGD correction of the positions q + disp of every simulation
 * (flowpm/tfpm.py:369-422 pgd): disp is updated in place.  params: (alpha,
 * kl, ks) per simulation, nsims x 3 doubles.  Synchronises the stream. */
int fpm_pgd(fpm_plan* plan, float* disp, const double* params, void* stream);

/* Eulerian binning of the forward leapfrog (replaces the particle order of
 * the reference's tf.scatter_nd / tf.gather_nd, flowpm/utils.py:87-89,
 * :207-209, which is arbitrary): with tile 8 or 16, fpm_nbody_run keeps the
 * particle state sorted by force-mesh cell, cell keys tile-major in tiles
 * of tile^3 cells, and re-sorts it every sort_every leapfrog steps (a
 * period longer than the run sorts once, at the start)
 * (counting sort carrying each particle's Lagrangian index).  mode
 * FPM_BIN_CHUNKS steps the sorted particles in equal chunks, painting into
 * the density directly with warp-summed deposits of neighbouring lanes;
 * FPM_BIN_TILES gives each tile to one block, which paints into a
 * shared-memory copy of the tile; FPM_BIN_FLOW re-sorts the particles at
 * every step without a sort pass: each step kernel writes every particle to
 * the next free slot of its cell in the other buffer and counts the cells
 * of the drifted particles for the next step (sort_every is ignored; runs
 * whose simulations take different step counts fall back to
 * FPM_BIN_CHUNKS); FPM_BIN_WALK keeps the forward on the
 * lattice walk and only provides the tiles and buffers for the reverse
 * sweep's binned order (fpm_plan_set_adjoint_binning).  The caller's
 * arrays stay in Lagrangian
 * order; the results equal the lattice walk's up to the order of the
 * density's FP32 sums.  tile 0 returns to the lattice walk.  Allocates 56
 * bytes per particle and 8 per force-mesh cell (freed by tile 0 or
 * fpm_plan_destroy), synchronising the device; every force mesh must divide
 * into tiles, and each simulation's lattice site must pack into 32 bits
 * (else FPM_ERR_UNSUPPORTED).  Plans with PGD switched on keep the lattice
 * walk.  Captured graphs of the plan must be captured again. */
enum {
  FPM_BIN_TILES = 0,
  FPM_BIN_CHUNKS = 1,
  FPM_BIN_WALK = 2,
  FPM_BIN_FLOW = 3
};
int fpm_plan_set_binning(fpm_plan* plan, int tile, int sort_every, int mode);

/* The reverse sweep (fpm_nbody_adjoint) of a plan with a potential tape in
 * the same binned order (no counterpart in the reference, whose gradient
 * is TensorFlow's tape over the scatter / gather ops above): the caller's
 * Lagrangian (disp, mom, lam_x, lam_p) are sorted by the cell of the final
 * position, each position's fused reverse drift and force VJP runs over
 * the sorted particles, which are re-sorted by their current cell every
 * sort_every positions, and the results go back to the caller's arrays in
 * Lagrangian order.  They equal the lattice walk's up to the order of the
 * FP32 sums into the adjoint meshes.  Needs an adjoint plan
 * (FPM_PLAN_ADJOINT) with binning on (fpm_plan_set_binning), else
 * FPM_ERR_STATE; without a tape, or with PGD on, the reverse sweep keeps
 * the lattice walk.  Allocates 48 bytes per particle (freed by sort_every
 * 0, by tile 0 or by fpm_plan_destroy), synchronising the device; the
 * setting survives a change of tile when the buffers still fit.  Captured
 * graphs of the plan must be captured again. */
int fpm_plan_set_adjoint_binning(fpm_plan* plan, int sort_every);

/* Autotuner of the forward step's particle traversal.  No counterpart in
 * the reference (TensorFlow picks its own kernels).  Times, on the plan's
 * current step tables (fpm_nbody_set_steps first) and on scratch copies of
 * the state (disp, mom: total_particles x 3, left unchanged), one graph
 * replay of fpm_nbody_run for each of FPM_TUNE_CONFIGS configurations --
 * the lattice walk; the binned step (fpm_plan_set_binning) in chunks with
 * keys in tiles of 16 cells re-sorted every 4, 6, 10 or 16 steps, or sorted
 * once at the start; re-sorted as the particles move (FPM_BIN_FLOW); in
 * shared-memory tiles of 16 cells every 4 steps -- keeping
 * the best of reps timed replays after one warm-up, and leaves the fastest
 * set on the plan.  choice[0..2] = its (tile, sort_every, mode); ms
 * (FPM_TUNE_CONFIGS
 * floats, or NULL) the times, -1 for configurations the plan's meshes do
 * not support.  The choice is cached per device, plan flags, step count,
 * PGD and tape setting and simulation shapes: a later call with the same
 * key and retune == 0 applies it without timing (ms all -1); with
 * retune == 0, disp and mom may be NULL to apply a cached choice only
 * (FPM_ERR_STATE, plan unchanged, when there is none).  Allocates scratch
 * state and synchronises the stream; captured graphs of the plan must be
 * captured again. */
#define FPM_TUNE_CONFIGS 8
int fpm_plan_autotune(fpm_plan* plan, const float* disp, const float* mom,
                      int reps, int retune, int32_t* choice, float* ms,
                      void* stream);

/* Checkpoints: when ckpt is not NULL, fpm_nbody_run stores the state
 * (disp, mom) at every position j (after the closing kick of step j-1,
 * j = 0 the initial state) with j % ckpt_every == 0 in slot j / ckpt_every
 * of ckpt, each slot 2 x total_particles x 3 floats (disp then mom). */

/* Reverse-time adjoint of fpm_nbody_run (the FastPM adjoint method; with
 * PGD on it needs a potential tape, fpm_nbody_set_tape, else
 * FPM_ERR_UNSUPPORTED):
 * given the final state (disp, mom, force = the outputs of the forward run)
 * and the cotangents lam_x = dL/dX, lam_p = dL/dp, lam_f = dL/dF (may be
 * NULL) at the final positions, integrate the leapfrog backwards --
 * rebuilding positions and momenta from the final state instead of storing
 * the trajectory, and resetting them to the checkpoints where ckpt is given
 * -- while propagating the cotangents through every kick, drift and force
 * (paint adjoint = gather with CIC weight derivatives, readout adjoint =
 * scatter, Fourier force adjoint = conjugate transfer function).  On return
 * lam_x, lam_p hold dL/dX_0, dL/dp_0 and disp, mom the rebuilt initial
 * state.  Needs FPM_PLAN_ADJOINT and fpm_nbody_set_steps. */
int fpm_nbody_adjoint(fpm_plan* plan, float* disp, float* mom,
                      const float* force, float* lam_x, float* lam_p,
                      const float* lam_f, const float* ckpt, int ckpt_every,
                      void* stream);

/* Potential tape (4-point gradient plans; FPM_ERR_UNSUPPORTED for order-0
 * plans): while tape is set, fpm_nbody_run stores the potential of the
 * force solve at every position it (0 .. max_steps) at
 * tape + it * total_mesh_cells, and fpm_nbody_adjoint takes the force
 * meshes of each position from the stencil of that potential instead of
 * painting the rebuilt positions and solving again; the forward values
 * replace the rebuilt ones, which removes the reconstruction drift from
 * the forces.  total_mesh_cells (Nc) is the sum over the simulations of
 * (pm_nc_factor)^3 nx ny nz; floats must be at least (max_steps + 1) Nc
 * (checked by both calls: FPM_ERR_ARG).  With PGD on (fpm_nbody_set_pgd)
 * the tape also holds, per step it < max_steps, the PGD potential at
 * (max_steps + 1 + it) Nc and the displacement before the PGD move at
 * (2 max_steps + 1) Nc + 3 it Np (Np = total particles): (2 max_steps + 1)
 * Nc + 3 max_steps Np floats in all.  This is what makes the PGD step
 * differentiable: the reverse sweep cannot undo the move, so it takes x'
 * from the tape and propagates the cotangents through the PGD readout,
 * its transfer function and its paint (flowpm/tfpm.py:369-422).  The
 * adjoint must follow a forward run with the same tape and steps.  NULL detaches; setting or
 * detaching a tape invalidates captured graphs (FPM_ERR_STATE).  This has
 * no counterpart in the reference, whose tape stores every TF op. */
int fpm_nbody_set_tape(fpm_plan* plan, float* tape, int64_t floats);

/* 2LPT initial conditions, flowpm/tfpm.py:148-180 lpt_init: from the real
 * linear field (the plan's lattice meshes concatenated) compute the 1LPT
 * and 2LPT displacements at the lattice points and
 *   d = D1 psi1 + D2 psi2, p = c[2] D1 psi1 + c[3] D2 psi2,
 *   f = c[4] D1 psi1 + c[5] D2 psi2
 * with coef[s*6 + 0..5] = {D1, D2, a^2 f1 E, a^2 f2 E, a^2 E gf / D1,
 * a^2 E gf2 / D2}.  order 1 skips the 2LPT term.  Needs FPM_PLAN_LPT. */
int fpm_lpt_init(fpm_plan* plan, const float* linear, const double* coef,
                 int order, float* disp, float* mom, float* force,
                 void* stream);

/* First-order LPT displacement read out at arbitrary positions,
 * flowpm/tfpm.py:66-95 lpt1: for each simulation s of the plan,
 *   psi_d = c2r3d(dlin_k * laplace_kernel * gradient_kernel_d)
 *   disp[s, p, d] = cic_readout(psi_d, pos[s, p]).
 * dlin_k is the full complex spectrum r2c3d(linear) (FFT / N^3) of each
 * simulation, (nx, ny, nz) complex64 concatenated; only l <= nz/2 is read
 * (the spectrum of a real field).  pos and disp are (nsims, npart, 3) in
 * lattice units.  Needs FPM_PLAN_LPT. */
int fpm_lpt1(fpm_plan* plan, const void* dlin_k, const float* pos,
             int64_t npart, float* disp, void* stream);

/* Second-order LPT source, flowpm/tfpm.py:98-145 lpt2_source:
 *   phi_ij = c2r3d(dlin_k * laplace_kernel * g_i g_j),
 *   source = 3/7 sum_{i<j} (phi_ii phi_jj - phi_ij^2),
 *   source_k = r2c3d(source) (FFT / N^3),
 * written as full complex spectra (nx, ny, nz) complex64 per simulation.
 * dlin_k as in fpm_lpt1.  Needs FPM_PLAN_LPT. */
int fpm_lpt2_source(fpm_plan* plan, const void* dlin_k, void* source_k,
                    void* stream);

/* CUDA graphs: capture one fpm_nbody_run (or fpm_nbody_adjoint) with the
 * given buffers into an executable graph, then replay it with
 * fpm_graph_launch on any stream, with one launch instead of ~10 per
 * leapfrog step.  The graph reads the plan's step tables at replay time,
 * so fpm_nbody_set_steps may change their values, but a call that changes
 * max_steps (or reallocates the tables) makes fpm_graph_launch return
 * FPM_ERR_STATE.  Capture runs on a private stream and executes nothing.
 * The graph must be destroyed before its plan. */
int fpm_graph_capture_nbody(fpm_plan* plan, float* disp, float* mom,
                            float* force, float* inter, unsigned flags,
                            float* ckpt, int ckpt_every, fpm_graph** graph);
int fpm_graph_capture_adjoint(fpm_plan* plan, float* disp, float* mom,
                              const float* force, float* lam_x, float* lam_p,
                              const float* lam_f, const float* ckpt,
                              int ckpt_every, fpm_graph** graph);
int fpm_graph_launch(fpm_graph* graph, void* stream);
int fpm_graph_destroy(fpm_graph* graph);

/* Vector-Jacobian product of fpm_lpt_init with respect to the linear
 * field: lam_linear = d/d(linear) of sum(lam_disp . d + lam_mom . p +
 * lam_force . f) (lam_mom, lam_force may be NULL).  Synchronises the
 * stream.  Needs FPM_PLAN_LPT. */
int fpm_lpt_adjoint(fpm_plan* plan, const float* linear, const double* coef,
                    int order, const float* lam_disp, const float* lam_mom,
                    const float* lam_force, float* lam_linear, void* stream);

/* Gaussian white noise N(0, sqrt(N^3)) per cell on every simulation's
 * lattice (Philox4x32-10 counter RNG + Box-Muller), then
 * linear = c2r(r2c(white) * amp), flowpm/tfpm.py:15-63 linear_field.
 * amp is the half-spectrum amplitude sqrt(P(|k|) / V) per simulation
 * (lattice half spectra concatenated, nx*ny*(nz/2+1) each).  white may be
 * NULL; when it is not NULL and generate == 0 it is read instead of
 * generated.  Needs FPM_PLAN_LPT. */
int fpm_linear_field(fpm_plan* plan, const float* amp, uint64_t seed,
                     int generate, float* white, float* linear,
                     void* stream);

/* out = in + sign * q for every particle of a uniform batch of lattices
 * (batch, nx*ny*nz, 3): sign -1 turns absolute positions X into lattice
 * displacements, +1 turns displacements back into X = q + d (the
 * reference's X = DX + Q, flowpm/tfpm.py:179).  in may equal out. */
int fpm_lattice_shift(const float* in, float* out, int batch, int nx, int ny,
                      int nz, int sign, void* stream);

/* y = y + a * x with the two roundings of the reference's kick and drift
 * updates (update = fac * F; state = state + update, flowpm/tfpm.py:287-292,
 * :309-314). */
int fpm_saxpy(float* y, const float* x, float a, int64_t n, void* stream);

/* ---------------------------------------------------------------------
 * Power spectrum, the estimator of flowpm/pk.py:7-103 (power_spectrum):
 * P[b][i] = sum W |F|^2 / sum W over the modes with
 * numpy.digitize(|k|, edges) == i + 1, times prod(boxsize) / ncell^2, for
 * i < nedges - 1, where edges[n] = kmin + n * dk, F the unnormalised FFT
 * of the field and W the reference's mode weights (1 on the z planes 0 and
 * nz - 1 of the full spectrum, 2 elsewhere).  boxsize holds 3 doubles;
 * power is (batch, nedges - 1) floats.
 * ------------------------------------------------------------------ */

/* From the unnormalised R2C half spectrum (batch, nx, ny, nz/2 + 1) of the
 * field.  Takes its bin accumulators (2 x batch x (nedges + 1) doubles)
 * from the stream-ordered allocator.  Any nedges >= 2: up to 3071 edges
 * the bins are summed in shared memory first, above that directly in the
 * accumulators. */
int fpm_pk_bin(const void* delta_k, int batch, int nx, int ny, int nz,
               const double* boxsize, double kmin, double dk, int nedges,
               float* power, void* stream);

/* Capacity, in doubles, of the fixed device array behind
 * fpm_pk_bin_noalloc: 2 * batch * (nedges + 1) must not exceed it. */
#define FPM_PK_NOALLOC_MAX_DOUBLES 16384

/* fpm_pk_bin without any device allocation.  No counterpart in the
 * reference.  For callers that cannot let a library allocate device memory:
 * applications that give all of a GPU's memory to their own pool or arena,
 * so that a cudaMalloc / cudaMallocAsync from here would fail or fragment
 * it, and loops that forbid allocation after start-up because allocating
 * can synchronise the device.  The bin sums live in a fixed 128 KiB array
 * inside this library (FPM_PK_NOALLOC_MAX_DOUBLES doubles), which every GPU
 * that loads the library holds until the process exits; requests with
 * 2 * batch * (nedges + 1) above that return FPM_ERR_LIMIT.  The caller
 * passes the inputs and the output as for fpm_pk_bin; every nedges that
 * fpm_pk_bin takes is accepted within that limit.  The first call on a
 * device looks up the array's device address (once per device) -- make
 * that first call before any stream capture; the address is kept for the
 * life of the process, so do not cudaDeviceReset in between.  All calls
 * share the one
 * array and each clears the part it uses before summing, so calls whose
 * execution overlaps on the GPU (several streams, several host threads)
 * race; order them on one stream. */
int fpm_pk_bin_noalloc(const void* delta_k, int batch, int nx, int ny, int nz,
                       const double* boxsize, double kmin, double dk,
                       int nedges, float* power, void* stream);

/* From the real field (batch, nx, ny, nz): R2C then fpm_pk_bin.  The
 * cuFFT plan of each (device, batch, nx, ny, nz) is created on first use
 * and kept, with its work area; at most 8 such plans are kept, and making
 * a ninth destroys the least recently used one (which waits for the work
 * queued on the device). */
int fpm_power_spectrum(const float* field, int batch, int nx, int ny, int nz,
                       const double* boxsize, double kmin, double dk,
                       int nedges, float* power, void* stream);

/* Gaussian white noise alone: out[e] = stddev * N(0,1) for e < n with the
 * generator of fpm_linear_field (counter = element index). */
int fpm_white_noise(float* out, int64_t n, uint64_t seed, double stddev,
                    void* stream);

/* 2-D CIC paint, flowpm/utils.py:94-160 cic_paint_2d: mesh (batch, nx, ny)
 * += the 4-neighbour CIC weights of part (batch, npart, 2) in mesh units,
 * times weight (batch, npart; NULL: 1), for the particles whose mask byte
 * (batch, npart; NULL: all) is non-zero.  Indices wrap modulo ny on both
 * axes, as the reference's; with nx < ny an x index may reach nx or more,
 * and such deposits are left out and reported as FPM_ERR_RANGE.
 * Synchronises the stream. */
int fpm_cic_paint_2d(float* mesh, int batch, int nx, int ny, const float* part,
                     int64_t npart, const float* weight, const uint8_t* mask,
                     void* stream);
/* Its adjoint for the mesh cotangent grad_mesh: grad_part (batch, npart, 2)
 * and grad_weight (batch, npart), either may be NULL (not written). */
int fpm_cic_paint_2d_adjoint(const float* grad_mesh, int batch, int nx,
                             int ny, const float* part, int64_t npart,
                             const float* weight, const uint8_t* mask,
                             float* grad_part, float* grad_weight,
                             void* stream);

/* Lensing density planes, flowpm/raytracing.py:49-109 density_plane, for
 * nplanes (<= 64) slabs at once: X (batch, npart, 3) positions in mesh
 * units; rotation (row-major 3x3, applied as R x) and shift (times
 * nx, ny, nz), each NULL for none; xy modulo nx, scaled by res / nx;
 * particles with center - width/2 < z <= center + width/2 painted into
 * slab p of planes (batch, nplanes, res, res), which is then divided by
 * (nx / res) (ny / res) width.  Synchronises the stream. */
int fpm_density_planes(const float* X, int batch, int64_t npart, int nx,
                       int ny, int nz, const double* rotation,
                       const double* shift, int nplanes, const double* centers,
                       const double* widths, int res, float* planes,
                       void* stream);
/* Its adjoint: grad_X (batch, npart, 3) for the plane cotangent. */
int fpm_density_planes_adjoint(const float* X, int batch, int64_t npart,
                               int nx, int ny, int nz, const double* rotation,
                               const double* shift, int nplanes,
                               const double* centers, const double* widths,
                               int res, const float* grad_planes,
                               float* grad_X, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FLOWPM_B200_H */
