// Adjoint (reverse-mode) kernels of the particle-mesh step: the
// vector-Jacobian products of CIC paint (a gather with the weight
// derivatives), CIC readout (a scatter), the Fourier force (the conjugate
// transfer function) and LPT, plus the reverse-time leapfrog that rebuilds
// the trajectory instead of storing it (FastPM adjoint method).
//
// CIC weight derivative: w = 1 - |y - n| per axis, dw/dy = -sign(y - n) with
// sign(0) = 0 (the convention of the reference's tape gradient of tf.abs):
// -1 for the lower neighbour when y is not on the cell face, 0 when it is,
// +1 for the upper neighbour.
#include <atomic>

#include "fpm_adjoint.cuh"

namespace fpm {

// Derivatives of the two axis weights.
struct DAxis {
  float d0, d1;
};
__device__ __forceinline__ DAxis cic_daxis(float y) {
  DAxis r;
  r.d0 = (y - floorf(y) > 0.f) ? -1.f : 0.f;
  r.d1 = 1.f;
  return r;
}

// acc += v * grad_y W for neighbour c.
__device__ __forceinline__ void grad_acc(const Axis& ax, const Axis& ay,
                                         const Axis& az, const DAxis& dx,
                                         const DAxis& dy, const DAxis& dz,
                                         int cx, int cy, int cz, float v,
                                         float3& acc) {
  const float wx = cx ? ax.w1 : ax.w0, wy = cy ? ay.w1 : ay.w0,
              wz = cz ? az.w1 : az.w0;
  const float gx = cx ? dx.d1 : dx.d0, gy = cy ? dy.d1 : dy.d0,
              gz = cz ? dz.d1 : dz.d0;
  acc.x += v * (gx * wy * wz);
  acc.y += v * (wx * gy * wz);
  acc.z += v * (wx * wy * gz);
}

// sum_c m[c] grad W(y - c)
__device__ __forceinline__ float3 gather_grad(const float* __restrict__ m,
                                              int mx, int my, int mz,
                                              float3 y) {
  const Axis ax = cic_axis(y.x, mx), ay = cic_axis(y.y, my),
             az = cic_axis(y.z, mz);
  const DAxis dx = cic_daxis(y.x), dy = cic_daxis(y.y), dz = cic_daxis(y.z);
  float3 acc = make_float3(0.f, 0.f, 0.f);
  // 32-bit offsets inside one simulation's mesh (< 2^31 cells)
  const unsigned rx0 = (unsigned)ax.i0 * (unsigned)my;
  const unsigned rx1 = (unsigned)ax.i1 * (unsigned)my;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int cx = conn_x(c), cy = conn_y(c), cz = conn_z(c);
    const unsigned o =
        ((cx ? rx1 : rx0) + (unsigned)(cy ? ay.i1 : ay.i0)) * (unsigned)mz +
        (unsigned)(cz ? az.i1 : az.i0);
    grad_acc(ax, ay, az, dx, dy, dz, cx, cy, cz, __ldg(m + o), acc);
  }
  return acc;
}

// ---------------------------------------------------------------------------
// Reverse-time leapfrog
// ---------------------------------------------------------------------------

// Transition from position it+1 to it of every sim with it < T:
//   lam_x += B * sum_c lam_rho[c] grad W   (paint adjoint at x_{it+1})
//   p_half = p - ke F_{it+1};  d -= dr p_half  (or the checkpoint)
//   lam_ph = lam_p + dr lam_x
// then paint x_it (also for the sims starting their reverse sweep, it == T).
// it = -1: only the final gather at position 0.
__global__ void __launch_bounds__(kThreads, FPM_STEP_MINBLOCKS)
k_adj_drift_paint(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
                  AdjArgs a) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kTraverse);
    const SimDev S = sims[s];
    const int T = a.nsteps[s];
    if (a.it > T) continue;
    const float* cf = a.coefs + (int64_t)s * a.max_steps * 3;
    const float b = (float)S.bf;
    const bool rec = a.it >= 0 && a.it < T;
    const float ke = rec ? cf[a.it * 3 + 2] : 0.f;
    const float dr = rec ? cf[a.it * 3 + 1] : 0.f;
    const float* lr = a.lrho + S.m_off;
    float* m = a.rho + S.m_off;
    const bool ck = rec && a.ckpt && (a.it % a.ckpt_every == 0);
    const float* ckd =
        ck ? a.ckpt + (int64_t)(a.it / a.ckpt_every) * 2 * a.total_np * 3
           : nullptr;
    const Walk w = walk_chunk(S, ch - traverse_first(S));
#pragma unroll 1
    for (int item = 0; item < S.wi; ++item) {
      int i, j, k;
      int64_t local;
      if (!walk_particle(S, w, item, i, j, k, local)) continue;
      const int64_t g = S.p_off + local;
      float3 d = ld3(a.disp, g);
      if (a.it < T) {
        const float3 gg = gather_grad(lr, S.mx, S.my, S.mz,
                                      mesh_pos(S, i, j, k, d));
        float3 lx = ld3(a.lam_x, g);
        lx.x += b * gg.x;
        lx.y += b * gg.y;
        lx.z += b * gg.z;
        if (rec) {
          const float3 f = ld3(a.fpart, g);
          const float3 p = ld3(a.mom, g);
          const float3 ph = make_float3(__fsub_rn(p.x, __fmul_rn(ke, f.x)),
                                        __fsub_rn(p.y, __fmul_rn(ke, f.y)),
                                        __fsub_rn(p.z, __fmul_rn(ke, f.z)));
          d = make_float3(__fsub_rn(d.x, __fmul_rn(dr, ph.x)),
                          __fsub_rn(d.y, __fmul_rn(dr, ph.y)),
                          __fsub_rn(d.z, __fmul_rn(dr, ph.z)));
          if (ckd) d = ld3(ckd, g);
          float3 lp = ld3(a.lam_p, g);
          lp.x += dr * lx.x;
          lp.y += dr * lx.y;
          lp.z += dr * lx.z;
          st3(a.mom, g, ph);
          st3(a.disp, g, d);
          st3(a.lam_p, g, lp);
        }
        st3(a.lam_x, g, lx);
      }
      if (a.it < 0) continue;
      const float3 x = mesh_pos(S, i, j, k, d);
      if (!finite3(x.x, x.y, x.z)) atomicOr(a.status, FPM_STATUS_NONFINITE_POS);
      paint8(m, S.mx, S.my, S.mz, cic_axis(x.x, S.mx), cic_axis(x.y, S.my),
             cic_axis(x.z, S.mz));
    }
  }
}

// At position it (force meshes of x_it ready): readout F_it, finish the
// momentum reconstruction p_it = p_half - ks F_it, and the force VJP with
// cotangent v = (ks_it + ke_{it-1}) lam_p (+ lam_F at the last position):
//   lam_x += fac * sum_c grad W * (v . f[c])            (readout weights)
//   lam_f[c] += (fac / B) * v * W                       (scatter)
template <int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
k_adj_vjp(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
          AdjArgs a) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kTraverse);
    const SimDev S = sims[s];
    const int T = a.nsteps[s];
    if (a.it > T) continue;
    const float* cf = a.coefs + (int64_t)s * a.max_steps * 3;
    const float ks = a.it < T ? cf[a.it * 3 + 0] : 0.f;
    const float kep = a.it >= 1 ? cf[(a.it - 1) * 3 + 2] : 0.f;
    const float cv = ks + kep;
    const bool last = a.it == T;
    const float fac = a.ffac[s];
    const float b = (float)S.bf;
    const float invb = 1.0f / b;
    const float uf = fac * invb;
    const int64_t mcells = (int64_t)S.mx * S.my * S.mz;
    const float* f0 = a.fmesh + 3 * S.m_off;
    float* l0 = a.lmesh + (a.lvec4 ? 4 : 3) * S.m_off;
    const bool ck = !last && a.ckpt && (a.it % a.ckpt_every == 0);
    const float* ckp =
        ck ? a.ckpt + (int64_t)(a.it / a.ckpt_every) * 2 * a.total_np * 3 +
                 a.total_np * 3
           : nullptr;
    const Walk w = walk_chunk(S, ch - traverse_first(S));
#pragma unroll 1
    for (int item = 0; item < S.wi; ++item) {
      int i, j, k;
      int64_t local;
      if (!walk_particle(S, w, item, i, j, k, local)) continue;
      const int64_t g = S.p_off + local;
      const float3 d = ld3(a.disp, g);
      const float3 lp = ld3(a.lam_p, g);
      float3 v = make_float3(cv * lp.x, cv * lp.y, cv * lp.z);
      if (last && a.lam_f) {
        const float3 lf = ld3(a.lam_f, g);
        v.x += lf.x;
        v.y += lf.y;
        v.z += lf.z;
      }
      const float3 y = mesh_pos(S, i, j, k, d);
      const Axis ax = cic_axis(y.x, S.mx), ay = cic_axis(y.y, S.my),
                 az = cic_axis(y.z, S.mz);
      const DAxis dx = cic_daxis(y.x), dy = cic_daxis(y.y),
                  dz = cic_daxis(y.z);
      float r0 = 0.f, r1 = 0.f, r2 = 0.f;
      float3 acc = make_float3(0.f, 0.f, 0.f);
      const float u0 = uf * v.x, u1 = uf * v.y, u2 = uf * v.z;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int cx = conn_x(c), cy = conn_y(c), cz = conn_z(c);
        const float w = cic_w(ax, ay, az, cx, cy, cz);
        const int ix = cx ? ax.i1 : ax.i0, iy = cy ? ay.i1 : ay.i0,
                  iz = cz ? az.i1 : az.i0;
        const int64_t o = ((int64_t)ix * S.my + iy) * S.mz + iz;
        const float a0 = __ldg(f0 + o), a1 = __ldg(f0 + mcells + o),
                    a2 = __ldg(f0 + 2 * mcells + o);
        r0 = __fadd_rn(r0, __fmul_rn(a0, w));
        r1 = __fadd_rn(r1, __fmul_rn(a1, w));
        r2 = __fadd_rn(r2, __fmul_rn(a2, w));
        grad_acc(ax, ay, az, dx, dy, dz, cx, cy, cz,
                 v.x * a0 + v.y * a1 + v.z * a2, acc);
        if (a.lvec4) {  // one 16-byte reduction for the three components
          red_add_v4(l0 + 4 * o, u0 * w, u1 * w, u2 * w);
        } else {
          red_add(l0 + o, u0 * w);
          red_add(l0 + mcells + o, u1 * w);
          red_add(l0 + 2 * mcells + o, u2 * w);
        }
      }
      const float3 f = make_float3(__fmul_rn(__fmul_rn(r0, fac), invb),
                                   __fmul_rn(__fmul_rn(r1, fac), invb),
                                   __fmul_rn(__fmul_rn(r2, fac), invb));
      float3 lx = ld3(a.lam_x, g);
      lx.x += fac * acc.x;
      lx.y += fac * acc.y;
      lx.z += fac * acc.z;
      st3(a.lam_x, g, lx);
      st3(a.fpart, g, f);
      if (!last) {
        float3 p = ld3(a.mom, g);
        p = make_float3(__fsub_rn(p.x, __fmul_rn(ks, f.x)),
                        __fsub_rn(p.y, __fmul_rn(ks, f.y)),
                        __fsub_rn(p.z, __fmul_rn(ks, f.z)));
        if (ckp) p = ld3(ckp, g);
        st3(a.mom, g, p);
      }
    }
  }
}

// Per-simulation constants of one reverse position of k_adj_position.
struct AdjPos {
  float b, dr, ks, kep, cv, fac, invb, uf;
  bool rec, last;
  int64_t mcells;
  const float* lr;
  const float* f0;
  float* l0;
  const float* ckd;
  const float* ckp;
};

// false when simulation s has no position a.it (it has fewer steps).
__device__ __forceinline__ bool adj_pos_setup(const SimDev& S, int s,
                                              const AdjArgs& a, AdjPos& c) {
  const int T = a.nsteps[s];
  if (a.it > T) return false;
  const float* cf = a.coefs + (int64_t)s * a.max_steps * 3;
  c.b = (float)S.bf;
  c.rec = a.it < T;  // a.it >= 0 here
  c.dr = c.rec ? cf[a.it * 3 + 1] : 0.f;
  c.ks = c.rec ? cf[a.it * 3 + 0] : 0.f;
  c.kep = a.it >= 1 ? cf[(a.it - 1) * 3 + 2] : 0.f;
  c.cv = c.ks + c.kep;
  c.last = !c.rec;
  c.fac = a.ffac[s];
  c.invb = 1.0f / c.b;
  c.uf = c.fac * c.invb;
  c.mcells = (int64_t)S.mx * S.my * S.mz;
  c.lr = a.lrho + S.m_off;
  c.f0 = a.fmesh + 3 * S.m_off;
  c.l0 = a.lmesh + (a.lvec4 ? 4 : 3) * S.m_off;
  const bool ck = c.rec && a.ckpt && (a.it % a.ckpt_every == 0);
  c.ckd = ck ? a.ckpt + (int64_t)(a.it / a.ckpt_every) * 2 * a.total_np * 3
             : nullptr;
  c.ckp = ck ? c.ckd + a.total_np * 3 : nullptr;
  return true;
}

// One particle of k_adj_position: its state in slot `slot` of the
// per-particle arrays, its lattice site (i, j, k), and g its Lagrangian
// slot in the checkpoints and lam_f.  AGG (particles sorted by cell, every
// lane of the warp calling together, `valid` false past the end): lanes
// whose force-VJP scatter starts from the same base cell sum their
// deposits with segmented shuffles, corner by corner, and the run's first
// lane deposits the sums once.
template <bool AGG>
__device__ __forceinline__ void adj_position_one(const SimDev& S,
                                                 const AdjArgs& a,
                                                 const AdjPos& c, int64_t slot,
                                                 int64_t g, int i, int j,
                                                 int k, bool valid = true) {
  const int lane = threadIdx.x & 31;
  float3 d = make_float3(0.f, 0.f, 0.f), lx = d, lp = d, ph = d;
  if (!AGG || valid) {
    d = ld3(a.disp, slot);
    lx = ld3(a.lam_x, slot);
    lp = ld3(a.lam_p, slot);
    // rec: p_half of step it (left by the position after); else p_T
    ph = ld3(a.mom, slot);
  }
  if (c.rec) {  // reverse drift from x_{it+1} (k_adj_drift_paint)
    const float3 gg = gather_grad(c.lr, S.mx, S.my, S.mz,
                                  mesh_pos(S, i, j, k, d));
    lx.x += c.b * gg.x;
    lx.y += c.b * gg.y;
    lx.z += c.b * gg.z;
    d = make_float3(__fsub_rn(d.x, __fmul_rn(c.dr, ph.x)),
                    __fsub_rn(d.y, __fmul_rn(c.dr, ph.y)),
                    __fsub_rn(d.z, __fmul_rn(c.dr, ph.z)));
    if (c.ckd) d = ld3(c.ckd, g);
    lp.x += c.dr * lx.x;
    lp.y += c.dr * lx.y;
    lp.z += c.dr * lx.z;
    if (!AGG || valid) {
      st3(a.disp, slot, d);
      st3(a.lam_p, slot, lp);
    }
  }
  // force VJP at x_it (k_adj_vjp)
  float3 v = make_float3(c.cv * lp.x, c.cv * lp.y, c.cv * lp.z);
  if (c.last && a.lam_f && (!AGG || valid)) {
    const float3 lf = ld3(a.lam_f, g);
    v.x += lf.x;
    v.y += lf.y;
    v.z += lf.z;
  }
  const float3 y = mesh_pos(S, i, j, k, d);
  if ((!AGG || valid) && !finite3(y.x, y.y, y.z))
    atomicOr(a.status, FPM_STATUS_NONFINITE_POS);
  const Axis ax = cic_axis(y.x, S.mx), ay = cic_axis(y.y, S.my),
             az = cic_axis(y.z, S.mz);
  const DAxis dx = cic_daxis(y.x), dy = cic_daxis(y.y), dz = cic_daxis(y.z);
  float r0 = 0.f, r1 = 0.f, r2 = 0.f;
  float3 acc = make_float3(0.f, 0.f, 0.f);
  const float u0 = c.uf * v.x, u1 = c.uf * v.y, u2 = c.uf * v.z;
  // 32-bit offsets inside the simulation's mesh (< 2^31 cells)
  const unsigned my = S.my, mz = S.mz;
  const unsigned rx0 = (unsigned)ax.i0 * my, rx1 = (unsigned)ax.i1 * my;
  unsigned heads = 0xffffffffu, longest = 1;
  if (AGG) {
    const unsigned key = valid ? (rx0 + (unsigned)ay.i0) * mz +
                                     (unsigned)az.i0
                               : 0xffffffffu - lane;
    heads = run_heads(key, lane);
    if (heads != 0xffffffffu)
      longest = __reduce_max_sync(
          0xffffffffu,
          (heads >> lane) & 1u ? (unsigned)run_length(heads, lane) : 1u);
  }
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int cx = conn_x(q), cy = conn_y(q), cz = conn_z(q);
    const float wc = cic_w(ax, ay, az, cx, cy, cz);
    const unsigned o =
        ((cx ? rx1 : rx0) + (unsigned)(cy ? ay.i1 : ay.i0)) * mz +
        (unsigned)(cz ? az.i1 : az.i0);
    const float a0 = __ldg(c.f0 + o), a1 = __ldg(c.f0 + c.mcells + o),
                a2 = __ldg(c.f0 + 2 * c.mcells + o);
    r0 = __fadd_rn(r0, __fmul_rn(a0, wc));
    r1 = __fadd_rn(r1, __fmul_rn(a1, wc));
    r2 = __fadd_rn(r2, __fmul_rn(a2, wc));
    grad_acc(ax, ay, az, dx, dy, dz, cx, cy, cz,
             v.x * a0 + v.y * a1 + v.z * a2, acc);
    float t0 = u0 * wc, t1 = u1 * wc, t2 = u2 * wc;
    if (AGG) {
      // segmented sums over the runs: lane + o is in this lane's run when
      // no run starts in (lane, lane + o]
#pragma unroll 1
      for (int off = 1; off < (int)longest; off <<= 1) {
        const bool same =
            lane + off < 32 &&
            ((unsigned long long)heads >> (lane + 1) & ((1ull << off) - 1)) ==
                0;
        const float s0 = __shfl_down_sync(0xffffffffu, t0, off);
        const float s1 = __shfl_down_sync(0xffffffffu, t1, off);
        const float s2 = __shfl_down_sync(0xffffffffu, t2, off);
        if (same) {
          t0 = __fadd_rn(t0, s0);
          t1 = __fadd_rn(t1, s1);
          t2 = __fadd_rn(t2, s2);
        }
      }
      if (!valid || !((heads >> lane) & 1u)) continue;
    }
    if (a.lvec4) {
      red_add_v4(c.l0 + 4 * o, t0, t1, t2);
    } else {
      red_add(c.l0 + o, t0);
      red_add(c.l0 + c.mcells + o, t1);
      red_add(c.l0 + 2 * c.mcells + o, t2);
    }
  }
  const float3 f = make_float3(__fmul_rn(__fmul_rn(r0, c.fac), c.invb),
                               __fmul_rn(__fmul_rn(r1, c.fac), c.invb),
                               __fmul_rn(__fmul_rn(r2, c.fac), c.invb));
  lx.x += c.fac * acc.x;
  lx.y += c.fac * acc.y;
  lx.z += c.fac * acc.z;
  if (AGG && !valid) return;
  st3(a.lam_x, slot, lx);
  // p_it (rec: p_half - ks F_it, or the checkpoint; else p_T), then
  // p_half of step it-1 for the next position
  float3 p = ph;
  if (c.rec) {
    p = make_float3(__fsub_rn(ph.x, __fmul_rn(c.ks, f.x)),
                    __fsub_rn(ph.y, __fmul_rn(c.ks, f.y)),
                    __fsub_rn(ph.z, __fmul_rn(c.ks, f.z)));
    if (c.ckp) p = ld3(c.ckp, g);
  }
  if (a.it >= 1)
    p = make_float3(__fsub_rn(p.x, __fmul_rn(c.kep, f.x)),
                    __fsub_rn(p.y, __fmul_rn(c.kep, f.y)),
                    __fsub_rn(p.z, __fmul_rn(c.kep, f.z)));
  if (c.rec || a.it >= 1) st3(a.mom, slot, p);
}

// k_adj_drift_paint (without its paint) and k_adj_vjp of the same position
// it in one pass over the particles, for reverse sweeps whose force meshes
// of x_it are ready before the reverse drift (the stencil of a stored
// potential): the state is read and written once instead of twice.  The
// arithmetic per particle is that of the two kernels in sequence, except
// that the momentum buffer carries p_half of the next (earlier) step,
// p_it - ke_{it-1} F_it, formed here with the same two roundings, instead
// of p_it and F_it in two buffers; the last position (it = 0) leaves p_0.
// The force buffer is not used.
template <int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
k_adj_position(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
               AdjArgs a) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kTraverse);
    const SimDev S = sims[s];
    AdjPos c;
    if (!adj_pos_setup(S, s, a, c)) continue;
    const Walk w = walk_chunk(S, ch - traverse_first(S));
#pragma unroll 1
    for (int item = 0; item < S.wi; ++item) {
      int i, j, k;
      int64_t local;
      if (!walk_particle(S, w, item, i, j, k, local)) continue;
      const int64_t g = S.p_off + local;
      adj_position_one<false>(S, a, c, g, g, i, j, k);
    }
  }
}

// k_adj_position over the particles in their binned order (sorted by the
// cell of x_{it+1}, or of a later position, keys tile-major): chunks of
// kChunk consecutive slots of one simulation.  Consecutive lanes then sit
// in the same or neighbouring cells, so the gathers and the vector
// reductions of a warp touch few L2 sectors at every time, where the
// lattice walk's warps spread over more and more of them as structure
// grows.  Per particle the arithmetic is k_adj_position's.
template <int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
k_adj_position_sorted(const SimDev* __restrict__ sims, int nsims,
                      int64_t nchunks, AdjArgs a) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kPart);
    const SimDev S = sims[s];
    AdjPos c;
    if (!adj_pos_setup(S, s, a, c)) continue;
    const int64_t first = S.p_off + (ch - S.ch_p) * kChunk;
    const int64_t end = S.p_off + S.np;
#pragma unroll 1
    for (int item = 0; item < kItems; ++item) {
      const int64_t i = first + item * kThreads + threadIdx.x;
      // every lane of the warp takes part (warp-uniform except in a sim's
      // last chunk, where lanes past the end only join the shuffles)
      const bool valid = i < end;
      if (!FPM_ADJ_SORTED_SEGSUM && !valid) break;  // no warp-wide steps
      int qi = 0, qj = 0, qk = 0;
      if (valid) unpack_site(a.lag[i], S.qkb, S.qjb, qi, qj, qk);
      adj_position_one<FPM_ADJ_SORTED_SEGSUM != 0>(
          S, a, c, i, S.p_off + site_local(S, qi, qj, qk), qi, qj, qk,
          valid);
    }
  }
}

// The PGD move of step it in reverse (flowpm/tfpm.py:369-422 apply_pgd,
// applied after the drift at :487-488): x_{it+1} = x' + (alpha / B) R(x'),
// R the readout of the PGD displacement meshes g = D phi_pgd(rho(x')).
// With lam = dL/dx_{it+1} (after the force's paint adjoint at x_{it+1}):
//   lam_x' = lam + alpha sum_c grad W(x' - c) (lam . g[c])   (readout weights)
//            + the paint adjoint of the mesh part, which starts here as the
//   scatter lf[c] += (alpha / B) lam W(x' - c)  (then divergence, PGD
//   filter, gather at x' by the next kernel).  x' comes from the tape.
__global__ void __launch_bounds__(kThreads, FPM_ADJ_MINBLOCKS)
k_adj_pgd(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
          AdjArgs a) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kTraverse);
    const SimDev S = sims[s];
    const int T = a.nsteps[s];
    if (a.it >= T) continue;  // no PGD move after position T
    const float alpha = a.pgd[((int64_t)s * a.pgd_stride + a.it) * 3];
    const float b = (float)S.bf;
    const float invb = 1.0f / b;
    const float uf = alpha * invb;
    const int64_t mcells = (int64_t)S.mx * S.my * S.mz;
    const float* lr = a.lrho + S.m_off;
    const float* f0 = a.fmesh + 3 * S.m_off;
    float* l0 = a.lmesh + (a.lvec4 ? 4 : 3) * S.m_off;
    const unsigned my = S.my, mz = S.mz;
    const Walk w = walk_chunk(S, ch - traverse_first(S));
#pragma unroll 1
    for (int item = 0; item < S.wi; ++item) {
      int i, j, k;
      int64_t local;
      if (!walk_particle(S, w, item, i, j, k, local)) continue;
      const int64_t g = S.p_off + local;
      const float3 d = ld3(a.disp, g);
      const float3 gg = gather_grad(lr, S.mx, S.my, S.mz,
                                    mesh_pos(S, i, j, k, d));
      float3 lx = ld3(a.lam_x, g);
      lx.x += b * gg.x;
      lx.y += b * gg.y;
      lx.z += b * gg.z;
      const float3 dp = ld3(a.pgd_disp, g);
      const float3 y = mesh_pos(S, i, j, k, dp);
      const Axis ax = cic_axis(y.x, S.mx), ay = cic_axis(y.y, S.my),
                 az = cic_axis(y.z, S.mz);
      const DAxis dx = cic_daxis(y.x), dy = cic_daxis(y.y),
                  dz = cic_daxis(y.z);
      float3 acc = make_float3(0.f, 0.f, 0.f);
      const float u0 = uf * lx.x, u1 = uf * lx.y, u2 = uf * lx.z;
      const unsigned rx0 = (unsigned)ax.i0 * my, rx1 = (unsigned)ax.i1 * my;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int cx = conn_x(c), cy = conn_y(c), cz = conn_z(c);
        const float wc = cic_w(ax, ay, az, cx, cy, cz);
        const unsigned o =
            ((cx ? rx1 : rx0) + (unsigned)(cy ? ay.i1 : ay.i0)) * mz +
            (unsigned)(cz ? az.i1 : az.i0);
        const float a0 = __ldg(f0 + o), a1 = __ldg(f0 + mcells + o),
                    a2 = __ldg(f0 + 2 * mcells + o);
        grad_acc(ax, ay, az, dx, dy, dz, cx, cy, cz,
                 lx.x * a0 + lx.y * a1 + lx.z * a2, acc);
        if (a.lvec4) {
          red_add_v4(l0 + 4 * o, u0 * wc, u1 * wc, u2 * wc);
        } else {
          red_add(l0 + o, u0 * wc);
          red_add(l0 + mcells + o, u1 * wc);
          red_add(l0 + 2 * mcells + o, u2 * wc);
        }
      }
      lx.x += alpha * acc.x;
      lx.y += alpha * acc.y;
      lx.z += alpha * acc.z;
      st3(a.lam_x, g, lx);
      st3(a.disp, g, dp);
    }
  }
}

// lam_rho_k = pre * w(k) * sum_d conj(i g_d) lam_f_d,k  (the transpose of
// the force transfer function; pre and w as in the forward kernel).
__global__ void __launch_bounds__(kThreads)
k_adj_fourier(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
              const float2* __restrict__ lk, float2* __restrict__ out,
              AxisTabs tabs, double r2, int deconv) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const SimDev S = sims[find_sim(sims, nsims, ch, kSpec)];
    const int64_t nmodes = (int64_t)S.mx * S.my * S.mzh;
    const int64_t mcells = (int64_t)S.mx * S.my * S.mz;
    const float pre = (float)((double)S.bf * S.bf * S.bf / (double)mcells);
    const double* kkx = tabs.kk + S.tab;
    const double* kky = kkx + S.mx;
    const double* kkz = kky + S.my;
    const float* gx = tabs.grad + S.tab;
    const float* gy = gx + S.mx;
    const float* gz = gy + S.my;
    const float* wx = tabs.win + S.tab;
    const float* wy = wx + S.mx;
    const float* wz = wy + S.my;
    const float2* l0 = lk + 3 * S.s_off;
    const int64_t base = (ch - S.ch_s) * kChunk + threadIdx.x;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const int64_t local = base + it * kThreads;
      if (local >= nmodes) break;
      int i, j, l;
      mode_ijl(local, S.my, S.mzh, i, j, l);
      const double kk = kkx[i] + kky[j] + kkz[l];
      float w = kk == 0.0 ? 0.f : (float)(1.0 / kk);
      if (r2 != 0.0) w *= (float)exp(-kk * r2);
      if (deconv) w *= wx[i] * wy[j] * wz[l];
      const float2 a0 = l0[local], a1 = l0[nmodes + local],
                   a2 = l0[2 * nmodes + local];
      const float g0 = gx[i], g1 = gy[j], g2 = gz[l];
      const float re = g0 * a0.y + g1 * a1.y + g2 * a2.y;
      const float im = -(g0 * a0.x + g1 * a1.x + g2 * a2.x);
      const float sc = pre * w;
      out[S.s_off + local] = make_float2(sc * re, sc * im);
    }
  }
}

// ---------------------------------------------------------------------------
// Stand-alone CIC adjoints (uniform batch)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads)
k_cic_paint_adjoint(const float* __restrict__ lmesh, int nx, int ny, int nz,
                    const float* __restrict__ part, int64_t npart,
                    int64_t total, const float* __restrict__ weight,
                    float* __restrict__ lpart, float* __restrict__ lweight) {
  const int64_t ncell = (int64_t)nx * ny * nz;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = g / npart;
    const float3 y = ld3(part, g);
    const float* m = lmesh + b * ncell;
    const float wt = weight ? weight[g] : 1.f;
    if (lpart) {
      const float3 gg = gather_grad(m, nx, ny, nz, y);
      st3(lpart, g, make_float3(wt * gg.x, wt * gg.y, wt * gg.z));
    }
    if (lweight) {
      const Axis ax = cic_axis(y.x, nx), ay = cic_axis(y.y, ny),
                 az = cic_axis(y.z, nz);
      float acc = 0.f;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int cx = conn_x(c), cy = conn_y(c), cz = conn_z(c);
        const int ix = cx ? ax.i1 : ax.i0, iy = cy ? ay.i1 : ay.i0,
                  iz = cz ? az.i1 : az.i0;
        acc += __ldg(m + ((int64_t)ix * ny + iy) * nz + iz) *
               cic_w(ax, ay, az, cx, cy, cz);
      }
      lweight[g] = acc;
    }
  }
}

__global__ void __launch_bounds__(kThreads)
k_cic_readout_adjoint(const float* __restrict__ mesh, int nx, int ny, int nz,
                      const float* __restrict__ part, int64_t npart,
                      int64_t total, const float* __restrict__ lout,
                      float* __restrict__ lmesh, float* __restrict__ lpart) {
  const int64_t ncell = (int64_t)nx * ny * nz;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = g / npart;
    const float3 y = ld3(part, g);
    const float lo = lout[g];
    if (lpart) {
      const float3 gg = gather_grad(mesh + b * ncell, nx, ny, nz, y);
      st3(lpart, g, make_float3(lo * gg.x, lo * gg.y, lo * gg.z));
    }
    if (lmesh) {
      const Axis ax = cic_axis(y.x, nx), ay = cic_axis(y.y, ny),
                 az = cic_axis(y.z, nz);
      paint_scaled(lmesh + b * ncell, nx, ny, nz, ax, ay, az, lo);
    }
  }
}

// ---------------------------------------------------------------------------
// LPT adjoint (flowpm/tfpm.py:148-180 lpt_init, :66-145 lpt1 / lpt2_source)
// ---------------------------------------------------------------------------

// lam_psi1 = D1 (lam_d + c2 lam_p + c4 lam_f), lam_psi2 = D2 (lam_d + c3
// lam_p + c5 lam_f); the particle index is the lattice cell index.
__global__ void __launch_bounds__(kThreads)
k_lpt_adj_particles(const SimDev* __restrict__ sims, int nsims,
                    int64_t nchunks, const float* __restrict__ ld,
                    const float* __restrict__ lp, const float* __restrict__ lf,
                    const float* __restrict__ coef, float* __restrict__ psi1,
                    int m1, float* __restrict__ psi2, int m2) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kPart);
    const SimDev S = sims[s];
    const int64_t ncells = (int64_t)S.nx * S.ny * S.nz;
    const float* c = coef + 6 * s;
    float* p1 = psi1 + (int64_t)m1 * S.l_off;
    float* p2 = psi2 ? psi2 + (int64_t)m2 * S.l_off : nullptr;
    const int64_t base = (ch - S.ch_p) * kChunk + threadIdx.x;
    for (int it = 0; it < kItems; ++it) {
      const int64_t local = base + it * kThreads;
      if (local >= S.np) break;
      const int64_t g = S.p_off + local;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float a = ld[3 * g + d], bp = lp ? lp[3 * g + d] : 0.f,
                    bf = lf ? lf[3 * g + d] : 0.f;
        p1[d * ncells + local] = c[0] * (a + c[2] * bp + c[4] * bf);
        if (p2) p2[d * ncells + local] = c[1] * (a + c[3] * bp + c[5] * bf);
      }
    }
  }
}

// out_k = pre * [sum_d conj(i g_d lap) L_d  (+ sum_q K_q L_{3+q})] with
// K_q = -lap g_i g_j the (real, even) LPT Hessian weights; nin = 3 or 9.
__global__ void __launch_bounds__(kThreads)
k_lpt_adj_fourier(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
                  const float2* __restrict__ in, int nin,
                  float2* __restrict__ out, AxisTabs tabs) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const SimDev S = sims[find_sim(sims, nsims, ch, kLatSpec)];
    const int64_t nmodes = (int64_t)S.nx * S.ny * S.lzh;
    const float pre = (float)(1.0 / ((double)S.nx * S.ny * S.nz));
    const double* kkx = tabs.kk + S.ltab;
    const double* kky = kkx + S.nx;
    const double* kkz = kky + S.ny;
    const float* gx = tabs.grad + S.ltab;
    const float* gy = gx + S.nx;
    const float* gz = gy + S.ny;
    const float2* L = in + (int64_t)nin * S.ls_off;
    const int64_t base = (ch - S.ch_ls) * kChunk + threadIdx.x;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const int64_t local = base + it * kThreads;
      if (local >= nmodes) break;
      int i, j, l;
      mode_ijl(local, S.ny, S.lzh, i, j, l);
      const double kk = kkx[i] + kky[j] + kkz[l];
      const float lap = kk == 0.0 ? 1.f : (float)(1.0 / kk);
      const float g[3] = {gx[i], gy[j], gz[l]};
      float re = 0.f, im = 0.f;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float gl = g[d] * lap;
        const float2 v = L[d * nmodes + local];
        re += gl * v.y;  // conj(i gl) v = -i gl (vr + i vi) = gl vi - i gl vr
        im -= gl * v.x;
      }
      if (nin == 9) {
        const int pi_[6] = {0, 1, 2, 1, 2, 0};
        const int pj_[6] = {0, 1, 2, 2, 0, 1};
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const float kq = -(lap * g[pi_[q]]) * g[pj_[q]];
          const float2 v = L[(3 + q) * nmodes + local];
          re += kq * v.x;
          im += kq * v.y;
        }
      }
      out[S.ls_off + local] = make_float2(pre * re, pre * im);
    }
  }
}

// lam_phi from lam_s = d/d(source) (3/7 [p1 p2 + p2 p0 + p0 p1 - q12^2 -
// q20^2 - q01^2]), in place over the phi meshes (slots 3..8 of 9).
__global__ void __launch_bounds__(kThreads)
k_lpt_adj_phi(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
              const float* __restrict__ ls, float* __restrict__ phi9) {
  const float c37 = (float)(3.0 / 7.0);
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const SimDev S = sims[find_sim(sims, nsims, ch, kLat)];
    const int64_t n = (int64_t)S.nx * S.ny * S.nz;
    float* ph = phi9 + 9 * S.l_off;
    const int64_t base = (ch - S.ch_l) * kChunk + threadIdx.x;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const int64_t c = base + it * kThreads;
      if (c >= n) break;
      const float l = c37 * ls[S.l_off + c];
      const float p0 = ph[3 * n + c], p1 = ph[4 * n + c], p2 = ph[5 * n + c];
      const float q12 = ph[6 * n + c], q20 = ph[7 * n + c],
                  q01 = ph[8 * n + c];
      ph[3 * n + c] = l * (p1 + p2);
      ph[4 * n + c] = l * (p2 + p0);
      ph[5 * n + c] = l * (p0 + p1);
      ph[6 * n + c] = -2.f * l * q12;
      ph[7 * n + c] = -2.f * l * q20;
      ph[8 * n + c] = -2.f * l * q01;
    }
  }
}

// ---------------------------------------------------------------------------
// Launch wrappers
// ---------------------------------------------------------------------------
void launch_adj_drift_paint(const SimDev* sims, int nsims, int64_t nchunks,
                            const AdjArgs& a, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_adj_drift_paint<<<grid_for(nchunks), kThreads, 0, st>>>(sims, nsims,
                                                            nchunks, a);
}

void launch_adj_vjp(const SimDev* sims, int nsims, int64_t nchunks,
                    const AdjArgs& a, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (a.long_walk)
    k_adj_vjp<FPM_ADJ_MINBLOCKS><<<grid_for(nchunks), kThreads, 0, st>>>(
        sims, nsims, nchunks, a);
  else
    k_adj_vjp<FPM_STEP_MINBLOCKS><<<grid_for(nchunks), kThreads, 0, st>>>(
        sims, nsims, nchunks, a);
}

void launch_adj_pgd(const SimDev* sims, int nsims, int64_t nchunks,
                    const AdjArgs& a, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_adj_pgd<<<grid_for(nchunks), kThreads, 0, st>>>(sims, nsims, nchunks, a);
}

void launch_adj_position(const SimDev* sims, int nsims, int64_t nchunks,
                         const AdjArgs& a, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (a.long_walk)
    k_adj_position<FPM_ADJ_MINBLOCKS><<<grid_for(nchunks), kThreads, 0, st>>>(
        sims, nsims, nchunks, a);
  else
    k_adj_position<FPM_STEP_MINBLOCKS>
        <<<grid_for(nchunks), kThreads, 0, st>>>(sims, nsims, nchunks, a);
}

void launch_adj_position_sorted(const SimDev* sims, int nsims,
                                int64_t nchunks, const AdjArgs& a,
                                cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_adj_position_sorted<FPM_ADJ_SORTED_MINBLOCKS>
      <<<grid_for(nchunks), kThreads, 0, st>>>(sims, nsims, nchunks, a);
}

void launch_adj_fourier(const SimDev* sims, int nsims, int64_t nchunks,
                        const float2* lk, float2* out, AxisTabs tabs,
                        double r_split2, int deconv, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_adj_fourier<<<grid_for(nchunks), kThreads, 0, st>>>(
      sims, nsims, nchunks, lk, out, tabs, r_split2, deconv);
}

void launch_lpt_adj_particles(const SimDev* sims, int nsims, int64_t nchunks,
                              const float* ld, const float* lp,
                              const float* lf, const float* coef, float* psi1,
                              int m1, float* psi2, int m2, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_lpt_adj_particles<<<grid_for(nchunks), kThreads, 0, st>>>(
      sims, nsims, nchunks, ld, lp, lf, coef, psi1, m1, psi2, m2);
}

void launch_lpt_adj_fourier(const SimDev* sims, int nsims, int64_t nchunks,
                            const float2* in, int nin, float2* out,
                            AxisTabs tabs, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_lpt_adj_fourier<<<grid_for(nchunks), kThreads, 0, st>>>(
      sims, nsims, nchunks, in, nin, out, tabs);
}

void launch_lpt_adj_phi(const SimDev* sims, int nsims, int64_t nchunks,
                        const float* ls, float* phi9, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_lpt_adj_phi<<<grid_for(nchunks), kThreads, 0, st>>>(sims, nsims, nchunks,
                                                        ls, phi9);
}

}  // namespace fpm

using namespace fpm;

static unsigned grid_elems_adj(int64_t n) {
  int64_t blocks = (n + kThreads - 1) / kThreads;
  const int64_t cap = (int64_t)kNumSMs * 32;
  if (blocks < 1) blocks = 1;
  return (unsigned)(blocks < cap ? blocks : cap);
}

extern "C" int fpm_cic_paint_adjoint(const float* lam_mesh, int batch, int nx,
                                     int ny, int nz, const float* part,
                                     int64_t npart, const float* weight,
                                     float* lam_part, float* lam_weight,
                                     void* stream) {
  if (!lam_mesh || batch < 1 || nx < 1 || ny < 1 || nz < 1 || npart < 0 ||
      (npart > 0 && !part) || (!lam_part && !lam_weight))
    return FPM_ERR_ARG;
  const int64_t total = (int64_t)batch * npart;
  if (total == 0) return FPM_OK;
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_cic_paint_adjoint<<<grid_elems_adj(total), kThreads, 0,
                        (cudaStream_t)stream>>>(lam_mesh, nx, ny, nz, part,
                                                npart, total, weight, lam_part,
                                                lam_weight);
  return cudaGetLastError() == cudaSuccess ? FPM_OK : FPM_ERR_CUDA;
}

extern "C" int fpm_cic_readout_adjoint(const float* mesh, int batch, int nx,
                                       int ny, int nz, const float* part,
                                       int64_t npart, const float* lam_out,
                                       float* lam_mesh, float* lam_part,
                                       void* stream) {
  if (batch < 1 || nx < 1 || ny < 1 || nz < 1 || npart < 0 ||
      (npart > 0 && (!part || !lam_out)) || (!lam_mesh && !lam_part) ||
      (lam_part && !mesh))
    return FPM_ERR_ARG;
  const int64_t total = (int64_t)batch * npart;
  if (total == 0) return FPM_OK;
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_cic_readout_adjoint<<<grid_elems_adj(total), kThreads, 0,
                          (cudaStream_t)stream>>>(mesh, nx, ny, nz, part,
                                                  npart, total, lam_out,
                                                  lam_mesh, lam_part);
  return cudaGetLastError() == cudaSuccess ? FPM_OK : FPM_ERR_CUDA;
}
