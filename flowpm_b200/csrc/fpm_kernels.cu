// Particle-mesh step kernels for sm_100a.
//
// All kernels are persistent grid-stride loops over "chunks" of kChunk
// elements; a chunk never straddles two simulations, and the owning
// simulation is found by binary search over the per-sim first chunk, so the
// same launch advances a batch of simulations of different sizes.
#include <atomic>

#include "fpm_kernels.cuh"

namespace fpm {

// ---------------------------------------------------------------------------
// Particle kernels
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kThreads, FPM_STEP_MINBLOCKS)
k_paint_lattice(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
                const float* __restrict__ disp, float* __restrict__ rho,
                int32_t* status) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const SimDev S = sims[find_sim(sims, nsims, ch, kTraverse)];
    const Walk w = walk_chunk(S, ch - traverse_first(S));
    float* m = rho + S.m_off;
#pragma unroll 4
    for (int it = 0; it < S.wi; ++it) {
      int i, j, k;
      int64_t local;
      if (!walk_particle(S, w, it, i, j, k, local)) continue;
      const float3 d = ld3(disp, S.p_off + local);
      const float3 x = mesh_pos(S, i, j, k, d);
      if (!finite3(x.x, x.y, x.z)) atomicOr(status, FPM_STATUS_NONFINITE_POS);
      paint8(m, S.mx, S.my, S.mz, cic_axis(x.x, S.mx), cic_axis(x.y, S.my),
             cic_axis(x.z, S.mz));
    }
  }
}

__global__ void __launch_bounds__(kThreads, FPM_STEP_MINBLOCKS)
k_step(const SimDev* __restrict__ sims, int nsims, int64_t ch0,
       int64_t nchunks, StepArgs a) {
  pdl_wait();  // the force meshes of the solve before
  for (int64_t ch = ch0 + blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kTraverse);
    const SimDev S = sims[s];
    const int T = a.nsteps[s];
    if (a.it > T) continue;  // this sim has finished
    const float* cf = a.coefs + (int64_t)s * a.max_steps * 3;
    const float ke = a.it >= 1 ? cf[(a.it - 1) * 3 + 2] : 0.f;
    const bool last = (a.it == T);
    const float ks = last ? 0.f : cf[a.it * 3 + 0];
    const float dr = last ? 0.f : cf[a.it * 3 + 1];
    const float fac = a.ffac[s];
    const float invb = 1.0f / (float)S.bf;
    const int64_t mcells = (int64_t)S.mx * S.my * S.mz;
    float* m = a.rho + S.m_off;
    const Walk w = walk_chunk(S, ch - traverse_first(S));
#pragma unroll 1
    for (int it = 0; it < S.wi; ++it) {
      int i, j, k;
      int64_t local;
      // missing particles of edge blocks skip their memory accesses
      const bool valid = walk_particle(S, w, it, i, j, k, local);
      const int64_t g = S.p_off + local;
      float3 d = make_float3(0.f, 0.f, 0.f), p = d;
      if (valid) {
        d = ld3(a.disp, g);
        p = ld3(a.mom, g);
      }
      const float3 x = mesh_pos(S, i, j, k, d);
      const Cic8 c0 = cic8(cic_axis(x.x, S.mx), cic_axis(x.y, S.my),
                           cic_axis(x.z, S.mz), S.my, S.mz);
      float3 f = valid ? readout_cic8(a.fmesh + 3 * S.m_off, mcells, c0)
                       : make_float3(0.f, 0.f, 0.f);
      // force = readout * factor / pm_nc_factor (flowpm/tfpm.py:218, :356)
      f.x = __fmul_rn(__fmul_rn(f.x, fac), invb);
      f.y = __fmul_rn(__fmul_rn(f.y, fac), invb);
      f.z = __fmul_rn(__fmul_rn(f.z, fac), invb);
      if (a.it >= 1) p = axpy(p, ke, f);  // closing kick of step it-1
      if (valid && a.ckpt && a.it % a.ckpt_every == 0) {
        float* o = a.ckpt + (int64_t)(a.it / a.ckpt_every) * 2 * a.total_np * 3;
        st3(o, g, d);
        st3(o + a.total_np * 3, g, p);
      }
      if (valid && a.inter && a.it >= 1) {
        float* o = a.inter + (int64_t)(a.it - 1) * 3 * a.total_np * 3;
        st3(o, g,
            make_float3(__fadd_rn(index_float(i), d.x),
                        __fadd_rn(index_float(j), d.y),
                        __fadd_rn(index_float(k), d.z)));
        st3(o + a.total_np * 3, g, p);
        st3(o + 2 * a.total_np * 3, g, f);
      }
      if (last) {  // uniform over the block: one sim per chunk
        if (valid) {
          st3(a.force_out, g, f);
          st3(a.mom, g, p);
          if (!finite3(p.x, p.y, p.z) || !finite3(f.x, f.y, f.z))
            atomicOr(a.status, FPM_STATUS_NONFINITE_MOM);
        }
        continue;
      }
      p = axpy(p, ks, f);  // opening kick of step it
      d = axpy(d, dr, p);  // drift of step it
      const float3 xn = mesh_pos(S, i, j, k, d);
      if (valid) {
        st3(a.mom, g, p);
        st3(a.disp, g, d);
        if (!finite3(xn.x, xn.y, xn.z))
          atomicOr(a.status, FPM_STATUS_NONFINITE_POS);
      }
      const Cic8 c1 = cic8(cic_axis(xn.x, S.mx), cic_axis(xn.y, S.my),
                           cic_axis(xn.z, S.mz), S.my, S.mz);
      if (valid) paint_cic8(m, c1, 1.f);
    }
  }
}

// PGD correction of one step (flowpm/tfpm.py:369-422, applied after the
// drift at :487-488): readout of the three PGD displacement meshes at
// (q + d) * bf, d += (alpha * R) / bf (the reference's update = readout *
// alpha / pm_nc_factor), then the paint of the moved particle into rho
// (zeroed by the PGD solve) for the force that follows.  pgd holds rows
// (alpha, kl, ks) of stride pgd_stride per sim; with nsteps, the row of
// step pos and only the sims with nsteps > pos (the ones that drifted).
__global__ void __launch_bounds__(kThreads, FPM_STEP_MINBLOCKS)
k_pgd(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
      float* __restrict__ disp, const float* __restrict__ fmesh,
      float* __restrict__ rho, const float* __restrict__ pgd, int pgd_stride,
      int pos, const int32_t* __restrict__ nsteps, int32_t* status) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kTraverse);
    if (nsteps && nsteps[s] <= pos) continue;
    const SimDev S = sims[s];
    const float alpha =
        pgd[((int64_t)s * pgd_stride + (nsteps ? pos : 0)) * 3];
    const float b = (float)S.bf;
    const int64_t mcells = (int64_t)S.mx * S.my * S.mz;
    float* m = rho + S.m_off;
    const Walk w = walk_chunk(S, ch - traverse_first(S));
#pragma unroll 1
    for (int it = 0; it < S.wi; ++it) {
      int i, j, k;
      int64_t local;
      if (!walk_particle(S, w, it, i, j, k, local)) continue;
      const int64_t g = S.p_off + local;
      float3 d = ld3(disp, g);
      const float3 x = mesh_pos(S, i, j, k, d);
      const float3 r = readout_cic8(fmesh + 3 * S.m_off, mcells,
                                    cic8(cic_axis(x.x, S.mx),
                                         cic_axis(x.y, S.my),
                                         cic_axis(x.z, S.mz), S.my, S.mz));
      d.x = __fadd_rn(d.x, __fdiv_rn(__fmul_rn(r.x, alpha), b));
      d.y = __fadd_rn(d.y, __fdiv_rn(__fmul_rn(r.y, alpha), b));
      d.z = __fadd_rn(d.z, __fdiv_rn(__fmul_rn(r.z, alpha), b));
      st3(disp, g, d);
      const float3 xn = mesh_pos(S, i, j, k, d);
      if (!finite3(xn.x, xn.y, xn.z)) atomicOr(status, FPM_STATUS_NONFINITE_POS);
      paint8(m, S.mx, S.my, S.mz, cic_axis(xn.x, S.mx), cic_axis(xn.y, S.my),
             cic_axis(xn.z, S.mz));
    }
  }
}

__global__ void __launch_bounds__(kThreads, FPM_STEP_MINBLOCKS)
k_force_readout(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
                const float* __restrict__ disp,
                const float* __restrict__ fmesh,
                const float* __restrict__ ffac, float* __restrict__ force) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kTraverse);
    const SimDev S = sims[s];
    const float fac = ffac[s];
    const float invb = 1.0f / (float)S.bf;
    const int64_t mcells = (int64_t)S.mx * S.my * S.mz;
    const Walk w = walk_chunk(S, ch - traverse_first(S));
    for (int it = 0; it < S.wi; ++it) {
      int i, j, k;
      int64_t local;
      if (!walk_particle(S, w, it, i, j, k, local)) continue;
      const int64_t g = S.p_off + local;
      const float3 x = mesh_pos(S, i, j, k, ld3(disp, g));
      float3 f = readout_cic8(
          fmesh + 3 * S.m_off, mcells,
          cic8(cic_axis(x.x, S.mx), cic_axis(x.y, S.my), cic_axis(x.z, S.mz),
               S.my, S.mz));
      f.x = __fmul_rn(__fmul_rn(f.x, fac), invb);
      f.y = __fmul_rn(__fmul_rn(f.y, fac), invb);
      f.z = __fmul_rn(__fmul_rn(f.z, fac), invb);
      st3(force, g, f);
    }
  }
}

// ---------------------------------------------------------------------------
// Fourier kernels
// ---------------------------------------------------------------------------

// Force spectra, flowpm/tfpm.py:199-215 apply_longrange:
//   pot_k = delta_k * lap * longrange;  force_d = pot_k * (i g_d)
// with delta_k = R2C(rho) / (nbar N^3), lap = 1/k^2 rounded to float (0 at
// k = 0, where the gradient vanishes anyway), g_d the 4-point gradient.
__global__ void __launch_bounds__(kThreads)
k_fourier_force(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
                const float2* __restrict__ dk, float2* __restrict__ fk,
                float* __restrict__ rho_zero, AxisTabs tabs, double r2,
                int deconv, const int32_t* __restrict__ nsteps, int pos,
                int skip_fused) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kSpec);
    if (nsteps && pos > nsteps[s]) continue;  // finished simulation
    const SimDev S = sims[s];
    if (skip_fused && S.fused) continue;
    const int64_t nmodes = (int64_t)S.mx * S.my * S.mzh;
    const int64_t mcells = (int64_t)S.mx * S.my * S.mz;
    // 1 / (nbar N^3) with nbar = Np / N^3 = 1 / bf^3.
    const float pre =
        (float)((double)S.bf * S.bf * S.bf / (double)mcells);
    const double* kkx = tabs.kk + S.tab;
    const double* kky = kkx + S.mx;
    const double* kkz = kky + S.my;
    const float* gx = tabs.grad + S.tab;
    const float* gy = gx + S.mx;
    const float* gz = gy + S.my;
    const float* wx = tabs.win + S.tab;
    const float* wy = wx + S.mx;
    const float* wz = wy + S.my;
    const int64_t base = (ch - S.ch_s) * kChunk + threadIdx.x;
    const float2* din = dk + S.s_off;
    float2* o0 = fk + 3 * S.s_off;
    float2* o1 = o0 + nmodes;
    float2* o2 = o1 + nmodes;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const int64_t local = base + it * kThreads;
      if (local < nmodes) {
        int i, j, l;
        mode_ijl(local, S.my, S.mzh, i, j, l);
        const double kk = kkx[i] + kky[j] + kkz[l];
        float w = kk == 0.0 ? 0.f : (float)(1.0 / kk);
        if (r2 != 0.0) w = __fmul_rn(w, (float)exp(-kk * r2));
        if (deconv) w = __fmul_rn(w, __fmul_rn(__fmul_rn(wx[i], wy[j]), wz[l]));
        float2 dv = din[local];
        dv.x = __fmul_rn(dv.x, pre);
        dv.y = __fmul_rn(dv.y, pre);
        const float pr = __fmul_rn(dv.x, w), pi = __fmul_rn(dv.y, w);
        const float g0 = gx[i], g1 = gy[j], g2 = gz[l];
        o0[local] = make_float2(-__fmul_rn(pi, g0), __fmul_rn(pr, g0));
        o1[local] = make_float2(-__fmul_rn(pi, g1), __fmul_rn(pr, g1));
        o2[local] = make_float2(-__fmul_rn(pi, g2), __fmul_rn(pr, g2));
      }
      // Zero the density mesh for the next paint (2 cells per mode slot).
      if (rho_zero) {
        for (int64_t c = local; c < mcells; c += nmodes)
          rho_zero[S.m_off + c] = 0.f;
      }
    }
  }
}

// Potential spectrum phi_k = delta_k * pre * w(k) with w = lap (0 at k = 0)
// times the optional Gaussian split and CIC deconvolution: the part of the
// force transfer function common to the three components.  The 4-point
// gradient i (8 sin k - sin 2k) / 6 of flowpm/kernels.py:72-76 is applied
// afterwards in real space, where it is exactly the stencil
// (8 (phi[x+1] - phi[x-1]) - (phi[x+2] - phi[x-2])) / 12 (k_stencil_grad).
// Also zeroes rho for the next paint.  Used unchanged (rho_zero = null) for
// the adjoint, the transfer function being real.
__global__ void __launch_bounds__(kThreads)
k_fourier_potential(const SimDev* __restrict__ sims, int nsims,
                    int64_t nchunks, const float2* dk, float2* out,
                    float* __restrict__ rho_zero,
                    AxisTabs tabs, Green G,
                    const int32_t* __restrict__ nsteps, int pos,
                    int skip_fused) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kSpec);
    if (nsteps && pos > nsteps[s]) continue;  // finished simulation
    const SimDev S = sims[s];
    if (skip_fused && (S.fused || S.xpass)) continue;
    const int64_t nmodes = (int64_t)S.mx * S.my * S.mzh;
    const int64_t mcells = (int64_t)S.mx * S.my * S.mz;
    const float pre = (float)((double)S.bf * S.bf * S.bf / (double)mcells);
    const double* kkx = tabs.kk + S.tab;
    const double* kky = kkx + S.mx;
    const double* kkz = kky + S.my;
    const float* wx = tabs.win + S.tab;
    const float* wy = wx + S.mx;
    const float* wz = wy + S.my;
    const int64_t base = (ch - S.ch_s) * kChunk + threadIdx.x;
    const float2* din = dk + S.s_off;
    float2* o = out + S.s_off;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const int64_t local = base + it * kThreads;
      if (local < nmodes) {
        int i, j, l;
        mode_ijl(local, S.my, S.mzh, i, j, l);
        const float w = green_w(G, s, kkx[i] + kky[j] + kkz[l], wx[i], wy[j],
                                wz[l]);
        float2 dv = din[local];
        dv.x = __fmul_rn(dv.x, pre);
        dv.y = __fmul_rn(dv.y, pre);
        o[local] = make_float2(__fmul_rn(dv.x, w), __fmul_rn(dv.y, w));
      }
      if (rho_zero) {
        for (int64_t c = local; c < mcells; c += nmodes)
          rho_zero[S.m_off + c] = 0.f;
      }
    }
  }
}

// 4-point central difference with periodic wrap:
// (8 (f[+1] - f[-1]) - (f[+2] - f[-2])) / 12.
__device__ __forceinline__ float stencil4(float m2, float m1, float p1,
                                          float p2) {
  return __fmul_rn(__fsub_rn(__fmul_rn(8.f, __fsub_rn(p1, m1)),
                             __fsub_rn(p2, m2)),
                   1.0f / 12.0f);
}

// k_stencil_grad with four z-consecutive cells per thread, for plans whose
// meshes all have mz % 4 == 0 and m_off % 4 == 0: 11 float4 loads (the 4
// x neighbours, the 4 y neighbours, and the z window [z0 - 4, z0 + 8) of
// the row) and 3 float4 stores per quad, one index decomposition per quad.
// One mesh chunk (kChunk cells) = one quad per thread.
__device__ __forceinline__ float4 stencil4v(float4 m2, float4 m1, float4 p1,
                                           float4 p2) {
  return make_float4(stencil4(m2.x, m1.x, p1.x, p2.x),
                     stencil4(m2.y, m1.y, p1.y, p2.y),
                     stencil4(m2.z, m1.z, p1.z, p2.z),
                     stencil4(m2.w, m1.w, p1.w, p2.w));
}

__global__ void __launch_bounds__(kThreads)
k_stencil_grad4(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
                const float* __restrict__ phi, float* __restrict__ fmesh,
                const int32_t* __restrict__ nsteps, int pos, int skip_fused) {
  static_assert(kChunk == 4 * kThreads, "one quad per thread and chunk");
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kMesh);
    if (nsteps && pos > nsteps[s]) continue;
    const SimDev S = sims[s];
    if (skip_fused && S.fused) continue;
    const unsigned my = S.my, mz = S.mz, mx = S.mx;
    const unsigned sx = my * mz, mcells = mx * sx;
    const unsigned c = ((unsigned)(ch - S.ch_m) * kThreads + threadIdx.x) * 4;
    if (c >= mcells) continue;
    const float* f = phi + S.m_off;
    const unsigned t = c / mz;
    const unsigned z = c - t * mz;
    const unsigned x = t / my;
    const unsigned y = t - x * my;
    const unsigned rx = c - x * sx, ry = c - y * mz, rz = c - z;
    const unsigned xm2 = (x >= 2 ? x - 2 : x + mx - 2) * sx;
    const unsigned xm1 = (x >= 1 ? x - 1 : x + mx - 1) * sx;
    const unsigned xp1 = (x + 1 < mx ? x + 1 : x + 1 - mx) * sx;
    const unsigned xp2 = (x + 2 < mx ? x + 2 : x + 2 - mx) * sx;
    const unsigned ym2 = (y >= 2 ? y - 2 : y + my - 2) * mz;
    const unsigned ym1 = (y >= 1 ? y - 1 : y + my - 1) * mz;
    const unsigned yp1 = (y + 1 < my ? y + 1 : y + 1 - my) * mz;
    const unsigned yp2 = (y + 2 < my ? y + 2 : y + 2 - my) * mz;
    const unsigned zl = z >= 4 ? z - 4 : z + mz - 4;
    const unsigned zr = z + 4 < mz ? z + 4 : z + 4 - mz;
    auto ld4 = [&](unsigned o) {
      return __ldg(reinterpret_cast<const float4*>(f + o));
    };
    const float4 gx = stencil4v(ld4(xm2 + rx), ld4(xm1 + rx), ld4(xp1 + rx),
                                ld4(xp2 + rx));
    const float4 gy = stencil4v(ld4(ym2 + ry), ld4(ym1 + ry), ld4(yp1 + ry),
                                ld4(yp2 + ry));
    const float4 L = ld4(rz + zl), C = ld4(c), R = ld4(rz + zr);
    // row window w[0..11] = L, C, R; cell z + i sits at w[4 + i]
    const float4 gz = make_float4(stencil4(L.z, L.w, C.y, C.z),
                                  stencil4(L.w, C.x, C.z, C.w),
                                  stencil4(C.x, C.y, C.w, R.x),
                                  stencil4(C.y, C.z, R.x, R.y));
    float* o0 = fmesh + 3 * S.m_off;
    reinterpret_cast<float4*>(o0 + c)[0] = gx;
    reinterpret_cast<float4*>(o0 + mcells + c)[0] = gy;
    reinterpret_cast<float4*>(o0 + 2 * mcells + c)[0] = gz;
  }
}

// Three force meshes f_d = D_d phi of each simulation (sim s: planes at
// fmesh + 3 m_off + d mcells).  With nsteps, finished simulations skip.
// 32-bit offsets inside a simulation's mesh.
__global__ void __launch_bounds__(kThreads)
k_stencil_grad(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
               const float* __restrict__ phi, float* __restrict__ fmesh,
               const int32_t* __restrict__ nsteps, int pos, int skip_fused) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kMesh);
    if (nsteps && pos > nsteps[s]) continue;
    const SimDev S = sims[s];
    if (skip_fused && S.fused) continue;
    const unsigned my = S.my, mz = S.mz, mx = S.mx;
    const unsigned sx = my * mz, mcells = mx * sx;
    const float* f = phi + S.m_off;
    float* o0 = fmesh + 3 * S.m_off;
    float* o1 = o0 + mcells;
    float* o2 = o1 + mcells;
    const unsigned base = (unsigned)(ch - S.ch_m) * kChunk + threadIdx.x;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const unsigned c = base + it * kThreads;
      if (c >= mcells) break;
      const unsigned t = c / mz;
      const unsigned z = c - t * mz;
      const unsigned x = t / my;
      const unsigned y = t - x * my;
      const unsigned rx = c - x * sx;           // y * mz + z
      const unsigned ry = c - y * mz;           // x * sx + z
      const unsigned rz = c - z;                // x * sx + y * mz
      const unsigned xm2 = (x >= 2 ? x - 2 : x + mx - 2) * sx;
      const unsigned xm1 = (x >= 1 ? x - 1 : x + mx - 1) * sx;
      const unsigned xp1 = (x + 1 < mx ? x + 1 : x + 1 - mx) * sx;
      const unsigned xp2 = (x + 2 < mx ? x + 2 : x + 2 - mx) * sx;
      const unsigned ym2 = (y >= 2 ? y - 2 : y + my - 2) * mz;
      const unsigned ym1 = (y >= 1 ? y - 1 : y + my - 1) * mz;
      const unsigned yp1 = (y + 1 < my ? y + 1 : y + 1 - my) * mz;
      const unsigned yp2 = (y + 2 < my ? y + 2 : y + 2 - my) * mz;
      const unsigned zm2 = z >= 2 ? z - 2 : z + mz - 2;
      const unsigned zm1 = z >= 1 ? z - 1 : z + mz - 1;
      const unsigned zp1 = z + 1 < mz ? z + 1 : z + 1 - mz;
      const unsigned zp2 = z + 2 < mz ? z + 2 : z + 2 - mz;
      o0[c] = stencil4(__ldg(f + xm2 + rx), __ldg(f + xm1 + rx),
                       __ldg(f + xp1 + rx), __ldg(f + xp2 + rx));
      o1[c] = stencil4(__ldg(f + ym2 + ry), __ldg(f + ym1 + ry),
                       __ldg(f + yp1 + ry), __ldg(f + yp2 + ry));
      o2[c] = stencil4(__ldg(f + rz + zm2), __ldg(f + rz + zm1),
                       __ldg(f + rz + zp1), __ldg(f + rz + zp2));
    }
  }
}

// Adjoint of k_stencil_grad: lphi = sum_d D_d^T lf_d = -sum_d D_d lf_d
// (the stencil is antisymmetric).  lf holds one float4 (lf_x, lf_y, lf_z, 0)
// per cell (the vector-reduction target of the readout adjoint).
__global__ void __launch_bounds__(kThreads)
k_stencil_div(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
              const float* __restrict__ lf, float* __restrict__ lphi,
              const int32_t* __restrict__ nsteps, int pos) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kMesh);
    if (nsteps && pos > nsteps[s]) continue;
    const SimDev S = sims[s];
    const unsigned my = S.my, mz = S.mz, mx = S.mx;
    const unsigned sx = my * mz, mcells = mx * sx;
    const float* l4 = lf + 4 * S.m_off;  // (x, y, z, 0) per cell
    float* o = lphi + S.m_off;
    const unsigned base = (unsigned)(ch - S.ch_m) * kChunk + threadIdx.x;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const unsigned c = base + it * kThreads;
      if (c >= mcells) break;
      const unsigned t = c / mz;
      const unsigned z = c - t * mz;
      const unsigned x = t / my;
      const unsigned y = t - x * my;
      const unsigned rx = c - x * sx, ry = c - y * mz, rz = c - z;
      const unsigned xm2 = (x >= 2 ? x - 2 : x + mx - 2) * sx;
      const unsigned xm1 = (x >= 1 ? x - 1 : x + mx - 1) * sx;
      const unsigned xp1 = (x + 1 < mx ? x + 1 : x + 1 - mx) * sx;
      const unsigned xp2 = (x + 2 < mx ? x + 2 : x + 2 - mx) * sx;
      const unsigned ym2 = (y >= 2 ? y - 2 : y + my - 2) * mz;
      const unsigned ym1 = (y >= 1 ? y - 1 : y + my - 1) * mz;
      const unsigned yp1 = (y + 1 < my ? y + 1 : y + 1 - my) * mz;
      const unsigned yp2 = (y + 2 < my ? y + 2 : y + 2 - my) * mz;
      const unsigned zm2 = z >= 2 ? z - 2 : z + mz - 2;
      const unsigned zm1 = z >= 1 ? z - 1 : z + mz - 1;
      const unsigned zp1 = z + 1 < mz ? z + 1 : z + 1 - mz;
      const unsigned zp2 = z + 2 < mz ? z + 2 : z + 2 - mz;
      const float a =
          stencil4(__ldg(l4 + 4 * (xm2 + rx)), __ldg(l4 + 4 * (xm1 + rx)),
                   __ldg(l4 + 4 * (xp1 + rx)), __ldg(l4 + 4 * (xp2 + rx)));
      const float b = stencil4(
          __ldg(l4 + 4 * (ym2 + ry) + 1), __ldg(l4 + 4 * (ym1 + ry) + 1),
          __ldg(l4 + 4 * (yp1 + ry) + 1), __ldg(l4 + 4 * (yp2 + ry) + 1));
      const float cz = stencil4(
          __ldg(l4 + 4 * (rz + zm2) + 2), __ldg(l4 + 4 * (rz + zm1) + 2),
          __ldg(l4 + 4 * (rz + zp1) + 2), __ldg(l4 + 4 * (rz + zp2) + 2));
      o[c] = -((a + b) + cz);
    }
  }
}

// k_stencil_div for large meshes (my % 16 == 0, mz % 64 == 0, mx % XC == 0,
// m_off % 4 == 0): a block owns a 16 x 64 (y, z) tile and marches over XC
// x planes.  The x stencil of lf_x comes from a window of five planes in
// registers; lf_y and lf_z of the current plane, with a halo of two cells
// in y (lf_y) and z (lf_z), from a ring of three planes in shared memory,
// so every float4 cell is read about once.  Thread (ty, tq) owns cells
// (y0 + ty, z0 + tq + 16 i), i < 4: consecutive lanes on consecutive
// cells for the loads and conflict-free shared reads.  Same arithmetic as
// k_stencil_div, bit for bit.
constexpr int kDivTY = 16, kDivTZ = 64;  // tile
constexpr int kDivRS = 80;               // shared row stride (floats)
constexpr int kDivRows = kDivTY + 4;

template <int XC>
__global__ void __launch_bounds__(256, 3)
k_stencil_div_tiled(const SimDev* __restrict__ sims, int first,
                    const float* __restrict__ lf, float* __restrict__ lphi,
                    const int32_t* __restrict__ nsteps, int pos) {
  __shared__ float sy[3][kDivRows][kDivRS];
  __shared__ float sz[3][kDivRows][kDivRS];
  const int s = first + blockIdx.y;
  if (nsteps && pos > nsteps[s]) return;
  const SimDev& S = sims[s];
  const int mx = S.mx, my = S.my, mz = S.mz;
  const int nzt = mz / kDivTZ, nyt = my / kDivTY;
  int b = blockIdx.x;
  const int z0 = (b % nzt) * kDivTZ;
  b /= nzt;
  const int y0 = (b % nyt) * kDivTY;
  const int x0 = (b / nyt) * XC;
  const int ty = threadIdx.x >> 4, tq = threadIdx.x & 15;
  const float4* L = reinterpret_cast<const float4*>(lf) + S.m_off;
  const unsigned sx = (unsigned)my * (unsigned)mz;
  const unsigned own = (unsigned)(y0 + ty) * mz + z0 + tq;
  // halo cells of this thread: y halo row hy (lf_y), z halo cell hz (lf_z)
  const int hr = threadIdx.x >> 6, hc = threadIdx.x & 63;
  const int hyrow = hr < 2 ? hr : kDivTY + hr;  // tile rows -2,-1,16,17
  const unsigned hyoff = (unsigned)((y0 - 2 + hyrow + my) % my) * mz + z0 + hc;
  const bool zh = threadIdx.x < 4 * kDivTY;
  const int zr = threadIdx.x >> 2, zk = threadIdx.x & 3;
  const int zcol = zk < 2 ? zk : kDivTZ + zk;   // tile cols -2,-1,64,65
  const unsigned zhoff =
      (unsigned)(y0 + (zh ? zr : 0)) * mz + (unsigned)((z0 - 2 + zcol + mz) % mz);
  auto plane = [&](int x) {
    return L + (size_t)(unsigned)((x % mx + mx) % mx) * sx;
  };
  float xw[5][4];
  float4 v[4];
  float hyv = 0.f, hzv = 0.f;
  auto load = [&](int x, bool halo) {
    const float4* P = plane(x);
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = __ldg(P + own + 16 * i);
    if (halo) {
      hyv = __ldg(reinterpret_cast<const float*>(P + hyoff) + 1);
      if (zh) hzv = __ldg(reinterpret_cast<const float*>(P + zhoff) + 2);
    }
  };
  auto put = [&](int slot) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      sy[slot][ty + 2][tq + 16 * i + 2] = v[i].y;
      sz[slot][ty + 2][tq + 16 * i + 2] = v[i].z;
    }
    sy[slot][hyrow][hc + 2] = hyv;
    if (zh) sz[slot][zr + 2][zcol] = hzv;
  };
#pragma unroll
  for (int k = 0; k < 5; ++k) {  // planes x0 - 2 .. x0 + 2
    load(x0 - 2 + k, k >= 2);
#pragma unroll
    for (int i = 0; i < 4; ++i) xw[k][i] = v[i].x;
    if (k >= 2) put(k - 2);
  }
  __syncthreads();
  float* out = lphi + S.m_off + own;
#pragma unroll 1
  for (int p = 0; p < XC; ++p) {
    const int slot = p % 3;
    const bool next = p + 3 <= XC + 1;  // plane x0 + p + 3 enters the window
    const bool next_slot = p + 3 < XC;  // and is processed
    if (next) load(x0 + p + 3, next_slot);
    const int r = ty + 2;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int c = tq + 16 * i + 2;
      const float a = stencil4(xw[0][i], xw[1][i], xw[3][i], xw[4][i]);
      const float bb = stencil4(sy[slot][r - 2][c], sy[slot][r - 1][c],
                                sy[slot][r + 1][c], sy[slot][r + 2][c]);
      const float cz = stencil4(sz[slot][r][c - 2], sz[slot][r][c - 1],
                                sz[slot][r][c + 1], sz[slot][r][c + 2]);
      out[(size_t)(unsigned)(x0 + p) * sx + 16 * i] = -((a + bb) + cz);
    }
    __syncthreads();  // every thread is done with this slot
    if (next) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        xw[0][i] = xw[1][i];
        xw[1][i] = xw[2][i];
        xw[2][i] = xw[3][i];
        xw[3][i] = xw[4][i];
        xw[4][i] = v[i].x;
      }
      if (next_slot) put(slot);
    }
    // the next plane reads another slot, written two planes ago
  }
}

// k_stencil_grad over the same 16 x 64 (y, z) tiles as k_stencil_div_tiled,
// marching over XC x planes: phi at x +- 1, x +- 2 of a block's cells from a
// window of five planes in registers, phi of the current plane with a halo
// of two cells in y and z from a ring of three planes in shared memory, so
// every phi value is read about once.  Same arithmetic as k_stencil_grad,
// bit for bit; three force planes out (sim s at fmesh + 3 m_off).
template <int XC>
__global__ void __launch_bounds__(256, 3)
k_stencil_grad_tiled(const SimDev* __restrict__ sims, int first,
                     const float* __restrict__ phi, float* __restrict__ fmesh,
                     const int32_t* __restrict__ nsteps, int pos) {
  __shared__ float sp[3][kDivRows][kDivRS];
  const int s = first + blockIdx.y;
  if (nsteps && pos > nsteps[s]) return;
  const SimDev& S = sims[s];
  const int mx = S.mx, my = S.my, mz = S.mz;
  const int nzt = mz / kDivTZ, nyt = my / kDivTY;
  int b = blockIdx.x;
  const int z0 = (b % nzt) * kDivTZ;
  b /= nzt;
  const int y0 = (b % nyt) * kDivTY;
  const int x0 = (b / nyt) * XC;
  const int ty = threadIdx.x >> 4, tq = threadIdx.x & 15;
  const float* F = phi + S.m_off;
  const unsigned sx = (unsigned)my * (unsigned)mz;
  const unsigned mcells = (unsigned)mx * sx;
  const unsigned own = (unsigned)(y0 + ty) * mz + z0 + tq;
  const int hr = threadIdx.x >> 6, hc = threadIdx.x & 63;
  const int hyrow = hr < 2 ? hr : kDivTY + hr;  // tile rows -2,-1,16,17
  const unsigned hyoff = (unsigned)((y0 - 2 + hyrow + my) % my) * mz + z0 + hc;
  const bool zh = threadIdx.x < 4 * kDivTY;
  const int zr = threadIdx.x >> 2, zk = threadIdx.x & 3;
  const int zcol = zk < 2 ? zk : kDivTZ + zk;   // tile cols -2,-1,64,65
  const unsigned zhoff =
      (unsigned)(y0 + (zh ? zr : 0)) * mz + (unsigned)((z0 - 2 + zcol + mz) % mz);
  auto plane = [&](int x) {
    return F + (size_t)(unsigned)((x % mx + mx) % mx) * sx;
  };
  float xw[5][4];
  float v[4];
  float hyv = 0.f, hzv = 0.f;
  auto load = [&](int x, bool halo) {
    const float* P = plane(x);
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = __ldg(P + own + 16 * i);
    if (halo) {
      hyv = __ldg(P + hyoff);
      if (zh) hzv = __ldg(P + zhoff);
    }
  };
  auto put = [&](int slot) {
#pragma unroll
    for (int i = 0; i < 4; ++i) sp[slot][ty + 2][tq + 16 * i + 2] = v[i];
    sp[slot][hyrow][hc + 2] = hyv;
    if (zh) sp[slot][zr + 2][zcol] = hzv;
  };
#pragma unroll
  for (int k = 0; k < 5; ++k) {  // planes x0 - 2 .. x0 + 2
    load(x0 - 2 + k, k >= 2);
#pragma unroll
    for (int i = 0; i < 4; ++i) xw[k][i] = v[i];
    if (k >= 2) put(k - 2);
  }
  __syncthreads();
  float* o = fmesh + 3 * S.m_off + own;
#pragma unroll 1
  for (int p = 0; p < XC; ++p) {
    const int slot = p % 3;
    const bool next = p + 3 <= XC + 1;  // plane x0 + p + 3 enters the window
    const bool next_slot = p + 3 < XC;  // and is processed
    if (next) load(x0 + p + 3, next_slot);
    const int r = ty + 2;
    const size_t base = (size_t)(unsigned)(x0 + p) * sx;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int c = tq + 16 * i + 2;
      o[base + 16 * i] = stencil4(xw[0][i], xw[1][i], xw[3][i], xw[4][i]);
      o[mcells + base + 16 * i] =
          stencil4(sp[slot][r - 2][c], sp[slot][r - 1][c],
                   sp[slot][r + 1][c], sp[slot][r + 2][c]);
      o[2 * (size_t)mcells + base + 16 * i] =
          stencil4(sp[slot][r][c - 2], sp[slot][r][c - 1],
                   sp[slot][r][c + 1], sp[slot][r][c + 2]);
    }
    __syncthreads();  // every thread is done with this slot
    if (next) {
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        xw[0][i] = xw[1][i];
        xw[1][i] = xw[2][i];
        xw[2][i] = xw[3][i];
        xw[3][i] = xw[4][i];
        xw[4][i] = v[i];
      }
      if (next_slot) put(slot);
    }
    // the next plane reads another slot, written two planes ago
  }
}

// LPT spectra (flowpm/tfpm.py:66-145 lpt1 / lpt2_source on the lattice).
// dk is the unnormalised R2C of the real field (normalised: already
// r2c3d's FFT / N^3, as the reference's lpt1 and lpt2_source take it).
__global__ void __launch_bounds__(kThreads)
k_lpt_fourier(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
              const float2* __restrict__ dk, float2* __restrict__ out,
              int mode, AxisTabs tabs, int normalised) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const SimDev S = sims[find_sim(sims, nsims, ch, kLatSpec)];
    const int64_t nmodes = (int64_t)S.nx * S.ny * S.lzh;
    const int64_t ncells = (int64_t)S.nx * S.ny * S.nz;
    const float pre = normalised ? 1.f : (float)(1.0 / (double)ncells);
    const double* kkx = tabs.kk + S.ltab;
    const double* kky = kkx + S.nx;
    const double* kkz = kky + S.ny;
    const float* gx = tabs.grad + S.ltab;
    const float* gy = gx + S.nx;
    const float* gz = gy + S.ny;
    const int nout = mode == 0 ? 9 : 3;
    float2* o = out + (int64_t)nout * S.ls_off;
    const int64_t base = (ch - S.ch_ls) * kChunk + threadIdx.x;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const int64_t local = base + it * kThreads;
      if (local >= nmodes) break;
      int i, j, l;
      mode_ijl(local, S.ny, S.lzh, i, j, l);
      const double kk = kkx[i] + kky[j] + kkz[l];
      // laplace_kernel is 1 at k = 0 in the reference (flowpm/kernels.py:
      // 42-48); every LPT weight also carries a gradient, which is 0 there.
      const float lap = kk == 0.0 ? 1.f : (float)(1.0 / kk);
      float2 dv = dk[S.ls_off + local];
      dv.x = __fmul_rn(dv.x, pre);
      dv.y = __fmul_rn(dv.y, pre);
      const float g[3] = {gx[i], gy[j], gz[l]};
      // psi_d: kweight = (i g_d) * lap = (0, g*lap); delta * kweight.
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float gl = __fmul_rn(g[d], lap);
        o[d * nmodes + local] =
            make_float2(-__fmul_rn(dv.y, gl), __fmul_rn(dv.x, gl));
      }
      if (mode == 0) {
        // phi_ij: kweight = lap * (i g_i) * (i g_j) = -(lap g_i) g_j.
        const int pi_[6] = {0, 1, 2, 1, 2, 0};
        const int pj_[6] = {0, 1, 2, 2, 0, 1};
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const float w = -__fmul_rn(__fmul_rn(lap, g[pi_[q]]), g[pj_[q]]);
          o[(3 + q) * nmodes + local] =
              make_float2(__fmul_rn(dv.x, w), __fmul_rn(dv.y, w));
        }
      }
    }
  }
}

// Full <-> half lattice spectra.  The reference's r2c3d / c2r3d
// (flowpm/utils.py:213-272) speak full complex spectra (nx, ny, nz); the
// library keeps the nz/2 + 1 half that a real field's Hermitian symmetry
// determines.  to_full == 0: half[i, j, l] = s * full[i, j, l], l <= nz/2
// (chunks over half-spectrum modes); to_full == 1: full[i, j, l] =
// s * half[i, j, l] for l <= nz/2, else s * conj(half[-i, -j, nz - l])
// (indices mod n; chunks over lattice cells).  s = 1/(nx ny nz) with
// inv_n, else 1.
__global__ void __launch_bounds__(kThreads)
k_lat_spectrum(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
               const float2* __restrict__ in, float2* __restrict__ out,
               int to_full, int inv_n) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const SimDev S =
        sims[find_sim(sims, nsims, ch, to_full ? kLat : kLatSpec)];
    const int64_t ncells = (int64_t)S.nx * S.ny * S.nz;
    const int64_t nmodes = (int64_t)S.nx * S.ny * S.lzh;
    const float s = inv_n ? (float)(1.0 / (double)ncells) : 1.f;
    const int64_t base =
        (ch - (to_full ? S.ch_l : S.ch_ls)) * kChunk + threadIdx.x;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const int64_t local = base + it * kThreads;
      if (local >= (to_full ? ncells : nmodes)) break;
      if (!to_full) {
        int i, j, l;
        mode_ijl(local, S.ny, S.lzh, i, j, l);
        const float2 v =
            in[S.l_off + ((int64_t)i * S.ny + j) * S.nz + l];
        out[S.ls_off + local] = make_float2(__fmul_rn(v.x, s), __fmul_rn(v.y, s));
      } else {
        int i, j, l;
        mode_ijl(local, S.ny, S.nz, i, j, l);
        float2 v;
        if (l < S.lzh) {
          v = in[S.ls_off + ((int64_t)i * S.ny + j) * S.lzh + l];
        } else {
          const int ci = i ? S.nx - i : 0, cj = j ? S.ny - j : 0;
          v = in[S.ls_off + ((int64_t)ci * S.ny + cj) * S.lzh + (S.nz - l)];
          v.y = -v.y;
        }
        out[S.l_off + local] = make_float2(__fmul_rn(v.x, s), __fmul_rn(v.y, s));
      }
    }
  }
}

// Three lattice meshes (psi_d of sim s at psi + 3 l_off + d ncells) read
// out at arbitrary positions: out[s, p, d] = cic_readout(psi_d, pos[s, p]),
// flowpm/tfpm.py:86-94 (lpt1's readout at pos).  One thread per particle.
__global__ void __launch_bounds__(kThreads)
k_lpt_readout(const SimDev* __restrict__ sims, int nsims,
              const float* __restrict__ psi, const float* __restrict__ pos,
              int64_t npart, float* __restrict__ out) {
  const int64_t total = (int64_t)nsims * npart;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const SimDev S = sims[g / npart];
    const int64_t ncells = (int64_t)S.nx * S.ny * S.nz;
    const float3 x = ld3(pos, g);
    const Cic8 c = cic8(cic_axis(x.x, S.nx), cic_axis(x.y, S.ny),
                        cic_axis(x.z, S.nz), S.ny, S.nz);
    st3(out, g, readout_cic8(psi + 3 * S.l_off, ncells, c));
  }
}

// source = 3/7 * [phi_1 phi_2 + phi_2 phi_0 + phi_0 phi_1
//                 - phi_12^2 - phi_20^2 - phi_01^2]  (flowpm/tfpm.py:128-144)
__global__ void __launch_bounds__(kThreads)
k_lpt2_source(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
              const float* __restrict__ phi9, float* __restrict__ source) {
  const float c37 = (float)(3.0 / 7.0);
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const SimDev S = sims[find_sim(sims, nsims, ch, kLat)];
    const int64_t ncells = (int64_t)S.nx * S.ny * S.nz;
    const float* ph = phi9 + 9 * S.l_off;
    const int64_t base = (ch - S.ch_l) * kChunk + threadIdx.x;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const int64_t c = base + it * kThreads;
      if (c >= ncells) break;
      const float p0 = ph[3 * ncells + c], p1 = ph[4 * ncells + c],
                  p2 = ph[5 * ncells + c];
      const float q12 = ph[6 * ncells + c], q20 = ph[7 * ncells + c],
                  q01 = ph[8 * ncells + c];
      float s = __fmul_rn(p1, p2);
      s = __fadd_rn(s, __fmul_rn(p2, p0));
      s = __fadd_rn(s, __fmul_rn(p0, p1));
      s = __fsub_rn(s, __fmul_rn(q12, q12));
      s = __fsub_rn(s, __fmul_rn(q20, q20));
      s = __fsub_rn(s, __fmul_rn(q01, q01));
      source[S.l_off + c] = __fmul_rn(s, c37);
    }
  }
}

// flowpm/tfpm.py:166-179: DX = D1 psi1 (+ D2 psi2), P and F likewise.  The
// readout at the lattice points returns the mesh value at the particle's own
// cell (weights 1, 0, ..., 0), so psi is read directly.
__global__ void __launch_bounds__(kThreads)
k_lpt_particles(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
                const float* __restrict__ psi1, int m1,
                const float* __restrict__ psi2, int m2,
                const float* __restrict__ coef, float* __restrict__ disp,
                float* __restrict__ mom, float* __restrict__ force) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kPart);
    const SimDev S = sims[s];
    const int64_t ncells = (int64_t)S.nx * S.ny * S.nz;
    const float* c = coef + 6 * s;
    const float* p1 = psi1 + (int64_t)m1 * S.l_off;
    const float* p2 = psi2 ? psi2 + (int64_t)m2 * S.l_off : nullptr;
    const int64_t base = (ch - S.ch_p) * kChunk + threadIdx.x;
    for (int it = 0; it < kItems; ++it) {
      const int64_t local = base + it * kThreads;
      if (local >= S.np) break;
      const int64_t g = S.p_off + local;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float dx1 = __fmul_rn(c[0], p1[d * ncells + local]);
        float dx = dx1;
        float pp = __fmul_rn(c[2], dx1);
        float ff = __fmul_rn(c[4], dx1);
        if (p2) {
          const float dx2 = __fmul_rn(c[1], p2[d * ncells + local]);
          dx = __fadd_rn(dx1, dx2);
          pp = __fadd_rn(pp, __fmul_rn(c[3], dx2));
          ff = __fadd_rn(ff, __fmul_rn(c[5], dx2));
        }
        disp[3 * g + d] = dx;
        mom[3 * g + d] = pp;
        force[3 * g + d] = ff;
      }
    }
  }
}

// lineark = whitec * amp, whitec = R2C(white) / N^3 (flowpm/tfpm.py:58-61).
__global__ void __launch_bounds__(kThreads)
k_linear_mul(const SimDev* __restrict__ sims, int nsims, int64_t nchunks,
             float2* __restrict__ wk, const float* __restrict__ amp) {
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const SimDev S = sims[find_sim(sims, nsims, ch, kLatSpec)];
    const int64_t nmodes = (int64_t)S.nx * S.ny * S.lzh;
    const float pre = (float)(1.0 / ((double)S.nx * S.ny * S.nz));
    const int64_t base = (ch - S.ch_ls) * kChunk + threadIdx.x;
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const int64_t local = base + it * kThreads;
      if (local >= nmodes) break;
      const int64_t o = S.ls_off + local;
      float2 v = wk[o];
      const float a = amp[o];
      v.x = __fmul_rn(__fmul_rn(v.x, pre), a);
      v.y = __fmul_rn(__fmul_rn(v.y, pre), a);
      wk[o] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11) + Box-Muller white noise.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += W0;
    k.y += W1;
  }
  return c;
}

// Uniform in (0, 1): (r + 0.5) / 2^32.
__device__ __forceinline__ double u01(uint32_t r) {
  return ((double)r + 0.5) * (1.0 / 4294967296.0);
}

// out[e - off] = stddev * z(e) for global element indices e in [off, off+n);
// z(4m + q) is lane q of the Box-Muller pairs of Philox block m.
__global__ void __launch_bounds__(kThreads)
k_white_noise(float* __restrict__ out, int64_t off, int64_t n, uint2 key,
              double stddev) {
  const int64_t g0 = off / 4, g1 = (off + n + 3) / 4;
  for (int64_t m = g0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
       m < g1; m += (int64_t)gridDim.x * blockDim.x) {
    const uint4 r = philox4x32_10(
        make_uint4((uint32_t)m, (uint32_t)((uint64_t)m >> 32), 0u, 0u), key);
    const double ra = sqrt(-2.0 * log(u01(r.x)));
    const double rb = sqrt(-2.0 * log(u01(r.z)));
    double sa, ca, sb, cb;
    sincospi(2.0 * u01(r.y), &sa, &ca);
    sincospi(2.0 * u01(r.w), &sb, &cb);
    const double z[4] = {ra * ca, ra * sa, rb * cb, rb * sb};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int64_t e = 4 * m + q;
      if (e >= off && e < off + n) out[e - off] = (float)(stddev * z[q]);
    }
  }
}

// ---------------------------------------------------------------------------
// Launch wrappers
// ---------------------------------------------------------------------------
std::atomic<int64_t> g_launches{0};

void launch_paint_lattice(const SimDev* sims, int nsims, int64_t nchunks,
                          const float* disp, float* rho, int32_t* status,
                          cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_paint_lattice<<<grid_for(nchunks), kThreads, 0, st>>>(sims, nsims, nchunks,
                                                          disp, rho, status);
}

void launch_fourier_force(const SimDev* sims, int nsims, int64_t nchunks,
                          const float2* dk, float2* fk, float* rho_zero,
                          AxisTabs tabs, double r_split2, int deconv,
                          const int32_t* nsteps, int pos, int skip_fused,
                          cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_fourier_force<<<grid_for(nchunks), kThreads, 0, st>>>(
      sims, nsims, nchunks, dk, fk, rho_zero, tabs, r_split2, deconv, nsteps,
      pos, skip_fused);
}

void launch_fourier_potential(const SimDev* sims, int nsims, int64_t nchunks,
                              const float2* dk, float2* out, float* rho_zero,
                              AxisTabs tabs, const Green& G,
                              const int32_t* nsteps, int pos, int skip_fused,
                              cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_fourier_potential<<<grid_for(nchunks), kThreads, 0, st>>>(
      sims, nsims, nchunks, dk, out, rho_zero, tabs, G, nsteps, pos,
      skip_fused);
}

void launch_stencil_grad(const SimDev* sims, int nsims, int64_t nchunks,
                         const float* phi, float* fmesh, const int32_t* nsteps,
                         int pos, int skip_fused, bool quads,
                         cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (quads)
    k_stencil_grad4<<<grid_for(nchunks), kThreads, 0, st>>>(
        sims, nsims, nchunks, phi, fmesh, nsteps, pos, skip_fused);
  else
    k_stencil_grad<<<grid_for(nchunks), kThreads, 0, st>>>(
        sims, nsims, nchunks, phi, fmesh, nsteps, pos, skip_fused);
}

void launch_stencil_div(const SimDev* sims, int nsims, int64_t nchunks,
                        const float* lf, float* lphi, const int32_t* nsteps,
                        int pos, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_stencil_div<<<grid_for(nchunks), kThreads, 0, st>>>(
      sims, nsims, nchunks, lf, lphi, nsteps, pos);
}

int stencil_div_chunk(int mx, int my, int mz, int64_t m_off, int count) {
  if (my % kDivTY != 0 || mz % kDivTZ != 0 || m_off % 4 != 0) return 0;
  const int64_t tiles = (int64_t)(my / kDivTY) * (mz / kDivTZ) * count;
  for (int xc : {32, 16})
    if (mx % xc == 0 && mx >= xc && tiles * (mx / xc) >= 2 * kNumSMs)
      return xc;
  return 0;
}

void launch_stencil_div_tiled(const SimDev* sims, int first, int count,
                              int mx, int my, int mz, int xc, const float* lf,
                              float* lphi, const int32_t* nsteps, int pos,
                              cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const dim3 grid((unsigned)((mx / xc) * (my / kDivTY) * (mz / kDivTZ)),
                  (unsigned)count);
  if (xc == 32)
    k_stencil_div_tiled<32><<<grid, 256, 0, st>>>(sims, first, lf, lphi,
                                                  nsteps, pos);
  else
    k_stencil_div_tiled<16><<<grid, 256, 0, st>>>(sims, first, lf, lphi,
                                                  nsteps, pos);
}

void launch_stencil_grad_tiled(const SimDev* sims, int first, int count,
                               int mx, int my, int mz, int xc,
                               const float* phi, float* fmesh,
                               const int32_t* nsteps, int pos,
                               cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const dim3 grid((unsigned)((mx / xc) * (my / kDivTY) * (mz / kDivTZ)),
                  (unsigned)count);
  if (xc == 32)
    k_stencil_grad_tiled<32><<<grid, 256, 0, st>>>(sims, first, phi, fmesh,
                                                   nsteps, pos);
  else
    k_stencil_grad_tiled<16><<<grid, 256, 0, st>>>(sims, first, phi, fmesh,
                                                   nsteps, pos);
}

void launch_step(const SimDev* sims, int nsims, int64_t ch0, int64_t ch1,
                 const StepArgs& a, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  launch_pdl(k_step, dim3(grid_for(ch1 - ch0)), dim3(kThreads), 0, st, sims,
             nsims, ch0, ch1, a);
}

void launch_pgd(const SimDev* sims, int nsims, int64_t nchunks, float* disp,
                const float* fmesh, float* rho, const float* pgd,
                int pgd_stride, int pos, const int32_t* nsteps,
                int32_t* status, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_pgd<<<grid_for(nchunks), kThreads, 0, st>>>(sims, nsims, nchunks, disp,
                                                fmesh, rho, pgd, pgd_stride,
                                                pos, nsteps, status);
}

void launch_force_readout(const SimDev* sims, int nsims, int64_t nchunks,
                          const float* disp, const float* fmesh,
                          const float* ffac, float* force, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_force_readout<<<grid_for(nchunks), kThreads, 0, st>>>(
      sims, nsims, nchunks, disp, fmesh, ffac, force);
}

void launch_lpt_fourier(const SimDev* sims, int nsims, int64_t nchunks,
                        const float2* dk, float2* out, int mode, AxisTabs tabs,
                        cudaStream_t st, int normalised) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_lpt_fourier<<<grid_for(nchunks), kThreads, 0, st>>>(
      sims, nsims, nchunks, dk, out, mode, tabs, normalised);
}

void launch_lat_spectrum(const SimDev* sims, int nsims, int64_t nchunks,
                         const float2* in, float2* out, int to_full,
                         int inv_n, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_lat_spectrum<<<grid_for(nchunks), kThreads, 0, st>>>(
      sims, nsims, nchunks, in, out, to_full, inv_n);
}

void launch_lpt_readout(const SimDev* sims, int nsims, const float* psi,
                        const float* pos, int64_t npart, float* out,
                        cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  int64_t blocks = ((int64_t)nsims * npart + kThreads - 1) / kThreads;
  const int64_t cap = (int64_t)kNumSMs * 32;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  k_lpt_readout<<<(unsigned)blocks, kThreads, 0, st>>>(sims, nsims, psi, pos,
                                                       npart, out);
}

void launch_lpt2_source(const SimDev* sims, int nsims, int64_t nchunks,
                        const float* phi9, float* source, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_lpt2_source<<<grid_for(nchunks), kThreads, 0, st>>>(sims, nsims, nchunks,
                                                        phi9, source);
}

void launch_lpt_particles(const SimDev* sims, int nsims, int64_t nchunks,
                          const float* psi1, int m1, const float* psi2, int m2,
                          const float* coef, float* disp, float* mom,
                          float* force, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_lpt_particles<<<grid_for(nchunks), kThreads, 0, st>>>(
      sims, nsims, nchunks, psi1, m1, psi2, m2, coef, disp, mom, force);
}

void launch_linear_mul(const SimDev* sims, int nsims, int64_t nchunks,
                       float2* wk, const float* amp, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_linear_mul<<<grid_for(nchunks), kThreads, 0, st>>>(sims, nsims, nchunks,
                                                       wk, amp);
}

void launch_white_noise(float* out, int64_t off, int64_t n, uint64_t seed,
                        double stddev, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const int64_t groups = (off + n + 3) / 4 - off / 4;
  int64_t blocks = (groups + kThreads - 1) / kThreads;
  const int64_t cap = (int64_t)kNumSMs * 32;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  k_white_noise<<<(unsigned)blocks, kThreads, 0, st>>>(
      out, off, n, make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)), stddev);
}

}  // namespace fpm

extern "C" int64_t fpm_launch_count(void) {
  return fpm::g_launches.load(std::memory_order_relaxed);
}
