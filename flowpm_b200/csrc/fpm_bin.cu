// Eulerian binning of the particles and the binned leapfrog step.
//
// The lattice-walk step (k_step) visits particles in Lagrangian order: as
// the run goes on, the 32 particles of a warp spread over many cells, so its
// CIC gathers and deposits touch many L2 sectors (at 128^3 the step grows
// from 63 us at the first leapfrog step to 114 us at the last, nearly all of
// it in the paint's reductions).  The binned step keeps the particle state
// sorted by force-mesh cell instead, cell keys tile-major (tiles of T^3
// cells, z fastest inside a tile), each particle carrying its Lagrangian
// index, so:
// * one block owns one tile: it reads its particles as one contiguous,
//   coalesced range, and consecutive lanes sit in the same or neighbouring
//   cells, so each CIC gather touches few sectors;
// * the block deposits the paint into a shared-memory copy of its tile plus
//   a halo, and adds that copy to the density with one 16-byte vector
//   reduction per four cells; only deposits that fall outside the halo (a
//   particle that drifted more than a cell out of its tile since the last
//   sort) go to global memory directly.
// Particles are re-sorted every few steps by a counting sort on the cell
// key (count, exclusive scan, scatter), which replaces tf.scatter_nd's role
// in flowpm/utils.py:87-89 (the reference deposits in arbitrary order).
// Outputs that the caller sees in Lagrangian order (final state, force,
// checkpoints, intermediate states) are written through the carried index.
#include "fpm_bin.cuh"

// Lanes of k_step_sorted that deposit into the same base cell sum their
// weights with a segmented shuffle reduction and deposit once (1), or each
// lane deposits its own (0).
#ifndef FPM_SORTED_SEGSUM
#define FPM_SORTED_SEGSUM 1
#endif
// Runs of k_step_sorted whose base cells are z-adjacent merge the four
// deposits they share (1), or each deposits its eight (0).  Measured on
// B200 (re-sorted every 16 steps; step kernels per 40-step simulation):
// 3.09 against 3.01 ms at 128^3, 21.4 against 20.7 ms at 256^3 -- the
// shuffles cost more than the reductions they save.
#ifndef FPM_SORTED_ZMERGE
#define FPM_SORTED_ZMERGE 0
#endif
// k_step_sorted paints through a shared-memory box of cells around its
// chunk (1) or straight into the density (0).  Measured on B200 (particles
// re-sorted every 16 steps; step kernels per 40-step simulation): 4.12 ms
// with the box against 2.99 ms without at 128^3, 28.9 against 20.7 ms at
// 256^3 -- the shared-memory atomics, the barriers and the flush of each
// chunk cost more than the L2 reductions they save, once runs of lanes in
// one cell already deposit once (the segmented sums; without them the
// step takes 3.46 ms at 128^3).
#ifndef FPM_SORTED_BOX
#define FPM_SORTED_BOX 0
#endif

namespace fpm {

namespace {

// Tile-major key of force-mesh cell (cx, cy, cz) inside its simulation.
template <int T>
__device__ __forceinline__ unsigned cell_key(const BinRun& R, int cx, int cy,
                                             int cz) {
  const unsigned tx = (unsigned)cx / T, ty = (unsigned)cy / T,
                 tz = (unsigned)cz / T;
  const unsigned lx = (unsigned)cx % T, ly = (unsigned)cy % T,
                 lz = (unsigned)cz % T;
  return ((tx * (unsigned)R.nty + ty) * (unsigned)R.ntz + tz) * (T * T * T) +
         (lx * T + ly) * T + lz;
}

// The same key from a simulation's tile counts, tiles of 2^lt cells.
__device__ __forceinline__ unsigned cell_key_lt(const SimDev& S, int lt,
                                                int cx, int cy, int cz) {
  const int tm = (1 << lt) - 1;
  const unsigned tile = ((unsigned)(cx >> lt) * (unsigned)S.nty +
                         (unsigned)(cy >> lt)) * (unsigned)S.ntz +
                        (unsigned)(cz >> lt);
  const unsigned local =
      ((unsigned)((cx & tm) << lt | (cy & tm)) << lt) | (unsigned)(cz & tm);
  return (tile << (3 * lt)) | local;
}

// Cell key of slot t of simulation r of the run (run-relative: + r *
// ncell) and its packed lattice site: from the carried index when lag is
// set, else t is the Lagrangian index itself.
template <int T>
__device__ __forceinline__ uint32_t particle_key(const BinRun& R,
                                                 const float3 dv,
                                                 const uint32_t* __restrict__ lag,
                                                 int r, int64_t slot,
                                                 uint32_t t, uint32_t& l) {
  int i, j, k;
  if (lag) {
    l = lag[slot];
    unpack_site(l, R.qkb, R.qjb, i, j, k);
  } else {
    const unsigned tt = t / (unsigned)R.nz;
    k = (int)(t - tt * (unsigned)R.nz);
    i = (int)(tt / (unsigned)R.ny);
    j = (int)(tt - (unsigned)i * (unsigned)R.ny);
    l = pack_site(i, j, k, R.qkb, R.qjb);
  }
  const float b = (float)R.bf;
  const float x = __fmul_rn(__fadd_rn(index_float(i), dv.x), b);
  const float y = __fmul_rn(__fadd_rn(index_float(j), dv.y), b);
  const float z = __fmul_rn(__fadd_rn(index_float(k), dv.z), b);
  const int cx = cic_axis(x, R.mx).i0, cy = cic_axis(y, R.my).i0,
            cz = cic_axis(z, R.mz).i0;
  return (uint32_t)r * (uint32_t)R.ncell + cell_key<T>(R, cx, cy, cz);
}

// Keys of lanes past the end of a sort's input (kSentinel - lane).
constexpr uint32_t kSentinel = 0xffffffffu;

// Chunks of kChunk slots per simulation: the sort kernels walk chunks, so
// that the simulation of a slot is known per chunk.
__device__ __forceinline__ int64_t sort_chunks_per_sim(const BinRun& R) {
  return (R.np + kChunk - 1) / kChunk;
}

// cnt[m0 + key] += 1 for every particle of the run, one atomic per run of
// equal keys.
template <int T>
__global__ void __launch_bounds__(kThreads)
k_bin_count(BinRun R, const float* __restrict__ d,
            const uint32_t* __restrict__ lag, int32_t* __restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  const int64_t cps = sort_chunks_per_sim(R);
  const int64_t nch = cps * R.count;
  for (int64_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
    const int r = (int)(ch / cps);
    const int64_t t0 = (ch - (int64_t)r * cps) * kChunk;
#pragma unroll
    for (int item = 0; item < kItems; ++item) {
      const int64_t t = t0 + item * kThreads + threadIdx.x;
      const bool valid = t < R.np;
      uint32_t key = kSentinel - lane, l;
      if (valid) {
        const int64_t slot = R.p0 + (int64_t)r * R.np + t;
        key = particle_key<T>(R, ld3(d, slot), lag, r, slot, (uint32_t)t, l);
      }
      const unsigned heads = run_heads(key, lane);
      if (valid && ((heads >> lane) & 1u))
        atomicAdd(cnt + R.m0 + key, (int32_t)run_length(heads, lane));
    }
  }
}

// Scatter: the head of each run claims the run's slots with one atomic on
// off[key] (lanes of a run keep their order), then every lane writes the
// NP float3 arrays of the payload (the first is the displacement the keys
// come from) and its packed lattice site.  The kItems claims of a thread
// are issued before any of them is used, so their latencies overlap.
template <int T, int NP>
__global__ void __launch_bounds__(kThreads)
k_bin_scatter(BinRun R, BinPayload pay, const uint32_t* __restrict__ lag,
              int32_t* __restrict__ off, uint32_t* __restrict__ lag_out) {
  const int lane = threadIdx.x & 31;
  const int64_t cps = sort_chunks_per_sim(R);
  const int64_t nch = cps * R.count;
  for (int64_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
    const int r = (int)(ch / cps);
    const int64_t t0 = (ch - (int64_t)r * cps) * kChunk;
    const int64_t s0 = R.p0 + (int64_t)r * R.np;
    uint32_t l[kItems];
    int base[kItems];
    unsigned heads[kItems];
    float3 dv[kItems];
#pragma unroll
    for (int item = 0; item < kItems; ++item) {
      const int64_t t = t0 + item * kThreads + threadIdx.x;
      const bool valid = t < R.np;
      uint32_t key = kSentinel - lane;
      l[item] = 0;
      dv[item] = make_float3(0.f, 0.f, 0.f);
      if (valid) {
        dv[item] = ld3(pay.src[0], s0 + t);
        key = particle_key<T>(R, dv[item], lag, r, s0 + t, (uint32_t)t,
                              l[item]);
      }
      heads[item] = run_heads(key, lane);
      base[item] = 0;
      if (valid && ((heads[item] >> lane) & 1u))
        base[item] = atomicAdd(off + R.m0 + key,
                               (int32_t)run_length(heads[item], lane));
    }
#pragma unroll
    for (int item = 0; item < kItems; ++item) {
      const int64_t t = t0 + item * kThreads + threadIdx.x;
      const int h = run_head(heads[item], lane);
      const int b = __shfl_sync(0xffffffffu, base[item], h);
      if (t >= R.np) continue;
      const int64_t dst = (int64_t)b + (lane - h);
      st3(pay.dst[0], dst, dv[item]);
#pragma unroll
      for (int q = 1; q < NP; ++q)
        st3(pay.dst[q], dst, ld3(pay.src[q], s0 + t));
      lag_out[dst] = l[item];
    }
  }
}

// Back to Lagrangian order: the slot of simulation r holding packed site
// (i, j, k) goes to p0 + r np + (i ny + j) nz + k.
template <int NP>
__global__ void __launch_bounds__(kThreads)
k_bin_unsort(BinRun R, BinPayload pay, const uint32_t* __restrict__ lag) {
  const int64_t cps = sort_chunks_per_sim(R);
  const int64_t nch = cps * R.count;
  for (int64_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
    const int r = (int)(ch / cps);
    const int64_t t0 = (ch - (int64_t)r * cps) * kChunk;
    const int64_t s0 = R.p0 + (int64_t)r * R.np;
#pragma unroll
    for (int item = 0; item < kItems; ++item) {
      const int64_t t = t0 + item * kThreads + threadIdx.x;
      if (t >= R.np) continue;
      int i, j, k;
      unpack_site(lag[s0 + t], R.qkb, R.qjb, i, j, k);
      const int64_t g =
          s0 + (int64_t)(((unsigned)i * (unsigned)R.ny + (unsigned)j) *
                             (unsigned)R.nz + (unsigned)k);
#pragma unroll
      for (int q = 0; q < NP; ++q) st3(pay.dst[q], g, ld3(pay.src[q], s0 + t));
    }
  }
}

// Exclusive scan of the counts cnt[0..n) into out (n a multiple of 4, both
// 16-byte aligned), plus base, zeroing cnt on the way: three passes over
// chunks of kScanChunk values.
constexpr int kScanThreads = 256, kScanPer = 16;
constexpr int kScanChunk = kScanThreads * kScanPer;

__device__ __forceinline__ int block_excl_scan(int v, int& total) {
  __shared__ int ws[kScanThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < kScanThreads / 32 ? ws[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kScanThreads / 32) ws[lane] = s;
  }
  __syncthreads();
  total = ws[kScanThreads / 32 - 1];
  const int excl = x - v + (w > 0 ? ws[w - 1] : 0);
  __syncthreads();  // ws is reused by the next call
  return excl;
}

__device__ __forceinline__ int4 load_part(const int32_t* v, int64_t i,
                                          int64_t n) {
  return i < n ? *reinterpret_cast<const int4*>(v + i) : make_int4(0, 0, 0, 0);
}

__global__ void __launch_bounds__(kScanThreads)
k_scan_sums(const int32_t* __restrict__ v, int64_t n, int32_t* sums) {
  const int64_t b0 = (int64_t)blockIdx.x * kScanChunk;
  int s = 0;
#pragma unroll
  for (int q = 0; q < kScanPer / 4; ++q) {
    const int4 a = load_part(v, b0 + (q * kScanThreads + threadIdx.x) * 4, n);
    s += a.x + a.y + a.z + a.w;
  }
  int total;
  block_excl_scan(s, total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// One block of 1024 threads: exclusive scan of the nb chunk sums, plus
// base (each thread sums a run of ceil(nb / 1024) of them; a two-level
// shuffle scan over the 32 warps combines the runs).
__global__ void __launch_bounds__(1024)
k_scan_top(int32_t* sums, int nb, int32_t base) {
  __shared__ int wsum[32];
  const int per = (nb + 1023) / 1024;
  const int b0 = threadIdx.x * per;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int s = 0;
  for (int i = 0; i < per && b0 + i < nb; ++i) s += sums[b0 + i];
  int x = s;  // inclusive scan over the warp
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    int t = wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    wsum[lane] = t;  // inclusive over warps
  }
  __syncthreads();
  int acc = base + (x - s) + (w > 0 ? wsum[w - 1] : 0);
  for (int i = 0; i < per && b0 + i < nb; ++i) {
    const int v = sums[b0 + i];
    sums[b0 + i] = acc;
    acc += v;
  }
}

// Thread t of block b scans the 16 values [b0 + 4 (q 256 + t), + 4) for
// q < 4 -- four int4 groups, strided for coalescing -- so its prefix runs
// over the groups in block order: group (q, t) precedes (q, t + 1) and
// (q + 1, 0).  The block scan runs once per q.
__global__ void __launch_bounds__(kScanThreads)
k_scan_apply(int32_t* __restrict__ cnt, int32_t* __restrict__ out, int64_t n,
             const int32_t* __restrict__ sums) {
  const int64_t b0 = (int64_t)blockIdx.x * kScanChunk;
  int carry = sums[blockIdx.x];
#pragma unroll
  for (int q = 0; q < kScanPer / 4; ++q) {
    const int64_t i = b0 + (q * kScanThreads + threadIdx.x) * 4;
    int4 a = load_part(cnt, i, n);
    const int s = a.x + a.y + a.z + a.w;
    int total;
    const int e = block_excl_scan(s, total) + carry;
    carry += total;
    if (i < n) {
      int4 o;
      o.x = e;
      o.y = e + a.x;
      o.z = o.y + a.y;
      o.w = o.z + a.z;
      *reinterpret_cast<int4*>(out + i) = o;
      // the counts start from zero at the next sort
      *reinterpret_cast<int4*>(cnt + i) = make_int4(0, 0, 0, 0);
    }
  }
}

// Offset of periodic cell c from the origin o of a tile of T cells: the
// representative of c - o (mod m) nearest the tile's centre, in
// [T/2 - m/2, T/2 + m/2) (so every cell of the tile maps into [0, T) even
// when m = T).
template <int T>
__device__ __forceinline__ int rel_cell(int c, int o, int m) {
  int r = c - o - T / 2;
  if (r >= (m >> 1)) r -= m;
  else if (r < -(m >> 1)) r += m;
  return r + T / 2;
}

// Offset of periodic cell c from a box origin o on an axis of m cells: the
// representative of c - o (mod m) in (-m/2, m/2], so a box no larger than
// the mesh sees every cell at most once; the caller tests 0 <= r < size.
__device__ __forceinline__ int box_rel(int c, int o, int m) {
  int r = c - o;
  if (r > (m >> 1)) r -= m;
  else if (r <= -(m >> 1)) r += m;
  return r;
}

// The binned leapfrog step: one tile of T^3 force-mesh cells per block
// iteration.  Per particle the arithmetic is k_step's (readout, closing
// kick, opening kick, drift, paint), in the same order and rounding.  The
// paint goes into a shared-memory copy of the cells [o - 1, o + T + 1] in
// x and y and [o - 4, o + T + 4) in z (z padded so that it flushes as
// aligned float4), then into rho with one vector reduction per nonzero
// group of four cells; a deposit outside that region goes to rho directly.
template <int T>
__global__ void __launch_bounds__(kThreads, FPM_STEP_MINBLOCKS)
k_step_binned(const SimDev* __restrict__ sims, int nsims, int64_t ch0,
              int64_t nchunks, BinStepArgs b) {
  constexpr int RX = T + 3, RZ = T + 8, RN = RX * RX * RZ;
  constexpr int T3 = T * T * T;
  __shared__ __align__(16) float tile[RN];
  pdl_wait();  // the force meshes of the solve before
  const StepArgs& a = b.a;
  for (int64_t ch = ch0 + blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kTile);
    const SimDev S = sims[s];
    const int Tn = a.nsteps[s];
    if (a.it > Tn) continue;  // this sim has finished
    const float* cf = a.coefs + (int64_t)s * a.max_steps * 3;
    const float ke = a.it >= 1 ? cf[(a.it - 1) * 3 + 2] : 0.f;
    const bool last = (a.it == Tn);
    const float ks = last ? 0.f : cf[a.it * 3 + 0];
    const float dr = last ? 0.f : cf[a.it * 3 + 1];
    const float fac = a.ffac[s];
    const float invb = 1.0f / (float)S.bf;
    const int64_t mcells = (int64_t)S.mx * S.my * S.mz;
    float* m = a.rho + S.m_off;
    const unsigned t = (unsigned)(ch - S.ch_t);
    const unsigned r = t / (unsigned)S.ntz;
    const int oz = (int)(t - r * (unsigned)S.ntz) * T;
    const int ox = (int)(r / (unsigned)S.nty) * T;
    const int oy = (int)(r - (unsigned)(ox / T) * (unsigned)S.nty) * T;
    const int64_t kf = S.m_off + (int64_t)t * T3;
    // a simulation's first tile starts at its first particle (the cell
    // before it belongs to another simulation, possibly of another run
    // whose sort may be in flight on another stream)
    const int begin = t == 0 ? (int)S.p_off : b.cell_end[kf - 1];
    const int end = b.cell_end[kf + T3 - 1];
    if (!last) {
      for (int q = threadIdx.x; q < RN / 4; q += blockDim.x)
        reinterpret_cast<float4*>(tile)[q] = make_float4(0.f, 0.f, 0.f, 0.f);
      __syncthreads();
    }
    for (int i = begin + (int)threadIdx.x; i < end; i += blockDim.x) {
      const uint32_t l = b.blag[i];
      int qi, qj, qk;
      unpack_site(l, S.qkb, S.qjb, qi, qj, qk);
      const int64_t g = S.p_off + site_local(S, qi, qj, qk);  // Lagrangian
      float3 d = ld3(b.bd, i), p = ld3(b.bp, i);
      const float3 x = mesh_pos(S, qi, qj, qk, d);
      const Cic8 c0 = cic8(cic_axis(x.x, S.mx), cic_axis(x.y, S.my),
                           cic_axis(x.z, S.mz), S.my, S.mz);
      float3 f = readout_cic8(a.fmesh + 3 * S.m_off, mcells, c0);
      // force = readout * factor / pm_nc_factor (flowpm/tfpm.py:218, :356)
      f.x = __fmul_rn(__fmul_rn(f.x, fac), invb);
      f.y = __fmul_rn(__fmul_rn(f.y, fac), invb);
      f.z = __fmul_rn(__fmul_rn(f.z, fac), invb);
      if (a.it >= 1) p = axpy(p, ke, f);  // closing kick of step it-1
      if (a.ckpt && a.it % a.ckpt_every == 0) {
        float* o = a.ckpt + (int64_t)(a.it / a.ckpt_every) * 2 * a.total_np * 3;
        st3(o, g, d);
        st3(o + a.total_np * 3, g, p);
      }
      if (a.inter && a.it >= 1) {
        float* o = a.inter + (int64_t)(a.it - 1) * 3 * a.total_np * 3;
        st3(o, g,
            make_float3(__fadd_rn(index_float(qi), d.x),
                        __fadd_rn(index_float(qj), d.y),
                        __fadd_rn(index_float(qk), d.z)));
        st3(o + a.total_np * 3, g, p);
        st3(o + 2 * a.total_np * 3, g, f);
      }
      if (last) {  // uniform over the block: one sim per tile
        st3(a.force_out, g, f);
        st3(a.mom, g, p);
        st3(a.disp, g, d);
        if (!finite3(p.x, p.y, p.z) || !finite3(f.x, f.y, f.z))
          atomicOr(a.status, FPM_STATUS_NONFINITE_MOM);
        continue;
      }
      p = axpy(p, ks, f);  // opening kick of step it
      d = axpy(d, dr, p);  // drift of step it
      st3(b.bp, i, p);
      st3(b.bd, i, d);
      const float3 xn = mesh_pos(S, qi, qj, qk, d);
      if (!finite3(xn.x, xn.y, xn.z))
        atomicOr(a.status, FPM_STATUS_NONFINITE_POS);
      const Axis ax = cic_axis(xn.x, S.mx), ay = cic_axis(xn.y, S.my),
                 az = cic_axis(xn.z, S.mz);
      const int rx = rel_cell<T>(ax.i0, ox, S.mx),
                ry = rel_cell<T>(ay.i0, oy, S.my),
                rz = rel_cell<T>(az.i0, oz, S.mz);
      const Cic8 c1 = cic8(ax, ay, az, S.my, S.mz);
      if (rx >= -1 && rx <= T && ry >= -1 && ry <= T && rz >= -4 &&
          rz <= T + 2) {
        float* t0 = tile + ((rx + 1) * RX + (ry + 1)) * RZ + (rz + 4);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float* tq = t0 + (q & 1) * (RX * RZ) + (q >> 1) * RZ;
          atomicAdd(tq, __fmul_rn(c1.wxy[q], c1.wz0));
          atomicAdd(tq + 1, __fmul_rn(c1.wxy[q], c1.wz1));
        }
      } else {
        paint_cic8(m, c1, 1.f);
      }
    }
    if (last) continue;
    __syncthreads();
    for (int q = threadIdx.x; q < RN / 4; q += blockDim.x) {
      const float4 v = reinterpret_cast<const float4*>(tile)[q];
      if (v.x == 0.f && v.y == 0.f && v.z == 0.f && v.w == 0.f) continue;
      const int zg = q % (RZ / 4), row = q / (RZ / 4);
      const int cy = wrap_near(oy - 1 + row % RX, S.my);
      const int cx = wrap_near(ox - 1 + row / RX, S.mx);
      const int cz = wrap_near(oz - 4 + 4 * zg, S.mz);
      red_add_f4(m + ((int64_t)cx * S.my + cy) * S.mz + cz, v);
    }
    __syncthreads();  // the next tile zeroes the shared copy
  }
}

// The step over the sorted particles in equal chunks (kChunk slots of one
// simulation per block iteration, the chunks of the lattice order, so the
// work per block does not depend on the clustering), CIC gathers and
// deposits straight from and to global memory.  Consecutive lanes sit in
// the same or neighbouring cells, so the gathers and reductions of a warp
// touch few sectors.  Lanes that deposit into the same base cell are
// contiguous in the sorted order: when a warp has such runs, each of the 8
// corner weights is summed over its run with a segmented shuffle reduction
// (5 steps) and only the run's first lane issues the reductions.  The sums
// of a run are formed in a different order than one deposit at a time
// (FP32 rounding, as any order of the reference's scatter).
template <bool BOX>
__global__ void __launch_bounds__(kThreads, FPM_STEP_MINBLOCKS)
k_step_sorted(const SimDev* __restrict__ sims, int nsims, int64_t ch0,
              int64_t nchunks, BinStepArgs b) {
  // BOX: the paint goes into a shared-memory box of cells around the
  // chunk (BX x-planes from the first particle's cell less two, and the
  // y and z extent of its 16^3 tile with a margin: z from four before, so
  // the box flushes as aligned float4), then into rho with one 16-byte
  // vector reduction per non-zero group of four; deposits outside the box
  // go to rho directly.
  constexpr int BX = 8, BY = 20, BZ = 24, BN = BX * BY * BZ;
  __shared__ __align__(16) float box[BOX ? BN : 4];
  __shared__ int box_org[3];
  pdl_wait();  // the force meshes of the solve before
  const StepArgs& a = b.a;
  const int lane = threadIdx.x & 31;
  for (int64_t ch = ch0 + blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int s = find_sim(sims, nsims, ch, kPart);
    const SimDev S = sims[s];
    const int Tn = a.nsteps[s];
    if (a.it > Tn) continue;  // this sim has finished
    const float* cf = a.coefs + (int64_t)s * a.max_steps * 3;
    const float ke = a.it >= 1 ? cf[(a.it - 1) * 3 + 2] : 0.f;
    const bool last = (a.it == Tn);
    const float ks = last ? 0.f : cf[a.it * 3 + 0];
    const float dr = last ? 0.f : cf[a.it * 3 + 1];
    const float fac = a.ffac[s];
    const float invb = 1.0f / (float)S.bf;
    const int64_t mcells = (int64_t)S.mx * S.my * S.mz;
    float* m = a.rho + S.m_off;
    const int64_t first = S.p_off + (ch - S.ch_p) * kChunk;
    const int64_t end = S.p_off + S.np;
    int bx0 = 0, by0 = 0, bz0 = 0;
    if (BOX && !last) {  // uniform over the block
      if (threadIdx.x == 0) {
        int fi, fj, fk;
        if (b.blag) {
          unpack_site(b.blag[first], S.qkb, S.qjb, fi, fj, fk);
        } else {
          lattice_ijk(S, first - S.p_off, fi, fj, fk);
        }
        const float3 fx = mesh_pos(S, fi, fj, fk, ld3(b.bd, first));
        box_org[0] = cic_axis(fx.x, S.mx).i0 - 2;
        box_org[1] = (cic_axis(fx.y, S.my).i0 & ~15) - 2;
        box_org[2] = (cic_axis(fx.z, S.mz).i0 & ~15) - 4;
      }
      for (int q = threadIdx.x; q < BN / 4; q += kThreads)
        reinterpret_cast<float4*>(box)[q] = make_float4(0.f, 0.f, 0.f, 0.f);
      __syncthreads();
      bx0 = box_org[0];
      by0 = box_org[1];
      bz0 = box_org[2];
    }
#pragma unroll 1
    for (int item = 0; item < kItems; ++item) {
      const int64_t i = first + item * kThreads + threadIdx.x;
      const bool valid = i < end;  // warp-uniform except in a sim's last chunk
      uint32_t l = 0;
      float3 d = make_float3(0.f, 0.f, 0.f), p = d;
      int qi = 0, qj = 0, qk = 0;
      if (valid) {
        d = ld3(b.bd, i);
        p = ld3(b.bp, i);
        if (b.blag) {
          l = b.blag[i];
          unpack_site(l, S.qkb, S.qjb, qi, qj, qk);
        } else {  // Lagrangian order: slot i is lattice site i - p_off
          lattice_ijk(S, i - S.p_off, qi, qj, qk);
          l = pack_site(qi, qj, qk, S.qkb, S.qjb);
        }
      }
      const int64_t g = S.p_off + site_local(S, qi, qj, qk);  // Lagrangian
      const float3 x = mesh_pos(S, qi, qj, qk, d);
      const Axis ax0 = cic_axis(x.x, S.mx), ay0 = cic_axis(x.y, S.my),
                 az0 = cic_axis(x.z, S.mz);
      const Cic8 c0 = cic8(ax0, ay0, az0, S.my, S.mz);
      // re-sorted as it moves: the run of lanes in this cell claims its
      // slots now; the claim's latency overlaps the readout
      int claim_base = 0;
      unsigned claim_heads = 0xffffffffu;
      if (b.claim && !last) {
        const unsigned k0 = valid ? c0.row[0] + c0.z0 : 0xffffffffu - lane;
        claim_heads = run_heads(k0, lane);
        if (valid && ((claim_heads >> lane) & 1u))
          claim_base = atomicAdd(
              b.claim + S.m_off +
                  cell_key_lt(S, b.tile_log2, ax0.i0, ay0.i0, az0.i0),
              (int32_t)run_length(claim_heads, lane));
      }
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
            make_float3(__fadd_rn(index_float(qi), d.x),
                        __fadd_rn(index_float(qj), d.y),
                        __fadd_rn(index_float(qk), d.z)));
        st3(o + a.total_np * 3, g, p);
        st3(o + 2 * a.total_np * 3, g, f);
      }
      if (last) {  // uniform over the block: one sim per chunk
        if (valid) {
          st3(a.force_out, g, f);
          st3(a.mom, g, p);
          st3(a.disp, g, d);
          if (!finite3(p.x, p.y, p.z) || !finite3(f.x, f.y, f.z))
            atomicOr(a.status, FPM_STATUS_NONFINITE_MOM);
        }
        continue;
      }
      p = axpy(p, ks, f);  // opening kick of step it
      d = axpy(d, dr, p);  // drift of step it
      const float3 xn = mesh_pos(S, qi, qj, qk, d);
      if (b.claim) {
        const int h = run_head(claim_heads, lane);
        const int base = __shfl_sync(0xffffffffu, claim_base, h);
        if (valid) {
          const int64_t o = (int64_t)base + (lane - h);
          st3(b.op, o, p);
          st3(b.od, o, d);
          b.olag[o] = l;
        }
      } else if (valid) {
        st3(b.bp, i, p);
        st3(b.bd, i, d);
      }
      if (valid && !finite3(xn.x, xn.y, xn.z))
        atomicOr(a.status, FPM_STATUS_NONFINITE_POS);
      const Axis nx1 = cic_axis(xn.x, S.mx), ny1 = cic_axis(xn.y, S.my),
                 nz1 = cic_axis(xn.z, S.mz);
      const Cic8 c1 = cic8(nx1, ny1, nz1, S.my, S.mz);
      // base cell of the deposit; a lane past the sim's end gets a key of
      // its own
      const unsigned key = valid ? c1.row[0] + c1.z0 : 0xffffffffu - lane;
      const unsigned up = __shfl_up_sync(0xffffffffu, key, 1);
      const bool head = lane == 0 || up != key;
      if (b.count) {
        // the sort after this step: one count per run of lanes in a cell
        const unsigned hs = __ballot_sync(0xffffffffu, head);
        if (valid && head)
          atomicAdd(b.count + S.m_off +
                        cell_key_lt(S, b.tile_log2, nx1.i0, ny1.i0, nz1.i0),
                    (int32_t)run_length(hs, lane));
      }
      float w[8];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        w[2 * q] = __fmul_rn(c1.wxy[q], c1.wz0);
        w[2 * q + 1] = __fmul_rn(c1.wxy[q], c1.wz1);
      }
      const unsigned heads =
          FPM_SORTED_SEGSUM ? __ballot_sync(0xffffffffu, head) : 0xffffffffu;
      if (heads != 0xffffffffu) {
        // segmented sums over runs of contiguous lanes with equal keys (a
        // key can recur in a later run after the particles drifted since
        // their sort; each run deposits its own sum): lane + o is in this
        // lane's run when no run starts in (lane, lane + o]; the longest
        // run of the warp bounds the rounds
        const unsigned longest = __reduce_max_sync(
            0xffffffffu, head ? (unsigned)run_length(heads, lane) : 1u);
#pragma unroll 1
        for (int o = 1; o < (int)longest; o <<= 1) {
          const bool same =
              lane + o < 32 &&
              ((unsigned long long)heads >> (lane + 1) & ((1ull << o) - 1)) == 0;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const float t = __shfl_down_sync(0xffffffffu, w[q], o);
            if (same) w[q] = __fadd_rn(w[q], t);
          }
        }
      }
      // z-adjacent runs share four cells: the run whose base cell is one z
      // step past the previous run's takes that run's upper-z weights into
      // its lower-z ones, and the previous run leaves them out
      bool skip_z1 = false;
      if (FPM_SORTED_ZMERGE) {
        const bool nowrap = valid && c1.z1 == c1.z0 + 1;
        const int ph = lane > 0 ? run_head(heads, lane - 1) : 0;
        const unsigned above = heads & ~((2u << lane) - 1u);
        const int nh = above ? __ffs(above) - 1 : lane;
        const unsigned kp = __shfl_sync(0xffffffffu, key, ph);
        const int pnw = __shfl_sync(0xffffffffu, (int)nowrap, ph);
        const unsigned kn = __shfl_sync(0xffffffffu, key, nh);
        const int nv = __shfl_sync(0xffffffffu, (int)valid, nh);
        const bool take = head && valid && lane > 0 && pnw && kp + 1u == key;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float t = __shfl_sync(0xffffffffu, w[2 * q + 1], ph);
          if (take) w[2 * q] = __fadd_rn(w[2 * q], t);
        }
        skip_z1 = nh != lane && nv && nowrap && key + 1u == kn;
      }
      if (valid && (head || !FPM_SORTED_SEGSUM)) {
        if (BOX) {
          const int rx0 = box_rel(nx1.i0, bx0, S.mx),
                    rx1 = box_rel(nx1.i1, bx0, S.mx),
                    ry0 = box_rel(ny1.i0, by0, S.my),
                    ry1 = box_rel(ny1.i1, by0, S.my),
                    rz0 = box_rel(nz1.i0, bz0, S.mz),
                    rz1 = box_rel(nz1.i1, bz0, S.mz);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int rx = (q & 1) ? rx1 : rx0, ry = (q >> 1) ? ry1 : ry0;
            const bool in = (unsigned)rx < (unsigned)BX &&
                            (unsigned)ry < (unsigned)BY;
            float* t = box + (rx * BY + ry) * BZ;
            if (in && (unsigned)rz0 < (unsigned)BZ)
              atomicAdd(t + rz0, w[2 * q]);
            else
              red_add(m + c1.row[q] + c1.z0, w[2 * q]);
            if (in && (unsigned)rz1 < (unsigned)BZ)
              atomicAdd(t + rz1, w[2 * q + 1]);
            else
              red_add(m + c1.row[q] + c1.z1, w[2 * q + 1]);
          }
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            red_add(m + c1.row[q] + c1.z0, w[2 * q]);
            if (!skip_z1) red_add(m + c1.row[q] + c1.z1, w[2 * q + 1]);
          }
        }
      }
    }
    if (BOX && !last) {  // flush the box
      __syncthreads();
      for (int q = threadIdx.x; q < BN / 4; q += kThreads) {
        const float4 v = reinterpret_cast<const float4*>(box)[q];
        if (v.x == 0.f && v.y == 0.f && v.z == 0.f && v.w == 0.f) continue;
        const int zg = q % (BZ / 4), row = q / (BZ / 4);
        const int cy = wrap_near(by0 + row % BY, S.my);
        const int cx = wrap_near(bx0 + row / BY, S.mx);
        const int cz = wrap_near(bz0 + 4 * zg, S.mz);
        red_add_f4(m + ((int64_t)cx * S.my + cy) * S.mz + cz, v);
      }
      __syncthreads();  // the next chunk zeroes the box
    }
  }
}

}  // namespace

void launch_step_sorted(const SimDev* sims, int nsims, int64_t ch0,
                        int64_t ch1, const BinStepArgs& b, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  // the shared-memory box follows tiles of 16 cells
  if (FPM_SORTED_BOX && b.tile_log2 == 4)
    launch_pdl(k_step_sorted<true>, dim3(grid_for(ch1 - ch0)), dim3(kThreads),
               0, st, sims, nsims, ch0, ch1, b);
  else
    launch_pdl(k_step_sorted<false>, dim3(grid_for(ch1 - ch0)),
               dim3(kThreads), 0, st, sims, nsims, ch0, ch1, b);
}

void launch_step_binned(int tile, const SimDev* sims, int nsims, int64_t ch0,
                        int64_t ch1, const BinStepArgs& b, cudaStream_t st) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (tile == 8)
    launch_pdl(k_step_binned<8>, dim3(grid_for(ch1 - ch0)), dim3(kThreads), 0,
               st, sims, nsims, ch0, ch1, b);
  else
    launch_pdl(k_step_binned<16>, dim3(grid_for(ch1 - ch0)), dim3(kThreads),
               0, st, sims, nsims, ch0, ch1, b);
}

namespace {
int bits_for(int n) {  // bits of the largest index n - 1
  int b = 0;
  while ((1ll << b) < (long long)n) ++b;
  return b;
}
}  // namespace

bool bin_run_supported(int nx, int ny, int nz, int64_t ncell, int count,
                       int* qkb, int* qjb) {
  const int ib = bits_for(nx), jb = bits_for(ny), kb = bits_for(nz);
  if (ib + jb + kb > 32 || jb + kb > 31) return false;
  // keys below the sentinels kSentinel - lane of lanes past the end
  if ((int64_t)count * ncell >= (int64_t)kSentinel - 64) return false;
  *qkb = kb;
  *qjb = jb;
  return true;
}

bool bin_tile_supported(int tile, int mx, int my, int mz) {
  if (tile != 8 && tile != 16) return false;
  return mx % tile == 0 && my % tile == 0 && mz % tile == 0;
}

size_t bin_scan_blocks(int64_t ncells) {
  return (size_t)((ncells + kScanChunk - 1) / kScanChunk);
}

namespace {

// Blocks of the sort kernels: one per chunk of kChunk slots of a
// simulation, at most 16 per SM (grid-stride beyond).
int64_t sort_blocks(const BinRun& R) {
  int64_t blocks = (R.np + kChunk - 1) / kChunk * R.count;
  const int64_t cap = (int64_t)kNumSMs * 16;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return blocks;
}

template <int NP>
void launch_scatter(int tile, unsigned blocks, const BinRun& R,
                    const BinPayload& pay, const uint32_t* lag, int32_t* cell,
                    uint32_t* lag_out, cudaStream_t st) {
  if (tile == 8)
    k_bin_scatter<8, NP>
        <<<blocks, kThreads, 0, st>>>(R, pay, lag, cell, lag_out);
  else
    k_bin_scatter<16, NP>
        <<<blocks, kThreads, 0, st>>>(R, pay, lag, cell, lag_out);
}

}  // namespace

#define FPM_RET(x)                 \
  do {                             \
    const int rc_ = (x);           \
    if (rc_ != FPM_OK) return rc_; \
  } while (0)

int launch_bin_scan(const BinRun& R, int32_t* count, int32_t* cell,
                    int32_t* sums, cudaStream_t st) {
  const int64_t ncells = (int64_t)R.count * R.ncell;
  const int nb = (int)bin_scan_blocks(ncells);
  g_launches.fetch_add(3, std::memory_order_relaxed);
  k_scan_sums<<<nb, kScanThreads, 0, st>>>(count + R.m0, ncells, sums);
  k_scan_top<<<1, 1024, 0, st>>>(sums, nb, (int32_t)R.p0);
  k_scan_apply<<<nb, kScanThreads, 0, st>>>(count + R.m0, cell + R.m0, ncells,
                                            sums);
  return cudaGetLastError() == cudaSuccess ? FPM_OK : FPM_ERR_CUDA;
}

int launch_bin_count_scan(int tile, const BinRun& R, const float* d,
                          const uint32_t* lag, int32_t* count, int32_t* cell,
                          int32_t* sums, cudaStream_t st) {
  const unsigned blocks = (unsigned)sort_blocks(R);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (tile == 8)
    k_bin_count<8><<<blocks, kThreads, 0, st>>>(R, d, lag, count);
  else
    k_bin_count<16><<<blocks, kThreads, 0, st>>>(R, d, lag, count);
  return launch_bin_scan(R, count, cell, sums, st);
}

int launch_bin_scan_scatter(int tile, const BinRun& R, const BinPayload& pay,
                            const uint32_t* lag, int32_t* count,
                            int32_t* cell, int32_t* sums, uint32_t* lag_out,
                            cudaStream_t st) {
  if (pay.n != 2 && pay.n != 4) return FPM_ERR_ARG;
  FPM_RET(launch_bin_scan(R, count, cell, sums, st));
  const unsigned blocks = (unsigned)sort_blocks(R);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (pay.n == 2)
    launch_scatter<2>(tile, blocks, R, pay, lag, cell, lag_out, st);
  else
    launch_scatter<4>(tile, blocks, R, pay, lag, cell, lag_out, st);
  return cudaGetLastError() == cudaSuccess ? FPM_OK : FPM_ERR_CUDA;
}

int launch_bin_sort(int tile, const BinRun& R, const BinPayload& pay,
                    const uint32_t* lag, int32_t* count, int32_t* cell,
                    int32_t* sums, uint32_t* lag_out, cudaStream_t st) {
  if (pay.n != 2 && pay.n != 4) return FPM_ERR_ARG;
  const unsigned blocks = (unsigned)sort_blocks(R);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (tile == 8)
    k_bin_count<8><<<blocks, kThreads, 0, st>>>(R, pay.src[0], lag, count);
  else
    k_bin_count<16><<<blocks, kThreads, 0, st>>>(R, pay.src[0], lag, count);
  return launch_bin_scan_scatter(tile, R, pay, lag, count, cell, sums,
                                 lag_out, st);
}

int launch_bin_sort(int tile, const BinRun& R, const float* d,
                    const float* p, const uint32_t* lag, int32_t* count,
                    int32_t* cell, int32_t* sums, float* d_out, float* p_out,
                    uint32_t* lag_out, bool counted, cudaStream_t st) {
  BinPayload pay;
  pay.n = 2;
  pay.src[0] = d;
  pay.src[1] = p;
  pay.dst[0] = d_out;
  pay.dst[1] = p_out;
  pay.src[2] = pay.src[3] = nullptr;
  pay.dst[2] = pay.dst[3] = nullptr;
  if (counted)
    return launch_bin_scan_scatter(tile, R, pay, lag, count, cell, sums,
                                   lag_out, st);
  return launch_bin_sort(tile, R, pay, lag, count, cell, sums, lag_out, st);
}

int launch_bin_unsort(const BinRun& R, const BinPayload& pay,
                      const uint32_t* lag, cudaStream_t st) {
  if (pay.n != 4) return FPM_ERR_ARG;
  const unsigned blocks = (unsigned)sort_blocks(R);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_bin_unsort<4><<<blocks, kThreads, 0, st>>>(R, pay, lag);
  return cudaGetLastError() == cudaSuccess ? FPM_OK : FPM_ERR_CUDA;
}

}  // namespace fpm
