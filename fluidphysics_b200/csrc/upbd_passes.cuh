// Pass bodies of the unified-particle substep (sm_100a). Each body restates
// one or more WGSL passes of the reference (src/gpu/wgsl.js, cited per body)
// and keeps their floating-point operand order; passes that only touch a
// particle's own slot are fused into one body. All of them are FP32 SIMT
// gathers over HBM-resident state: there is no dense contraction on this
// path, so the tensor cores have no role here. The scalar type is `real`
// (upbd_device.cuh): float, or double in the test-only FP64 build that
// re-runs these same bodies as the drift reference.
//
// A body processes one block-sized tile `vb` of one scene (thread index
// vb * blockDim.x + threadIdx.x). The single-scene kernels (upbd_kernels.cuh)
// call it with vb = blockIdx.x; the batched kernels (upbd_batch.cu) call it
// for every tile of every scene from a persistent grid, so one scene's
// arithmetic is the same whichever way it is stepped.
#pragma once
#include "upbd_device.cuh"

namespace upbd {

#define UPBD_VTID (vb * blockDim.x + threadIdx.x)

// --------------------------------------------------- integrate + grid count
// integrate (src/gpu/wgsl.js:121-160) fused with gridCount
// (src/gpu/wgsl.js:173-178). The count keeps each particle's arrival ticket
// and bumps its scan tile's total, so the scan needs no second pass.
template <bool INTEGRATE, bool COUNT>
__device__ __forceinline__ void b_integrate_count(const SimView& v, const DevParams* __restrict__ P, uint32_t vb) {
  const int i = UPBD_VTID;
  if (i >= v.N) return;
  uint32_t f = v.flags[i];
  if (!(f & F_ACTIVE)) return;
  real4 p4 = v.pos[i];
  if (INTEGRATE) {
    const real h = P->h;
    const real4 vv = v.vel[i];
    const real vx = vv.x, vz = vv.z;
    const real vy = vv.y + P->gravity * h;
    const real px = p4.x, py = p4.y, pz = p4.z;
    real nx = px + vx * h, ny = py + vy * h, nz = pz + vz * h;
    const real4 pv = v.prev[i];
    real tw = pv.w;
    bool slipped = false;
    if (f & F_GRABBED) {
      const float4 gd = P->grab_delta;
      const real2 dn = v.density[i];
      real tx = pv.w, ty = vv.w, tz = dn.x;
      tx = tx + gd.x; ty = ty + gd.y; tz = tz + gd.z;
      const real ex = nx - tx, ey = ny - ty, ez = nz - tz;
      if (r_sqrt(dot3(ex, ey, ez, ex, ey, ez)) > 1.0f) {
        f &= ~F_GRABBED;
        v.flags[i] = f;
        v.vel[i] = make_real4(vx, vy, vz, 0.f);
        slipped = true;
      } else {
        const real k = P->grab_k * dn.y;
        real cx = (tx - nx) * k, cy = (ty - ny) * k, cz = (tz - nz) * k;
        const real cl = r_sqrt(dot3(cx, cy, cz, cx, cy, cz));
        const real maxC = 0.05f;
        if (cl > maxC) {
          const real g = maxC / cl;
          cx = cx * g; cy = cy * g; cz = cz * g;
        }
        nx = nx + cx; ny = ny + cy; nz = nz + cz;
        tw = tx;
        v.vel[i] = make_real4(vx, vy, vz, ty);
        v.density[i] = make_real2(tz, dn.y);
      }
    } else {
      v.vel[i] = make_real4(vx, vy, vz, vv.w);
    }
    (void)slipped;
    v.prev[i] = make_real4(px, py, pz, tw);
    p4 = make_real4(nx, ny, nz, p4.w);
    v.pos[i] = p4;
    if (i >= v.S) v.mark[i] = 0u;  // contact marks of this substep start clear
  }
  if (COUNT) {
    const uint32_t h = cell_of(p4.x, p4.y, p4.z, P->inv_cell, (uint32_t)v.T - 1u);
    v.cell[i] = h;
    v.ticket[i] = atomicAdd(&v.counts[h], 1u);
    const int rep = (i >> 5) & (tile_reps(v.num_tiles) - 1);  // a power of two
    atomicAdd(&v.tile_sum[rep * v.num_tiles + (int)(h / SCAN_TILE)], 1u);
  }
}

// ------------------------------------------------------------ exclusive scan
// scanBlocks/scanPartials/scanApply (src/gpu/wgsl.js:180-236) as one launch:
// block b scans its own 2048 counts (8 consecutive ones per thread), adds the
// totals of tiles < b (the count's tile counters, all replicas), writes
// start[], and clears the counts it read. The counts and the earlier totals
// are loaded up front so that their latencies overlap, and one block barrier
// publishes both per-warp sums.
__device__ __forceinline__ void b_scan(const SimView& v, uint32_t vb) {
  __shared__ uint32_t s_scan[SCAN_THREADS / 32];  // per-warp sums of this tile's counts
  __shared__ uint32_t s_prev[SCAN_THREADS / 32];  // per-warp sums of earlier tiles' totals
  const int tid = threadIdx.x;
  const int lane = tid & 31, wid = tid >> 5;
  const long long t0 = (long long)vb * SCAN_TILE + (long long)tid * 8;
  // 16-byte rows when the tile is whole and the arrays allow it (start[] may
  // be a caller's buffer at any 4-byte offset)
  const bool vec = t0 + 8 <= (long long)v.T && ((reinterpret_cast<uintptr_t>(v.counts) | reinterpret_cast<uintptr_t>(v.start) |
                                                 reinterpret_cast<uintptr_t>(v.fend)) & 15u) == 0;
  uint32_t c[8];
  if (vec) {
    const uint4 a = *reinterpret_cast<const uint4*>(v.counts + t0);
    const uint4 b = *reinterpret_cast<const uint4*>(v.counts + t0 + 4);
    c[0] = a.x; c[1] = a.y; c[2] = a.z; c[3] = a.w;
    c[4] = b.x; c[5] = b.y; c[6] = b.z; c[7] = b.w;
  } else {
#pragma unroll
    for (int k = 0; k < 8; k++) c[k] = (t0 + k < (long long)v.T) ? v.counts[t0 + k] : 0u;
  }
  // earlier tiles: word j holds replica j / num_tiles of tile j % num_tiles
  const int nt = v.num_tiles, words = tile_words(nt);
  uint32_t acc = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int j = tid + k * SCAN_THREADS;
    if (j < words && (uint32_t)(j % nt) < vb) acc += v.tile_sum[j];
  }
  for (int j = tid + 8 * SCAN_THREADS; j < words; j += SCAN_THREADS)  // past 2^22 buckets only
    if ((uint32_t)(j % nt) < vb) acc += v.tile_sum[j];
  uint32_t sum = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) sum += c[k];
  uint32_t x = sum;  // inclusive scan of the thread sums within the warp
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  acc = __reduce_add_sync(0xffffffffu, acc);
  if (lane == 31) s_scan[wid] = x;
  if (lane == 0) s_prev[wid] = acc;
  __syncthreads();
  uint32_t run = x - sum;
#pragma unroll
  for (int w = 0; w < SCAN_THREADS / 32; w++) {
    run += s_prev[w];
    if (w < wid) run += s_scan[w];
  }
  uint32_t r[8];
#pragma unroll
  for (int k = 0; k < 8; k++) {
    r[k] = run;
    run += c[k];
  }
  if (vec) {
    const uint4 a = make_uint4(r[0], r[1], r[2], r[3]), b = make_uint4(r[4], r[5], r[6], r[7]);
    *reinterpret_cast<uint4*>(v.start + t0) = a;
    *reinterpret_cast<uint4*>(v.start + t0 + 4) = b;
    if (v.fend) {  // empty buckets; rankfix sets occupied ones
      *reinterpret_cast<uint4*>(v.fend + t0) = a;
      *reinterpret_cast<uint4*>(v.fend + t0 + 4) = b;
    }
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);  // ready for the next count
    *reinterpret_cast<uint4*>(v.counts + t0) = z;
    *reinterpret_cast<uint4*>(v.counts + t0 + 4) = z;
    if (v.bmove) {  // no movement recorded yet this substep
      *reinterpret_cast<uint4*>(v.bmove + t0) = z;
      *reinterpret_cast<uint4*>(v.bmove + t0 + 4) = z;
    }
  } else {
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const long long idx = t0 + k;
      if (idx < v.T) {
        v.start[idx] = r[k];
        if (v.fend) v.fend[idx] = r[k];
        v.counts[idx] = 0u;
        if (v.bmove) v.bmove[idx] = 0u;
      }
    }
  }
  if (vb == (uint32_t)v.num_tiles - 1u && tid == SCAN_THREADS - 1) v.start[v.T] = run;
  if (vb == 0 && tid == 0 && v.bmove) v.scratch[SCR_XMOVE] = 0u;
}

// Scatter by ticket (gridScatter, src/gpu/wgsl.js:238-245, without its
// second atomic), and clear the tile totals for the next count.
__device__ __forceinline__ void b_scatter(const SimView& v, uint32_t vb) {
  const int i = UPBD_VTID;
  if (i < tile_words(v.num_tiles)) v.tile_sum[i] = 0u;
  if (i >= v.N) return;
  if (!(v.flags[i] & F_ACTIVE)) return;
  const uint32_t h = v.cell[i];
  const uint32_t at = v.start[h] + v.ticket[i];
  if (UPBD_IDX_OK(v, at, v.N)) v.tmp[at] = (uint32_t)i;
}

// Deterministic membership: particle i goes to start[h] + #{j in bucket : j > i},
// i.e. descending index inside a bucket, the order Solver._buildGrid's
// `--cellStart[h]` scatter leaves (src/solver.js:182-183).
__device__ __forceinline__ void b_rankfix(const SimView& v, uint32_t vb) {
  const int i = UPBD_VTID;
  if (i >= v.N) return;
  if (!(v.flags[i] & F_ACTIVE)) return;
  const uint32_t h = v.cell[i];
  const uint32_t s = v.start[h], e = v.start[h + 1];
  uint32_t rank = 0, solids = 0;
  if (!UPBD_IDX_OK(v, e, (uint32_t)v.N + 1u)) return;
  for (uint32_t k = s; k < e; k++) {
    const uint32_t j = v.tmp[k];
    rank += (j > (uint32_t)i) ? 1u : 0u;
    solids += (j < (uint32_t)v.S) ? 1u : 0u;
  }
  if (!UPBD_IDX_OK(v, s + rank, v.N)) return;
  v.entries[s + rank] = (uint32_t)i;
  if (v.spos) {  // the stateless grid build has no bucket-ordered copies
    v.slot[i] = s + rank;
    v.spos[s + rank] = v.pos[i];
    v.fend[h] = e - solids;  // every member writes the same value
  }
}

// ------------------------------------------------------------------ fluid
// The fluid-fluid gathers run GLF lanes per particle (see lane_strided): a
// warp holds 32/GLF particles, every lane reaches the shuffles, and lane 0
// writes. Groups take the particles in slot order (group g: the particle at
// slot g of this substep's grid, entries[g]): the particles of one bucket sit
// in consecutive slots and share their 27 neighbour buckets, so a warp's
// candidate loads mostly hit L1. A particle's own arithmetic does not depend
// on which group runs it. Groups whose slot holds a solid, or lies past the
// active count start[T], have no work.
__device__ __forceinline__ void slot_group(const SimView& v, uint32_t t, uint32_t& e0, uint32_t& i, bool& fluid) {
  e0 = t / GLF;
  const uint32_t nact = __ldg(&v.start[v.T]);
  i = (e0 < nact) ? v.entries[e0] : 0u;
  fluid = e0 < nact && i >= (uint32_t)v.S;
}

// fluidDensity, src/gpu/wgsl.js:254-279. Every grid entry is active (the
// grid is built from the active particles of this substep, before bounds).
__device__ __forceinline__ void b_density(const SimView& v, const DevParams* __restrict__ P, uint32_t vb) {
  const uint32_t t = UPBD_VTID;
  const int lane = threadIdx.x & (GLF - 1);
  uint32_t myslot, i;
  bool act;
  slot_group(v, t, myslot, i, act);
  if (!__any_sync(0xffffffffu, act)) return;  // a warp of solid slots (or past the active count)
  real rho = 0.f, rhoNear = 0.f;
  const real4 pi = act ? v.spos[myslot] : make_real4(0.f, 0.f, 0.f, 0.f);
  CellHash ch;
  group_cell_hash<GLF>(pi.x, pi.y, pi.z, P->inv_cell, ch);
  const real H = P->fluid_h, H2 = H * H;
  const real HS = H * (1.0f + XSKIN), HS2 = HS * HS;  // list radius (for xsph)
  const real4* __restrict__ spos = v.spos;
  // lane l's c-th listed candidate goes to row l*NL + c, column myslot
  const uint32_t NS = (uint32_t)v.N;
  uint32_t* __restrict__ nbr = v.nbr + (size_t)lane * NL * NS + myslot;
  uint32_t cnt = 0;
#ifndef UPBD_PARITY_BUILD
  const real invH = 1.0f / H;
#endif
  lane_strided<0, GLF>(v, ch, lane, act, [&](uint32_t e) { return spos[e]; }, [&](uint32_t e, const real4& pj) {
    const real ex = pj.x - pi.x, ey = pj.y - pi.y, ez = pj.z - pi.z;
    const real d2 = dot3(ex, ey, ez, ex, ey, ez);
#ifdef UPBD_PARITY_BUILD
    if (e == myslot) return;
    if (d2 >= HS2) return;
    if (cnt < NL) nbr[cnt * NS] = e | ((d2 < H2) ? NBR_IN : 0u);  // for fluidDisp (same positions) and xsph
    cnt++;
    if (d2 >= H2) return;
    const real q = 1.0f - r_sqrt(d2) / H;
    rho = rho + q * q;
    rhoNear = rhoNear + q * q * q;
#else
    // branch-free: every lane of the warp takes the same path per candidate
    const bool in = (e != myslot) && (d2 < H2);
    const bool listed = (e != myslot) && (d2 < HS2);
    const real q = 1.0f - approx_sqrt(d2) * invH;
    const real qq = in ? q * q : 0.0f;
    rho = rho + qq;
    rhoNear = rhoNear + qq * q;
    if (listed && cnt < NL) nbr[cnt * NS] = e | (in ? NBR_IN : 0u);  // for fluidDisp (same positions) and xsph
    cnt += listed ? 1u : 0u;
#endif
  });
  if (act) v.ncount[lane * NS + myslot] = cnt;
  rho = lane_sum<GLF>(rho);
  rhoNear = lane_sum<GLF>(rhoNear);
  if (act && lane == 0) {
    const real2 d = make_real2(rho, rhoNear);
    v.density[i] = d;
    v.sdens[myslot] = d;
  }
}

// Contact marks (mark_fluid_near below) find a fluid particle from the
// solid's side, through the bucket the grid build put it in; the particle's
// own contact walk runs around the cell it is in after its displacement. A
// displacement that carries it into another cell can bring it within contact
// range of a solid two cells from its grid cell, which no mark walk reaches,
// so the pass that applies the fluid's move (from o, the position the grid
// was built from, to p) marks such a particle itself and it walks. Every
// particle that kept its cell and is in range of a solid is in a bucket of
// the 27 around that solid's cell, where the mark walk finds it.
__device__ __forceinline__ void mark_if_cell_changed(const SimView& v, const DevParams* __restrict__ P, int i,
                                                     const real4& o, const real4& p) {
  if (!P->use_mark) return;
  const double inv = P->inv_cell;
  const bool same = floor(__dmul_rn((double)o.x, inv)) == floor(__dmul_rn((double)p.x, inv)) &&
                    floor(__dmul_rn((double)o.y, inv)) == floor(__dmul_rn((double)p.y, inv)) &&
                    floor(__dmul_rn((double)o.z, inv)) == floor(__dmul_rn((double)p.z, inv));
  if (!same) v.mark[i] = 1u;  // also for a coordinate that is not finite
}

// fluidDisp, src/gpu/wgsl.js:281-316, DL threads per slot over the density
// pass's lists (same positions). Thread h of a slot takes lanes h*GLF/DL ..
// (h+1)*GLF/DL - 1: lane l's in-range neighbours (its NBR_IN entries) in its
// walk order, then the next lane's, summed one after another; the DL partials combine by the xor
// butterfly. A thread whose lists overflowed walks the 27 buckets for its
// lanes' shares instead, in the same order. With APPLY it also applies the
// displacement (applyDeltaFluid, src/gpu/wgsl.js:318-323): pos[i] and the own
// sfp slot are written, while every thread reads neighbours from spos, so no
// read sees a moved particle.
template <bool APPLY>
__device__ __forceinline__ void b_disp(const SimView& v, const DevParams* __restrict__ P, uint32_t vb) {
  constexpr int LPT = GLF / DL;  // lanes' lists per thread
  const uint32_t e0 = UPBD_VTID / DL;
  const int h = (int)(threadIdx.x & (DL - 1));
  const uint32_t nact = __ldg(&v.start[v.T]);
  const uint32_t i = (e0 < nact) ? v.entries[e0] : 0u;
  const bool act = e0 < nact && i >= (uint32_t)v.S;
  if (DL > 1) {
    if (!__any_sync(0xffffffffu, act)) return;
  } else if (!act) {
    return;
  }
  const real H = P->fluid_h, H2 = H * H;
  real sx = 0.f, sy = 0.f, sz = 0.f;
  const real4* __restrict__ spos = v.spos;
  const real2* __restrict__ sdens = v.sdens;
  const real4 pi = act ? spos[e0] : make_real4(0.f, 0.f, 0.f, 0.f);
  if (act) {
    const real maxPair = 0.05f * H;
    const real k = P->stiffness, kn = P->near_stiffness, rho0 = P->rest_density;
    const real2 di = sdens[e0];
    const real Pi = k * (di.x - rho0);
    const real PNi = kn * di.y;
#ifndef UPBD_PARITY_BUILD
    const real invH = 1.0f / H;
#endif
    auto pair = [&](const real4& pj, const real2& dj) {
      const real ex = pj.x - pi.x, ey = pj.y - pi.y, ez = pj.z - pi.z;
      const real d2 = dot3(ex, ey, ez, ex, ey, ez);
      if (d2 >= H2 || d2 < 1e-12f) return;
#ifdef UPBD_PARITY_BUILD
      const real d = r_sqrt(d2);
      const real q = 1.0f - d / H;
#else
      const real rd = r_rsqrt(d2);  // d2 >= 1e-12 here
      const real d = d2 * rd;
      const real q = 1.0f - d * invH;
#endif
      const real Pj = k * (dj.x - rho0);
      const real PNj = kn * dj.y;
      real D = 0.25f * ((Pi + Pj) * q + (PNi + PNj) * q * q);
      D = clampf(D, -maxPair, maxPair);
#ifdef UPBD_PARITY_BUILD
      const real f = D / d;
#else
      const real f = D * rd;
#endif
      sx = sx - ex * f; sy = sy - ey * f; sz = sz - ez * f;
    };
    const uint32_t NS = (uint32_t)v.N;
    const int l0 = h * LPT;
    uint32_t cnt[LPT];
    bool over = false;
#pragma unroll
    for (int u = 0; u < LPT; u++) {
      cnt[u] = v.ncount[(l0 + u) * NS + e0];
      over = over || cnt[u] > NL;
    }
    if (!over) {
      const uint32_t* __restrict__ nbr = v.nbr + e0;
#pragma unroll
      for (int u = 0; u < LPT; u++) {
        // four entries at a time: their list, position and density loads are
        // in flight together (a lane list holds ~4)
        for (uint32_t c = 0; c < cnt[u]; c += 4) {
          uint32_t e[4];
          real4 pj[4];
          real2 dj[4];
#pragma unroll
          for (int w = 0; w < 4; w++) {
            // entries beyond H (listed for xsph) and past the count become the
            // own slot, which pair() skips (d2 = 0)
            const uint32_t r = (c + w < cnt[u]) ? __ldg(&nbr[((uint32_t)(l0 + u) * NL + c + w) * NS]) : e0;
            e[w] = (r & NBR_IN) ? (r & ~NBR_IN) : e0;
            if (!UPBD_IDX_OK(v, e[w], NS)) e[w] = e0;  // out of range: the own slot (skipped, reported)
          }
#pragma unroll
          for (int w = 0; w < 4; w++) {
            pj[w] = spos[e[w]];
            dj[w] = sdens[e[w]];
          }
#pragma unroll
          for (int w = 0; w < 4; w++)
            if (c + w < cnt[u]) pair(pj[w], dj[w]);
        }
      }
    } else {
      // lane l's share of the walk: candidates c = l, l+GLF, ... of the sequence
      CellHash ch;
      ch.init(pi.x, pi.y, pi.z, P->inv_cell);
      const uint32_t mask = (uint32_t)v.T - 1u;
      for (int l = l0; l < l0 + LPT; l++) {
        uint32_t c = 0;
        for (int kk = 0; kk < 27; kk++) {
          const uint32_t hb = ch.bucket_k(kk, mask);
          const uint32_t s0 = __ldg(&v.start[hb]), s1 = __ldg(&v.fend[hb]);
          for (uint32_t e = s0; e < s1; e++, c++)
            if ((c & (GLF - 1)) == (uint32_t)l && e != e0) pair(spos[e], sdens[e]);
        }
      }
    }
  }
#pragma unroll
  for (int d = DL / 2; d > 0; d >>= 1) {
    sx = sx + __shfl_xor_sync(0xffffffffu, sx, d);
    sy = sy + __shfl_xor_sync(0xffffffffu, sy, d);
    sz = sz + __shfl_xor_sync(0xffffffffu, sz, d);
  }
  if (!act || h != 0) return;
  const real maxTotal = 0.35f * H;
  const real s2 = dot3(sx, sy, sz, sx, sy, sz);
  if (s2 > maxTotal * maxTotal) {
    const real f = maxTotal / r_sqrt(s2);
    sx = sx * f; sy = sy * f; sz = sz * f;
  }
  if (APPLY) {  // pi is pos[i]: the grid build copied it and nothing moved it since
    const real4 p = make_real4(pi.x + sx, pi.y + sy, pi.z + sz, pi.w);
    v.pos[i] = p;
    v.sfp[e0] = p;
    mark_if_cell_changed(v, P, (int)i, pi, p);
  } else {
    v.delta[i] = make_real4(sx, sy, sz, 1.0f);
  }
}

// applyDeltaFluid, src/gpu/wgsl.js:318-323 (standalone form)
__device__ __forceinline__ void b_apply_fluid(const SimView& v, const DevParams* __restrict__ P, uint32_t vb) {
  const int i = v.S + (int)UPBD_VTID;
  if (i >= v.N) return;
  if (!(v.flags[i] & F_ACTIVE)) return;
  const real4 o = v.pos[i];
  real4 p = o;
  const real4 d = v.delta[i];
  p.x = p.x + d.x; p.y = p.y + d.y; p.z = p.z + d.z;
  v.pos[i] = p;
  v.sfp[v.slot[i]] = p;
  mark_if_cell_changed(v, P, i, o, p);
}

// ------------------------------------------------------------------ solids
// Marks the fluid particles within contact range of solid i at position p
// (G lanes per solid). The bound is widened by 1e-5 so the set only grows:
// the contacts pass makes the exact test.
// Every lane of the warp calls it (the hash is shared by shuffles); only
// active solids walk.
// FROM_GRID: the fluid's positions are those of the grid build (spos), from
// before its displacement, which moves a particle by at most 0.35 H (the
// displacement pass's clamp): the reach grows by that much (and a relative
// 1e-3, far above the rounding of the positions), so every particle that
// ends within contact range is marked, and the marks need not wait for the
// displacement pass.
template <int G = GL, bool FROM_GRID = false>
__device__ __forceinline__ void mark_fluid_near(const SimView& v, const DevParams* __restrict__ P, real4 p,
                                                bool act, int lane) {
  CellHash ch;
  group_cell_hash<G>(p.x, p.y, p.z, P->inv_cell, ch);
  const real rsum = P->solid_radius + P->fluid_radius;
  const real reach = FROM_GRID ? (rsum + 0.35f * P->fluid_h) * 1.001f : rsum;
  const real lim2 = reach * reach * 1.00001f;
  // without FROM_GRID the fluid has moved by its displacement (sfp)
  const real4* __restrict__ sfp = FROM_GRID ? v.spos : v.sfp;
  uint32_t* __restrict__ mark = v.mark;
  lane_strided<0, G>(v, ch, lane, act, [&](uint32_t e) { return sfp[e]; }, [&](uint32_t e, const real4& pj) {
    const real ex = p.x - pj.x, ey = p.y - pj.y, ez = p.z - pj.z;
    if (ex * ex + ey * ey + ez * ez < lim2) {
      const uint32_t j = v.entries[e];
      if (UPBD_IDX_OK(v, j, v.N)) mark[j] = 1u;
    }
  });
}

// solidSolve, src/gpu/wgsl.js:326-359, GL lanes per solid: lane l takes the
// incident constraints k = st+l, st+l+GL, ... of the static CSR, whose other
// endpoint and pair scale 1/max(deg_i, deg_j) are precomputed (both are fixed
// for the life of the scene); the partials combine like lane_sum.
// Threads from solid_pad on (a warp multiple, so the solve's warps are whole)
// apply the fluid displacement when APPLY_FLUID (applyDeltaFluid,
// src/gpu/wgsl.js:318-323): the solve reads solid positions only.
//
// OUT selects what the solve does with solid i's correction:
//   SOLVE_DELTA  writes delta[i] for b_apply_solid (the reference's split).
//   SOLVE_STEP   applies it too (applyDeltaSolid, src/gpu/wgsl.js:361-366)
//                into a ping-pong copy of the solid positions: iteration `it`
//                reads pos (it 0) or sbuf[(it-1)&1] and writes sbuf[it&1],
//                inactive solids carried over unchanged.
//   SOLVE_LAST   applies it into pos and the slot copy, then marks the fluid
//                near the final position (b_apply_solid<true>'s work).
//   SOLVE_FINAL  as SOLVE_LAST without the marks (b_contact_mark follows).
// Every solve reads the previous iteration's positions only, as with the
// split passes, and pos + omega * delta is the same expression, so the
// folded iterations give the split ones' results bit for bit; they need at
// least two iterations (the first may not write what it reads).
constexpr int SOLVE_DELTA = 0, SOLVE_STEP = 1, SOLVE_LAST = 2, SOLVE_FINAL = 3;
template <bool APPLY_FLUID, int OUT = SOLVE_DELTA>
__device__ __forceinline__ void b_solid_solve(const SimView& v, const DevParams* __restrict__ P, int solid_pad, int it,
                                              uint32_t vb) {
  const int t = UPBD_VTID;
  if (t >= solid_pad) {
    const int i = v.S + (t - solid_pad);
    if (APPLY_FLUID && i < v.N && (v.flags[i] & F_ACTIVE)) {
      const real4 o = v.pos[i];
      real4 p = o;
      const real4 d = v.delta[i];
      p.x = p.x + d.x; p.y = p.y + d.y; p.z = p.z + d.z;
      v.pos[i] = p;
      v.sfp[v.slot[i]] = p;
      mark_if_cell_changed(v, P, i, o, p);
    }
    return;
  }
  const int i = t / GL;
  const int lane = threadIdx.x & (GL - 1);
  const bool act = i < v.S && (v.flags[i] & F_ACTIVE);
  const real4* __restrict__ pos = (OUT == SOLVE_DELTA || it == 0) ? v.pos : v.sbuf + (size_t)((it - 1) & 1) * v.S;
  const real4 pi = (i < v.S) ? pos[i] : make_real4(0.f, 0.f, 0.f, 0.f);
  real cx = 0.f, cy = 0.f, cz = 0.f;
  if (act) {
    const real wi = pi.w;
    const real h = P->h;
    const real alpha = P->compliance / (h * h);
    const uint32_t st = v.adj[i], en = v.adj[i + 1];
    const uint32_t* __restrict__ ids = v.adj + v.S + 1;
    const uint4* __restrict__ cons = v.cons;
#pragma unroll 2
    for (uint32_t k = st + lane; k < en; k += GL) {
      const uint32_t ci = __ldg(&ids[k]);
      const uint32_t other = __ldg(&v.adj_other[k]);
      if (!UPBD_IDX_OK(v, ci, v.C) || !UPBD_IDX_OK(v, other, v.S)) continue;
      const real s = __ldg(&v.adj_scale[k]);
      const real4 po = pos[other];
      const uint2 rw = *reinterpret_cast<const uint2*>(&cons[ci].z);  // rest bits, alive
      if (rw.y == 0u) continue;
      const real rest = __uint_as_float(rw.x);
      const real ex = pi.x - po.x, ey = pi.y - po.y, ez = pi.z - po.z;
      const real d = r_sqrt(dot3(ex, ey, ez, ex, ey, ez));
      if (d < 1e-9f) continue;
      const real wsum = wi + po.w;
      if (wsum == 0.f) continue;
      const real dl = -(d - rest) / (wsum + alpha);
      const real f = dl * wi / d * s;
      cx = cx + ex * f; cy = cy + ey * f; cz = cz + ez * f;
    }
  }
  cx = lane_sum(cx);
  cy = lane_sum(cy);
  cz = lane_sum(cz);
  if (OUT == SOLVE_DELTA) {
    if (act && lane == 0) v.delta[i] = make_real4(cx, cy, cz, 1.0f);
    return;
  }
  // applyDeltaSolid on the correction just summed (the delta b_apply_solid reads)
  const real w = P->omega;
  real4 p = pi;
  if (act) {
    p.x = p.x + cx * w; p.y = p.y + cy * w; p.z = p.z + cz * w;
  }
  if (OUT == SOLVE_STEP) {
    if (i < v.S && lane == 0) v.sbuf[(size_t)(it & 1) * v.S + i] = p;
    return;
  }
  if (act && lane == 0) {
    v.pos[i] = p;
    v.spos[v.slot[i]] = p;
  }
  if (OUT == SOLVE_LAST && P->use_mark) mark_fluid_near(v, P, act ? p : make_real4(0.f, 0.f, 0.f, 0.f), act, lane);
}

// applyDeltaSolid, src/gpu/wgsl.js:361-366. With MARK (last iteration of the
// solve) GL lanes per solid also mark the fluid near its final position for
// the contacts pass; the fluid positions are final by then.
template <bool MARK>
__device__ __forceinline__ void b_apply_solid(const SimView& v, const DevParams* __restrict__ P, uint32_t vb) {
  const int t = UPBD_VTID;
  const int i = MARK ? t / GL : t;
  const bool act = i < v.S && (v.flags[i] & F_ACTIVE);
  if (!MARK && !act) return;
  const real w = P->omega;
  real4 p = make_real4(0.f, 0.f, 0.f, 0.f);
  if (act) {
    p = v.pos[i];
    const real4 d = v.delta[i];
    p.x = p.x + d.x * w; p.y = p.y + d.y * w; p.z = p.z + d.z * w;
  }
  if (!MARK) {
    v.pos[i] = p;
    v.spos[v.slot[i]] = p;
    return;
  }
  const int lane = threadIdx.x & (GL - 1);
  if (act && lane == 0) {
    v.pos[i] = p;
    v.spos[v.slot[i]] = p;
  }
  if (P->use_mark) mark_fluid_near(v, P, p, act, lane);
}

// Contact marking on its own (when the solve's last position update does not
// carry it), G lanes per solid. Marks are a set, so the lane count is free:
// a whole warp per solid makes the 27 bucket lookups one round.
template <int G = GL, bool FROM_GRID = false>
__device__ __forceinline__ void b_contact_mark(const SimView& v, const DevParams* __restrict__ P, uint32_t vb) {
  if (!P->use_mark) return;
  const int t = UPBD_VTID;
  const int i = t / G;
  const bool act = i < v.S && (v.flags[i] & F_ACTIVE);
  mark_fluid_near<G, FROM_GRID>(v, P, act ? v.pos[i] : make_real4(0.f, 0.f, 0.f, 0.f), act, threadIdx.x & (G - 1));
}

// latticeRest, src/gpu/wgsl.js:373-381
__device__ __forceinline__ real lattice_rest(const SimView& v, real spacing, uint32_t a0, uint32_t b0) {
  uint32_t a = a0, b = b0, D = (uint32_t)v.dim1;
  if (a0 >= (uint32_t)v.N1) { a = a0 - v.N1; b = b0 - v.N1; D = (uint32_t)(v.dim2 > 1 ? v.dim2 : 1); }
  const real ax = (real)(a / (D * D)), ay = (real)((a / D) % D), az = (real)(a % D);
  const real bx = (real)(b / (D * D)), by = (real)((b / D) % D), bz = (real)(b % D);
  const real dx = ax - bx, dy = ay - by, dz = az - bz;
  return spacing * r_sqrt(dx * dx + dy * dy + dz * dz);
}

// latticeAdjacent, src/gpu/wgsl.js:409-416
__device__ __forceinline__ bool lattice_adjacent(const SimView& v, uint32_t i, uint32_t j) {
  if ((i >= (uint32_t)v.N1) != (j >= (uint32_t)v.N1)) return false;
  uint32_t a = i, b = j, D = (uint32_t)v.dim1;
  if (i >= (uint32_t)v.N1) { a = i - v.N1; b = j - v.N1; D = (uint32_t)(v.dim2 > 1 ? v.dim2 : 1); }
  const int ax = (int)(a / (D * D)), ay = (int)((a / D) % D), az = (int)(a % D);
  const int bx = (int)(b / (D * D)), by = (int)((b / D) % D), bz = (int)(b % D);
  return abs(ax - bx) <= 1 && abs(ay - by) <= 1 && abs(az - bz) <= 1;
}

// isBonded, src/gpu/wgsl.js:599-607
__device__ __forceinline__ bool is_bonded(const SimView& v, uint32_t i, uint32_t j) {
  const uint32_t* ids = v.adj + v.S + 1;
  for (uint32_t k = v.adj[i]; k < v.adj[i + 1]; k++) {
    if (!UPBD_IDX_OK(v, ids[k], v.C)) continue;
    const uint4 c = v.cons[ids[k]];
    if (c.w != 0u && (c.x == j || c.y == j)) return true;
  }
  return false;
}

__device__ __forceinline__ real solid_rsum(const SimView& v, const DevParams* __restrict__ P,
                                            uint32_t i, uint32_t j) {
  const real rsum = 2.0f * P->solid_radius;
  if (lattice_adjacent(v, i, j)) return mn(rsum, P->spacing * 0.97f);
  return rsum;
}

// collectContacts, src/gpu/wgsl.js:532-560
__device__ __forceinline__ void b_collect_contacts(const SimView& v, const DevParams* __restrict__ P, uint32_t vb) {
  const int i = UPBD_VTID;
  if (i >= v.S) return;
  uint32_t cnt = 0;
  if (v.flags[i] & F_ACTIVE) {
    const real4 pi = v.pos[i];
    const real margin = 2.0f * P->solid_radius;
    const uint32_t mask = (uint32_t)v.T - 1u;
    CellHash ch;
    ch.init(pi.x, pi.y, pi.z, P->inv_cell);
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        for (int c = 0; c < 3; c++) {
          const uint32_t hb = ch.bucket(a, b, c, mask);
          const uint32_t e1 = v.start[hb + 1];
          for (uint32_t e = v.start[hb]; e < e1; e++) {
            const uint32_t j = v.entries[e];
            if (j == (uint32_t)i || j >= (uint32_t)v.S || cnt >= C_K) continue;
            const real4 pj = v.pos[j];
            const real ex = pi.x - pj.x, ey = pi.y - pj.y, ez = pi.z - pj.z;
            const real lim = solid_rsum(v, P, i, j) + margin;
            if (dot3(ex, ey, ez, ex, ey, ez) >= lim * lim) continue;
            if (is_bonded(v, i, j)) continue;
            v.clist[(size_t)i * C_K + cnt] = j;
            cnt++;
          }
        }
  }
  v.ccount[i] = cnt;
}

// solidContacts, src/gpu/wgsl.js:562-585
__device__ __forceinline__ void b_solid_contacts(const SimView& v, const DevParams* __restrict__ P, uint32_t vb) {
  const int i = UPBD_VTID;
  if (i >= v.S) return;
  if (!(v.flags[i] & F_ACTIVE)) return;
  const real4 pi = v.pos[i];
  const real wi = pi.w;
  real cx = 0.f, cy = 0.f, cz = 0.f;
  const uint32_t n = v.ccount[i];
  for (uint32_t k = 0; k < n; k++) {
    const uint32_t j = v.clist[(size_t)i * C_K + k];
    if (!UPBD_IDX_OK(v, j, v.S)) continue;
    const real4 pj = v.pos[j];
    const real ex = pi.x - pj.x, ey = pi.y - pj.y, ez = pi.z - pj.z;
    const real rsum = solid_rsum(v, P, i, j);
    const real d2 = dot3(ex, ey, ez, ex, ey, ez);
    if (d2 >= rsum * rsum || d2 < 1e-12f) continue;
    const real wsum = wi + pj.w;
    if (wsum == 0.f) continue;
    const real d = r_sqrt(d2);
    const real f = (rsum - d) / d * wi / wsum * 0.5f;
    cx = cx + ex * f; cy = cy + ey * f; cz = cz + ez * f;
  }
  v.delta[i] = make_real4(cx, cy, cz, 1.0f);
}

// applySolidContacts, src/gpu/wgsl.js:587-596
__device__ __forceinline__ void b_apply_solid_contacts(const SimView& v, const DevParams* __restrict__ P, uint32_t vb) {
  const int i = UPBD_VTID;
  if (i >= v.S) return;
  if (!(v.flags[i] & F_ACTIVE)) return;
  const real maxC = 0.5f * P->solid_radius;
  const real4 dd = v.delta[i];
  real dx = dd.x, dy = dd.y, dz = dd.z;
  const real m2 = dot3(dx, dy, dz, dx, dy, dz);
  if (m2 > maxC * maxC) {
    const real f = maxC / r_sqrt(m2);
    dx = dx * f; dy = dy * f; dz = dz * f;
  }
  real4 p = v.pos[i];
  p.x = p.x + dx; p.y = p.y + dy; p.z = p.z + dz;
  v.pos[i] = p;
  v.spos[v.slot[i]] = p;
}

__device__ __forceinline__ void cross3(real ax, real ay, real az, real bx, real by, real bz,
                                       real& x, real& y, real& z) {
  x = ay * bz - az * by;
  y = az * bx - ax * bz;
  z = ax * by - ay * bx;
}

// solveTets, src/gpu/wgsl.js:423-468
__device__ __forceinline__ void b_solve_tets(const SimView& v, const DevParams* __restrict__ P, uint32_t vb) {
  const int i = UPBD_VTID;
  if (i >= v.S) return;
  if (!(v.flags[i] & F_ACTIVE)) return;
  const uint32_t* ids = v.tet_adj + v.S + 1;
  real cx = 0.f, cy = 0.f, cz = 0.f;
  for (uint32_t k = v.tet_adj[i]; k < v.tet_adj[i + 1]; k++) {
    const uint32_t t = ids[k];
    if (!UPBD_IDX_OK(v, t, v.NT)) continue;
    const uint32_t ia = v.tet_idx[4 * t], ib = v.tet_idx[4 * t + 1], ic = v.tet_idx[4 * t + 2],
                   id = v.tet_idx[4 * t + 3];
    if (!UPBD_IDX_OK(v, ia, v.S) || !UPBD_IDX_OK(v, ib, v.S) || !UPBD_IDX_OK(v, ic, v.S) ||
        !UPBD_IDX_OK(v, id, v.S))
      continue;
    const real V0 = v.tet_vol[t];
    if (V0 <= 0.f) continue;
    const real4 pa = v.pos[ia], pb = v.pos[ib], pc = v.pos[ic], pd = v.pos[id];
    const real bax = pb.x - pa.x, bay = pb.y - pa.y, baz = pb.z - pa.z;
    const real cax = pc.x - pa.x, cay = pc.y - pa.y, caz = pc.z - pa.z;
    const real dax = pd.x - pa.x, day = pd.y - pa.y, daz = pd.z - pa.z;
    real xx, xy, xz;
    cross3(bax, bay, baz, cax, cay, caz, xx, xy, xz);
    const real V = dot3(xx, xy, xz, dax, day, daz) / 6.0f;
    const real Cv = V - V0;
    real gbx, gby, gbz, gcx, gcy, gcz, gdx, gdy, gdz;
    cross3(cax, cay, caz, dax, day, daz, gbx, gby, gbz);
    gbx = gbx / 6.0f; gby = gby / 6.0f; gbz = gbz / 6.0f;
    cross3(dax, day, daz, bax, bay, baz, gcx, gcy, gcz);
    gcx = gcx / 6.0f; gcy = gcy / 6.0f; gcz = gcz / 6.0f;
    cross3(bax, bay, baz, cax, cay, caz, gdx, gdy, gdz);
    gdx = gdx / 6.0f; gdy = gdy / 6.0f; gdz = gdz / 6.0f;
    const real gax = -((gbx + gcx) + gdx), gay = -((gby + gcy) + gdy), gaz = -((gbz + gcz) + gdz);
    const real w = pa.w;
    const real denom = w * (dot3(gax, gay, gaz, gax, gay, gaz) + dot3(gbx, gby, gbz, gbx, gby, gbz) +
                             dot3(gcx, gcy, gcz, gcx, gcy, gcz) + dot3(gdx, gdy, gdz, gdx, gdy, gdz));
    if (denom < 1e-12f) continue;
    const real dl = -Cv / denom;
    const uint32_t da = v.tet_adj[ia + 1] - v.tet_adj[ia], db = v.tet_adj[ib + 1] - v.tet_adj[ib];
    const uint32_t dc = v.tet_adj[ic + 1] - v.tet_adj[ic], dd = v.tet_adj[id + 1] - v.tet_adj[id];
    const uint32_t m1 = (da < db) ? db : da, m2 = (dc < dd) ? dd : dc;
    uint32_t dm = (m1 < m2) ? m2 : m1;
    if (dm < 1u) dm = 1u;
    const real s = 1.0f / (real)dm;
    real gx = gax, gy = gay, gz = gaz;
    if ((uint32_t)i == ib) { gx = gbx; gy = gby; gz = gbz; }
    else if ((uint32_t)i == ic) { gx = gcx; gy = gcy; gz = gcz; }
    else if ((uint32_t)i == id) { gx = gdx; gy = gdy; gz = gdz; }
    const real f = w * dl * s;
    real c1x = gx * f, c1y = gy * f, c1z = gz * f;
    const real cl2 = dot3(c1x, c1y, c1z, c1x, c1y, c1z);
    const real lim = 0.5f * P->solid_radius;
    if (cl2 > lim * lim) {
      const real g = lim / r_sqrt(cl2);
      c1x = c1x * g; c1y = c1y * g; c1z = c1z * g;
    }
    cx = cx + c1x; cy = cy + c1y; cz = cz + c1z;
  }
  v.delta[i] = make_real4(cx, cy, cz, 1.0f);
}

// -------------------------------------------- bond update + contacts
// Threads [0, nb) run bondUpdate (src/gpu/wgsl.js:383-404) on one constraint
// each, threads [nb, nb+nt) run tetUpdate (src/gpu/wgsl.js:472-491), threads
// [nb+nt, nb+nt+nc) run the solid↔fluid coupling gather `contacts`
// (src/gpu/wgsl.js:609-646). All three read positions only; their outputs
// (constraints, tets, delta) are disjoint.
__device__ __forceinline__ void bond_update(const SimView& v, const DevParams* __restrict__ P, int ci) {
  const uint4 c = v.cons[ci];
  if (c.w == 0u) return;
  if (!UPBD_IDX_OK(v, c.x, v.S) || !UPBD_IDX_OK(v, c.y, v.S)) return;
  const real4 pa = v.pos[c.x], pb = v.pos[c.y];
  const real ex = pa.x - pb.x, ey = pa.y - pb.y, ez = pa.z - pb.z;
  const real d = r_sqrt(dot3(ex, ey, ez, ex, ey, ez));
  const real rest = __uint_as_float(c.z);
  const bool tear = (P->tear_mode == 1) ? (d > rest * P->break_strain)
                                        : (d > rest + P->tear_gap * 2.0f * P->solid_radius);
  if (tear) {
    v.cons[ci].w = 0u;
    return;
  }
  const real strain = (d - rest) / rest;
  real nr = rest;
  if (r_fabs(strain) > P->plastic_threshold) nr = rest + (d - rest) * P->plastic_rate;
  if (P->plastic_clamp) {
    const real r0 = lattice_rest(v, P->spacing, c.x, c.y);
    nr = clampf(nr, 0.9f * r0, 1.25f * r0);
  }
  if (nr != rest) v.cons[ci].z = __float_as_uint((float)nr);
}

__device__ __forceinline__ void tet_update(const SimView& v, const DevParams* __restrict__ P, int t) {
  const real V0 = v.tet_vol[t];
  if (V0 <= 0.f) return;
  const real gap = P->tear_gap * 2.0f * P->solid_radius;
  for (int p = 0; p < 3; p++)
    for (int q = p + 1; q < 4; q++) {
      const uint32_t a = v.tet_idx[4 * t + p], b = v.tet_idx[4 * t + q];
      if (!UPBD_IDX_OK(v, a, v.S) || !UPBD_IDX_OK(v, b, v.S)) return;
      const real4 pa = v.pos[a], pb = v.pos[b];
      const real ex = pa.x - pb.x, ey = pa.y - pb.y, ez = pa.z - pb.z;
      const real d = r_sqrt(dot3(ex, ey, ez, ex, ey, ez));
      if (d > lattice_rest(v, P->spacing, a, b) + gap) {
        v.tet_vol[t] = -V0;
        return;
      }
    }
}

// contacts for particle i, lane `lane` of its GL; every lane reaches the
// shuffles. Fluid particles that no solid marked have no contact and skip the
// walk (their correction is zero either way).
__device__ __forceinline__ void contacts_lane(const SimView& v, const DevParams* __restrict__ P, int i, int lane,
                                              int nc) {
  const bool act = i < nc && (v.flags[i] & F_ACTIVE);
  const bool iSolid = i < v.S;
  const bool walk = act && (iSolid || !P->use_mark || v.mark[i] != 0u);
  const unsigned FULL = 0xffffffffu;
  if (!__any_sync(FULL, walk)) {  // most fluid warps: nothing near a solid, no hash to compute
    if (act && lane == 0) v.delta[i] = make_real4(0.f, 0.f, 0.f, 0.f);
    return;
  }
  real cx = 0.f, cy = 0.f, cz = 0.f, cnt = 0.f;
  const real4 pi = walk ? v.pos[i] : make_real4(0.f, 0.f, 0.f, 0.f);
  CellHash ch;
  group_cell_hash(pi.x, pi.y, pi.z, P->inv_cell, ch);
  const real wi = pi.w;
  const real rs = P->solid_radius, rf = P->fluid_radius, scale = P->contact_scale;
  // a solid meets the fluid part of each bucket, a fluid particle the solid
  // part (fluid-fluid is DDR's job, solid-solid the contact cache's)
  const real ri = iSolid ? rs : rf;
  const real rsum = ri + (iSolid ? rf : rs);
  const real4* __restrict__ spos = v.spos;
  const real4* __restrict__ sfp = v.sfp;
  auto load_fluid = [&](uint32_t e) { return sfp[e]; };  // after the displacement
  auto load_solid = [&](uint32_t e) { return spos[e]; };  // after the solve
  auto pair = [&](uint32_t, const real4& pj) {
    const real ex = pi.x - pj.x, ey = pi.y - pj.y, ez = pi.z - pj.z;
    const real d2 = dot3(ex, ey, ez, ex, ey, ez);
    if (d2 >= rsum * rsum || d2 < 1e-12f) return;
    const real wsum = wi + pj.w;
    if (wsum == 0.f) return;
#ifdef UPBD_PARITY_BUILD
    const real d = r_sqrt(d2);
    const real f = (rsum - d) / d * wi / wsum * scale;
#else
    const real rd = r_rsqrt(d2);  // d2 >= 1e-12 here
    const real f = (rsum - d2 * rd) * rd * r_fdiv(wi, wsum) * scale;
#endif
    cx = cx + ex * f; cy = cy + ey * f; cz = cz + ez * f;
    cnt = cnt + 1.0f;
  };
  // a warp holds solids or fluid or both (at the S boundary): the two walks
  // are separate calls, each with every lane of the warp
  if (__any_sync(FULL, walk && iSolid)) lane_strided<0>(v, ch, lane, walk && iSolid, load_fluid, pair);
  if (__any_sync(FULL, walk && !iSolid)) lane_strided<1>(v, ch, lane, walk && !iSolid, load_solid, pair);
  cx = lane_sum(cx);
  cy = lane_sum(cy);
  cz = lane_sum(cz);
  cnt = lane_sum(cnt);
  if (act && lane == 0) v.delta[i] = make_real4(cx, cy, cz, cnt);
}

// nb_pad is nb + nt rounded up to a multiple of 32, so the contact threads
// start on a warp boundary and whole warps reach lane_sum's shuffles.
__device__ __forceinline__ void b_bond_contacts(const SimView& v, const DevParams* __restrict__ P,
                                                       int nb, int nt, int nb_pad, int nc, uint32_t vb) {
  const int t = UPBD_VTID;
  if (t < nb_pad) {
    if (t < nb)
      bond_update(v, P, t);
    else if (t < nb + nt)
      tet_update(v, P, t - nb);
    return;
  }
  const int c = t - nb_pad;
  contacts_lane(v, P, c / GL, c & (GL - 1), nc);
}

// -------------------------------- apply + bounds + velocity (per particle)
// The movement allowance of xsph's list test (XSKIN above), the same float on
// both sides of the test.
__device__ __forceinline__ real xsph_allowance(const DevParams* __restrict__ P) {
  return XSKIN * P->fluid_h * XMOVE_FRAC;
}

// Records how far fluid particle i (at slot sl) moved since the density pass
// (o: the position that pass saw, which its slot copy holds until the bounds
// pass writes p there): smove gets the distance (+inf when the particle left
// its cell or a coordinate is not finite), its grid bucket's bmove and the
// scene's SCR_XMOVE the largest distance above the recording threshold (the
// latter one atomic per warp).
__device__ __forceinline__ void record_move(const SimView& v, const DevParams* __restrict__ P, int i, uint32_t sl,
                                            const real4& o, const real4& p) {
  const real dx = p.x - o.x, dy = p.y - o.y, dz = p.z - o.z;
  const real INF = __int_as_float(0x7f800000);
  real m = r_sqrt(dot3(dx, dy, dz, dx, dy, dz));
  if (!(m <= 3.0e38f)) m = INF;  // NaN or inf
  const double inv = P->inv_cell;
  const bool same = floor(__dmul_rn((double)o.x, inv)) == floor(__dmul_rn((double)p.x, inv)) &&
                    floor(__dmul_rn((double)o.y, inv)) == floor(__dmul_rn((double)p.y, inv)) &&
                    floor(__dmul_rn((double)o.z, inv)) == floor(__dmul_rn((double)p.z, inv));
  v.smove[sl] = same ? r_to_float_up(m) : __int_as_float(0x7f800000);
  const bool rec = m > XMOVE_REC * xsph_allowance(P);
  if (rec) atomicMax(&v.bmove[v.cell[i]], __float_as_uint(r_to_float_up(m)));
  const unsigned am = __activemask();
  const uint32_t wm = __reduce_max_sync(am, rec ? __float_as_uint(r_to_float_up(m)) : 0u);
  if (wm != 0u && (int)(threadIdx.x & 31) == __ffs(am) - 1) atomicMax(&v.scratch[SCR_XMOVE], wm);
}

// applyDeltaAll (src/gpu/wgsl.js:648-660), bounds (src/gpu/wgsl.js:663-697)
// and velocityUpdate (src/gpu/wgsl.js:700-710): each touches only its own
// particle, so one launch runs all three. stage 1/2/3 stops after the first,
// second or third.
__device__ __forceinline__ void b_apply_bounds_vel(const SimView& v, const DevParams* __restrict__ P,
                                                          int stage, uint32_t vb) {
  const int i = UPBD_VTID;
  if (i >= v.N) return;
  uint32_t f = v.flags[i];
  if (!(f & F_ACTIVE)) return;
  const bool iSolid = i < v.S;
  const real r = iSolid ? P->solid_radius : P->fluid_radius;
  real4 p = v.pos[i];
  const uint32_t sl = v.slot[i];
  const real4 o = iSolid ? p : v.spos[sl];  // a fluid particle's density-pass position, read before any store
  // applyDeltaAll
  {
    const real4 dd = v.delta[i];
    real dx = dd.x, dy = dd.y, dz = dd.z;
    const real m2 = dot3(dx, dy, dz, dx, dy, dz);
    if (m2 > r * r) {
      const real g = r / r_sqrt(m2);
      dx = dx * g; dy = dy * g; dz = dz * g;
    }
    p.x = p.x + dx; p.y = p.y + dy; p.z = p.z + dz;
  }
  if (stage < 2) {
    v.pos[i] = p;
    if (!iSolid) record_move(v, P, i, sl, o, p);
    v.spos[sl] = p;
    return;
  }
  // bounds
  const real4 pv = v.prev[i];
  real px = p.x, py = p.y, pz = p.z;
  if (py < r) {
    py = r;
    const real mu = iSolid ? P->friction_solid : P->friction_fluid;
    px = px - (px - pv.x) * mu;
    pz = pz - (pz - pv.z) * mu;
  }
  if (py < P->wall_h + r) {
    const real lim = r + P->wall_t;
    const real wx = P->wall_x, wz = P->wall_z;
    if (r_fabs(r_fabs(px) - wx) < lim) {
      const real side = signf(px);
      px = (r_fabs(px) < wx) ? side * (wx - lim) : side * (wx + lim);
    }
    if (r_fabs(r_fabs(pz) - wz) < lim) {
      const real side = signf(pz);
      pz = (r_fabs(pz) < wz) ? side * (wz - lim) : side * (wz + lim);
    }
  }
  bool culled = false;
  if (!iSolid) {
    const real cr = P->cull_r;
    if (py < -3.0f || px * px + pz * pz > cr * cr) {
      v.flags[i] = 0u;
      culled = true;
    }
  }
  p.x = px; p.y = py; p.z = pz;
  v.pos[i] = p;
  if (!iSolid) record_move(v, P, i, sl, o, p);
  v.spos[sl] = p;
  if (stage < 3) return;
  if (culled) {
    // xsph still reads a culled neighbour's velocity (src/gpu/wgsl.js:761
    // does not test its flag): its slot keeps the unchanged velocity
    v.svel[sl] = v.vel[i];
    return;
  }
  // velocityUpdate
  const real h = P->h;
  real vx = (p.x - pv.x) / h, vy = (p.y - pv.y) / h, vz = (p.z - pv.z) / h;
  const real damp = iSolid ? P->damp_solid : P->damp_fluid;
  const real g = mx(0.0f, 1.0f - damp * h);
  vx = vx * g; vy = vy * g; vz = vz * g;
  const real sp2 = dot3(vx, vy, vz, vx, vy, vz);
  const real ms = P->max_speed;
  if (sp2 > ms * ms) {
    const real q = ms / r_sqrt(sp2);
    vx = vx * q; vy = vy * q; vz = vz * q;
  }
  if (!isfinite(vx) || !isfinite(vy) || !isfinite(vz)) atomicOr(&v.scratch[SCR_HEALTH], 1u);
  const real vw = v.vel[i].w;
  const real4 nv = make_real4(vx, vy, vz, vw);
  v.vel[i] = nv;
  v.svel[sl] = nv;
}

// solidVisc, src/gpu/wgsl.js:717-735
__device__ __forceinline__ void b_solid_visc(const SimView& v, const DevParams* __restrict__ P, uint32_t vb) {
  const int i = UPBD_VTID;
  if (i >= v.S) return;
  if (!(v.flags[i] & F_ACTIVE)) return;
  const uint32_t* ids = v.adj + v.S + 1;
  real sx = 0.f, sy = 0.f, sz = 0.f, m = 0.f;
  for (uint32_t k = v.adj[i]; k < v.adj[i + 1]; k++) {
    const uint4 c = v.cons[ids[k]];
    if (c.w == 0u) continue;
    const uint32_t other = (c.x == (uint32_t)i) ? c.y : c.x;
    const real4 vo = v.vel[other];
    sx = sx + vo.x; sy = sy + vo.y; sz = sz + vo.z;
    m = m + 1.0f;
  }
  const real4 vi = v.vel[i];
  real vx = vi.x, vy = vi.y, vz = vi.z;
  if (m > 0.f) {
    const real mu = P->solid_viscosity;
    vx = vx + mu * (sx / m - vx);
    vy = vy + mu * (sy / m - vy);
    vz = vz + mu * (sz / m - vz);
  }
  v.delta[i] = make_real4(vx, vy, vz, 0.f);
}

// solidViscApply, src/gpu/wgsl.js:737-742
__device__ __forceinline__ void b_solid_visc_apply(const SimView& v, uint32_t vb) {
  const int i = UPBD_VTID;
  if (i >= v.S) return;
  if (!(v.flags[i] & F_ACTIVE)) return;
  const real4 d = v.delta[i];
  const real w = v.vel[i].w;
  v.vel[i] = make_real4(d.x, d.y, d.z, w);
}

// xsph, src/gpu/wgsl.js:745-771 (slot-ordered groups, as b_density). The
// grid still holds the particles bounds culled this substep: they are
// neighbours (the reference does not test their flag) but have no pass of
// their own. Neighbour velocities come from the slot copies (svel), so with
// APPLY the blended velocity goes straight to vel[i] (xsphApply's result,
// src/gpu/wgsl.js:773-778) and the copy pass is not needed; without it the
// result waits in delta, where the reference's xsph pass leaves it.
// A group whose particle passes the list test (XSKIN) reads its lanes'
// density-pass lists instead of walking the 27 buckets: each lane's listed
// candidates are a subsequence, in order, of its walk share that holds every
// candidate within H now, so both forms add the same terms in the same order.
// list entries whose loads are in flight together: 2 in the list-only
// launch (48 registers: more warps hide the latency), 4 where one launch also
// walks
constexpr int XCH_LIST = 2, XCH_BOTH = 4;
constexpr int XWU = 4;  // candidates in flight per step of a walk beside the lists
// ROLE 0 runs both forms; ROLE 1 only the groups that read lists, ROLE 2
// only those that walk (two launches that run side by side, each with the
// registers its own form needs).
template <bool APPLY, int ROLE = 0>
__device__ __forceinline__ void b_xsph(const SimView& v, const DevParams* __restrict__ P, uint32_t vb) {
  const uint32_t t = UPBD_VTID;
  const int lane = threadIdx.x & (GLF - 1);
  uint32_t myslot, i;
  bool fluid;
  slot_group(v, t, myslot, i, fluid);
  const bool act = fluid && (v.flags[i] & F_ACTIVE);
  if (!__any_sync(0xffffffffu, act)) return;
  real sx = 0.f, sy = 0.f, sz = 0.f, m = 0.f;
  const real4 pi = act ? v.spos[myslot] : make_real4(0.f, 0.f, 0.f, 0.f);
  const real H = P->fluid_h, H2 = H * H;
  const real4* __restrict__ spos = v.spos;
  const real4* __restrict__ svel = v.svel;
  // position and velocity of every candidate are loaded together, before the
  // range test, and out-of-range ones add zero (the sums start at +0, so +0
  // leaves them unchanged): no load waits on the test
  struct PV {
    real4 p, v;
  };
  auto load = [&](uint32_t e) { return PV{spos[e], svel[e]}; };
  auto use = [&](uint32_t e, const PV& c) {
    const real ex = c.p.x - pi.x, ey = c.p.y - pi.y, ez = c.p.z - pi.z;
    const bool in = (e != myslot) && (dot3(ex, ey, ez, ex, ey, ez) < H2);
    sx = sx + (in ? c.v.x : 0.f); sy = sy + (in ? c.v.y : 0.f); sz = sz + (in ? c.v.z : 0.f);
    m = m + (in ? 1.0f : 0.f);
  };
  // the list test: the particle kept its cell (smove finite), it and every
  // particle of its 27 buckets moved within the allowance, and no lane's list
  // overflowed. The scene's largest recorded movement bounds every bucket's,
  // so when it passes the buckets are not looked at (nor hashed, unless the
  // group walks).
  const uint32_t NS = (uint32_t)v.N;
  const real allow = xsph_allowance(P), rec = XMOVE_REC * allow;
  const real sm = act ? v.smove[myslot] : 0.f;
  const uint32_t cnt = act ? v.ncount[lane * NS + myslot] : 0u;
  uint32_t over = (cnt > NL) ? 1u : 0u;
#pragma unroll
  for (int d = 1; d < GLF; d <<= 1) over |= __shfl_xor_sync(0xffffffffu, over, d);
  const bool quick = act && over == 0u && sm + r_fmax(rec, (real)__uint_as_float(v.scratch[SCR_XMOVE])) <= allow;
  const bool need = act && !quick;  // its buckets' movement, or the walk
  CellHash ch;
  bool listed = quick;
  if (__any_sync(0xffffffffu, need)) {
    group_cell_hash<GLF>(pi.x, pi.y, pi.z, P->inv_cell, ch);
    uint32_t bm = 0;
    if (need) {
      const uint32_t mask = (uint32_t)v.T - 1u;
#pragma unroll
      for (int r = 0; r < (27 + GLF - 1) / GLF; r++) {
        const int k = lane + GLF * r;
        if (k < 27) bm = max(bm, v.bmove[ch.bucket_k(k, mask)]);
      }
    }
#pragma unroll
    for (int d = 1; d < GLF; d <<= 1) bm = max(bm, __shfl_xor_sync(0xffffffffu, bm, d));
    // bm holds a finite distance or +inf
    listed = quick || (need && over == 0u && sm + r_fmax(rec, (real)__uint_as_float(bm)) <= allow);
  }
  const bool walks = act && !listed;
  const bool mine = (ROLE == 0) ? act : ((ROLE == 1) ? listed : walks);
  if (ROLE != 0 && !__any_sync(0xffffffffu, mine)) return;
  // with both forms in one launch the groups that walk keep XWU candidates'
  // loads in flight: while most groups read lists, the few walks are the
  // kernel's tail
  if (ROLE == 0 && __any_sync(0xffffffffu, walks)) lane_strided<0, GLF, XWU>(v, ch, lane, walks, load, use);
  // the walking launch: where one or two groups of a warp walk, the warp's
  // lanes load their candidates for them; where more do, each walks its own
  // (staged walks take turns, so they cost more than they save there)
  if (ROLE == 2) {
    const unsigned wg = __ballot_sync(0xffffffffu, walks && lane == 0);
    if (wg != 0u && __popc(wg) <= 2) lane_staged<0, GLF>(v, ch, lane, walks, load, use);
    else if (wg != 0u) lane_strided<0, GLF, 1>(v, ch, lane, walks, load, use);
  }
  if (ROLE != 2 && listed) {
    constexpr int XCH = (ROLE == 1) ? XCH_LIST : XCH_BOTH;
    const uint32_t* __restrict__ nbr = v.nbr + (size_t)lane * NL * NS + myslot;
    for (uint32_t c = 0; c < cnt; c += XCH) {  // XCH entries' loads in flight
      uint32_t e[XCH];
      PV pv[XCH];
#pragma unroll
      for (int w = 0; w < XCH; w++) {
        e[w] = (c + w < cnt) ? (__ldg(&nbr[(c + w) * NS]) & ~NBR_IN) : myslot;
        if (!UPBD_IDX_OK(v, e[w], NS)) e[w] = myslot;  // out of range: the own slot (skipped, reported)
      }
#pragma unroll
      for (int w = 0; w < XCH; w++) pv[w] = load(e[w]);
#pragma unroll
      for (int w = 0; w < XCH; w++)
        if (c + w < cnt) use(e[w], pv[w]);
    }
  }
  sx = lane_sum<GLF>(sx);
  sy = lane_sum<GLF>(sy);
  sz = lane_sum<GLF>(sz);
  m = lane_sum<GLF>(m);
  if (mine && lane == 0) {
    const real4 vi = v.vel[i];
    real vx = vi.x, vy = vi.y, vz = vi.z;
    if (m > 0.f) {
      const real mu = P->viscosity;
      vx = vx + mu * (sx / m - vx);
      vy = vy + mu * (sy / m - vy);
      vz = vz + mu * (sz / m - vz);
    }
    if (APPLY)
      v.vel[i] = make_real4(vx, vy, vz, 0.f);
    else
      v.delta[i] = make_real4(vx, vy, vz, m);
  }
}

// countActive (src/gpu/wgsl.js:874-879) with a last-block epilogue that
// publishes the count and the health bits to mapped host memory.
__device__ __forceinline__ void b_count_active(const SimView& v, uint32_t vb, uint32_t nblk) {
  const int i = v.S + (int)UPBD_VTID;
  uint32_t a = (i < v.N && (v.flags[i] & F_ACTIVE)) ? 1u : 0u;
  a = __reduce_add_sync(0xffffffffu, a);
  __shared__ uint32_t s_sum;
  if (threadIdx.x == 0) s_sum = 0;
  __syncthreads();
  if ((threadIdx.x & 31) == 0 && a) atomicAdd(&s_sum, a);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_sum) atomicAdd(&v.scratch[SCR_ACTIVE], s_sum);
    __threadfence();
    const uint32_t done = atomicAdd(&v.scratch[SCR_DONE], 1u);
    if (done == nblk - 1u) {
      __threadfence();
      const uint32_t total = atomicExch(&v.scratch[SCR_ACTIVE], 0u);
      v.scratch[SCR_DONE] = 0u;
      volatile uint32_t* hm = v.host_mapped;
      hm[HM_ACTIVE] = total;
      hm[HM_HEALTH] = atomicOr(&v.scratch[SCR_HEALTH], 0u);
    }
  }
}

}  // namespace upbd
