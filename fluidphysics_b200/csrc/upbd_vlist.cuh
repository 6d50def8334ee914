// Product-build fluid gathers over neighbour lists kept across substeps
// (Verlet lists): fluidDensity, fluidDisp and xsph of src/gpu/wgsl.js
// (254-279, 281-323, 745-778) with the same pair sets as the 27-bucket walks
// and their own summation order (the parity build keeps the walk order of
// upbd_passes.cuh and matches the oracle bit for bit; this build stays within
// the stated per-substep tolerance of it).
//
// Which pairs the reference counts. Its gathers visit the members of the 27
// hash buckets around a particle's cell, so particle j enters i's sum once
// per occurrence of j's bucket among i's 27 buckets, when within H. With no
// two of those 27 buckets equal (PF_DUP / PF_DUPF clear) and every pair
// within H in adjacent cells (fluid_h at most the cell size), that is: every
// fluid j within H, once. xsph runs after the fluid moved but on the grid
// built before: j counts when its grid-time bucket is among the 27 buckets
// of i's current cell; for a j that kept its cell since the grid build that
// holds whenever j is within H, and the others (evel[.].w = 1) are checked
// against the 27 buckets explicitly.
//
// When lists are complete. A rebuild (density pass, SCR_REBUILD) lists every
// fluid particle within R = H * (1 + VSKIN): it walks the 27 cells and the
// cells beyond them that R reaches (R is below two cell sizes), and takes a
// candidate only at the visit of its own cell, so buckets met through two
// cells list it once; it records the position. A list may be read when the
// particle's movement since then, plus the largest movement of any particle
// that can be within H of it, stays within the allowance VMOVE_FRAC * VSKIN
// * H. The scene-wide largest movement of the particles below VFAST * the
// allowance (SCR_XMOVE) settles most particles; the faster ones mark the 27
// buckets around them (bfast), and a particle in a marked bucket, or one
// that the scene-wide bound does not settle, takes the largest movement
// recorded in its 27 buckets (every particle the reference could count sits
// in one of them). Particles that fail walk the buckets (without touching
// their lists). A rebuild follows a substep where more than F / VWALK_DIV
// particles walked for want of a usable list (particles whose 27 buckets
// coincide walk regardless and are not counted), and any change the lists
// cannot follow (emit, drain, a state write, a cull: SCR_DIRTY).
//
// Order. The gathers run their groups in the rank order of the last rebuild
// (the grid's slot order then: group r takes particle ep[r]) and read their
// own and their neighbours' data from rank-ordered copies, so list entries
// and neighbour loads stay close together in memory between rebuilds.
#pragma once
#include "upbd_device.cuh"

namespace upbd {

// list entries whose loads are in flight together per lane (the list
// kernels run at 32 registers so that all their blocks are resident at once)
constexpr int VLF = 2;

__device__ __forceinline__ float vl_allowance(const DevParams* __restrict__ P) {
  return VSKIN * P->fluid_h * VMOVE_FRAC;
}

__device__ __forceinline__ float vl_dist(const float4& a, const float4& b) {
  const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
  const float m = sqrtf(dot3(dx, dy, dz, dx, dy, dz));
  return (m <= 3.0e38f) ? m : __int_as_float(0x7f800000);  // NaN / inf -> +inf
}

// Largest recorded movement (float bits) in the 27 buckets of ch, reduced
// over the GLF lanes of each group. Every lane of the warp calls it.
__device__ __forceinline__ uint32_t vl_bucket_move(const SimView& v, const CellHash& ch, bool need, int lane) {
  uint32_t bm = 0;
  if (need) {
    const uint32_t mask = (uint32_t)v.T - 1u;
#pragma unroll
    for (int r = 0; r < (27 + GLF - 1) / GLF; r++) {
      const int k = lane + GLF * r;
      if (k < 27) bm = max(bm, __ldg(&v.bmove[ch.bucket_k(k, mask)]));
    }
  }
#pragma unroll
  for (int d = 1; d < GLF; d <<= 1) bm = max(bm, __shfl_xor_sync(0xffffffffu, bm, d));
  return bm;
}

// Walkers of this warp's groups (lane 0 of each) into the scene's counter.
__device__ __forceinline__ void vl_count_walkers(const SimView& v, bool walks, int lane) {
  const unsigned b = __ballot_sync(0xffffffffu, walks && lane == 0);
  if (b != 0u && (threadIdx.x & 31) == 0) atomicAdd(&v.scratch[SCR_WALKERS], (uint32_t)__popc(b));
}

// Records movement m of a fluid particle whose cell is that of p and grid
// bucket h: above VMOVE_REC * the allowance into bmove[h]; above VFAST * the
// allowance it marks the 27 buckets around p's cell, else it raises the
// scene-wide SCR_XMOVE (one atomic per warp). am: the lanes that call it.
__device__ __forceinline__ void vl_note_move(const SimView& v, const DevParams* __restrict__ P, unsigned am, float m,
                                             uint32_t h, const float4& p) {
  const float allow = vl_allowance(P);
  const bool rec = m > VMOVE_REC * allow;
  const bool fast = m > VFAST * allow;
  if (rec) atomicMax(&v.bmove[h], __float_as_uint(m));
  if (fast) {
    CellHash ch;
    ch.init(p.x, p.y, p.z, P->inv_cell);
    const uint32_t mask = (uint32_t)v.T - 1u;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++)
#pragma unroll
        for (int c = 0; c < 3; c++) v.bfast[ch.bucket(a, b, c, mask)] = 1u;
  }
  const uint32_t wm = __reduce_max_sync(am, (rec && !fast) ? __float_as_uint(m) : 0u);
  if (wm != 0u && (int)(threadIdx.x & 31) == __ffs(am) - 1) atomicMax(&v.scratch[SCR_XMOVE], wm);
}

// Grid-time record by the rank fix-up (not at a rebuild, when the density
// rebuild writes them): the rank record, the position copy for the density
// and displacement passes, and the movement since the list build.
__device__ __forceinline__ void vl_record_grid(const SimView& v, const DevParams* __restrict__ P, int i, uint32_t h,
                                               uint32_t slot) {
  const unsigned am = __activemask();  // the lanes that reach the warp reduction below
  const uint32_t r = v.erank[i];
  float m = 0.f;
  float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
  if (r != NO_RANK) {
    p = v.pos[i];
    v.epos[r] = p;
    v.erec[r] = make_uint4((uint32_t)i, slot, h, v.pfl[i] & (PF_DUP | PF_LOK));
    m = vl_dist(p, v.xlist[r]);
  }
  vl_note_move(v, P, am, m, h, p);
}

// Final-time record by the bounds pass for fluid particle i of rank r: its
// final position copy, how far it moved since its list was built (smove[r]
// and the bucket / scene records), whether its final cell differs from its
// grid-time cell o (returned; PF_MOVED, and then PF_DUPF is tested for the
// new cell) and whether it was culled (PF_CULLED), into the rank record.
__device__ __forceinline__ bool vl_record(const SimView& v, const DevParams* __restrict__ P, int i, uint32_t r,
                                          const float4& o, const float4& p, bool culled) {
  const unsigned am = __activemask();  // the lanes that reach the warp reduction below
  v.epos[r] = p;
  const float m = vl_dist(p, v.xlist[r]);
  v.smove[r] = m;
  vl_note_move(v, P, am, m, v.cell[i], p);
  const double inv = P->inv_cell;
  const bool same = floor(__dmul_rn((double)o.x, inv)) == floor(__dmul_rn((double)p.x, inv)) &&
                    floor(__dmul_rn((double)o.y, inv)) == floor(__dmul_rn((double)p.y, inv)) &&
                    floor(__dmul_rn((double)o.z, inv)) == floor(__dmul_rn((double)p.z, inv));
  const uint32_t pf = v.erec[r].w;
  bool dupf = (pf & PF_DUP) != 0u;
  if (!same) {
    CellHash ch;
    ch.init(p.x, p.y, p.z, inv);
    dupf = buckets_coincide(ch, (uint32_t)v.T - 1u);
  }
  uint32_t npf = pf & ~(PF_DUPF | PF_MOVED | PF_CULLED);
  npf |= (dupf ? PF_DUPF : 0u) | (same ? 0u : PF_MOVED) | (culled ? PF_CULLED : 0u);
  v.erec[r].w = npf;
  return !same;
}

// Cell (cx, cy, cz) is the cell of p (Solver._hashPos's floor(p * (1/cs))).
__device__ __forceinline__ bool vl_in_cell(const float4& p, double inv, double cx, double cy, double cz) {
  return floor(__dmul_rn((double)p.x, inv)) == cx && floor(__dmul_rn((double)p.y, inv)) == cy &&
         floor(__dmul_rn((double)p.z, inv)) == cz;
}

// Hash component (Solver._hash) of cell coordinate c + o, o in -2..2, from
// the five precomputed ones.
__device__ __forceinline__ int32_t vl_sel(int o, int32_t m2, int32_t m1, int32_t z0, int32_t p1, int32_t p2) {
  return (o == -2) ? m2 : ((o == -1) ? m1 : ((o == 0) ? z0 : ((o == 1) ? p1 : p2)));
}

// The particle of group r (rank r of the last rebuild, or slot r of this
// substep's grid when `slots`), its slot, and whether it is active fluid.
__device__ __forceinline__ void vl_group(const SimView& v, uint32_t r, bool slots, uint32_t& i, uint32_t& slot,
                                         bool& fluid) {
  const uint32_t nact = __ldg(&v.start[v.T]);
  if (slots) {
    i = (r < nact) ? v.entries[r] : NO_RANK;
    slot = r;
  } else {
    i = (r < (uint32_t)v.N) ? v.ep[r] : NO_RANK;
    slot = (i != NO_RANK) ? v.slot[i] : 0u;
  }
  fluid = i != NO_RANK && i >= (uint32_t)v.S;
}

// Density of one group over its list (lane l: entries l, l + GLF, ...,
// VLF entries' loads in flight).
__device__ __forceinline__ void vl_density_list(const SimView& v, uint32_t r, int lane, const float4& pi, float H2,
                                                float invH, float& rho, float& rhoNear) {
  const uint32_t NS = (uint32_t)v.N;
  const uint32_t n = v.ncount[r];
  const uint32_t* __restrict__ lst = v.nbr + r;
  const float4* __restrict__ epos = v.epos;
  for (uint32_t c = (uint32_t)lane; c < n; c += VLF * GLF) {
    uint32_t j[VLF];
#pragma unroll
    for (int w = 0; w < VLF; w++) {
      const uint32_t cw = c + (uint32_t)(w * GLF);
      j[w] = (cw < n) ? __ldg(&lst[(size_t)cw * NS]) : NO_RANK;
    }
    float4 pj[VLF];
#pragma unroll
    for (int w = 0; w < VLF; w++) pj[w] = epos[(j[w] != NO_RANK) ? j[w] : j[0]];
#pragma unroll
    for (int w = 0; w < VLF; w++) {
      const float ex = pj[w].x - pi.x, ey = pj[w].y - pi.y, ez = pj[w].z - pi.z;
      const float d2 = dot3(ex, ey, ez, ex, ey, ez);
      const float q = 1.0f - approx_sqrt(d2) * invH;
      const float qq = (d2 < H2 && j[w] != NO_RANK) ? q * q : 0.0f;
      rho = rho + qq;
      rhoNear = rhoNear + qq * q;
    }
  }
}

// Per-lane partial sums of a walk (K floats).
template <int K>
struct VAcc {
  float v[K];
};

// Lane src's copy of x (a struct of 32-bit words).
template <class T>
__device__ __forceinline__ T vl_shfl(const T& x, int src) {
  static_assert(sizeof(T) % 4 == 0, "32-bit fields only");
  T y;
  const uint32_t* a = reinterpret_cast<const uint32_t*>(&x);
  uint32_t* b = reinterpret_cast<uint32_t*>(&y);
#pragma unroll
  for (int k = 0; k < (int)(sizeof(T) / 4); k++) b[k] = __shfl_sync(0xffffffffu, a[k], src);
  return y;
}

// Walk of the groups that cannot read their lists: all 32 lanes of the warp
// walk each walking group's 27-bucket sequence in turn (candidate c to lane
// c mod 32), with the group's own data `st` broadcast from its first lane;
// term(st, e, load(e)) gives a candidate's contribution, and the warp's sum
// is added to `out` on the group's first lane (the other lanes add nothing).
// A walk then costs about seven steps instead of fifty, so the few particles
// that walk do not hold the launch open. Every lane of the warp calls it.
template <int K, class St, class Load, class Term>
__device__ __forceinline__ void vl_walk(const SimView& v, const CellHash& ch, int lane, bool walks, const St& st,
                                        Load&& load, Term&& term, VAcc<K>& out) {
  const unsigned FULL = 0xffffffffu;
  const unsigned todo0 = __ballot_sync(FULL, walks && lane == 0);  // one bit per walking group
  if (todo0 == 0u) return;
  const int L = (int)(threadIdx.x & 31), w = (int)(threadIdx.x >> 5);
  const int g = w * (32 / GLF) + L / GLF;
  walk_tables<0, GLF>(v, ch, lane, walks, g);
  unsigned todo = todo0;
  while (todo) {
    const int first = __ffs(todo) - 1;  // the group's lane 0
    todo &= todo - 1u;
    const int gw = w * (32 / GLF) + first / GLF;
    const St sw = vl_shfl(st, first);
    const uint32_t run = s_walk_off[gw][27];
    uint32_t k = 0, next = s_walk_off[gw][1], base = s_walk_base[gw][0];
    VAcc<K> acc;
#pragma unroll
    for (int q = 0; q < K; q++) acc.v[q] = 0.f;
    for (uint32_t c = (uint32_t)L; c < run; c += 32) {
      while (c >= next) {
        k++;
        next = s_walk_off[gw][k + 1];
        base = s_walk_base[gw][k];
      }
      const uint32_t e = base + c;
      const VAcc<K> t = term(sw, e, load(e));
#pragma unroll
      for (int q = 0; q < K; q++) acc.v[q] = acc.v[q] + t.v[q];
    }
#pragma unroll
    for (int q = 0; q < K; q++) {
      float x = acc.v[q];
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) x = x + __shfl_xor_sync(FULL, x, d);
      if (L == first) out.v[q] = out.v[q] + x;
    }
  }
  __syncwarp();  // the next call may rewrite this warp's table rows
}

// fluidDensity (src/gpu/wgsl.js:254-279) at a rebuild for the particle of
// rank r (its slot in this substep's grid), with the whole warp: its density
// and its list.
//
// The reference's density over the 27 cells (every bucket visit counted,
// coinciding buckets included) and, for the list, every fluid candidate
// within R of the cells that R reaches: the 27 and those past them. When two
// of the visited cells share a bucket, a candidate is taken only at the
// visit of its own cell (so it is listed once); otherwise every candidate
// within R lies in the cell it was met through. The lanes place their entries
// by a ballot, so a list holds its candidates in walk order (deterministic
// sums). At a rebuild a candidate's rank is its slot.
__device__ __forceinline__ void vl_rebuild_one(const SimView& v, const DevParams* __restrict__ P, uint32_t r,
                                               int lane, int g) {
  const unsigned FULL = 0xffffffffu;
  uint32_t i, myslot;
  bool act;
  vl_group(v, r, true, i, myslot, act);  // the same for every lane of the warp
  if (lane == 0 && r < (uint32_t)v.N) {  // the new rank order
    v.ep[r] = i;
    if (i != NO_RANK) v.erank[i] = r;
  }
  if (!act) return;  // the whole warp
  const float4 pi = v.spos[myslot];
  const float H = P->fluid_h, H2 = H * H, invH = 1.0f / H;
  const float R = H * (1.0f + VSKIN), R2 = R * R;
  const double inv = P->inv_cell;
  const double cx = floor(__dmul_rn((double)pi.x, inv)), cy = floor(__dmul_rn((double)pi.y, inv)),
               cz = floor(__dmul_rn((double)pi.z, inv));
  CellHash ch;
  group_cell_hash<32>(pi.x, pi.y, pi.z, inv, ch);
  const uint32_t mask = (uint32_t)v.T - 1u;
  // the box of cells that R reaches (R is below two cells)
  const double ext = (double)R * inv - 1.0 + 1e-3, rc2 = ((double)R * inv) * ((double)R * inv) * 1.0001;
  const double fx = __dmul_rn((double)pi.x, inv) - cx, fy = __dmul_rn((double)pi.y, inv) - cy,
               fz = __dmul_rn((double)pi.z, inv) - cz;
  const int lox = (fx < ext) ? -2 : -1, hix = (1.0 - fx < ext) ? 2 : 1;
  const int loy = (fy < ext) ? -2 : -1, hiy = (1.0 - fy < ext) ? 2 : 1;
  const int loz = (fz < ext) ? -2 : -1, hiz = (1.0 - fz < ext) ? 2 : 1;
  const int ny = hiy - loy + 1, nz = hiz - loz + 1, nbox = (hix - lox + 1) * ny * nz;  // <= 64
  const int32_t xm2 = js_toint32(__dmul_rn(__dadd_rn(cx, -2.0), 92837111.0));
  const int32_t xp2 = js_toint32(__dmul_rn(__dadd_rn(cx, 2.0), 92837111.0));
  const int32_t ym2 = js_toint32(__dmul_rn(__dadd_rn(cy, -2.0), 689287499.0));
  const int32_t yp2 = js_toint32(__dmul_rn(__dadd_rn(cy, 2.0), 689287499.0));
  const int32_t zm2 = js_toint32(__dmul_rn(__dadd_rn(cz, -2.0), 283923481.0));
  const int32_t zp2 = js_toint32(__dmul_rn(__dadd_rn(cz, 2.0), 283923481.0));
  // box cells k = lane and lane + 32: visited (one of the 27, or past them and
  // within R) -> bucket and fluid range; bv = NO_RANK for cells not visited
  uint32_t bv[2], s0[2], n[2];
  bool extra[2];
#pragma unroll
  for (int half = 0; half < 2; half++) {
    const int k = lane + 32 * half;
    bv[half] = NO_RANK;
    s0[half] = 0u;
    n[half] = 0u;
    extra[half] = false;
    if (k < nbox) {
      const int a = lox + k / (ny * nz), b = loy + (k / nz) % ny, c = loz + k % nz;
      const bool core = a >= -1 && a <= 1 && b >= -1 && b <= 1 && c >= -1 && c <= 1;
      const double gx = (a < 0) ? fx + (double)(-a - 1) : ((a > 0) ? (1.0 - fx) + (double)(a - 1) : 0.0);
      const double gy = (b < 0) ? fy + (double)(-b - 1) : ((b > 0) ? (1.0 - fy) + (double)(b - 1) : 0.0);
      const double gz = (c < 0) ? fz + (double)(-c - 1) : ((c > 0) ? (1.0 - fz) + (double)(c - 1) : 0.0);
      if (core || gx * gx + gy * gy + gz * gz <= rc2) {
        bv[half] = (uint32_t)(vl_sel(a, xm2, ch.hx[0], ch.hx[1], ch.hx[2], xp2) ^
                              vl_sel(b, ym2, ch.hy[0], ch.hy[1], ch.hy[2], yp2) ^
                              vl_sel(c, zm2, ch.hz[0], ch.hz[1], ch.hz[2], zp2)) & mask;
        if (!core) {
          extra[half] = true;
          s0[half] = __ldg(&v.start[bv[half]]);
          n[half] = __ldg(&v.fend[bv[half]]) - s0[half];
        }
      }
    }
  }
  // do two visited cells share a bucket?
  bool dup = false;
#pragma unroll
  for (int half = 0; half < 2; half++) {
    const unsigned same = __match_any_sync(FULL, bv[half]);
    dup = dup || (bv[half] != NO_RANK && __popc(same) > 1);
  }
  for (int d = 0; d < 32; d++) {
    const uint32_t o = __shfl_sync(FULL, bv[1], d);
    dup = dup || (bv[0] != NO_RANK && bv[0] == o);
  }
  const bool check = __any_sync(FULL, dup);
  const float4* __restrict__ spos = v.spos;
  const uint32_t NS = (uint32_t)v.N;
  uint32_t* __restrict__ lst = v.nbr + r;
  const unsigned lt = (1u << lane) - 1u;
  uint32_t lcount = 0;
  auto place = [&](bool kp, uint32_t e) {
    const unsigned bal = __ballot_sync(FULL, kp);
    if (kp) {
      const uint32_t c = lcount + (uint32_t)__popc(bal & lt);
      if (c < NLT) lst[(size_t)c * NS] = e;
    }
    lcount += (uint32_t)__popc(bal);
  };
  float rho = 0.f, rhoNear = 0.f;
  {  // the 27 cells
    const uint32_t run = walk_tables<0, 32>(v, ch, lane, true, g);
    uint32_t k = 0, next = s_walk_off[g][1], base = s_walk_base[g][0];
    for (uint32_t c0 = 0; c0 < run; c0 += 32) {
      const uint32_t c = c0 + (uint32_t)lane;
      bool kp = false;
      uint32_t e = 0;
      if (c < run) {
        while (c >= next) {
          k++;
          next = s_walk_off[g][k + 1];
          base = s_walk_base[g][k];
        }
        e = base + c;
        const float4 pj = spos[e];
        const float ex = pj.x - pi.x, ey = pj.y - pi.y, ez = pj.z - pi.z;
        const float d2 = dot3(ex, ey, ez, ex, ey, ez);
        const bool in = (e != myslot) && (d2 < H2);
        const float q = 1.0f - approx_sqrt(d2) * invH;
        const float qq = in ? q * q : 0.0f;
        rho = rho + qq;
        rhoNear = rhoNear + qq * q;
        kp = e != myslot && d2 < R2;
        if (kp && check) {
          const int a = (int)k / 9 - 1, b = ((int)k / 3) % 3 - 1, cc = (int)k % 3 - 1;
          kp = vl_in_cell(pj, inv, cx + a, cy + b, cz + cc);
        }
      }
      place(kp, e);
    }
    __syncwarp();
  }
  if (__any_sync(FULL, extra[0] || extra[1])) {
    // the cells past the 27 as one sequence (offsets by a warp scan) in the
    // warp's spare walk-table rows, read as flat arrays
    uint32_t* xb = &s_walk_base[g + 1][0];  // 7 rows x 28 >= 65 entries
    uint32_t* xo = &s_walk_off[g + 1][0];
    uint32_t run = 0;
#pragma unroll
    for (int half = 0; half < 2; half++) {
      const int k = lane + 32 * half;
      uint32_t x = n[half];  // inclusive scan over the warp
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL, x, d);
        if (lane >= d) x += y;
      }
      const uint32_t off = run + x - n[half];
      run += __shfl_sync(FULL, x, 31);
      xb[k] = s0[half] - off;
      xo[k] = off;
    }
    if (lane == 0) xo[64] = run;
    __syncwarp();
    uint32_t k = 0, next = xo[1], base = xb[0];
    for (uint32_t c0 = 0; c0 < run; c0 += 32) {
      const uint32_t c = c0 + (uint32_t)lane;
      bool kp = false;
      uint32_t e = 0;
      if (c < run) {
        while (c >= next) {
          k++;
          next = xo[k + 1];
          base = xb[k];
        }
        e = base + c;
        const float4 pj = spos[e];
        const float ex = pj.x - pi.x, ey = pj.y - pi.y, ez = pj.z - pi.z;
        kp = dot3(ex, ey, ez, ex, ey, ez) < R2;
        if (kp && check) {
          const int a = lox + (int)k / (ny * nz), b = loy + ((int)k / nz) % ny, cc = loz + (int)k % nz;
          kp = vl_in_cell(pj, inv, cx + (double)a, cy + (double)b, cz + (double)cc);
        }
      }
      place(kp, e);
    }
    __syncwarp();
  }
  rho = lane_sum<32>(rho);
  rhoNear = lane_sum<32>(rhoNear);
  if (lane == 0) {
    const uint32_t pf = v.pfl[i];
    const float2 d = make_float2(rho, rhoNear);
    v.density[i] = d;
    v.sdens[myslot] = d;
    v.edens[r] = d;
    v.ncount[r] = lcount;  // may exceed NLT: then the list is not used
    v.xlist[r] = pi;
    v.epos[r] = pi;
    const bool ok = lcount <= NLT;
    const uint32_t npf = ok ? (pf | PF_LOK) : (pf & ~PF_LOK);
    v.pfl[i] = npf;
    // the fresh list holds exactly this substep's pairs when complete and no
    // two of the 27 buckets coincide: the displacement pass reads it
    const uint32_t rpf = (npf & (PF_DUP | PF_LOK)) | ((ok && !(pf & PF_DUP)) ? PF_LIST : 0u);
    v.erec[r] = make_uint4(i, myslot, v.cell[i], rpf);
  }
  __syncwarp();  // the walk tables are reused by the next rank
}

// fluidDensity (src/gpu/wgsl.js:254-279) at a rebuild substep: sets the rank
// order to this substep's grid order and writes the lists (the list kernel
// below has nothing to do then); returns at once on other substeps. Tile vb
// covers ranks vb * blockDim.x / GLF onwards, each warp 32 / GLF of them in
// turn, each with all 32 lanes.
__device__ __forceinline__ void b_density_rebuild_vl(const SimView& v, const DevParams* __restrict__ P,
                                                     uint32_t vb) {
  if (v.scratch[SCR_REBUILD] == 0u) return;  // one value for the whole scene
  if (vb == 0 && threadIdx.x == 0) v.scratch[SCR_DIRTY] = 0u;
  const int lane = threadIdx.x & 31;
  const int g = (int)(threadIdx.x >> 5) * (32 / GLF);  // this warp's first walk-table row
  const uint32_t r0 = (UPBD_VTID >> 5) * (32 / GLF);
  for (int k = 0; k < 32 / GLF; k++) vl_rebuild_one(v, P, r0 + (uint32_t)k, lane, g);
}

// fluidDensity (src/gpu/wgsl.js:254-279) on the substeps without a rebuild:
// each group reads its list when the movement test allows and walks the 27
// buckets otherwise (every group walks when lists are off).
__device__ __forceinline__ void b_density_vl(const SimView& v, const DevParams* __restrict__ P, uint32_t vb) {
  const unsigned FULL = 0xffffffffu;
  if (v.scratch[SCR_REBUILD] != 0u) return;  // the rebuild kernel did this substep's density
  const uint32_t t = UPBD_VTID;
  const int lane = threadIdx.x & (GLF - 1);
  const uint32_t r = t / GLF;  // this group's rank (or slot, lists off)
  const bool slots = !P->use_lists;
  uint32_t i, myslot, h = 0, pf = 0;
  bool act;
  if (slots) {
    vl_group(v, r, true, i, myslot, act);
  } else {
    const uint4 rc = (r < (uint32_t)v.N) ? v.erec[r] : make_uint4(NO_RANK, 0u, 0u, 0u);
    i = rc.x; myslot = rc.y; h = rc.z; pf = rc.w;
    act = i != NO_RANK && i >= (uint32_t)v.S && r < (uint32_t)v.N && v.ep[r] == i;
  }
  if (!__any_sync(FULL, act)) return;
  const float4 pi = act ? (slots ? v.spos[myslot] : v.epos[r]) : make_float4(0.f, 0.f, 0.f, 0.f);
  const float H = P->fluid_h, H2 = H * H, invH = 1.0f / H;
  const float allow = vl_allowance(P), rec = VMOVE_REC * allow;
  const bool cand = act && !slots && (pf & (PF_LOK | PF_DUP)) == PF_LOK;
  const float mv = cand ? vl_dist(pi, v.xlist[r]) : 0.f;
  const bool quick = cand && mv + fmaxf(rec, __uint_as_float(v.scratch[SCR_XMOVE])) <= allow &&
                     v.bfast[h] == 0u;
  const bool need = cand && !quick && mv + rec <= allow;
  bool listed = quick;
  CellHash ch;
  if (__any_sync(FULL, act && !quick)) {
    group_cell_hash<GLF>(pi.x, pi.y, pi.z, P->inv_cell, ch);
    const uint32_t bm = vl_bucket_move(v, ch, need, lane);
    listed = quick || (need && mv + fmaxf(rec, __uint_as_float(bm)) <= allow);
  }
  const bool walks = act && !listed;
  float rho = 0.f, rhoNear = 0.f;
  {
    struct St {
      float4 p;
      uint32_t slot;
    };
    const float4* __restrict__ spos = v.spos;
    VAcc<2> wsum = {{0.f, 0.f}};
    vl_walk(v, ch, lane, walks, St{pi, myslot}, [&](uint32_t e) { return spos[e]; },
            [&](const St& s, uint32_t e, const float4& pj) {
              const float ex = pj.x - s.p.x, ey = pj.y - s.p.y, ez = pj.z - s.p.z;
              const float d2 = dot3(ex, ey, ez, ex, ey, ez);
              const bool in = (e != s.slot) && (d2 < H2);
              const float q = 1.0f - approx_sqrt(d2) * invH;
              const float qq = in ? q * q : 0.0f;
              return VAcc<2>{{qq, qq * q}};
            },
            wsum);
    rho = rho + wsum.v[0];
    rhoNear = rhoNear + wsum.v[1];
  }
  if (listed) vl_density_list(v, r, lane, pi, H2, invH, rho, rhoNear);
  rho = lane_sum<GLF>(rho);
  rhoNear = lane_sum<GLF>(rhoNear);
  // a particle whose buckets coincide walks whatever the lists hold: it does
  // not count towards a rebuild
  if (!slots) vl_count_walkers(v, walks && !(pf & PF_DUP), lane);
  if (act && lane == 0) {
    const float2 d = make_float2(rho, rhoNear);
    v.density[i] = d;
    v.sdens[myslot] = d;
    if (!slots) {
      v.edens[r] = d;
      v.erec[r].w = listed ? (pf | PF_LIST) : (pf & ~PF_LIST);
    }
  }
}

// fluidDisp (src/gpu/wgsl.js:281-316) over the same pairs as the density
// pass; with APPLY also applyDeltaFluid (src/gpu/wgsl.js:318-323) into the
// particle's slot copy sfp (pos[i] is left for the bounds pass to write).
template <bool APPLY>
__device__ __forceinline__ void b_disp_vl(const SimView& v, const DevParams* __restrict__ P, uint32_t vb) {
  const unsigned FULL = 0xffffffffu;
  const uint32_t t = UPBD_VTID;
  const int lane = threadIdx.x & (GLF - 1);
  const uint32_t r = t / GLF;
  const bool slots = !P->use_lists;
  uint32_t i, myslot, pf = 0;
  bool act;
  if (slots) {
    vl_group(v, r, true, i, myslot, act);
  } else {
    const uint4 rc = (r < (uint32_t)v.N) ? v.erec[r] : make_uint4(NO_RANK, 0u, 0u, 0u);
    i = rc.x; myslot = rc.y; pf = rc.w;
    act = i != NO_RANK && i >= (uint32_t)v.S && r < (uint32_t)v.N && v.ep[r] == i;
  }
  if (!__any_sync(FULL, act)) return;
  const bool listed = act && (pf & PF_LIST);
  const bool walks = act && !listed;
  const float H = P->fluid_h, H2 = H * H, invH = 1.0f / H;
  const float4 pi = act ? (slots ? v.spos[myslot] : v.epos[r]) : make_float4(0.f, 0.f, 0.f, 0.f);
  const float2 di = act ? (slots ? v.sdens[myslot] : v.edens[r]) : make_float2(0.f, 0.f);
  const float maxPair = 0.05f * H;
  const float k = P->stiffness, kn = P->near_stiffness, rho0 = P->rest_density;
  const float Pi = k * (di.x - rho0);
  const float PNi = kn * di.y;
  float sx = 0.f, sy = 0.f, sz = 0.f;
  auto pair = [&](const float4& pj, const float2& dj) {
    const float ex = pj.x - pi.x, ey = pj.y - pi.y, ez = pj.z - pi.z;
    const float d2 = dot3(ex, ey, ez, ex, ey, ez);
    if (d2 >= H2 || d2 < 1e-12f) return;
    const float rd = rsqrtf(d2);
    const float q = 1.0f - d2 * rd * invH;
    const float Pj = k * (dj.x - rho0);
    const float PNj = kn * dj.y;
    float D = 0.25f * ((Pi + Pj) * q + (PNi + PNj) * q * q);
    D = clampf(D, -maxPair, maxPair);
    const float f = D * rd;
    sx = sx - ex * f; sy = sy - ey * f; sz = sz - ez * f;
  };
  if (__any_sync(FULL, walks)) {
    CellHash ch;
    group_cell_hash<GLF>(pi.x, pi.y, pi.z, P->inv_cell, ch);
    struct PD {
      float4 p;
      float2 d;
    };
    struct St {
      float4 p;
      uint32_t slot;
      float Pi, PNi;
    };
    const float4* __restrict__ spos = v.spos;
    const float2* __restrict__ sdens = v.sdens;
    VAcc<3> wsum = {{0.f, 0.f, 0.f}};
    vl_walk(v, ch, lane, walks, St{pi, myslot, Pi, PNi}, [&](uint32_t e) { return PD{spos[e], sdens[e]}; },
            [&](const St& s, uint32_t e, const PD& c) {
              VAcc<3> t = {{0.f, 0.f, 0.f}};
              const float ex = c.p.x - s.p.x, ey = c.p.y - s.p.y, ez = c.p.z - s.p.z;
              const float d2 = dot3(ex, ey, ez, ex, ey, ez);
              if (e == s.slot || d2 >= H2 || d2 < 1e-12f) return t;
              const float rd = rsqrtf(d2);
              const float q = 1.0f - d2 * rd * invH;
              const float Pj = k * (c.d.x - rho0);
              const float PNj = kn * c.d.y;
              float D = 0.25f * ((s.Pi + Pj) * q + (s.PNi + PNj) * q * q);
              D = clampf(D, -maxPair, maxPair);
              const float f = D * rd;
              t.v[0] = -ex * f; t.v[1] = -ey * f; t.v[2] = -ez * f;
              return t;
            },
            wsum);
    sx = sx + wsum.v[0]; sy = sy + wsum.v[1]; sz = sz + wsum.v[2];
  }
  if (listed) {  // lane l reads entries l, l + GLF, ...
    const uint32_t NS = (uint32_t)v.N;
    const uint32_t n = v.ncount[r];
    const uint32_t* __restrict__ lst = v.nbr + r;
    const float4* __restrict__ epos = v.epos;
    const float2* __restrict__ edens = v.edens;
    for (uint32_t c = (uint32_t)lane; c < n; c += VLF * GLF) {  // VLF entries' loads in flight
      uint32_t j[VLF];
#pragma unroll
      for (int w = 0; w < VLF; w++) {
        const uint32_t cw = c + (uint32_t)(w * GLF);
        j[w] = (cw < n) ? __ldg(&lst[(size_t)cw * NS]) : NO_RANK;
      }
      float4 pj[VLF];
      float2 dj[VLF];
#pragma unroll
      for (int w = 0; w < VLF; w++) {
        const uint32_t jj = (j[w] != NO_RANK) ? j[w] : j[0];
        pj[w] = epos[jj];
        dj[w] = edens[jj];
      }
#pragma unroll
      for (int w = 0; w < VLF; w++)
        if (j[w] != NO_RANK) pair(pj[w], dj[w]);
    }
  }
#pragma unroll
  for (int d = 1; d < GLF; d <<= 1) {
    sx = sx + __shfl_xor_sync(FULL, sx, d);
    sy = sy + __shfl_xor_sync(FULL, sy, d);
    sz = sz + __shfl_xor_sync(FULL, sz, d);
  }
  if (!act || lane != 0) return;
  const float maxTotal = 0.35f * H;
  const float s2 = dot3(sx, sy, sz, sx, sy, sz);
  if (s2 > maxTotal * maxTotal) {
    const float f = maxTotal / sqrtf(s2);
    sx = sx * f; sy = sy * f; sz = sz * f;
  }
  if (APPLY)
    v.sfp[myslot] = make_float4(pi.x + sx, pi.y + sy, pi.z + sz, pi.w);
  else
    v.delta[i] = make_float4(sx, sy, sz, 1.0f);
}

// Particle j's grid-time bucket is one of the 27 around the cell of p.
static __device__ __noinline__ bool vl_member(const SimView& v, const DevParams* __restrict__ P, const float4& p,
                                              uint32_t j) {
  CellHash ch;
  ch.init(p.x, p.y, p.z, P->inv_cell);
  const uint32_t mask = (uint32_t)v.T - 1u, h = v.cell[j];
  bool hit = false;
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++)
#pragma unroll
      for (int c = 0; c < 3; c++) hit |= (ch.bucket(a, b, c, mask) == h);
  return hit;
}

// xsph (src/gpu/wgsl.js:745-771) at the final positions; with APPLY the
// blended velocity goes to vel[i] (xsphApply, src/gpu/wgsl.js:773-778), the
// neighbours' velocities being read from the copies the velocity pass wrote
// (svel by slot for walks, evel by rank for lists).
template <bool APPLY>
__device__ __forceinline__ void b_xsph_vl(const SimView& v, const DevParams* __restrict__ P, uint32_t vb) {
  const unsigned FULL = 0xffffffffu;
  const uint32_t t = UPBD_VTID;
  const int lane = threadIdx.x & (GLF - 1);
  const uint32_t r = t / GLF;
  const bool slots = !P->use_lists;
  uint32_t i, myslot, h = 0, pf = 0;
  bool act;
  if (slots) {
    bool fluid;
    vl_group(v, r, true, i, myslot, fluid);
    act = fluid && (v.flags[i] & F_ACTIVE);
  } else {
    const uint4 rc = (r < (uint32_t)v.N) ? v.erec[r] : make_uint4(NO_RANK, 0u, 0u, 0u);
    i = rc.x; myslot = rc.y; h = rc.z; pf = rc.w;
    // culled by this substep's bounds pass: no xsph of its own
    act = i != NO_RANK && i >= (uint32_t)v.S && r < (uint32_t)v.N && v.ep[r] == i && !(pf & PF_CULLED);
  }
  if (!__any_sync(FULL, act)) return;
  // the bounds pass wrote the final position to both copies
  const float4 pi = act ? (slots ? v.spos[myslot] : v.epos[r]) : make_float4(0.f, 0.f, 0.f, 0.f);
  const float H = P->fluid_h, H2 = H * H;
  const float allow = vl_allowance(P), rec = VMOVE_REC * allow;
  const float mv = (act && !slots) ? v.smove[r] : 0.f;
  const bool cand = act && !slots && (pf & (PF_LOK | PF_DUPF)) == PF_LOK && mv + rec <= allow;
  // a particle that kept its cell reads its grid bucket's fast mark; one that
  // changed cell takes the per-bucket test
  const bool quick = cand && !(pf & PF_MOVED) && v.bfast[h] == 0u &&
                     mv + fmaxf(rec, __uint_as_float(v.scratch[SCR_XMOVE])) <= allow;
  const bool need = cand && !quick;
  bool listed = quick;
  CellHash ch;
  if (__any_sync(FULL, act && !quick)) {
    group_cell_hash<GLF>(pi.x, pi.y, pi.z, P->inv_cell, ch);
    const uint32_t bm = vl_bucket_move(v, ch, need, lane);
    listed = quick || (need && mv + fmaxf(rec, __uint_as_float(bm)) <= allow);
  }
  const bool walks = act && !listed;
  float sx = 0.f, sy = 0.f, sz = 0.f, m = 0.f;
  if (__any_sync(FULL, walks)) {
    struct PV {
      float4 p, v;
    };
    struct St {
      float4 p;
      uint32_t slot;
    };
    const float4* __restrict__ spos = v.spos;
    const float4* __restrict__ svel = v.svel;
    VAcc<4> wsum = {{0.f, 0.f, 0.f, 0.f}};
    vl_walk(v, ch, lane, walks, St{pi, myslot}, [&](uint32_t e) { return PV{spos[e], svel[e]}; },
            [&](const St& s, uint32_t e, const PV& c) {
              const float ex = c.p.x - s.p.x, ey = c.p.y - s.p.y, ez = c.p.z - s.p.z;
              const bool in = (e != s.slot) && (dot3(ex, ey, ez, ex, ey, ez) < H2);
              return VAcc<4>{{in ? c.v.x : 0.f, in ? c.v.y : 0.f, in ? c.v.z : 0.f, in ? 1.0f : 0.f}};
            },
            wsum);
    sx = sx + wsum.v[0]; sy = sy + wsum.v[1]; sz = sz + wsum.v[2]; m = m + wsum.v[3];
  }
  if (listed) {  // lane l reads entries l, l + GLF, ...
    const uint32_t NS = (uint32_t)v.N;
    const uint32_t n = v.ncount[r];
    const uint32_t* __restrict__ lst = v.nbr + r;
    const float4* __restrict__ epos = v.epos;
    const float4* __restrict__ evel = v.evel;
    for (uint32_t c = (uint32_t)lane; c < n; c += VLF * GLF) {  // VLF entries' loads in flight
      uint32_t j[VLF];
#pragma unroll
      for (int w = 0; w < VLF; w++) {
        const uint32_t cw = c + (uint32_t)(w * GLF);
        j[w] = (cw < n) ? __ldg(&lst[(size_t)cw * NS]) : NO_RANK;
      }
      float4 pj[VLF], uj[VLF];
#pragma unroll
      for (int w = 0; w < VLF; w++) {
        const uint32_t jj = (j[w] != NO_RANK) ? j[w] : j[0];
        pj[w] = epos[jj];
        uj[w] = evel[jj];
      }
#pragma unroll
      for (int w = 0; w < VLF; w++) {
        const float ex = pj[w].x - pi.x, ey = pj[w].y - pi.y, ez = pj[w].z - pi.z;
        bool in = j[w] != NO_RANK && dot3(ex, ey, ez, ex, ey, ez) < H2;
        // a neighbour that changed cell after the grid build counts when its
        // grid bucket is one of this particle's 27
        if (in && uj[w].w != 0.f) in = vl_member(v, P, pi, v.ep[j[w]]);
        sx = sx + (in ? uj[w].x : 0.f); sy = sy + (in ? uj[w].y : 0.f); sz = sz + (in ? uj[w].z : 0.f);
        m = m + (in ? 1.0f : 0.f);
      }
    }
  }
  sx = lane_sum<GLF>(sx);
  sy = lane_sum<GLF>(sy);
  sz = lane_sum<GLF>(sz);
  m = lane_sum<GLF>(m);
  if (!slots) vl_count_walkers(v, walks && !(pf & PF_DUPF), lane);
  if (act && lane == 0) {
    const float4 vi = slots ? v.vel[i] : v.evel[r];  // the velocity pass's result either way
    float vx = vi.x, vy = vi.y, vz = vi.z;
    if (m > 0.f) {
      const float mu = P->viscosity;
      vx = vx + mu * (sx / m - vx);
      vy = vy + mu * (sy / m - vy);
      vz = vz + mu * (sz / m - vz);
    }
    if (APPLY)
      v.vel[i] = make_float4(vx, vy, vz, 0.f);
    else
      v.delta[i] = make_float4(vx, vy, vz, m);
  }
}

}  // namespace upbd
