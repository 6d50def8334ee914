// Device-side types and helpers of the unified-particle step (sm_100a).
//
// State layout in HBM (structure of arrays, 16-byte aligned rows, the field
// meanings of src/gpu/wgsl.js:92-98; float4/float2 rows are `real` rows, which
// are double4/double2 in the test-only FP64 build):
//   pos[N]     float4  xyz + inverse mass
//   prev[N]    float4  xyz + grab target x
//   vel[N]     float4  xyz + grab target y
//   density[N] float2  (rho, rho_near) or (grab target z, grip weight)
//   delta[N]   float4  per-pass private correction (xyz + count)
//   flags[N]   uint32  bit0 ACTIVE, bit1 GRABBED
//   cons[C]    uint4   {a, b, rest float bits, alive}
//   adj        uint32  [S+1 offsets][2C constraint ids]  (static CSR)
// Hash grid (rebuilt every substep):
//   counts[T], start[T+1], entries[N], tmp[N], ticket[N], cell[N], tile_sum
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "upbd_grid_layout.h"

namespace upbd {

constexpr uint32_t F_ACTIVE = 1u;
constexpr uint32_t F_GRABBED = 2u;
constexpr uint32_t C_K = 40u;           // solid contact cache width, src/gpu/wgsl.js:25
constexpr int SCAN_THREADS = 256;       // 8 counts per thread (SCAN_TILE / 8)

// scratch words (device)
constexpr int SCR_PICK_T = 0;      // uint64 bits of the best t (words 0-1)
constexpr int SCR_PICK_I = 2;      // best index
constexpr int SCR_CUT = 3;         // constraints cut by the last wedge
constexpr int SCR_ACTIVE = 4;      // active-fluid partial sums
constexpr int SCR_DONE = 5;        // blocks finished (last-block pattern)
constexpr int SCR_HEALTH = 6;      // UPBD_HEALTH_* bits
constexpr int SCR_XMOVE = 7;       // largest movement the bounds pass recorded this substep (float bits)
constexpr int SCR_WORDS = 16;
// mapped host words
constexpr int HM_ACTIVE = 0;
constexpr int HM_HEALTH = 1;
constexpr int HM_WORDS = 8;

// Scalar type of the particle state and of the pass arithmetic: float in
// the product and parity builds (the reference's f32 buffers); double in the
// test-only FP64 build (UPBD_FP64_BUILD), which instantiates these same pass
// bodies on double as the reference trajectory for long-run drift. The
// uniforms, the constraint rest lengths (float bits in cons.z, the buffer
// layout of the reference), tet rest volumes and the movement bounds stay
// float in every build.
#ifdef UPBD_FP64_BUILD
using real = double;
using real2 = double2;
using real4 = double4;
__host__ __device__ __forceinline__ real4 make_real4(real x, real y, real z, real w) { return make_double4(x, y, z, w); }
__host__ __device__ __forceinline__ real2 make_real2(real x, real y) { return make_double2(x, y); }
#else
using real = float;
using real2 = float2;
using real4 = float4;
__host__ __device__ __forceinline__ real4 make_real4(real x, real y, real z, real w) { return make_float4(x, y, z, w); }
__host__ __device__ __forceinline__ real2 make_real2(real x, real y) { return make_float2(x, y); }
#endif
// Math on the scalar type: the float overloads call exactly what the FP32
// builds always called.
__device__ __forceinline__ float r_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double r_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float r_rsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double r_rsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float r_fabs(float x) { return fabsf(x); }
__device__ __forceinline__ double r_fabs(double x) { return fabs(x); }
__device__ __forceinline__ float r_fmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double r_fmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float r_fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double r_fdiv(double a, double b) { return a / b; }
// a float no smaller than x (movement bounds kept as float bits); x >= 0
__device__ __forceinline__ float r_to_float_up(float x) { return x; }
__device__ __forceinline__ float r_to_float_up(double x) { return __double2float_ru(x); }

// Uniforms of one frame (Params of src/gpu/wgsl.js:36-90), in device memory
// so captured graphs read the values current at replay.
struct DevParams {
  float h, gravity, solid_radius, fluid_radius;
  float fluid_h, rest_density, stiffness, near_stiffness;
  float viscosity, compliance, omega, plastic_threshold;
  float plastic_rate, tear_gap, max_speed, wall_x;
  float wall_z, wall_h, wall_t, cull_r;
  float damp_solid, damp_fluid, friction_solid, friction_fluid;
  float grab_k, spacing, solid_viscosity, break_strain;
  float contact_scale, pad0, pad1, pad2;
  double inv_cell;
  int32_t tear_mode, plastic_clamp;
  // 1 when solid_radius + fluid_radius is below the cell size: every
  // solid↔fluid contact then lies in adjacent cells, so the solids can mark
  // the fluid particles that have one and the rest skip their gather.
  int32_t use_mark, pad4;
  float4 grab_delta;  // per-substep share of the frame's grab motion
  uint32_t emit_count, emit_start, grab_lattice, pad3;
  float4 emit_pos, emit_dir, emit_side, emit_up;
  float4 grab_c;
  double cut_o[4], cut_d1[4], cut_d2[4];
  double pick_o[4], pick_d[4];  // pick_o[3] = max perpendicular distance
};

// Device pointers and sizes of one scene (passed by value to kernels).
struct SimView {
  real4* pos;
  real4* prev;
  real4* vel;
  real4* delta;
  real2* density;
  uint32_t* flags;
  uint4* cons;
  const uint32_t* adj;
  uint32_t* counts;
  uint32_t* start;
  uint32_t* entries;
  uint32_t* tmp;
  uint32_t* ticket;
  uint32_t* cell;
  uint32_t* tile_sum;
  uint32_t* tet_idx;   // 4 per tet
  float* tet_vol;      // rest volume, negative = dead
  const uint32_t* tet_adj;  // [S+1 offsets][4NT ids]
  // Bucket-ordered copies, slot e matching entries[e]: neighbour gathers read
  // a candidate's data with one load at its slot instead of entries -> pos.
  // Every pass that moves a particle also writes its slot's copy.
  real4* spos;         // position + inverse mass
  real2* sdens;        // (rho, rho_near) of the density pass
  real4* svel;         // velocity after velocityUpdate
  uint32_t* slot;      // slot of particle i in this substep's grid
  // Inside a bucket, entries run in descending index, so fluid (indices >= S)
  // precede solids: fend[h] splits bucket h into [start[h], fend[h]) fluid and
  // [fend[h], start[h+1]) solid.
  uint32_t* fend;
  // Density-pass neighbour lists: lane l (of GLF) of the fluid particle at
  // slot e records the slots of its fluid candidates within the list radius
  // H * (1 + XSKIN), in its walk order, at nbr[(l*NL + c) * N + e] (c < NL),
  // those within H flagged with NBR_IN, and their number in ncount[l*N + e].
  uint32_t* nbr;
  uint32_t* ncount;
  // Movement between the density pass and xsph (written by the bounds pass):
  // smove[e] for the fluid particle at slot e (+inf when it left its cell),
  // bmove[h] the largest movement above XMOVE_REC * the allowance among the
  // particles of bucket h (float bits; cleared by the scan).
  float* smove;
  uint32_t* bmove;
  const uint32_t* adj_other;  // CSR-parallel: the other endpoint of constraint ids[k]
  const float* adj_scale;     // CSR-parallel: 1 / max(deg_i, deg_other) (static)
  uint32_t* mark;      // per particle: a solid is within contact range (fluid only)
  real4* sbuf;         // 2 x S: solid positions between folded solve iterations
  // Slot-ordered fluid positions after applyDeltaFluid: the contact passes
  // (marks, solid-fluid contacts) read the fluid there, while spos keeps the
  // positions the fluid gathers saw until the bounds pass rewrites it.
  real4* sfp;
  uint32_t* ccount;
  uint32_t* clist;
  uint32_t* scratch;
  uint32_t* host_mapped;
#ifdef UPBD_FP64_BUILD
  float* conv;  // N x 4 floats: host rows staged on their way to or from the double state
#endif
  int S, N1, dim1, dim2, F, N, C, NT, T, num_tiles;
};

// ---------------------------------------------------------------------------
// ECMAScript ToInt32 of an integer-valued double (the operands of `^` in
// Solver._hash, src/solver.js:162-164). Values below 2^63 in magnitude convert
// exactly through int64; larger finite values reduce mod 2^32 with fmod.
__device__ __forceinline__ int32_t js_toint32(double x) {
  if (!isfinite(x)) return 0;
  if (fabs(x) < 9.0e18) return (int32_t)(uint32_t)(unsigned long long)(long long)x;
  double m = fmod(trunc(x), 4294967296.0);
  if (m < 0) m += 4294967296.0;
  if (m >= 2147483648.0) m -= 4294967296.0;
  return (int32_t)m;
}

// Bucket hashes of the 27 cells around a position: Solver._hashPos /
// Solver._hash (src/solver.js:162-172) — floor(p * (1/cellSize)) in double,
// products in double, ToInt32, xor, mask.
struct CellHash {
  int32_t hx[3], hy[3], hz[3];
  __device__ __forceinline__ void init(real px, real py, real pz, double inv) {
    const double cx = floor(__dmul_rn((double)px, inv));
    const double cy = floor(__dmul_rn((double)py, inv));
    const double cz = floor(__dmul_rn((double)pz, inv));
#pragma unroll
    for (int d = 0; d < 3; d++) {
      hx[d] = js_toint32(__dmul_rn(__dadd_rn(cx, (double)(d - 1)), 92837111.0));
      hy[d] = js_toint32(__dmul_rn(__dadd_rn(cy, (double)(d - 1)), 689287499.0));
      hz[d] = js_toint32(__dmul_rn(__dadd_rn(cz, (double)(d - 1)), 283923481.0));
    }
  }
  __device__ __forceinline__ uint32_t bucket(int a, int b, int c, uint32_t mask) const {
    return (uint32_t)(hx[a] ^ hy[b] ^ hz[c]) & mask;
  }
  // Bucket of neighbour cell k = (dx+1)*9 + (dy+1)*3 + (dz+1) with a runtime
  // k: selects keep the nine hashes in registers.
  __device__ __forceinline__ uint32_t bucket_k(int k, uint32_t mask) const {
    const int a = k / 9, r = k - 9 * a, b = r / 3, c = r - 3 * b;
    const int32_t X = (a == 0) ? hx[0] : ((a == 1) ? hx[1] : hx[2]);
    const int32_t Y = (b == 0) ? hy[0] : ((b == 1) ? hy[1] : hy[2]);
    const int32_t Z = (c == 0) ? hz[0] : ((c == 1) ? hz[1] : hz[2]);
    return (uint32_t)(X ^ Y ^ Z) & mask;
  }
};

// Index guard of the checked build (UPBD_CHECKED_BUILD, libupbd_checked.so):
// the indices the gathers read from device arrays (bucket members, list
// entries, CSR constraint ids and other endpoints, bucket slots, tet
// corners, contact-cache entries) are tested against their array's extent
// before use; an index out of range sets UPBD_HEALTH_BOUNDS in the scene's
// health word (upbd_health, upbd_sync) and its access is skipped instead of
// faulting. In the product and parity builds the guard is the constant true
// and generates no code.
#ifdef UPBD_CHECKED_BUILD
__device__ __forceinline__ bool idx_ok(uint32_t* scratch, uint64_t idx, uint64_t n) {
  if (idx < n) return true;
  if (scratch) atomicOr(&scratch[SCR_HEALTH], 8u);  // UPBD_HEALTH_BOUNDS (the stateless grid build has none)
  return false;
}
#define UPBD_IDX_OK(v, idx, n) (::upbd::idx_ok((v).scratch, (uint64_t)(idx), (uint64_t)(n)))
#else
#define UPBD_IDX_OK(v, idx, n) (true)
#endif

// Neighbour gathers run G lanes per particle (lane_strided below deals the
// candidates to the lanes); each lane accumulates its own partial sums from
// zero and the G partials are combined by a fixed xor butterfly, so the
// result is deterministic: for G = 8 ((p0+p4)+(p2+p6)) + ((p1+p5)+(p3+p7)),
// for G = 4 (p0+p2) + (p1+p3). The contact gathers and the solid solve use
// GL = 8 lanes; the fluid-fluid gathers (density, xsph) GLF = 4: each lane
// walks the whole 27-cell sequence, so fewer lanes per particle cross fewer
// cell boundaries in all.
constexpr int GL = 8;
constexpr int GLF = 4;
constexpr uint32_t NL = 32;  // density-pass neighbour-list entries kept per fluid lane (GLF * NL per particle)
constexpr int DL = 2;        // threads per particle in the displacement pass

// xsph sums over the fluid candidates within H at its own time, after the
// displacement, contact and bounds passes moved the fluid. The density pass
// lists every candidate within H * (1 + XSKIN), so when the particle kept its
// cell (the same 27 buckets, the same candidate sequence) and it and every
// particle of those buckets moved by at most `allowance` = XSKIN * H *
// XMOVE_FRAC in total, every candidate within H at xsph time is on its lanes'
// lists, in walk order: xsph reads the lists instead of walking the buckets,
// and the sums are the walk's sums bit for bit (each lane's skipped candidates
// would add +0 to sums that start at +0). The rest of the allowance (1 -
// XMOVE_FRAC) covers the rounding of the distance tests. Movements at or
// below XMOVE_REC * allowance are not recorded per bucket: a bucket counts
// them as that much.
constexpr float XSKIN = 0.05f;
constexpr float XMOVE_FRAC = 0.9f;
constexpr float XMOVE_REC = 0.25f;
constexpr uint32_t NBR_IN = 0x80000000u;  // list entry flag: within H at density time (slots stay below 2^31)

template <int G = GL>
__device__ __forceinline__ real lane_sum(real x) {
#pragma unroll
  for (int d = G / 2; d > 0; d >>= 1) x = x + __shfl_xor_sync(0xffffffffu, x, d);
  return x;
}

// The nine hash components of the cells around p (CellHash::init's values),
// component j computed by lane j mod G of a G-lane group and exchanged by
// shuffles. Every lane of the warp must call it (inactive groups pass any
// position).
template <int G = GL>
__device__ __forceinline__ void group_cell_hash(real px, real py, real pz, double inv, CellHash& ch) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & (G - 1);
  const int base = (threadIdx.x & 31) & ~(G - 1);
  // component j: axis j / 3 (x, y, z), cell offset j % 3 - 1
  int32_t mine[(9 + G - 1) / G];
#pragma unroll
  for (int m = 0; m < (9 + G - 1) / G; m++) {
    const int j = lane + G * m;
    const int axis = (j < 9) ? j / 3 : 2;
    const real pa = (axis == 0) ? px : ((axis == 1) ? py : pz);
    const double K = (axis == 0) ? 92837111.0 : ((axis == 1) ? 689287499.0 : 283923481.0);
    const double c = floor(__dmul_rn((double)pa, inv));
    mine[m] = js_toint32(__dmul_rn(__dadd_rn(c, (double)(j - 3 * axis - 1)), K));
  }
  int32_t comp[9];
#pragma unroll
  for (int j = 0; j < 9; j++) comp[j] = __shfl_sync(FULL, mine[j / G], base + (j % G));
#pragma unroll
  for (int d = 0; d < 3; d++) {
    ch.hx[d] = comp[d];
    ch.hy[d] = comp[3 + d];
    ch.hz[d] = comp[6 + d];
  }
}

// Walk the candidates of the 27 neighbour buckets as ONE sequence: cells in
// the reference's order k = (dx+1)*9 + (dy+1)*3 + (dz+1), each bucket's PART
// entries in bucket order (PART 0: its fluid entries, PART 1: its solids);
// lane l of the G group takes candidates c = l, l+G, l+2G, ... so the
// lanes' shares differ by at most one. For each slot e of its share, in
// order, a lane calls use(e, load(e)); with U > 1 it issues the loads of U
// slots before their uses. The bucket ranges are looked up by
// their round-robin lanes (cell k by lane k mod G), scanned into sequence
// offsets by shuffles, and handed over in shared memory. Every lane of the
// warp must call it; a group with `walk` false has an empty sequence. At most
// 256 threads per block.
static __shared__ uint32_t s_walk_base[256 / GLF][28];  // slot of candidate 0 of cell k, minus its offset
static __shared__ uint32_t s_walk_off[256 / GLF][28];   // sequence offset of cell k ([27] = total)

// The shared tables of a walk: row g (this lane's group) gets the slot base
// and sequence offset of each of the 27 cells; returns the sequence length.
template <int PART, int G>
__device__ __forceinline__ uint32_t walk_tables(const SimView& v, const CellHash& ch, int lane, bool walk, int g) {
  auto& s_base = s_walk_base;  // shared by every instantiation
  auto& s_off = s_walk_off;
  const unsigned FULL = 0xffffffffu;
  const uint32_t mask = (uint32_t)v.T - 1u;
  uint32_t run = 0;
#pragma unroll
  for (int m = 0; m < (27 + G - 1) / G; m++) {
    const int k = lane + G * m;
    uint32_t s = 0, n = 0;
    if (walk && k < 27) {
      const uint32_t hb = ch.bucket_k(k, mask);
      const uint32_t f = __ldg(&v.fend[hb]);
      if (PART == 0) {
        s = __ldg(&v.start[hb]);
        n = f - s;
      } else {
        s = f;
        n = __ldg(&v.start[hb + 1]) - f;
      }
    }
    uint32_t x = n;  // inclusive scan over the group's lanes (cell order within the round)
#pragma unroll
    for (int d = 1; d < G; d <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, x, d, G);
      if (lane >= d) x += y;
    }
    const uint32_t off = run + x - n;
    run += __shfl_sync(FULL, x, G - 1, G);
    if (k < 27) {
      s_base[g][k] = s - off;
      s_off[g][k] = off;
    }
  }
  if (lane == 0) s_off[g][27] = run;
  __syncwarp();
  return run;
}

template <int PART, int G = GL, int U = 1, class Load, class Use>
__device__ __forceinline__ void lane_strided(const SimView& v, const CellHash& ch, int lane, bool walk, Load&& load,
                                             Use&& use) {
  static_assert(G <= 32 && GLF <= G, "walk tables are sized for GLF..32 lanes");
  auto& s_base = s_walk_base;
  auto& s_off = s_walk_off;
  // each warp owns 32/GLF rows, its groups the first 32/G of them: warps of
  // one block may walk with different G (a 32-lane solid warp beside 8-lane
  // fluid warps), and rows taken as threadIdx.x / G would then overlap
  const int g = (int)(threadIdx.x >> 5) * (32 / GLF) + (int)(threadIdx.x & 31) / G;
  const uint32_t run = walk_tables<PART, G>(v, ch, lane, walk, g);
  uint32_t k = 0, next = s_off[g][1], base = s_base[g][0];
  if (U == 1) {
    // one candidate per step: where every group walks, unrolling to keep
    // several loads in flight costs more in registers (occupancy) than it
    // wins in latency on B200
    for (uint32_t c = (uint32_t)lane; c < run; c += G) {
      while (c >= next) {  // next non-empty cell (the total ends the sequence)
        k++;
        next = s_off[g][k + 1];
        base = s_base[g][k];
      }
      const uint32_t e = base + c;
      if (UPBD_IDX_OK(v, e, v.N)) use(e, load(e));
    }
  } else {
    // U candidates per step, their loads in flight together (for the few
    // groups that walk while the rest of the kernel reads lists)
    for (uint32_t c0 = (uint32_t)lane; c0 < run; c0 += G * U) {
      uint32_t e[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const uint32_t c = c0 + (uint32_t)(u * G);
        if (c < run) {
          while (c >= next) {
            k++;
            next = s_off[g][k + 1];
            base = s_base[g][k];
          }
          e[u] = base + c;
          if (!UPBD_IDX_OK(v, e[u], v.N)) e[u] = 0u;  // out of range: slot 0 instead (reported)
        } else {
          e[u] = e[0];  // c0 < run: a valid slot, loaded again and not used
        }
      }
      decltype(load(0u)) x[U];
#pragma unroll
      for (int u = 0; u < U; u++) x[u] = load(e[u]);
#pragma unroll
      for (int u = 0; u < U; u++)
        if (c0 + (uint32_t)(u * G) < run) use(e[u], x[u]);
    }
  }
  __syncwarp();  // the next call may rewrite this group's cells
}

// The same walk for warps where only a few groups walk: for each walking
// group in turn, all 32 lanes of the warp load its next 32 candidates (one
// each, all in flight together) into shared memory, and the group's lanes
// then use them in their own order (lane l: candidates l, l+G, ..., as in
// lane_strided, so the results are the same bit for bit). Every lane of the
// warp must call it; at most 256 threads per block.
template <int PART, int G, class Load, class Use>
__device__ __forceinline__ void lane_staged(const SimView& v, const CellHash& ch, int lane, bool walk, Load&& load,
                                            Use&& use) {
  static_assert(G <= 32 && GLF <= G && 32 % G == 0, "walk tables are sized for GLF..32 lanes");
  using X = decltype(load(0u));
  __shared__ X s_x[256 / 32][32];
  __shared__ uint32_t s_e[256 / 32][32];
  auto& s_base = s_walk_base;
  auto& s_off = s_walk_off;
  const int w = (int)(threadIdx.x >> 5), L = (int)(threadIdx.x & 31);
  const int g = w * (32 / GLF) + L / G;
  walk_tables<PART, G>(v, ch, lane, walk, g);
  unsigned todo = __ballot_sync(0xffffffffu, walk && lane == 0);  // one bit per walking group
  while (todo) {
    const int first = __ffs(todo) - 1;  // the group's lane 0
    todo &= todo - 1u;
    const int gw = w * (32 / GLF) + first / G;
    const bool mine = (L / G) == (first / G);
    const uint32_t run = s_off[gw][27];
    uint32_t k = 0, next = s_off[gw][1], base = s_base[gw][0];
    for (uint32_t c0 = 0; c0 < run; c0 += 32) {
      const uint32_t c = c0 + (uint32_t)L;
      if (c < run) {
        while (c >= next) {
          k++;
          next = s_off[gw][k + 1];
          base = s_base[gw][k];
        }
        uint32_t e = base + c;
        if (!UPBD_IDX_OK(v, e, v.N)) e = 0u;  // out of range: slot 0 instead (reported)
        s_e[w][L] = e;
        s_x[w][L] = load(e);
      }
      __syncwarp();
      if (mine)
        for (uint32_t j = (uint32_t)lane; j < 32u && c0 + j < run; j += G) use(s_e[w][j], s_x[w][j]);
      __syncwarp();
    }
  }
  __syncwarp();  // the next call may rewrite this warp's rows
}

// Square roots inside the gathers' candidate loops. The parity build keeps
// the correctly rounded operations of the reference's expressions (its results
// match the oracle bit for bit); the product build uses the hardware
// approximation (sqrt.approx.f32, exact at 0) and reciprocal square root, which
// stay within the stated per-substep tolerance and keep the loops short.
__device__ __forceinline__ float approx_sqrt(float x) {
  float y;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double approx_sqrt(double x) { return sqrt(x); }

__device__ __forceinline__ uint32_t cell_of(real px, real py, real pz, double inv, uint32_t mask) {
  const double cx = floor(__dmul_rn((double)px, inv));
  const double cy = floor(__dmul_rn((double)py, inv));
  const double cz = floor(__dmul_rn((double)pz, inv));
  const int32_t a = js_toint32(__dmul_rn(cx, 92837111.0));
  const int32_t b = js_toint32(__dmul_rn(cy, 689287499.0));
  const int32_t c = js_toint32(__dmul_rn(cz, 283923481.0));
  return (uint32_t)(a ^ b ^ c) & mask;
}

// std::max / std::min / clamp with the operand order of the oracle (so -0.0
// and NaN resolve the same way on both sides).
__device__ __forceinline__ real mx(real a, real b) { return (a < b) ? b : a; }
__device__ __forceinline__ real mn(real a, real b) { return (b < a) ? b : a; }
__device__ __forceinline__ real clampf(real e, real lo, real hi) { return mn(mx(e, lo), hi); }
__device__ __forceinline__ real signf(real x) { return x > 0 ? real(1) : (x < 0 ? real(-1) : real(0)); }
__device__ __forceinline__ real dot3(real ax, real ay, real az, real bx, real by, real bz) {
  return ax * bx + ay * by + az * bz;
}

}  // namespace upbd
