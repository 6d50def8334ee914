// Device-side types and helpers of the unified-particle step (sm_100a).
//
// State layout in HBM (structure of arrays, 16-byte aligned rows, the field
// meanings of src/gpu/wgsl.js:92-98):
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

namespace upbd {

constexpr uint32_t F_ACTIVE = 1u;
constexpr uint32_t F_GRABBED = 2u;
constexpr uint32_t C_K = 40u;           // solid contact cache width, src/gpu/wgsl.js:25
constexpr int SCAN_TILE = 2048;         // counts scanned per block
constexpr int SCAN_THREADS = 256;       // 8 counts per thread

// scratch words (device)
constexpr int SCR_PICK_T = 0;      // uint64 bits of the best t (words 0-1)
constexpr int SCR_PICK_I = 2;      // best index
constexpr int SCR_CUT = 3;         // constraints cut by the last wedge
constexpr int SCR_ACTIVE = 4;      // active-fluid partial sums
constexpr int SCR_DONE = 5;        // blocks finished (last-block pattern)
constexpr int SCR_HEALTH = 6;      // UPBD_HEALTH_* bits
constexpr int SCR_WORDS = 16;
// mapped host words
constexpr int HM_ACTIVE = 0;
constexpr int HM_HEALTH = 1;
constexpr int HM_WORDS = 8;

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
  float4 grab_delta;  // per-substep share of the frame's grab motion
  uint32_t emit_count, emit_start, grab_lattice, pad3;
  float4 emit_pos, emit_dir, emit_side, emit_up;
  float4 grab_c;
  double cut_o[4], cut_d1[4], cut_d2[4];
  double pick_o[4], pick_d[4];  // pick_o[3] = max perpendicular distance
};

// Device pointers and sizes of one scene (passed by value to kernels).
struct SimView {
  float4* pos;
  float4* prev;
  float4* vel;
  float4* delta;
  float2* density;
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
  uint32_t* ccount;
  uint32_t* clist;
  uint32_t* scratch;
  uint32_t* host_mapped;
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
  __device__ __forceinline__ void init(float px, float py, float pz, double inv) {
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
};

__device__ __forceinline__ uint32_t cell_of(float px, float py, float pz, double inv, uint32_t mask) {
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
__device__ __forceinline__ float mx(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float mn(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float clampf(float e, float lo, float hi) { return mn(mx(e, lo), hi); }
__device__ __forceinline__ float signf(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }
__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
  return ax * bx + ay * by + az * bz;
}

}  // namespace upbd
