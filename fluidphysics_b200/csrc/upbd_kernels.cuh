// Single-scene sm_100a kernels of libupbd: the per-pass wrappers around the
// pass bodies of upbd_passes.cuh, and the tool kernels (emit, wedge cut,
// pick, grab, drain) that run on demand.
#pragma once
#include "upbd_passes.cuh"

namespace upbd {

#define UPBD_TID (blockIdx.x * blockDim.x + threadIdx.x)

// ------------------------------------------------------------------ emit
// emit, src/gpu/wgsl.js:781-801 (hose ring buffer)
__global__ void __launch_bounds__(64) k_emit(SimView v, const DevParams* __restrict__ P) {
  const uint32_t k = UPBD_TID;
  if (k >= P->emit_count) return;
  const int slot = v.S + (int)((P->emit_start + k) % (uint32_t)v.F);
  const float4 E_pos = P->emit_pos, E_dir = P->emit_dir, E_side = P->emit_side, E_up = P->emit_up;
  const real phase = E_dir.w + (real)k * 2.39996f;
  const real spacing = P->fluid_radius * 2.2f;
  const real fk = (real)k * 0.618034f;
  const real rad = spacing * (0.4f + 1.6f * (fk - floorf(fk)));
  const real c = cosf(phase), s = sinf(phase);
  const real along = (real)(k % 8u) * spacing * 0.5f;
  const real offx = E_side.x * (c * rad) + E_up.x * (s * rad) + E_dir.x * along;
  const real offy = E_side.y * (c * rad) + E_up.y * (s * rad) + E_dir.y * along;
  const real offz = E_side.z * (c * rad) + E_up.z * (s * rad) + E_dir.z * along;
  const real px = E_pos.x + offx, py = E_pos.y + offy, pz = E_pos.z + offz;
  const real a = sinf(phase * 12.9898f) * 43758.547f;
  const real b = sinf(phase * 78.233f) * 12543.123f;
  const real d = sinf(phase * 39.425f) * 26781.897f;
  const real jx = ((a - floorf(a)) - 0.5f) * 0.5f;
  const real jy = ((b - floorf(b)) - 0.5f) * 0.5f;
  const real jz = ((d - floorf(d)) - 0.5f) * 0.5f;
  const real speed = E_pos.w;
  const real w = v.pos[slot].w;
  v.pos[slot] = make_real4(px, py, pz, w);
  v.prev[slot] = make_real4(px, py, pz, 0.f);
  v.vel[slot] = make_real4(E_dir.x * speed + jx, E_dir.y * speed + jy, E_dir.z * speed + jz, 0.f);
  v.flags[slot] = F_ACTIVE;
}

// Solver.emitFluid for a batch, src/solver.js:139-149 (ring buffer).
__global__ void k_emit_particles(SimView v, const float* __restrict__ p3,
                                 const float* __restrict__ v3, int n, int start, float inv_mass) {
  const int k = UPBD_TID;
  if (k >= n) return;
  const int slot = v.S + (int)(((long long)start + k) % v.F);
  const real x = p3[3 * k], y = p3[3 * k + 1], z = p3[3 * k + 2];
  v.pos[slot] = make_real4(x, y, z, inv_mass);
  v.prev[slot] = make_real4(x, y, z, 0.f);
  v.vel[slot] = make_real4(v3[3 * k], v3[3 * k + 1], v3[3 * k + 2], 0.f);
  v.flags[slot] = F_ACTIVE;
}

// ------------------------------------------------- single-scene kernels
// One launch per pass over one scene: tile vb = blockIdx.x.
template <bool INTEGRATE, bool COUNT>
__global__ void __launch_bounds__(256) k_integrate_count(SimView v, const DevParams* __restrict__ P) {
  b_integrate_count<INTEGRATE, COUNT>(v, P, blockIdx.x);
}
__global__ void __launch_bounds__(SCAN_THREADS) k_scan(SimView v) { b_scan(v, blockIdx.x); }
__global__ void __launch_bounds__(256) k_scatter(SimView v) { b_scatter(v, blockIdx.x); }
__global__ void __launch_bounds__(256) k_rankfix(SimView v) { b_rankfix(v, blockIdx.x); }
__global__ void __launch_bounds__(256) k_density(SimView v, const DevParams* __restrict__ P) {
  b_density(v, P, blockIdx.x);
}
template <bool APPLY>
__global__ void __launch_bounds__(256) k_disp(SimView v, const DevParams* __restrict__ P) {
  b_disp<APPLY>(v, P, blockIdx.x);
}
__global__ void __launch_bounds__(256) k_apply_fluid(SimView v, const DevParams* __restrict__ P) {
  b_apply_fluid(v, P, blockIdx.x);
}
template <bool APPLY_FLUID, int OUT>
__global__ void __launch_bounds__(256) k_solid_solve(SimView v, const DevParams* __restrict__ P, int solid_pad, int it) {
  b_solid_solve<APPLY_FLUID, OUT>(v, P, solid_pad, it, blockIdx.x);
}
template <bool MARK>
__global__ void __launch_bounds__(256) k_apply_solid(SimView v, const DevParams* __restrict__ P) {
  b_apply_solid<MARK>(v, P, blockIdx.x);
}
template <int G, bool FROM_GRID = false>
__global__ void __launch_bounds__(256) k_contact_mark(SimView v, const DevParams* __restrict__ P) {
  b_contact_mark<G, FROM_GRID>(v, P, blockIdx.x);
}
__global__ void __launch_bounds__(256) k_collect_contacts(SimView v, const DevParams* __restrict__ P) {
  b_collect_contacts(v, P, blockIdx.x);
}
__global__ void __launch_bounds__(256) k_solid_contacts(SimView v, const DevParams* __restrict__ P) {
  b_solid_contacts(v, P, blockIdx.x);
}
__global__ void __launch_bounds__(256) k_apply_solid_contacts(SimView v, const DevParams* __restrict__ P) {
  b_apply_solid_contacts(v, P, blockIdx.x);
}
__global__ void __launch_bounds__(256) k_solve_tets(SimView v, const DevParams* __restrict__ P) {
  b_solve_tets(v, P, blockIdx.x);
}
__global__ void __launch_bounds__(256) k_bond_contacts(SimView v, const DevParams* __restrict__ P, int nb, int nt,
                                                       int nb_pad, int nc) {
  b_bond_contacts(v, P, nb, nt, nb_pad, nc, blockIdx.x);
}
__global__ void __launch_bounds__(256) k_apply_bounds_vel(SimView v, const DevParams* __restrict__ P, int stage) {
  b_apply_bounds_vel(v, P, stage, blockIdx.x);
}
__global__ void __launch_bounds__(256) k_solid_visc(SimView v, const DevParams* __restrict__ P) {
  b_solid_visc(v, P, blockIdx.x);
}
__global__ void __launch_bounds__(256) k_solid_visc_apply(SimView v) { b_solid_visc_apply(v, blockIdx.x); }
template <bool APPLY, int ROLE = 0>
__global__ void __launch_bounds__(256) k_xsph(SimView v, const DevParams* __restrict__ P) {
  b_xsph<APPLY, ROLE>(v, P, blockIdx.x);
}
__global__ void __launch_bounds__(256) k_count_active(SimView v) { b_count_active(v, blockIdx.x, gridDim.x); }

// ------------------------------------------------------------------ tools
// Wedge cut over the constraint buffer (kernel shape of src/gpu/wgsl.js:804-823)
// with the double-precision arithmetic of Solver.cut, src/solver.js:458-486.
// Every operation is an explicit round-to-nearest intrinsic so no multiply-add
// is fused and the alive flags match the CPU solver bit for bit.
__global__ void __launch_bounds__(256) k_cut(SimView v, const DevParams* __restrict__ P) {
  const int c = UPBD_TID;
  if (c >= v.C) return;
  const uint4 cc = v.cons[c];
  if (cc.w == 0u) return;
  const double ox = P->cut_o[0], oy = P->cut_o[1], oz = P->cut_o[2];
  const double d1x = P->cut_d1[0], d1y = P->cut_d1[1], d1z = P->cut_d1[2];
  const double d2x = P->cut_d2[0], d2y = P->cut_d2[1], d2z = P->cut_d2[2];
  const double nx = __dsub_rn(__dmul_rn(d1y, d2z), __dmul_rn(d1z, d2y));
  const double ny = __dsub_rn(__dmul_rn(d1z, d2x), __dmul_rn(d1x, d2z));
  const double nz = __dsub_rn(__dmul_rn(d1x, d2y), __dmul_rn(d1y, d2x));
  const double nl = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(nx, nx), __dmul_rn(ny, ny)), __dmul_rn(nz, nz)));
  if (nl < 1e-8) return;
  if (!UPBD_IDX_OK(v, cc.x, v.S) || !UPBD_IDX_OK(v, cc.y, v.S)) return;
  const real4 A = v.pos[cc.x], B = v.pos[cc.y];
  const double ax = A.x, ay = A.y, az = A.z, bx = B.x, by = B.y, bz = B.z;
  const double sa = __dadd_rn(__dadd_rn(__dmul_rn(__dsub_rn(ax, ox), nx), __dmul_rn(__dsub_rn(ay, oy), ny)),
                              __dmul_rn(__dsub_rn(az, oz), nz));
  const double sb = __dadd_rn(__dadd_rn(__dmul_rn(__dsub_rn(bx, ox), nx), __dmul_rn(__dsub_rn(by, oy), ny)),
                              __dmul_rn(__dsub_rn(bz, oz), nz));
  if (__dmul_rn(sa, sb) >= 0.0) return;
  const double t = __ddiv_rn(sa, __dsub_rn(sa, sb));
  const double px = __dsub_rn(__dadd_rn(ax, __dmul_rn(__dsub_rn(bx, ax), t)), ox);
  const double py = __dsub_rn(__dadd_rn(ay, __dmul_rn(__dsub_rn(by, ay), t)), oy);
  const double pz = __dsub_rn(__dadd_rn(az, __dmul_rn(__dsub_rn(bz, az), t)), oz);
  const double c1 = __dadd_rn(__dadd_rn(__dmul_rn(__dsub_rn(__dmul_rn(d1y, pz), __dmul_rn(d1z, py)), nx),
                                        __dmul_rn(__dsub_rn(__dmul_rn(d1z, px), __dmul_rn(d1x, pz)), ny)),
                              __dmul_rn(__dsub_rn(__dmul_rn(d1x, py), __dmul_rn(d1y, px)), nz));
  const double c2 = __dadd_rn(__dadd_rn(__dmul_rn(__dsub_rn(__dmul_rn(py, d2z), __dmul_rn(pz, d2y)), nx),
                                        __dmul_rn(__dsub_rn(__dmul_rn(pz, d2x), __dmul_rn(px, d2z)), ny)),
                              __dmul_rn(__dsub_rn(__dmul_rn(px, d2y), __dmul_rn(py, d2x)), nz));
  if (c1 < 0.0 || c2 < 0.0) return;
  v.cons[c].w = 0u;
  atomicAdd(&v.scratch[SCR_CUT], 1u);
}

// cutTets, src/gpu/wgsl.js:494-519 (f32 wedge, as the reference kernel)
__global__ void __launch_bounds__(256) k_cut_tets(SimView v, const DevParams* __restrict__ P) {
  const int t = UPBD_TID;
  if (t >= v.NT) return;
  const real V0 = v.tet_vol[t];
  if (V0 <= 0.f) return;
  const real ox = (real)P->cut_o[0], oy = (real)P->cut_o[1], oz = (real)P->cut_o[2];
  const real ax1 = (real)P->cut_d1[0], ay1 = (real)P->cut_d1[1], az1 = (real)P->cut_d1[2];
  const real ax2 = (real)P->cut_d2[0], ay2 = (real)P->cut_d2[1], az2 = (real)P->cut_d2[2];
  real nx, ny, nz;
  cross3(ax1, ay1, az1, ax2, ay2, az2, nx, ny, nz);
  if (dot3(nx, ny, nz, nx, ny, nz) < 1e-16f) return;
  for (int p = 0; p < 3; p++)
    for (int q = p + 1; q < 4; q++) {
      const uint32_t ta = v.tet_idx[4 * t + p], tb = v.tet_idx[4 * t + q];
      if (!UPBD_IDX_OK(v, ta, v.S) || !UPBD_IDX_OK(v, tb, v.S)) return;
      const real4 A = v.pos[ta];
      const real4 B = v.pos[tb];
      const real pax = A.x - ox, pay = A.y - oy, paz = A.z - oz;
      const real pbx = B.x - ox, pby = B.y - oy, pbz = B.z - oz;
      const real sa = dot3(pax, pay, paz, nx, ny, nz);
      const real sb = dot3(pbx, pby, pbz, nx, ny, nz);
      if (sa * sb >= 0.f) continue;
      const real tt = sa / (sa - sb);
      const real ppx = pax + (pbx - pax) * tt, ppy = pay + (pby - pay) * tt, ppz = paz + (pbz - paz) * tt;
      real cx, cy, cz;
      cross3(ax1, ay1, az1, ppx, ppy, ppz, cx, cy, cz);
      if (dot3(cx, cy, cz, nx, ny, nz) < 0.f) continue;
      cross3(ppx, ppy, ppz, ax2, ay2, az2, cx, cy, cz);
      if (dot3(cx, cy, cz, nx, ny, nz) < 0.f) continue;
      v.tet_vol[t] = -V0;
      return;
    }
}

// Pick, pass 1: smallest t (Solver.pickSolid, src/solver.js:502-515, in
// double). t >= 0, so its IEEE bits order like unsigned integers.
__device__ __forceinline__ bool pick_t(const SimView& v, const DevParams* __restrict__ P, int i, double& t) {
  if (!(v.flags[i] & F_ACTIVE)) return false;
  const real4 p = v.pos[i];
  const double ox = P->pick_o[0], oy = P->pick_o[1], oz = P->pick_o[2], mp = P->pick_o[3];
  const double dx = P->pick_d[0], dy = P->pick_d[1], dz = P->pick_d[2];
  const double px = __dsub_rn((double)p.x, ox), py = __dsub_rn((double)p.y, oy), pz = __dsub_rn((double)p.z, oz);
  t = __dadd_rn(__dadd_rn(__dmul_rn(px, dx), __dmul_rn(py, dy)), __dmul_rn(pz, dz));
  if (!(t >= 0.0)) return false;
  const double qx = __dsub_rn(px, __dmul_rn(dx, t)), qy = __dsub_rn(py, __dmul_rn(dy, t)),
               qz = __dsub_rn(pz, __dmul_rn(dz, t));
  const double q2 = __dadd_rn(__dadd_rn(__dmul_rn(qx, qx), __dmul_rn(qy, qy)), __dmul_rn(qz, qz));
  if (q2 > __dmul_rn(mp, mp)) return false;
  return true;
}

__global__ void __launch_bounds__(256) k_pick_min_t(SimView v, const DevParams* __restrict__ P) {
  const int i = UPBD_TID;
  unsigned long long best = ~0ull;
  double t;
  if (i < v.S && pick_t(v, P, i, t)) best = (unsigned long long)__double_as_longlong(t);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_down_sync(0xffffffffu, best, o);
    best = (y < best) ? y : best;
  }
  if ((threadIdx.x & 31) == 0 && best != ~0ull)
    atomicMin(reinterpret_cast<unsigned long long*>(&v.scratch[SCR_PICK_T]), best);
}

// Pick, pass 2: lowest index among the particles at the smallest t.
__global__ void __launch_bounds__(256) k_pick_min_i(SimView v, const DevParams* __restrict__ P) {
  const int i = UPBD_TID;
  const unsigned long long best = *reinterpret_cast<const unsigned long long*>(&v.scratch[SCR_PICK_T]);
  double t;
  if (i < v.S && best != ~0ull && pick_t(v, P, i, t) &&
      (unsigned long long)__double_as_longlong(t) == best)
    atomicMin(&v.scratch[SCR_PICK_I], (uint32_t)i);
}

// grabSelect, src/gpu/wgsl.js:843-865
__global__ void __launch_bounds__(256) k_grab_select(SimView v, const DevParams* __restrict__ P) {
  const int i = UPBD_TID;
  if (i >= v.S) return;
  uint32_t f = v.flags[i];
  if (!(f & F_ACTIVE)) return;
  const uint32_t lat = (i >= v.N1) ? 1u : 0u;
  if (P->grab_lattice != 0xffffu && lat != P->grab_lattice) return;
  const float4 c = P->grab_c;
  const real4 p = v.pos[i];
  const real dx = p.x - c.x, dy = p.y - c.y, dz = p.z - c.z;
  const real q2 = dot3(dx, dy, dz, dx, dy, dz) / (c.w * c.w);
  if (q2 < 1.0f) {
    v.flags[i] = f | F_GRABBED;
    const real w = (1.0f - q2) * (1.0f - q2) * 0.95f + 0.05f;
    v.prev[i].w = p.x;
    v.vel[i].w = p.y;
    v.density[i] = make_real2(p.z, w);
  }
}

// Explicit-list grab: spring target given or at the current position.
__global__ void k_grab_indices(SimView v, const uint32_t* __restrict__ idx, const float* __restrict__ w,
                               const float* __restrict__ t3, int n) {
  const int k = UPBD_TID;
  if (k >= n) return;
  const uint32_t i = idx[k];
  if (i >= (uint32_t)v.S) return;
  const uint32_t f = v.flags[i];
  if (!(f & F_ACTIVE)) return;
  const real4 p = v.pos[i];
  const real tx = t3 ? t3[3 * k] : p.x, ty = t3 ? t3[3 * k + 1] : p.y, tz = t3 ? t3[3 * k + 2] : p.z;
  v.flags[i] = f | F_GRABBED;
  v.prev[i].w = tx;
  v.vel[i].w = ty;
  v.density[i] = make_real2(tz, w ? w[k] : 1.0f);
}

// grabRelease, src/gpu/wgsl.js:867-871
__global__ void k_grab_release(SimView v) {
  const int i = UPBD_TID;
  if (i < v.S) v.flags[i] &= ~F_GRABBED;
}

// GpuSim.clearFluid, src/gpu/sim.js:294-297
// the body of every kernel node in upbd_profile_graph_floor's copy of a frame
__global__ void k_empty() {}

__global__ void k_drain(SimView v) {
  const int i = v.S + (int)UPBD_TID;
  if (i < v.N) v.flags[i] = 0u;
}

}  // namespace upbd
