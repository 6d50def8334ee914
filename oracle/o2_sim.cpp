// ORACLE — test infrastructure only (checker, never the product path).
// O2 kernel restatements; the WGSL line cited above each pass is the kernel
// it restates (src/gpu/wgsl.js), the sim.js line the host code.
#include "o2_sim.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "js_numerics.h"

namespace oracle {

// A literal as WGSL sees it: an abstract float converted to the kernel's type.
template <class R> inline R lit(float f, double d);
template <> inline float lit<float>(float f, double) { return f; }
template <> inline double lit<double>(float, double d) { return d; }
#define LIT(x) lit<R>(x##f, x)

template <class R> static inline R dot3(R ax, R ay, R az, R bx, R by, R bz) {
  return ax * bx + ay * by + az * bz;
}
template <class R> static inline R clampR(R e, R lo, R hi) { return std::min(std::max(e, lo), hi); }
template <class R> static inline R fractR(R x) { return x - std::floor(x); }
template <class R> static inline R signR(R x) { return x > 0 ? R(1) : (x < 0 ? R(-1) : R(0)); }

static constexpr uint32_t F_ACTIVE = 1u, F_GRABBED = 2u;
static constexpr uint32_t C_K = 40u;  // src/gpu/wgsl.js:25

// Summation order of the neighbour gathers (fluidDensity, fluidDisp, xsph,
// contacts). The reference sums one particle's neighbours in any order its
// invocation takes; this restatement fixes the order the CUDA kernels use, so
// the two agree bit for bit. The candidates of one part (fluid entries, or
// solid entries) of the 27 neighbour buckets, cells k = (dx+1)*9 + (dy+1)*3 +
// (dz+1) in order and each bucket's entries in order, form one sequence c =
// 0, 1, ...; candidate c goes to lane c mod L, every lane sums from zero, and
// the partials combine by an xor butterfly: for the contacts L = GL = 8,
// ((p0+p4)+(p2+p6)) + ((p1+p5)+(p3+p7)); for fluidDensity and xsph L = GLF =
// 4, (p0+p2) + (p1+p3). fluidDisp instead sums the GLF lanes' shares in lane
// order, DL partial sums of GLF/DL lanes each, combined by the same kind of
// butterfly.
static constexpr int GL = 8;
static constexpr int GLF = 4;
static constexpr int DL = 2;  // fluidDisp threads per particle
template <class R> static inline R lane_reduce(const R* p) {
  return ((p[0] + p[4]) + (p[2] + p[6])) + ((p[1] + p[5]) + (p[3] + p[7]));
}
// the butterfly for any power-of-two lane count G: after the step of width d,
// lane l holds its value plus lane l+d's (what lane 0 ends with is returned)
template <int G, class R> static inline R lane_reduce_g(const R* p) {
  R t[G];
  for (int l = 0; l < G; l++) t[l] = p[l];
  for (int d = G / 2; d > 0; d /= 2)
    for (int l = 0; l < d; l++) t[l] = t[l] + t[l + d];
  return t[0];
}
template <class Sim, class V, class Fn>
static inline void strided_walk(const Sim& s, const V& pi, bool solid_part, Fn&& fn, uint32_t lanes = GL) {
  uint32_t c = 0;
  for (int k = 0; k < 27; k++) {
    const uint32_t h = s.cellHashOf(pi, k / 9 - 1, (k / 3) % 3 - 1, k % 3 - 1);
    for (uint32_t e = s.start[h]; e < s.start[h + 1]; e++) {
      const uint32_t j = s.entries[e];
      if ((j < (uint32_t)s.S) != solid_part) continue;
      fn((int)(c % lanes), j);
      c++;
    }
  }
}

template <class R> int O2Sim<R>::create(const upbd_scene_desc& d, const upbd_params& p) {
  desc = d;
  if (d.solid_dim < 0 || d.solid_dim2 < 0 || d.max_fluid < 0) return UPBD_ERR_INVALID;
  if (d.table_size < 1 || (d.table_size & (d.table_size - 1))) return UPBD_ERR_INVALID;
  dim1 = d.solid_dim;
  dim2 = d.solid_dim2;
  N1 = dim1 * dim1 * dim1;
  S = N1 + dim2 * dim2 * dim2;
  F = d.max_fluid;
  N = S + F;
  T = d.table_size;
  substeps = d.substeps;
  iters = d.solid_iters;
  features = d.features;

  // _buildHostData, src/gpu/sim.js:98-214 (JS doubles, f32 buffers)
  std::vector<float> hpos(4 * (size_t)N, 0.f);
  std::vector<uint32_t> ca, cb;
  std::vector<double> crest;
  std::vector<std::vector<uint32_t>> incident(S);
  const double spacing = d.spacing;
  const double maxD2 = 3 * spacing * spacing + 1e-9;
  int id = 0;
  auto addLattice = [&](int dim, const double* center) {
    const int base = id;
    const double half = (dim - 1) * spacing / 2;
    for (int ix = 0; ix < dim; ix++)
      for (int iy = 0; iy < dim; iy++)
        for (int iz = 0; iz < dim; iz++) {
          hpos[4 * id + 0] = (float)(center[0] - half + ix * spacing);
          hpos[4 * id + 1] = (float)(center[1] - half + iy * spacing);
          hpos[4 * id + 2] = (float)(center[2] - half + iz * spacing);
          hpos[4 * id + 3] = (float)(1 / d.solid_mass);
          id++;
        }
    auto idx = [&](int ix, int iy, int iz) { return base + (ix * dim + iy) * dim + iz; };
    for (int ix = 0; ix < dim; ix++)
      for (int iy = 0; iy < dim; iy++)
        for (int iz = 0; iz < dim; iz++)
          for (int dx = -1; dx <= 1; dx++)
            for (int dy = -1; dy <= 1; dy++)
              for (int dz = -1; dz <= 1; dz++) {
                const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
                if (jx < 0 || jy < 0 || jz < 0 || jx >= dim || jy >= dim || jz >= dim) continue;
                const int a = idx(ix, iy, iz), b = idx(jx, jy, jz);
                if (b <= a) continue;
                const double d2 = (double)(dx * dx + dy * dy + dz * dz) * spacing * spacing;
                if (d2 > maxD2) continue;
                const uint32_t c = (uint32_t)ca.size();
                ca.push_back(a); cb.push_back(b); crest.push_back(std::sqrt(d2));
                incident[a].push_back(c); incident[b].push_back(c);
              }
  };
  // tets, src/gpu/sim.js:147-166
  std::vector<uint32_t> tets;
  std::vector<double> tvol;
  auto signedVol = [&](int a, int b, int c, int dd) {
    auto v = [&](int p0, int q, int k) { return (double)hpos[q * 4 + k] - hpos[p0 * 4 + k]; };
    const double abx = v(a, b, 0), aby = v(a, b, 1), abz = v(a, b, 2);
    const double acx = v(a, c, 0), acy = v(a, c, 1), acz = v(a, c, 2);
    const double adx = v(a, dd, 0), ady = v(a, dd, 1), adz = v(a, dd, 2);
    return (aby * acz - abz * acy) * adx + (abz * acx - abx * acz) * ady +
           (abx * acy - aby * acx) * adz;
  };
  auto addTets = [&](int dim, int base) {
    auto idx = [&](int ix, int iy, int iz) { return base + (ix * dim + iy) * dim + iz; };
    for (int ix = 0; ix < dim - 1; ix++)
      for (int iy = 0; iy < dim - 1; iy++)
        for (int iz = 0; iz < dim - 1; iz++) {
          auto c = [&](int dx, int dy, int dz) { return idx(ix + dx, iy + dy, iz + dz); };
          const int A = c(0, 0, 0), B = c(1, 0, 0), Cc = c(1, 1, 0), D = c(0, 1, 0);
          const int E = c(0, 0, 1), Fv = c(1, 0, 1), G = c(1, 1, 1), H = c(0, 1, 1);
          int five[5][4];
          if ((ix + iy + iz) % 2 == 0) {
            const int f[5][4] = {{A, Cc, Fv, H}, {A, B, Cc, Fv}, {A, Cc, D, H}, {A, E, Fv, H}, {Cc, Fv, G, H}};
            std::memcpy(five, f, sizeof(f));
          } else {
            const int f[5][4] = {{B, D, E, G}, {A, B, D, E}, {B, Cc, D, G}, {D, E, H, G}, {B, E, Fv, G}};
            std::memcpy(five, f, sizeof(f));
          }
          for (auto& t : five) {
            for (int q = 0; q < 4; q++) tets.push_back(t[q]);
            tvol.push_back(signedVol(t[0], t[1], t[2], t[3]) / 6);
          }
        }
  };
  if (dim1 > 0) {
    addLattice(dim1, d.cube_center);
    addTets(dim1, 0);
  }
  if (dim2 > 0) {
    addLattice(dim2, d.cube2_center);
    addTets(dim2, N1);
  }
  for (int i = S; i < N; i++) hpos[i * 4 + 3] = (float)(1 / d.fluid_mass);
  C = (int)ca.size();
  NT = (int)tvol.size();

  pos.assign(N, V4<R>{0, 0, 0, 0});
  prev.assign(N, V4<R>{0, 0, 0, 0});
  vel.assign(N, V4<R>{0, 0, 0, 0});
  delta.assign(N, V4<R>{0, 0, 0, 0});
  density.assign(N, V2<R>{0, 0});
  flags.assign(N, 0);
  initPos.resize(N);
  for (int i = 0; i < N; i++)
    initPos[i] = V4<R>{(R)hpos[4 * i], (R)hpos[4 * i + 1], (R)hpos[4 * i + 2], (R)hpos[4 * i + 3]};
  consA = ca;
  consB = cb;
  initRest.resize(C);
  for (int c = 0; c < C; c++) initRest[c] = (R)(float)crest[c];  // f32 buffer (sim.js:201)
  adj.assign(S + 1 + 2 * (size_t)C, 0);
  {
    uint32_t off = 0;
    for (int i = 0; i < S; i++) {
      adj[i] = off;
      for (uint32_t c : incident[i]) adj[S + 1 + off++] = c;
    }
    adj[S] = off;
  }
  tetIdx = tets;
  initTetVol.resize(NT);
  for (int t = 0; t < NT; t++) initTetVol[t] = (R)(float)tvol[t];
  {
    std::vector<std::vector<uint32_t>> tinc(S);
    for (int t = 0; t < NT; t++)
      for (int q = 0; q < 4; q++) tinc[tets[4 * t + q]].push_back(t);
    tetAdj.assign(S + 1 + 4 * (size_t)NT, 0);
    uint32_t off = 0;
    for (int i = 0; i < S; i++) {
      tetAdj[i] = off;
      for (uint32_t t : tinc[i]) tetAdj[S + 1 + off++] = t;
    }
    tetAdj[S] = off;
  }
  ccount.assign(S, 0);
  clist.assign((size_t)S * C_K, 0);
  counts.assign(T, 0);
  start.assign(T + 1, 0);
  entries.assign(N, 0);
  setParams(p);
  // fluid slots carry their inverse mass but start inactive (src/gpu/sim.js:174,288)
  resetSolid();
  return UPBD_OK;
}

template <class R> void O2Sim<R>::setParams(const upbd_params& p) {
  prm = p;
  // _writeParams, src/gpu/sim.js:300-330 (f32 buffer for R = float)
  P.h = (R)p.h; P.gravity = (R)p.gravity; P.solidRadius = (R)p.solid_radius;
  P.fluidRadius = (R)p.fluid_radius; P.cellSize = (R)p.cell_size; P.fluidH = (R)p.fluid_h;
  P.restDensity = (R)p.rest_density; P.stiffness = (R)p.stiffness;
  P.nearStiffness = (R)p.near_stiffness; P.viscosity = (R)p.viscosity;
  P.compliance = (R)p.compliance; P.omega = (R)p.omega;
  P.plasticThreshold = (R)p.plastic_threshold; P.plasticRate = (R)p.plastic_rate;
  P.tearGap = (R)p.tear_gap; P.maxSpeed = (R)p.max_speed; P.wallX = (R)p.wall_x;
  P.wallZ = (R)p.wall_z; P.wallH = (R)p.wall_h; P.wallT = (R)p.wall_t; P.cullR = (R)p.cull_r;
  P.dampSolid = (R)p.damp_solid; P.dampFluid = (R)p.damp_fluid;
  P.frictionSolid = (R)p.friction_solid; P.frictionFluid = (R)p.friction_fluid;
  P.grabK = (R)p.grab_k; P.sleepSpeed = (R)p.sleep_speed; P.spacing = (R)desc.spacing;
  P.solidViscosity = (R)p.solid_viscosity; P.breakStrain = (R)p.break_strain;
  P.contactScale = (R)p.contact_scale;
  P.invCell = 1.0 / p.cell_size;
  P.tearMode = p.tear_mode;
  P.plasticClamp = p.plastic_clamp;
}

// GpuSim.resetSolid, src/gpu/sim.js:283-292: pos and prev of every slot
// (fluid slots included) back to the initial buffer, every velocity zeroed,
// flags and density of the solids reset, constraints and tets pristine.
template <class R> void O2Sim<R>::resetSolid() {
  for (int i = 0; i < N; i++) {
    pos[i] = initPos[i];
    prev[i] = initPos[i];
    vel[i] = V4<R>{0, 0, 0, 0};
  }
  for (int i = 0; i < S; i++) {
    flags[i] = F_ACTIVE;
    density[i] = V2<R>{0, 0};
  }
  consRest = initRest;
  consAlive.assign(C, 1);
  tetVol = initTetVol;
}

// GpuSim.clearFluid, src/gpu/sim.js:294-297
template <class R> void O2Sim<R>::drain() {
  for (int i = S; i < N; i++) flags[i] = 0;
}

// countActive, src/gpu/wgsl.js:874-879
template <class R> uint32_t O2Sim<R>::activeCount() const {
  uint32_t n = 0;
  for (int i = S; i < N; i++) n += (flags[i] & F_ACTIVE) ? 1 : 0;
  return n;
}

template <class R>
uint32_t O2Sim<R>::cellHashOf(const V4<R>& p, int dx, int dy, int dz) const {
  const double xi = js_cell((double)p.x, P.invCell), yi = js_cell((double)p.y, P.invCell),
               zi = js_cell((double)p.z, P.invCell);
  return js_hash(xi + dx, yi + dy, zi + dz, (uint32_t)T);
}

// emit, src/gpu/wgsl.js:781-801
template <class R> void O2Sim<R>::passEmit() {
  const Emit& E = emit;
  for (int k = 0; k < E.count; k++) {
    const int slot = S + (int)(((uint32_t)E.start + (uint32_t)k) % (uint32_t)F);
    const R phase = E.dir.w + (R)k * LIT(2.39996);
    const R spacing = P.fluidRadius * LIT(2.2);
    const R rad = spacing * (LIT(0.4) + LIT(1.6) * fractR((R)k * LIT(0.618034)));
    const R c = std::cos(phase), s = std::sin(phase);
    const R along = (R)(k % 8) * spacing * LIT(0.5);
    const R offx = E.side.x * (c * rad) + E.up.x * (s * rad) + E.dir.x * along;
    const R offy = E.side.y * (c * rad) + E.up.y * (s * rad) + E.dir.y * along;
    const R offz = E.side.z * (c * rad) + E.up.z * (s * rad) + E.dir.z * along;
    const R px = E.pos.x + offx, py = E.pos.y + offy, pz = E.pos.z + offz;
    const R jx = (fractR(std::sin(phase * LIT(12.9898)) * LIT(43758.547)) - LIT(0.5)) * LIT(0.5);
    const R jy = (fractR(std::sin(phase * LIT(78.233)) * LIT(12543.123)) - LIT(0.5)) * LIT(0.5);
    const R jz = (fractR(std::sin(phase * LIT(39.425)) * LIT(26781.897)) - LIT(0.5)) * LIT(0.5);
    const R speed = E.pos.w;
    pos[slot] = V4<R>{px, py, pz, pos[slot].w};
    prev[slot] = V4<R>{px, py, pz, 0};
    vel[slot] = V4<R>{E.dir.x * speed + jx, E.dir.y * speed + jy, E.dir.z * speed + jz, 0};
    flags[slot] = F_ACTIVE;
  }
}

// integrate, src/gpu/wgsl.js:121-160
template <class R> void O2Sim<R>::passIntegrate() {
  for (int i = 0; i < N; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    R vx = vel[i].x, vy = vel[i].y, vz = vel[i].z;
    vy = vy + P.gravity * P.h;
    const R px = pos[i].x, py = pos[i].y, pz = pos[i].z;
    R nx = px + vx * P.h, ny = py + vy * P.h, nz = pz + vz * P.h;
    R tw = prev[i].w;
    if (flags[i] & F_GRABBED) {
      R tx = prev[i].w, ty = vel[i].w, tz = density[i].x;
      tx = tx + grabDeltaSub.x; ty = ty + grabDeltaSub.y; tz = tz + grabDeltaSub.z;
      const R ex = nx - tx, ey = ny - ty, ez = nz - tz;
      if (std::sqrt(dot3(ex, ey, ez, ex, ey, ez)) > LIT(1.0)) {
        flags[i] &= ~F_GRABBED;
        prev[i] = V4<R>{px, py, pz, tw};
        pos[i] = V4<R>{nx, ny, nz, pos[i].w};
        vel[i] = V4<R>{vx, vy, vz, 0};
        continue;
      }
      const R k = P.grabK * density[i].y;
      R cx = (tx - nx) * k, cy = (ty - ny) * k, cz = (tz - nz) * k;
      const R cl = std::sqrt(dot3(cx, cy, cz, cx, cy, cz));
      const R maxC = LIT(0.05);
      if (cl > maxC) {
        const R f = maxC / cl;
        cx = cx * f; cy = cy * f; cz = cz * f;
      }
      nx = nx + cx; ny = ny + cy; nz = nz + cz;
      tw = tx;
      vel[i] = V4<R>{vx, vy, vz, ty};
      density[i] = V2<R>{tz, density[i].y};
    } else {
      vel[i] = V4<R>{vx, vy, vz, vel[i].w};
    }
    prev[i] = V4<R>{px, py, pz, tw};
    pos[i] = V4<R>{nx, ny, nz, pos[i].w};
  }
}

// gridClear/gridCount/scan*/gridScatter, src/gpu/wgsl.js:163-245, with the
// membership order of Solver._buildGrid (src/solver.js:174-184).
template <class R> void O2Sim<R>::passGrid() {
  std::fill(counts.begin(), counts.end(), 0u);
  std::vector<uint32_t> hs(N);
  for (int i = 0; i < N; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    hs[i] = cellHashOf(pos[i], 0, 0, 0);
    counts[hs[i]]++;
  }
  uint32_t sum = 0;
  for (int k = 0; k < T; k++) {
    start[k] = sum;
    sum += counts[k];
  }
  start[T] = sum;
  std::vector<uint32_t> end(start.begin() + 1, start.end());
  for (int i = 0; i < N; i++)
    if (flags[i] & F_ACTIVE) entries[--end[hs[i]]] = (uint32_t)i;
}

// fluidDensity, src/gpu/wgsl.js:254-279
template <class R> void O2Sim<R>::passDensity() {
  const R H = P.fluidH, H2 = H * H;
#pragma omp parallel for schedule(static)
  for (int i = S; i < N; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    const V4<R> pi = pos[i];
    R rho[GLF] = {}, rhoNear[GLF] = {};
    strided_walk(*this, pi, false, [&](int l, uint32_t j) {
      if (j == (uint32_t)i || j < (uint32_t)S) return;
      const R ex = pos[j].x - pi.x, ey = pos[j].y - pi.y, ez = pos[j].z - pi.z;
      const R d2 = dot3(ex, ey, ez, ex, ey, ez);
      if (d2 >= H2) return;
      const R q = LIT(1.0) - std::sqrt(d2) / H;
      rho[l] = rho[l] + q * q;
      rhoNear[l] = rhoNear[l] + q * q * q;
    }, GLF);
    density[i] = V2<R>{lane_reduce_g<GLF>(rho), lane_reduce_g<GLF>(rhoNear)};
  }
}

// fluidDisp, src/gpu/wgsl.js:281-316
template <class R> void O2Sim<R>::passDisp() {
  const R H = P.fluidH, H2 = H * H;
  const R maxPair = LIT(0.05) * H, maxTotal = LIT(0.35) * H;
#pragma omp parallel for schedule(static)
  for (int i = S; i < N; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    const V4<R> pi = pos[i];
    const R Pi = P.stiffness * (density[i].x - P.restDensity);
    const R PNi = P.nearStiffness * density[i].y;
    // DL sums over the neighbours in lane-major order: part h takes lanes
    // h*GLF/DL .. (h+1)*GLF/DL - 1, lane l's share of the walk being candidates
    // c = l, l+GLF, ... (the CUDA pass reads them from the density pass's
    // per-lane lists in that order); the parts combine by the xor butterfly
    std::vector<uint32_t> share[GLF];
    strided_walk(*this, pi, false, [&](int l, uint32_t j) {
      if (j != (uint32_t)i && j >= (uint32_t)S) share[l].push_back(j);
    }, GLF);
    R part[DL][3] = {};
    for (int l = 0; l < GLF; l++) {
      R& sx = part[l / (GLF / DL)][0];
      R& sy = part[l / (GLF / DL)][1];
      R& sz = part[l / (GLF / DL)][2];
      for (uint32_t j : share[l]) {
        const R ex = pos[j].x - pi.x, ey = pos[j].y - pi.y, ez = pos[j].z - pi.z;
        const R d2 = dot3(ex, ey, ez, ex, ey, ez);
        if (d2 >= H2 || d2 < LIT(1e-12)) continue;
        const R d = std::sqrt(d2);
        const R q = LIT(1.0) - d / H;
        const R Pj = P.stiffness * (density[j].x - P.restDensity);
        const R PNj = P.nearStiffness * density[j].y;
        R D = LIT(0.25) * ((Pi + Pj) * q + (PNi + PNj) * q * q);
        D = clampR(D, -maxPair, maxPair);
        const R f = D / d;
        sx = sx - ex * f; sy = sy - ey * f; sz = sz - ez * f;
      }
    }
    for (int dd = DL / 2; dd > 0; dd /= 2)  // the CUDA pass's xor butterfly
      for (int a = 0; a < dd; a++)
        for (int c = 0; c < 3; c++) part[a][c] = part[a][c] + part[a + dd][c];
    R sx = part[0][0], sy = part[0][1], sz = part[0][2];
    const R s2 = dot3(sx, sy, sz, sx, sy, sz);
    if (s2 > maxTotal * maxTotal) {
      const R f = maxTotal / std::sqrt(s2);
      sx = sx * f; sy = sy * f; sz = sz * f;
    }
    delta[i] = V4<R>{sx, sy, sz, LIT(1.0)};
  }
}

// applyDeltaFluid, src/gpu/wgsl.js:318-323
template <class R> void O2Sim<R>::passApplyFluid() {
  for (int i = S; i < N; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    pos[i].x = pos[i].x + delta[i].x;
    pos[i].y = pos[i].y + delta[i].y;
    pos[i].z = pos[i].z + delta[i].z;
  }
}

// latticeRest, src/gpu/wgsl.js:373-381
template <class R> R O2Sim<R>::latticeRest(uint32_t a0, uint32_t b0) const {
  uint32_t a = a0, b = b0, D = (uint32_t)dim1;
  if (a0 >= (uint32_t)N1) { a = a0 - N1; b = b0 - N1; D = (uint32_t)std::max(1, dim2); }
  const R ax = (R)(a / (D * D)), ay = (R)((a / D) % D), az = (R)(a % D);
  const R bx = (R)(b / (D * D)), by = (R)((b / D) % D), bz = (R)(b % D);
  const R dx = ax - bx, dy = ay - by, dz = az - bz;
  return P.spacing * std::sqrt(dx * dx + dy * dy + dz * dz);
}

// latticeAdjacent, src/gpu/wgsl.js:409-416
template <class R> bool O2Sim<R>::latticeAdjacent(uint32_t i, uint32_t j) const {
  if ((i >= (uint32_t)N1) != (j >= (uint32_t)N1)) return false;
  uint32_t a = i, b = j, D = (uint32_t)dim1;
  if (i >= (uint32_t)N1) { a = i - N1; b = j - N1; D = (uint32_t)std::max(1, dim2); }
  const int ax = (int)(a / (D * D)), ay = (int)((a / D) % D), az = (int)(a % D);
  const int bx = (int)(b / (D * D)), by = (int)((b / D) % D), bz = (int)(b % D);
  return std::abs(ax - bx) <= 1 && std::abs(ay - by) <= 1 && std::abs(az - bz) <= 1;
}

// isBonded, src/gpu/wgsl.js:599-607
template <class R> bool O2Sim<R>::isBonded(uint32_t i, uint32_t j) const {
  for (uint32_t k = adj[i]; k < adj[i + 1]; k++) {
    const uint32_t c = adj[S + 1 + k];
    if (consAlive[c] != 0 && (consA[c] == j || consB[c] == j)) return true;
  }
  return false;
}

// solidRsum, src/gpu/wgsl.js:526-530
template <class R> R O2Sim<R>::solidRsum(uint32_t i, uint32_t j) const {
  const R rsum = LIT(2.0) * P.solidRadius;
  if (latticeAdjacent(i, j)) return std::min(rsum, P.spacing * LIT(0.97));
  return rsum;
}

// collectContacts, src/gpu/wgsl.js:532-560
template <class R> void O2Sim<R>::passCollectContacts() {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S; i++) {
    uint32_t cnt = 0;
    if (flags[i] & F_ACTIVE) {
      const V4<R> pi = pos[i];
      const R margin = LIT(2.0) * P.solidRadius;
      for (int dx = -1; dx <= 1; dx++)
        for (int dy = -1; dy <= 1; dy++)
          for (int dz = -1; dz <= 1; dz++) {
            const uint32_t h = cellHashOf(pi, dx, dy, dz);
            for (uint32_t e = start[h]; e < start[h + 1]; e++) {
              const uint32_t j = entries[e];
              if (j == (uint32_t)i || j >= (uint32_t)S || cnt >= C_K) continue;
              const R ex = pi.x - pos[j].x, ey = pi.y - pos[j].y, ez = pi.z - pos[j].z;
              const R lim = solidRsum(i, j) + margin;
              if (dot3(ex, ey, ez, ex, ey, ez) >= lim * lim) continue;
              if (isBonded(i, j)) continue;
              clist[(size_t)i * C_K + cnt] = j;
              cnt++;
            }
          }
    }
    ccount[i] = cnt;
  }
}

// solidSolve, src/gpu/wgsl.js:326-359
template <class R> void O2Sim<R>::passSolidSolve() {
  const R alpha = P.compliance / (P.h * P.h);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    const V4<R> pi = pos[i];
    const R wi = pi.w;
    // incident constraint k of the CSR goes to lane (k - st) % GL; lanes
    // combine like the neighbour gathers (see lane_reduce)
    R cx[GL] = {}, cy[GL] = {}, cz[GL] = {};
    const uint32_t st = adj[i], en = adj[i + 1];
    const uint32_t degI = en - st;
    for (uint32_t k = st; k < en; k++) {
      const int l = (int)((k - st) % GL);
      const uint32_t ci = adj[S + 1 + k];
      if (consAlive[ci] == 0) continue;
      const uint32_t other = (consA[ci] == (uint32_t)i) ? consB[ci] : consA[ci];
      const R rest = consRest[ci];
      const R ex = pi.x - pos[other].x, ey = pi.y - pos[other].y, ez = pi.z - pos[other].z;
      const R d = std::sqrt(dot3(ex, ey, ez, ex, ey, ez));
      if (d < LIT(1e-9)) continue;
      const R wo = pos[other].w;
      const R wsum = wi + wo;
      if (wsum == 0) continue;
      const uint32_t degJ = adj[other + 1] - adj[other];
      const R s = LIT(1.0) / (R)std::max(degI, degJ);
      const R dl = -(d - rest) / (wsum + alpha);
      const R f = dl * wi / d * s;
      cx[l] = cx[l] + ex * f; cy[l] = cy[l] + ey * f; cz[l] = cz[l] + ez * f;
    }
    delta[i] = V4<R>{lane_reduce(cx), lane_reduce(cy), lane_reduce(cz), LIT(1.0)};
  }
}

// applyDeltaSolid, src/gpu/wgsl.js:361-366
template <class R> void O2Sim<R>::passApplySolid() {
  for (int i = 0; i < S; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    pos[i].x = pos[i].x + delta[i].x * P.omega;
    pos[i].y = pos[i].y + delta[i].y * P.omega;
    pos[i].z = pos[i].z + delta[i].z * P.omega;
  }
}

template <class R> static inline void cross3(R ax, R ay, R az, R bx, R by, R bz, R& x, R& y, R& z) {
  x = ay * bz - az * by;
  y = az * bx - ax * bz;
  z = ax * by - ay * bx;
}

// solveTets, src/gpu/wgsl.js:423-468
template <class R> void O2Sim<R>::passSolveTets() {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    R cx = 0, cy = 0, cz = 0;
    for (uint32_t k = tetAdj[i]; k < tetAdj[i + 1]; k++) {
      const uint32_t t = tetAdj[S + 1 + k];
      const uint32_t ia = tetIdx[4 * t], ib = tetIdx[4 * t + 1], ic = tetIdx[4 * t + 2],
                     id = tetIdx[4 * t + 3];
      const R V0 = tetVol[t];
      if (V0 <= 0) continue;
      const V4<R> pa = pos[ia], pb = pos[ib], pc = pos[ic], pd = pos[id];
      const R bax = pb.x - pa.x, bay = pb.y - pa.y, baz = pb.z - pa.z;
      const R cax = pc.x - pa.x, cay = pc.y - pa.y, caz = pc.z - pa.z;
      const R dax = pd.x - pa.x, day = pd.y - pa.y, daz = pd.z - pa.z;
      R xx, xy, xz;
      cross3(bax, bay, baz, cax, cay, caz, xx, xy, xz);
      const R V = dot3(xx, xy, xz, dax, day, daz) / LIT(6.0);
      const R Cv = V - V0;
      R gbx, gby, gbz, gcx, gcy, gcz, gdx, gdy, gdz;
      cross3(cax, cay, caz, dax, day, daz, gbx, gby, gbz);
      gbx = gbx / LIT(6.0); gby = gby / LIT(6.0); gbz = gbz / LIT(6.0);
      cross3(dax, day, daz, bax, bay, baz, gcx, gcy, gcz);
      gcx = gcx / LIT(6.0); gcy = gcy / LIT(6.0); gcz = gcz / LIT(6.0);
      cross3(bax, bay, baz, cax, cay, caz, gdx, gdy, gdz);
      gdx = gdx / LIT(6.0); gdy = gdy / LIT(6.0); gdz = gdz / LIT(6.0);
      const R gax = -((gbx + gcx) + gdx), gay = -((gby + gcy) + gdy), gaz = -((gbz + gcz) + gdz);
      const R w = pa.w;
      const R denom = w * (dot3(gax, gay, gaz, gax, gay, gaz) + dot3(gbx, gby, gbz, gbx, gby, gbz) +
                           dot3(gcx, gcy, gcz, gcx, gcy, gcz) + dot3(gdx, gdy, gdz, gdx, gdy, gdz));
      if (denom < LIT(1e-12)) continue;
      const R dl = -Cv / denom;
      auto deg = [&](uint32_t q) { return tetAdj[q + 1] - tetAdj[q]; };
      const uint32_t dm = std::max(std::max(deg(ia), deg(ib)), std::max(deg(ic), deg(id)));
      const R s = LIT(1.0) / (R)std::max(dm, 1u);
      R mx = gax, my = gay, mz = gaz;
      if ((uint32_t)i == ib) { mx = gbx; my = gby; mz = gbz; }
      else if ((uint32_t)i == ic) { mx = gcx; my = gcy; mz = gcz; }
      else if ((uint32_t)i == id) { mx = gdx; my = gdy; mz = gdz; }
      const R f = w * dl * s;
      R c1x = mx * f, c1y = my * f, c1z = mz * f;
      const R cl2 = dot3(c1x, c1y, c1z, c1x, c1y, c1z);
      const R lim = LIT(0.5) * P.solidRadius;
      if (cl2 > lim * lim) {
        const R g = lim / std::sqrt(cl2);
        c1x = c1x * g; c1y = c1y * g; c1z = c1z * g;
      }
      cx = cx + c1x; cy = cy + c1y; cz = cz + c1z;
    }
    delta[i] = V4<R>{cx, cy, cz, LIT(1.0)};
  }
}

// solidContacts, src/gpu/wgsl.js:562-585
template <class R> void O2Sim<R>::passSolidContacts() {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < S; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    const V4<R> pi = pos[i];
    const R wi = pi.w;
    R cx = 0, cy = 0, cz = 0;
    for (uint32_t k = 0; k < ccount[i]; k++) {
      const uint32_t j = clist[(size_t)i * C_K + k];
      const R ex = pi.x - pos[j].x, ey = pi.y - pos[j].y, ez = pi.z - pos[j].z;
      const R rsum = solidRsum(i, j);
      const R d2 = dot3(ex, ey, ez, ex, ey, ez);
      if (d2 >= rsum * rsum || d2 < LIT(1e-12)) continue;
      const R wj = pos[j].w;
      const R wsum = wi + wj;
      if (wsum == 0) continue;
      const R d = std::sqrt(d2);
      const R f = (rsum - d) / d * wi / wsum * LIT(0.5);
      cx = cx + ex * f; cy = cy + ey * f; cz = cz + ez * f;
    }
    delta[i] = V4<R>{cx, cy, cz, LIT(1.0)};
  }
}

// applySolidContacts, src/gpu/wgsl.js:587-596
template <class R> void O2Sim<R>::passApplySolidContacts() {
  const R maxC = LIT(0.5) * P.solidRadius;
  for (int i = 0; i < S; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    R dx = delta[i].x, dy = delta[i].y, dz = delta[i].z;
    const R m2 = dot3(dx, dy, dz, dx, dy, dz);
    if (m2 > maxC * maxC) {
      const R f = maxC / std::sqrt(m2);
      dx = dx * f; dy = dy * f; dz = dz * f;
    }
    pos[i].x = pos[i].x + dx; pos[i].y = pos[i].y + dy; pos[i].z = pos[i].z + dz;
  }
}

// bondUpdate, src/gpu/wgsl.js:383-404 (tear_mode 1 = the strain rule of
// src/solver.js:370; plastic_clamp 0 = unclamped like src/solver.js:377-379)
template <class R> void O2Sim<R>::passBondUpdate() {
  for (int ci = 0; ci < C; ci++) {
    if (consAlive[ci] == 0) continue;
    const V4<R> pa = pos[consA[ci]], pb = pos[consB[ci]];
    const R ex = pa.x - pb.x, ey = pa.y - pb.y, ez = pa.z - pb.z;
    const R d = std::sqrt(dot3(ex, ey, ez, ex, ey, ez));
    const R rest = consRest[ci];
    const bool tear = (P.tearMode == 1) ? (d > rest * P.breakStrain)
                                        : (d > rest + P.tearGap * LIT(2.0) * P.solidRadius);
    if (tear) {
      consAlive[ci] = 0;
      continue;
    }
    const R strain = (d - rest) / rest;
    R nr = rest;
    if (std::fabs(strain) > P.plasticThreshold) nr = rest + (d - rest) * P.plasticRate;
    if (P.plasticClamp) {
      const R r0 = latticeRest(consA[ci], consB[ci]);
      nr = clampR(nr, LIT(0.9) * r0, LIT(1.25) * r0);
    }
    if (nr != rest) consRest[ci] = nr;
  }
}

// tetUpdate, src/gpu/wgsl.js:472-491
template <class R> void O2Sim<R>::passTetUpdate() {
  const R gap = P.tearGap * LIT(2.0) * P.solidRadius;
  for (int t = 0; t < NT; t++) {
    const R V0 = tetVol[t];
    if (V0 <= 0) continue;
    bool dead = false;
    for (int p = 0; p < 3 && !dead; p++)
      for (int q = p + 1; q < 4; q++) {
        const uint32_t a = tetIdx[4 * t + p], b = tetIdx[4 * t + q];
        const R ex = pos[a].x - pos[b].x, ey = pos[a].y - pos[b].y, ez = pos[a].z - pos[b].z;
        const R d = std::sqrt(dot3(ex, ey, ez, ex, ey, ez));
        if (d > latticeRest(a, b) + gap) {
          dead = true;
          break;
        }
      }
    if (dead) tetVol[t] = -V0;
  }
}

// contacts, src/gpu/wgsl.js:609-646
template <class R> void O2Sim<R>::passContacts() {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < N; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    const bool iSolid = i < S;
    const V4<R> pi = pos[i];
    const R wi = pi.w;
    const R ri = iSolid ? P.solidRadius : P.fluidRadius;
    R cx[GL] = {}, cy[GL] = {}, cz[GL] = {}, cnt[GL] = {};
    // a solid walks the fluid part of each bucket, a fluid particle the solids
    strided_walk(*this, pi, !iSolid, [&](int l, uint32_t j) {
      if (j == (uint32_t)i) return;
      const bool jSolid = j < (uint32_t)S;
      if (iSolid == jSolid) return;
      const R ex = pi.x - pos[j].x, ey = pi.y - pos[j].y, ez = pi.z - pos[j].z;
      const R rj = jSolid ? P.solidRadius : P.fluidRadius;
      const R rsum = ri + rj;
      const R d2 = dot3(ex, ey, ez, ex, ey, ez);
      if (d2 >= rsum * rsum || d2 < LIT(1e-12)) return;
      const R wj = pos[j].w;
      const R wsum = wi + wj;
      if (wsum == 0) return;
      const R d = std::sqrt(d2);
      const R f = (rsum - d) / d * wi / wsum * P.contactScale;
      cx[l] = cx[l] + ex * f; cy[l] = cy[l] + ey * f; cz[l] = cz[l] + ez * f;
      cnt[l] = cnt[l] + LIT(1.0);
    });
    delta[i] = V4<R>{lane_reduce(cx), lane_reduce(cy), lane_reduce(cz), lane_reduce(cnt)};
  }
}

// applyDeltaAll, src/gpu/wgsl.js:648-660
template <class R> void O2Sim<R>::passApplyAll() {
  for (int i = 0; i < N; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    R dx = delta[i].x, dy = delta[i].y, dz = delta[i].z;
    const R r = (i < S) ? P.solidRadius : P.fluidRadius;
    const R m2 = dot3(dx, dy, dz, dx, dy, dz);
    if (m2 > r * r) {
      const R f = r / std::sqrt(m2);
      dx = dx * f; dy = dy * f; dz = dz * f;
    }
    pos[i].x = pos[i].x + dx; pos[i].y = pos[i].y + dy; pos[i].z = pos[i].z + dz;
  }
}

// bounds, src/gpu/wgsl.js:663-697
template <class R> void O2Sim<R>::passBounds() {
  for (int i = 0; i < N; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    const bool iSolid = i < S;
    R px = pos[i].x, py = pos[i].y, pz = pos[i].z;
    const R pvx = prev[i].x, pvz = prev[i].z;
    const R r = iSolid ? P.solidRadius : P.fluidRadius;
    if (py < r) {
      py = r;
      const R mu = iSolid ? P.frictionSolid : P.frictionFluid;
      px = px - (px - pvx) * mu;
      pz = pz - (pz - pvz) * mu;
    }
    if (py < P.wallH + r) {
      const R lim = r + P.wallT;
      if (std::fabs(std::fabs(px) - P.wallX) < lim) {
        const R side = signR(px);
        px = (std::fabs(px) < P.wallX) ? side * (P.wallX - lim) : side * (P.wallX + lim);
      }
      if (std::fabs(std::fabs(pz) - P.wallZ) < lim) {
        const R side = signR(pz);
        pz = (std::fabs(pz) < P.wallZ) ? side * (P.wallZ - lim) : side * (P.wallZ + lim);
      }
    }
    if (!iSolid) {
      if (py < LIT(-3.0) || px * px + pz * pz > P.cullR * P.cullR) flags[i] = 0u;
    }
    pos[i].x = px; pos[i].y = py; pos[i].z = pz;
  }
}

// velocityUpdate, src/gpu/wgsl.js:700-710
template <class R> void O2Sim<R>::passVelocity() {
  for (int i = 0; i < N; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    R vx = (pos[i].x - prev[i].x) / P.h, vy = (pos[i].y - prev[i].y) / P.h,
      vz = (pos[i].z - prev[i].z) / P.h;
    const R damp = (i < S) ? P.dampSolid : P.dampFluid;
    const R g = std::max(LIT(0.0), LIT(1.0) - damp * P.h);
    vx = vx * g; vy = vy * g; vz = vz * g;
    const R sp2 = dot3(vx, vy, vz, vx, vy, vz);
    if (sp2 > P.maxSpeed * P.maxSpeed) {
      const R f = P.maxSpeed / std::sqrt(sp2);
      vx = vx * f; vy = vy * f; vz = vz * f;
    }
    if (!std::isfinite(vx) || !std::isfinite(vy) || !std::isfinite(vz)) healthBits |= UPBD_HEALTH_NAN;
    vel[i] = V4<R>{vx, vy, vz, vel[i].w};
  }
}

// solidVisc, src/gpu/wgsl.js:717-735
template <class R> void O2Sim<R>::passSolidVisc() {
  for (int i = 0; i < S; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    R sx = 0, sy = 0, sz = 0, m = 0;
    for (uint32_t k = adj[i]; k < adj[i + 1]; k++) {
      const uint32_t c = adj[S + 1 + k];
      if (consAlive[c] == 0) continue;
      const uint32_t other = (consA[c] == (uint32_t)i) ? consB[c] : consA[c];
      sx = sx + vel[other].x; sy = sy + vel[other].y; sz = sz + vel[other].z;
      m = m + LIT(1.0);
    }
    R vx = vel[i].x, vy = vel[i].y, vz = vel[i].z;
    if (m > 0) {
      vx = vx + P.solidViscosity * (sx / m - vx);
      vy = vy + P.solidViscosity * (sy / m - vy);
      vz = vz + P.solidViscosity * (sz / m - vz);
    }
    delta[i] = V4<R>{vx, vy, vz, 0};
  }
}

// solidViscApply, src/gpu/wgsl.js:737-742
template <class R> void O2Sim<R>::passSolidViscApply() {
  for (int i = 0; i < S; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    vel[i] = V4<R>{delta[i].x, delta[i].y, delta[i].z, vel[i].w};
  }
}

// xsph, src/gpu/wgsl.js:745-771
template <class R> void O2Sim<R>::passXsph() {
  const R H2 = P.fluidH * P.fluidH;
#pragma omp parallel for schedule(static)
  for (int i = S; i < N; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    const V4<R> pi = pos[i];
    R qx[GLF] = {}, qy[GLF] = {}, qz[GLF] = {}, qm[GLF] = {};
    strided_walk(*this, pi, false, [&](int l, uint32_t j) {
      if (j == (uint32_t)i || j < (uint32_t)S) return;
      const R ex = pos[j].x - pi.x, ey = pos[j].y - pi.y, ez = pos[j].z - pi.z;
      if (dot3(ex, ey, ez, ex, ey, ez) >= H2) return;
      qx[l] = qx[l] + vel[j].x; qy[l] = qy[l] + vel[j].y; qz[l] = qz[l] + vel[j].z;
      qm[l] = qm[l] + LIT(1.0);
    }, GLF);
    const R sx = lane_reduce_g<GLF>(qx), sy = lane_reduce_g<GLF>(qy), sz = lane_reduce_g<GLF>(qz),
            m = lane_reduce_g<GLF>(qm);
    R vx = vel[i].x, vy = vel[i].y, vz = vel[i].z;
    if (m > 0) {
      vx = vx + P.viscosity * (sx / m - vx);
      vy = vy + P.viscosity * (sy / m - vy);
      vz = vz + P.viscosity * (sz / m - vz);
    }
    delta[i] = V4<R>{vx, vy, vz, m};
  }
}

// xsphApply, src/gpu/wgsl.js:773-778
template <class R> void O2Sim<R>::passXsphApply() {
  for (int i = S; i < N; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    vel[i] = V4<R>{delta[i].x, delta[i].y, delta[i].z, 0};
  }
}

// Wedge cut with the arithmetic of Solver.cut, src/solver.js:458-486, over
// the constraint buffer (kernel shape of src/gpu/wgsl.js:804-823).
template <class R> uint32_t O2Sim<R>::passCut(const Cut& k) {
  const double ox = k.o[0], oy = k.o[1], oz = k.o[2];
  const double d1x = k.d1[0], d1y = k.d1[1], d1z = k.d1[2];
  const double d2x = k.d2[0], d2y = k.d2[1], d2z = k.d2[2];
  const double nx = d1y * d2z - d1z * d2y;
  const double ny = d1z * d2x - d1x * d2z;
  const double nz = d1x * d2y - d1y * d2x;
  const double nLen = std::sqrt(nx * nx + ny * ny + nz * nz);
  if (nLen < 1e-8) return 0;
  uint32_t cuts = 0;
  for (int c = 0; c < C; c++) {
    if (!consAlive[c]) continue;
    const V4<R>& A = pos[consA[c]];
    const V4<R>& B = pos[consB[c]];
    const double ax = (double)A.x, ay = (double)A.y, az = (double)A.z;
    const double bx = (double)B.x, by = (double)B.y, bz = (double)B.z;
    const double sa = (ax - ox) * nx + (ay - oy) * ny + (az - oz) * nz;
    const double sb = (bx - ox) * nx + (by - oy) * ny + (bz - oz) * nz;
    if (sa * sb >= 0) continue;
    const double t = sa / (sa - sb);
    const double px = ax + (bx - ax) * t - ox;
    const double py = ay + (by - ay) * t - oy;
    const double pz = az + (bz - az) * t - oz;
    const double c1 = (d1y * pz - d1z * py) * nx + (d1z * px - d1x * pz) * ny +
                      (d1x * py - d1y * px) * nz;
    const double c2 = (py * d2z - pz * d2y) * nx + (pz * d2x - px * d2z) * ny +
                      (px * d2y - py * d2x) * nz;
    if (c1 < 0 || c2 < 0) continue;
    consAlive[c] = 0;
    cuts++;
  }
  return cuts;
}

// cutTets, src/gpu/wgsl.js:494-519 (f32 wedge, as the reference kernel)
template <class R> void O2Sim<R>::passCutTets(const Cut& k) {
  const R ox = (R)(float)k.o[0], oy = (R)(float)k.o[1], oz = (R)(float)k.o[2];
  const R ax1 = (R)(float)k.d1[0], ay1 = (R)(float)k.d1[1], az1 = (R)(float)k.d1[2];
  const R ax2 = (R)(float)k.d2[0], ay2 = (R)(float)k.d2[1], az2 = (R)(float)k.d2[2];
  R nx, ny, nz;
  cross3(ax1, ay1, az1, ax2, ay2, az2, nx, ny, nz);
  if (dot3(nx, ny, nz, nx, ny, nz) < LIT(1e-16)) return;
  for (int t = 0; t < NT; t++) {
    const R V0 = tetVol[t];
    if (V0 <= 0) continue;
    bool dead = false;
    for (int p = 0; p < 3 && !dead; p++)
      for (int q = p + 1; q < 4; q++) {
        const V4<R>& A = pos[tetIdx[4 * t + p]];
        const V4<R>& B = pos[tetIdx[4 * t + q]];
        const R pax = A.x - ox, pay = A.y - oy, paz = A.z - oz;
        const R pbx = B.x - ox, pby = B.y - oy, pbz = B.z - oz;
        const R sa = dot3(pax, pay, paz, nx, ny, nz);
        const R sb = dot3(pbx, pby, pbz, nx, ny, nz);
        if (sa * sb >= 0) continue;
        const R tt = sa / (sa - sb);
        const R ppx = pax + (pbx - pax) * tt, ppy = pay + (pby - pay) * tt, ppz = paz + (pbz - paz) * tt;
        R cx, cy, cz;
        cross3(ax1, ay1, az1, ppx, ppy, ppz, cx, cy, cz);
        if (dot3(cx, cy, cz, nx, ny, nz) < 0) continue;
        cross3(ppx, ppy, ppz, ax2, ay2, az2, cx, cy, cz);
        if (dot3(cx, cy, cz, nx, ny, nz) < 0) continue;
        dead = true;
        break;
      }
    if (dead) tetVol[t] = -V0;
  }
}

// One substep, GpuSim.encode's loop body, src/gpu/sim.js:354-385.
template <class R> void O2Sim<R>::substep(R h, int lastPass) {
  P.h = h;
  const bool tets = (features & UPBD_FEAT_TETS) != 0;
  const bool scc = (features & UPBD_FEAT_SOLID_CONTACTS) != 0;
  if (lastPass < UPBD_PASS_INTEGRATE) return;
  passIntegrate();
  if (lastPass < UPBD_PASS_GRID) return;
  passGrid();
  if (lastPass < UPBD_PASS_DENSITY) return;
  passDensity();
  if (lastPass < UPBD_PASS_DISP) return;
  passDisp();
  if (lastPass < UPBD_PASS_APPLY_FLUID) return;
  passApplyFluid();
  if (lastPass < UPBD_PASS_SOLID) return;
  if (scc) passCollectContacts();
  for (int it = 0; it < iters; it++) {
    passSolidSolve();
    passApplySolid();
    if (tets) {
      passSolveTets();
      passApplySolidContacts();
    }
    if (scc) {
      passSolidContacts();
      passApplySolidContacts();
    }
  }
  if (lastPass < UPBD_PASS_BONDS) return;
  passBondUpdate();
  if (tets) passTetUpdate();
  if (lastPass < UPBD_PASS_CONTACTS) return;
  passContacts();
  if (lastPass < UPBD_PASS_APPLY_ALL) return;
  passApplyAll();
  if (lastPass < UPBD_PASS_BOUNDS) return;
  passBounds();
  if (lastPass < UPBD_PASS_VELOCITY) return;
  passVelocity();
  if (lastPass < UPBD_PASS_SOLID_VISC) return;
  if (P.solidViscosity > 0) {
    passSolidVisc();
    passSolidViscApply();
  }
  if (lastPass < UPBD_PASS_XSPH) return;
  passXsph();
  if (lastPass < UPBD_PASS_XSPH_APPLY) return;
  passXsphApply();
}

// One frame: GpuSim.encode, src/gpu/sim.js:333-398, with substep hd.
template <class R> void O2Sim<R>::step(double dt, int nsub) { stepH(dt / nsub, nsub); }

template <class R> void O2Sim<R>::stepH(double hd, int nsub) {
  bool cutThisFrame = false;
  Cut cutNow{};
  if (!cuts.empty()) {
    cutNow = cuts.front();
    cuts.pop_front();
    cutThisFrame = true;
  }
  grabDeltaSub = V3<R>{(R)(grabDelta[0] / nsub), (R)(grabDelta[1] / nsub), (R)(grabDelta[2] / nsub)};
  if (emitPending && emit.count > 0) passEmit();
  for (int s = 0; s < nsub; s++) substep((R)hd);
  if (cutThisFrame) {
    passCut(cutNow);
    if (features & UPBD_FEAT_TETS) passCutTets(cutNow);
  }
  if (emitPending) {
    fluidNext = (fluidNext + emit.count) % F;
    emitPending = false;
  }
  grabDelta[0] = grabDelta[1] = grabDelta[2] = 0;
  grabDeltaSub = V3<R>{0, 0, 0};
  frames++;
}

template <class R> void O2Sim<R>::frame() { stepH(prm.h, substeps); }

// Solver.pickSolid, src/solver.js:502-515 (active solids).
template <class R>
int O2Sim<R>::pick(const double ro[3], const double rd[3], double maxPerp, double* tOut) const {
  int best = -1;
  double bestT = INFINITY;
  for (int i = 0; i < S; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    const double px = (double)pos[i].x - ro[0], py = (double)pos[i].y - ro[1],
                 pz = (double)pos[i].z - ro[2];
    const double t = px * rd[0] + py * rd[1] + pz * rd[2];
    if (t < 0 || t >= bestT) continue;
    const double qx = px - rd[0] * t, qy = py - rd[1] * t, qz = pz - rd[2] * t;
    if (qx * qx + qy * qy + qz * qz > maxPerp * maxPerp) continue;
    best = i;
    bestT = t;
  }
  if (tOut) *tOut = bestT;
  return best;
}

// grabSelect, src/gpu/wgsl.js:843-865
template <class R> void O2Sim<R>::grabSelect(const float c[3], float radius, uint32_t lattice) {
  const R cx = c[0], cy = c[1], cz = c[2], cw = radius;
  for (int i = 0; i < S; i++) {
    if (!(flags[i] & F_ACTIVE)) continue;
    const uint32_t lat = (i >= N1) ? 1u : 0u;
    if (lattice != 0xffffu && lat != lattice) continue;
    const R dx = pos[i].x - cx, dy = pos[i].y - cy, dz = pos[i].z - cz;
    const R q2 = dot3(dx, dy, dz, dx, dy, dz) / (cw * cw);
    if (q2 < LIT(1.0)) {
      flags[i] |= F_GRABBED;
      const R w = (LIT(1.0) - q2) * (LIT(1.0) - q2) * LIT(0.95) + LIT(0.05);
      prev[i].w = pos[i].x;
      vel[i].w = pos[i].y;
      density[i] = V2<R>{pos[i].z, w};
    }
  }
}

template <class R>
void O2Sim<R>::grabIndices(const uint32_t* idx, int n, const float* w, const float* t3) {
  for (int k = 0; k < n; k++) {
    const uint32_t i = idx[k];
    if (i >= (uint32_t)S || !(flags[i] & F_ACTIVE)) continue;
    flags[i] |= F_GRABBED;
    prev[i].w = t3 ? (R)t3[3 * k] : pos[i].x;
    vel[i].w = t3 ? (R)t3[3 * k + 1] : pos[i].y;
    density[i] = V2<R>{t3 ? (R)t3[3 * k + 2] : pos[i].z, w ? (R)w[k] : LIT(1.0)};
  }
}

// grabRelease, src/gpu/wgsl.js:867-871
template <class R> void O2Sim<R>::release() {
  for (int i = 0; i < S; i++) flags[i] &= ~F_GRABBED;
}

// Solver.emitFluid, src/solver.js:139-149, for n particles.
template <class R>
void O2Sim<R>::emitParticles(int n, const float* p3, const float* v3, double mass) {
  for (int k = 0; k < n; k++) {
    const int i = S + fluidNext;
    fluidNext = (fluidNext + 1) % F;
    const R x = p3[3 * k], y = p3[3 * k + 1], z = p3[3 * k + 2];
    pos[i] = V4<R>{x, y, z, (R)(float)(1 / mass)};
    prev[i] = V4<R>{x, y, z, 0};
    vel[i] = V4<R>{(R)v3[3 * k], (R)v3[3 * k + 1], (R)v3[3 * k + 2], 0};
    flags[i] = F_ACTIVE;
  }
}

// Solver._recomputeGroups, src/solver.js:488-499
template <class R> void O2Sim<R>::groups(int32_t* out) const {
  std::vector<int32_t> parent(S);
  std::iota(parent.begin(), parent.end(), 0);
  auto find = [&parent](int x) {
    while (parent[x] != x) {
      parent[x] = parent[parent[x]];
      x = parent[x];
    }
    return x;
  };
  for (int c = 0; c < C; c++) {
    if (!consAlive[c]) continue;
    const int ra = find((int)consA[c]), rb = find((int)consB[c]);
    if (ra != rb) parent[ra] = rb;
  }
  for (int i = 0; i < S; i++) out[i] = find(i);
}

template struct O2Sim<float>;
template struct O2Sim<double>;

}  // namespace oracle
