// Host-side scene construction shared by the single-scene handle and the
// batch of scenes (declarations and contracts in upbd_scene.h).
#include "upbd_scene.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>

namespace upbd {

void build_scene(const upbd_scene_desc& d, HostScene& out) {
  const int n1 = d.solid_dim, n2 = d.solid_dim2;
  out.N1 = n1 * n1 * n1;
  out.S = out.N1 + n2 * n2 * n2;
  out.N = out.S + d.max_fluid;
  out.pos.assign(out.N, make_float4(0, 0, 0, 0));
  const double sp = d.spacing;
  const double maxD2 = 3 * sp * sp + 1e-9;
  std::vector<uint32_t> ca, cb;
  std::vector<double> crest;
  std::vector<std::vector<uint32_t>> inc(out.S);
  int id = 0;
  auto add_lattice = [&](int dim, const double* c) {
    const int base = id;
    const double half = (dim - 1) * sp / 2;
    for (int ix = 0; ix < dim; ix++)
      for (int iy = 0; iy < dim; iy++)
        for (int iz = 0; iz < dim; iz++) {
          out.pos[id] = make_float4((float)(c[0] - half + ix * sp), (float)(c[1] - half + iy * sp),
                                    (float)(c[2] - half + iz * sp), (float)(1 / d.solid_mass));
          id++;
        }
    for (int ix = 0; ix < dim; ix++)
      for (int iy = 0; iy < dim; iy++)
        for (int iz = 0; iz < dim; iz++)
          for (int dx = -1; dx <= 1; dx++)
            for (int dy = -1; dy <= 1; dy++)
              for (int dz = -1; dz <= 1; dz++) {
                const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
                if (jx < 0 || jy < 0 || jz < 0 || jx >= dim || jy >= dim || jz >= dim) continue;
                const int a = base + (ix * dim + iy) * dim + iz;
                const int b = base + (jx * dim + jy) * dim + jz;
                if (b <= a) continue;
                const double d2 = (double)(dx * dx + dy * dy + dz * dz) * sp * sp;
                if (d2 > maxD2) continue;
                const uint32_t cidx = (uint32_t)ca.size();
                ca.push_back(a);
                cb.push_back(b);
                crest.push_back(std::sqrt(d2));
                inc[a].push_back(cidx);
                inc[b].push_back(cidx);
              }
  };
  auto signed_vol = [&](int a, int b, int c, int e) {
    auto comp = [&](int p, int q, int k) {
      const float* fp = &out.pos[p].x;
      const float* fq = &out.pos[q].x;
      return (double)fq[k] - fp[k];
    };
    const double abx = comp(a, b, 0), aby = comp(a, b, 1), abz = comp(a, b, 2);
    const double acx = comp(a, c, 0), acy = comp(a, c, 1), acz = comp(a, c, 2);
    const double adx = comp(a, e, 0), ady = comp(a, e, 1), adz = comp(a, e, 2);
    return (aby * acz - abz * acy) * adx + (abz * acx - abx * acz) * ady + (abx * acy - aby * acx) * adz;
  };
  auto add_tets = [&](int dim, int base) {
    auto idx = [&](int x, int y, int z) { return base + (x * dim + y) * dim + z; };
    for (int ix = 0; ix < dim - 1; ix++)
      for (int iy = 0; iy < dim - 1; iy++)
        for (int iz = 0; iz < dim - 1; iz++) {
          const int A = idx(ix, iy, iz), B = idx(ix + 1, iy, iz), C = idx(ix + 1, iy + 1, iz),
                    D = idx(ix, iy + 1, iz), E = idx(ix, iy, iz + 1), F = idx(ix + 1, iy, iz + 1),
                    G = idx(ix + 1, iy + 1, iz + 1), H = idx(ix, iy + 1, iz + 1);
          // five tets per cell, mirrored on checkerboard parity (sim.js:161-163)
          const int even[5][4] = {{A, C, F, H}, {A, B, C, F}, {A, C, D, H}, {A, E, F, H}, {C, F, G, H}};
          const int odd[5][4] = {{B, D, E, G}, {A, B, D, E}, {B, C, D, G}, {D, E, H, G}, {B, E, F, G}};
          const int(*five)[4] = ((ix + iy + iz) % 2 == 0) ? even : odd;
          for (int t = 0; t < 5; t++) {
            for (int q = 0; q < 4; q++) out.tet_idx.push_back((uint32_t)five[t][q]);
            out.tet_vol.push_back((float)(signed_vol(five[t][0], five[t][1], five[t][2], five[t][3]) / 6));
          }
        }
  };
  if (n1 > 0) {
    add_lattice(n1, d.cube_center);
    add_tets(n1, 0);
  }
  if (n2 > 0) {
    add_lattice(n2, d.cube2_center);
    add_tets(n2, out.N1);
  }
  for (int i = out.S; i < out.N; i++) out.pos[i].w = (float)(1 / d.fluid_mass);
  const int C = (int)ca.size();
  out.cons.resize(C);
  for (int c = 0; c < C; c++) {
    const float r = (float)crest[c];
    uint32_t bits;
    std::memcpy(&bits, &r, 4);
    out.cons[c] = make_uint4(ca[c], cb[c], bits, 1u);
  }
  out.adj.assign(out.S + 1 + 2 * (size_t)C, 0);
  uint32_t off = 0;
  for (int i = 0; i < out.S; i++) {
    out.adj[i] = off;
    for (uint32_t c : inc[i]) out.adj[out.S + 1 + off++] = c;
  }
  out.adj[out.S] = off;
  // CSR-parallel static data of the Jacobi gather: the other endpoint of each
  // incident constraint and the pair scale 1/max(deg_i, deg_j) of
  // src/gpu/wgsl.js:340-354 (endpoints and degrees never change)
  out.adj_other.assign(2 * (size_t)C, 0);
  out.adj_scale.assign(2 * (size_t)C, 0.f);
  for (int i = 0; i < out.S; i++) {
    const uint32_t degI = out.adj[i + 1] - out.adj[i];
    for (uint32_t k = out.adj[i]; k < out.adj[i + 1]; k++) {
      const uint32_t c = out.adj[out.S + 1 + k];
      const uint32_t other = (ca[c] == (uint32_t)i) ? cb[c] : ca[c];
      const uint32_t degJ = out.adj[other + 1] - out.adj[other];
      out.adj_other[k] = other;
      out.adj_scale[k] = 1.0f / (float)((degI < degJ) ? degJ : degI);
    }
  }
  const int NT = (int)out.tet_vol.size();
  std::vector<std::vector<uint32_t>> tinc(out.S);
  for (int t = 0; t < NT; t++)
    for (int q = 0; q < 4; q++) tinc[out.tet_idx[4 * t + q]].push_back(t);
  out.tet_adj.assign(out.S + 1 + 4 * (size_t)NT, 0);
  off = 0;
  for (int i = 0; i < out.S; i++) {
    out.tet_adj[i] = off;
    for (uint32_t t : tinc[i]) out.tet_adj[out.S + 1 + off++] = t;
  }
  out.tet_adj[out.S] = off;
}

namespace {
struct Carver {
  size_t off = 0;
  template <class T> size_t take(size_t count) {
    const size_t o = off;
    off += ((count * sizeof(T) + 255) / 256) * 256;
    return o;
  }
};
}  // namespace

SceneLayout layout_scene(const upbd_scene_desc& d, const HostScene& hs, SimView& v) {
  v = SimView{};
  v.S = hs.S;
  v.N1 = hs.N1;
  v.dim1 = d.solid_dim;
  v.dim2 = d.solid_dim2;
  v.F = d.max_fluid;
  v.N = hs.S + d.max_fluid;
  v.C = (int)hs.cons.size();
  v.NT = (int)hs.tet_vol.size();
  v.T = d.table_size;
  v.num_tiles = (v.T + SCAN_TILE - 1) / SCAN_TILE;
  const bool scc = (d.features & UPBD_FEAT_SOLID_CONTACTS) != 0;
  Carver cv;
  SceneLayout L{};
  L.pos = cv.take<real4>(v.N);
  L.prev = cv.take<real4>(v.N);
  L.vel = cv.take<real4>(v.N);
  L.delta = cv.take<real4>(v.N);
  L.dens = cv.take<real2>(v.N);
  L.flags = cv.take<uint32_t>(v.N);
  L.cons = cv.take<uint4>(std::max(v.C, 1));
  L.adj = cv.take<uint32_t>(hs.adj.size());
  L.counts = cv.take<uint32_t>(v.T);
  L.start = cv.take<uint32_t>(v.T + 1);
  L.entries = cv.take<uint32_t>(v.N);
  L.tmp = cv.take<uint32_t>(v.N);
  L.ticket = cv.take<uint32_t>(v.N);
  L.cell = cv.take<uint32_t>(v.N);
  L.tiles = cv.take<uint32_t>(tile_words(v.num_tiles));
  L.tidx = cv.take<uint32_t>(4 * (size_t)std::max(v.NT, 1));
  L.tvol = cv.take<float>(std::max(v.NT, 1));
  L.tadj = cv.take<uint32_t>(hs.tet_adj.size());
  L.mark = cv.take<uint32_t>(v.N);
  L.spos = cv.take<real4>(v.N);
  L.sdens = cv.take<real2>(v.N);
  L.svel = cv.take<real4>(v.N);
  L.slot = cv.take<uint32_t>(v.N);
  L.fend = cv.take<uint32_t>(v.T);
  L.nbr = cv.take<uint32_t>(std::max<size_t>((size_t)v.N * GLF * NL, 1));
  L.ncount = cv.take<uint32_t>(std::max<size_t>((size_t)v.N * GLF, 1));
  L.aoth = cv.take<uint32_t>(std::max<size_t>(hs.adj_other.size(), 1));
  L.ascl = cv.take<float>(std::max<size_t>(hs.adj_scale.size(), 1));
  L.ccount = cv.take<uint32_t>(scc ? std::max(v.S, 1) : 1);
  L.clist = cv.take<uint32_t>(scc ? (size_t)std::max(v.S, 1) * C_K : 1);
  L.sbuf = cv.take<real4>(2 * (size_t)std::max(v.S, 1));
  L.sfp = cv.take<real4>(v.N);
  L.smove = cv.take<float>(v.N);
  L.bmove = cv.take<uint32_t>(v.T);
  L.scr = cv.take<uint32_t>(SCR_WORDS);
  L.par = cv.take<DevParams>(1);
#ifdef UPBD_FP64_BUILD
  L.conv = cv.take<float4>(v.N);
#else
  L.conv = 0;
#endif
  L.bytes = cv.off;
  return L;
}

void bind_scene(const SceneLayout& L, char* base, SimView& v, DevParams** params) {
  v.pos = (real4*)(base + L.pos);
  v.prev = (real4*)(base + L.prev);
  v.vel = (real4*)(base + L.vel);
  v.delta = (real4*)(base + L.delta);
  v.density = (real2*)(base + L.dens);
  v.flags = (uint32_t*)(base + L.flags);
  v.cons = (uint4*)(base + L.cons);
  v.adj = (const uint32_t*)(base + L.adj);
  v.counts = (uint32_t*)(base + L.counts);
  v.start = (uint32_t*)(base + L.start);
  v.entries = (uint32_t*)(base + L.entries);
  v.tmp = (uint32_t*)(base + L.tmp);
  v.ticket = (uint32_t*)(base + L.ticket);
  v.cell = (uint32_t*)(base + L.cell);
  v.tile_sum = (uint32_t*)(base + L.tiles);
  v.tet_idx = (uint32_t*)(base + L.tidx);
  v.tet_vol = (float*)(base + L.tvol);
  v.tet_adj = (const uint32_t*)(base + L.tadj);
  v.mark = (uint32_t*)(base + L.mark);
  v.spos = (real4*)(base + L.spos);
  v.sdens = (real2*)(base + L.sdens);
  v.svel = (real4*)(base + L.svel);
  v.slot = (uint32_t*)(base + L.slot);
  v.fend = (uint32_t*)(base + L.fend);
  v.nbr = (uint32_t*)(base + L.nbr);
  v.ncount = (uint32_t*)(base + L.ncount);
  v.adj_other = (const uint32_t*)(base + L.aoth);
  v.adj_scale = (const float*)(base + L.ascl);
  v.ccount = (uint32_t*)(base + L.ccount);
  v.clist = (uint32_t*)(base + L.clist);
  v.sbuf = (real4*)(base + L.sbuf);
  v.sfp = (real4*)(base + L.sfp);
  v.smove = (float*)(base + L.smove);
  v.bmove = (uint32_t*)(base + L.bmove);
  v.scratch = (uint32_t*)(base + L.scr);
#ifdef UPBD_FP64_BUILD
  v.conv = (float*)(base + L.conv);
#endif
  if (params) *params = (DevParams*)(base + L.par);
}

#ifdef UPBD_FP64_BUILD
namespace {
__global__ void k_widen(double* dst, const float* src, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (double)src[i];
}
__global__ void k_narrow(float* dst, const double* src, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (float)src[i];
}
unsigned conv_blocks(size_t n) { return (unsigned)((n + 255) / 256); }
}  // namespace

cudaError_t state_to_device(real* dst, const float* src_host, size_t rows, int comps, const SimView& v,
                            cudaStream_t st) {
  const size_t n = rows * (size_t)comps;
  if (n == 0) return cudaSuccess;
  if (n > (size_t)v.N * 4) return cudaErrorInvalidValue;
  cudaError_t e = cudaMemcpyAsync(v.conv, src_host, n * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  k_widen<<<conv_blocks(n), 256, 0, st>>>(dst, v.conv, n);
  return cudaPeekAtLastError();
}

cudaError_t state_to_host(float* dst_host, const real* src, size_t rows, int comps, const SimView& v,
                          cudaStream_t st) {
  const size_t n = rows * (size_t)comps;
  if (n == 0) return cudaSuccess;
  if (n > (size_t)v.N * 4) return cudaErrorInvalidValue;
  k_narrow<<<conv_blocks(n), 256, 0, st>>>(v.conv, src, n);
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) return e;
  return cudaMemcpyAsync(dst_host, v.conv, n * sizeof(float), cudaMemcpyDeviceToHost, st);
}

cudaError_t state_to_f32(float* dst_dev, const real* src, size_t rows, int comps, cudaStream_t st) {
  const size_t n = rows * (size_t)comps;
  if (n == 0) return cudaSuccess;
  k_narrow<<<conv_blocks(n), 256, 0, st>>>(dst_dev, src, n);
  return cudaPeekAtLastError();
}
#else
cudaError_t state_to_device(real* dst, const float* src_host, size_t rows, int comps, const SimView&,
                            cudaStream_t st) {
  const size_t bytes = rows * (size_t)comps * sizeof(float);
  return bytes ? cudaMemcpyAsync(dst, src_host, bytes, cudaMemcpyHostToDevice, st) : cudaSuccess;
}

cudaError_t state_to_host(float* dst_host, const real* src, size_t rows, int comps, const SimView&,
                          cudaStream_t st) {
  const size_t bytes = rows * (size_t)comps * sizeof(float);
  return bytes ? cudaMemcpyAsync(dst_host, src, bytes, cudaMemcpyDeviceToHost, st) : cudaSuccess;
}

cudaError_t state_to_f32(float* dst_dev, const real* src, size_t rows, int comps, cudaStream_t st) {
  const size_t bytes = rows * (size_t)comps * sizeof(float);
  return bytes ? cudaMemcpyAsync(dst_dev, src, bytes, cudaMemcpyDeviceToDevice, st) : cudaSuccess;
}
#endif

cudaError_t upload_scene(const HostScene& hs, const SimView& v, cudaStream_t st) {
  cudaError_t e = cudaMemcpyAsync((void*)v.adj, hs.adj.data(), hs.adj.size() * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !hs.adj_other.empty())
    e = cudaMemcpyAsync((void*)v.adj_other, hs.adj_other.data(), hs.adj_other.size() * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !hs.adj_scale.empty())
    e = cudaMemcpyAsync((void*)v.adj_scale, hs.adj_scale.data(), hs.adj_scale.size() * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !hs.tet_adj.empty())
    e = cudaMemcpyAsync((void*)v.tet_adj, hs.tet_adj.data(), hs.tet_adj.size() * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !hs.tet_idx.empty())
    e = cudaMemcpyAsync(v.tet_idx, hs.tet_idx.data(), hs.tet_idx.size() * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = state_to_device((real*)v.pos, (const float*)hs.pos.data(), hs.pos.size(), 4, v, st);
  if (e == cudaSuccess) e = state_to_device((real*)v.prev, (const float*)hs.pos.data(), hs.pos.size(), 4, v, st);
  if (e == cudaSuccess && v.C > 0)
    e = cudaMemcpyAsync(v.cons, hs.cons.data(), (size_t)v.C * 16, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && v.NT > 0)
    e = cudaMemcpyAsync(v.tet_vol, hs.tet_vol.data(), (size_t)v.NT * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && v.S > 0) {
    // solids active; a fill kernel would do, but this keeps the unit host-only
    std::vector<uint32_t> f((size_t)v.S, F_ACTIVE);
    e = cudaMemcpyAsync(v.flags, f.data(), (size_t)v.S * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // f is a stack buffer
  }
  return e;
}

namespace {
struct LatticeKey {
  int dim1, dim2;
  double spacing, solid_mass, c1[3], c2[3];
  bool operator<(const LatticeKey& o) const { return std::memcmp(this, &o, sizeof(*this)) < 0; }
};
std::mutex g_lat_mu;
std::map<LatticeKey, std::shared_ptr<const HostScene>> g_lat;
constexpr size_t kLatticeCacheMax = 128;
}  // namespace

std::shared_ptr<const HostScene> lattice_of(const upbd_scene_desc& d) {
  LatticeKey k;
  std::memset(&k, 0, sizeof(k));
  k.dim1 = d.solid_dim;
  k.dim2 = d.solid_dim2;
  k.spacing = d.spacing;
  k.solid_mass = d.solid_mass;
  for (int i = 0; i < 3; i++) {
    k.c1[i] = d.cube_center[i];
    k.c2[i] = d.solid_dim2 > 0 ? d.cube2_center[i] : 0.0;
  }
  {
    std::lock_guard<std::mutex> lk(g_lat_mu);
    auto it = g_lat.find(k);
    if (it != g_lat.end()) return it->second;
  }
  upbd_scene_desc ld = d;
  ld.max_fluid = 0;
  auto hs = std::make_shared<HostScene>();
  build_scene(ld, *hs);
  std::lock_guard<std::mutex> lk(g_lat_mu);
  if (g_lat.size() >= kLatticeCacheMax) g_lat.clear();
  return g_lat.emplace(k, std::move(hs)).first->second;
}

const char* prepare_scene(const upbd_scene_desc& d, const upbd_params& p, int n_fluid, const float* pos3,
                          const float* vel3, double mass, PreparedScene& out) {
  if (const char* why = check_desc(&d, &p)) return why;
  if (n_fluid < 0 || n_fluid > d.max_fluid) return "n_fluid exceeds max_fluid";
  if (n_fluid > 0 && (!pos3 || !(mass > 0))) return "fluid positions and a positive mass are required";
  out.desc = d;
  out.prm = p;
  out.lat = lattice_of(d);
  out.n_fluid = n_fluid;
  const float w_slot = d.max_fluid > 0 ? (float)(1 / d.fluid_mass) : 0.f;
  const float w_placed = n_fluid > 0 ? (float)(1 / mass) : 0.f;
  out.fluid_pos.assign(d.max_fluid, make_float4(0.f, 0.f, 0.f, w_slot));
  out.fluid_prev.assign(d.max_fluid, make_float4(0.f, 0.f, 0.f, w_slot));
  for (int k = 0; k < n_fluid; k++) {
    const float x = pos3[3 * k], y = pos3[3 * k + 1], z = pos3[3 * k + 2];
    out.fluid_pos[k] = make_float4(x, y, z, w_placed);
    out.fluid_prev[k] = make_float4(x, y, z, 0.f);
  }
  out.fluid_vel.clear();
  if (vel3 && n_fluid > 0) {
    out.fluid_vel.resize(n_fluid);
    for (int k = 0; k < n_fluid; k++)
      out.fluid_vel[k] = make_float4(vel3[3 * k], vel3[3 * k + 1], vel3[3 * k + 2], 0.f);
  }
  return nullptr;
}

cudaError_t upload_prepared(const PreparedScene& ps, const SimView& v, cudaStream_t st) {
  const HostScene& L = *ps.lat;
  const int S = v.S;
  auto up = [&](void* dst, const void* src, size_t bytes) {
    return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st) : cudaSuccess;
  };
  cudaError_t e = up((void*)v.adj, L.adj.data(), L.adj.size() * 4);
  if (e == cudaSuccess) e = up((void*)v.adj_other, L.adj_other.data(), L.adj_other.size() * 4);
  if (e == cudaSuccess) e = up((void*)v.adj_scale, L.adj_scale.data(), L.adj_scale.size() * 4);
  if (e == cudaSuccess) e = up((void*)v.tet_adj, L.tet_adj.data(), L.tet_adj.size() * 4);
  if (e == cudaSuccess) e = up(v.tet_idx, L.tet_idx.data(), L.tet_idx.size() * 4);
  if (e == cudaSuccess) e = up(v.cons, L.cons.data(), L.cons.size() * 16);
  if (e == cudaSuccess) e = up(v.tet_vol, L.tet_vol.data(), L.tet_vol.size() * 4);
  auto rows = [&](real4* dst, const std::vector<float4>& src, size_t n) {
    return n ? state_to_device((real*)dst, (const float*)src.data(), n, 4, v, st) : cudaSuccess;
  };
  if (e == cudaSuccess) e = rows(v.pos, L.pos, (size_t)S);
  if (e == cudaSuccess) e = rows(v.prev, L.pos, (size_t)S);
  if (e == cudaSuccess) e = rows(v.pos + S, ps.fluid_pos, ps.fluid_pos.size());
  if (e == cudaSuccess) e = rows(v.prev + S, ps.fluid_prev, ps.fluid_prev.size());
  if (e == cudaSuccess) e = rows(v.vel + S, ps.fluid_vel, ps.fluid_vel.size());
  if (e == cudaSuccess && S + ps.n_fluid > 0) {
    // solids and placed fluid active (a pageable copy: staged before return)
    std::vector<uint32_t> f((size_t)S + ps.n_fluid, F_ACTIVE);
    e = up(v.flags, f.data(), f.size() * 4);
  }
  return e;
}

const char* check_desc(const upbd_scene_desc* d, const upbd_params* p) {
  if (!d || !p) return "null descriptor";
  if (d->solid_dim < 0 || d->solid_dim > 256 || d->solid_dim2 < 0 || d->solid_dim2 > 256)
    return "solid_dim out of range [0, 256]";
  if (d->max_fluid < 0 || d->max_fluid > (1 << 28)) return "max_fluid out of range";
  if (d->table_size < 1 || (d->table_size & (d->table_size - 1)) || d->table_size > (1 << 28))
    return "table_size must be a power of two <= 2^28";
  if (d->substeps < 1 || d->solid_iters < 0 || d->solid_iters > 1000) return "substeps/solid_iters out of range";
  if (d->solid_dim > 0 && !(d->solid_mass > 0)) return "solid_mass must be > 0";
  if (d->max_fluid > 0 && !(d->fluid_mass > 0)) return "fluid_mass must be > 0";
  if (!(p->cell_size > 0)) return "cell_size must be > 0";
  const long long total = (long long)d->solid_dim * d->solid_dim * d->solid_dim +
                          (long long)d->solid_dim2 * d->solid_dim2 * d->solid_dim2 + d->max_fluid;
  if (total < 1 || total > (1ll << 29)) return "particle count out of range";
  return nullptr;
}

void fill_dev_params(const upbd_params& p, const upbd_scene_desc& desc, DevParams& d) {
  d.h = (float)p.h;
  d.gravity = (float)p.gravity;
  d.solid_radius = (float)p.solid_radius;
  d.fluid_radius = (float)p.fluid_radius;
  d.fluid_h = (float)p.fluid_h;
  d.rest_density = (float)p.rest_density;
  d.stiffness = (float)p.stiffness;
  d.near_stiffness = (float)p.near_stiffness;
  d.viscosity = (float)p.viscosity;
  d.compliance = (float)p.compliance;
  d.omega = (float)p.omega;
  d.plastic_threshold = (float)p.plastic_threshold;
  d.plastic_rate = (float)p.plastic_rate;
  d.tear_gap = (float)p.tear_gap;
  d.max_speed = (float)p.max_speed;
  d.wall_x = (float)p.wall_x;
  d.wall_z = (float)p.wall_z;
  d.wall_h = (float)p.wall_h;
  d.wall_t = (float)p.wall_t;
  d.cull_r = (float)p.cull_r;
  d.damp_solid = (float)p.damp_solid;
  d.damp_fluid = (float)p.damp_fluid;
  d.friction_solid = (float)p.friction_solid;
  d.friction_fluid = (float)p.friction_fluid;
  d.grab_k = (float)p.grab_k;
  d.spacing = (float)desc.spacing;
  d.solid_viscosity = (float)p.solid_viscosity;
  d.break_strain = (float)p.break_strain;
  d.contact_scale = (float)p.contact_scale;
  d.inv_cell = 1.0 / p.cell_size;  // Solver._hashPos: 1 / cellSize in double
  d.tear_mode = p.tear_mode;
  d.plastic_clamp = p.plastic_clamp;
  // solid<->fluid contacts only within adjacent cells: the marking shortcut is
  // exact (the marked set only grows by the 1e-5 slack of mark_fluid_near)
  const double rsum = (double)(d.solid_radius + d.fluid_radius);
  d.use_mark = (rsum * 1.0001 < p.cell_size * (1.0 - 1e-6)) ? 1 : 0;
}

}  // namespace upbd
