// Scene batch of libupbd.so (C ABI in include/upbd_batch.h).
//
// Every pass of the substep runs once per frame substep for all live scenes:
// a persistent grid (ctas_per_sm x SMs CTAs) walks the "virtual blocks" of
// the pass, tile 0..k0-1 of scene 0, then scene 1's, and so on, through a
// per-scene offset table (prefix sums of each scene's tile count, one row per
// tile domain). For each virtual block a CTA finds its scene by binary search
// in the row, loads the scene's SimView and uniform block, and runs the same
// pass body the single-scene kernels run (upbd_passes.cuh) on that tile.
//
// The table, the SimViews and the uniform blocks live in one device buffer
// whose address never changes; the frame is captured once per shape into a
// CUDA graph whose kernels read the scene count from that buffer, so adding
// or removing scenes only rewrites the table (one stream-ordered copy before
// the next replay). Scene arenas come from a first-fit pool of large device
// chunks, bounded by the HBM budget.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/upbd_batch.h"
#include "upbd_batch_internal.h"
#include "upbd_kinds.h"
#include "upbd_passes.cuh"
#include "upbd_scene.h"

using namespace upbd;

namespace {

// Tile domains: which per-scene extent a pass's threads cover.
enum Domain {
  D_N,        // particles (integrate/count, rankfix, apply+bounds+velocity)
  D_TILES,    // scan tiles of the bucket table (SCAN_THREADS per block)
  D_SCATTER,  // max(particles, scan tiles)
  D_FGL,      // GLF lanes per grid slot (density, xsph)
  D_DISP,     // DL threads per grid slot (displacement)
  D_F,        // fluid particles (apply, xsph apply, active count)
  D_SOLVE0,   // solve lanes rounded to warps + fluid (first iteration)
  D_SOLVE,    // solve lanes rounded to warps
  D_SGL,      // GL lanes per solid (apply + contact marks)
  D_S,        // solids
  D_BC,       // bond/tet updates rounded to warps + GL lanes per particle
  NUM_DOMAINS
};

constexpr int kMetaWords = 64;

struct BatchArgs {
  const SimView* __restrict__ views;
  const DevParams* __restrict__ params;
  const uint32_t* __restrict__ prefix;  // [NUM_DOMAINS][stride]
  const uint32_t* __restrict__ meta;    // meta[0] = live scenes
  uint32_t stride;                      // max_scenes + 1
};

// Scene s with pre[s] <= vb < pre[s+1] (pre is non-decreasing, pre[0] = 0,
// pre[n] > vb); scenes with no tile in the domain are never returned.
__device__ __forceinline__ uint32_t find_scene(const uint32_t* __restrict__ pre, uint32_t n, uint32_t vb) {
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1u) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(pre + mid) <= vb) lo = mid;
    else hi = mid;
  }
  return lo;
}

// The persistent loop: virtual block vb = blockIdx.x, += gridDim.x, is
// uniform across the CTA, so pass bodies keep whole warps and may
// synchronize the CTA (SYNC bodies use shared memory between iterations).
// The body sees the scene's SimView as a copy or, with BYREF, in place in
// the table (its fields loaded where the body uses them): which one needs
// fewer registers depends on the body, and the kernels below choose by
// measurement.
template <int D, bool SYNC, bool BYREF = false, class Fn>
__device__ __forceinline__ void batch_loop(const BatchArgs& a, Fn&& fn) {
  const uint32_t n = __ldg(a.meta);
  const uint32_t* __restrict__ pre = a.prefix + (size_t)D * a.stride;
  const uint32_t total = (n > 0) ? __ldg(pre + n) : 0u;
  for (uint32_t vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const uint32_t s = find_scene(pre, n, vb);
    const uint32_t b0 = __ldg(pre + s);
    if constexpr (BYREF) {
      const SimView& v = a.views[s];
      fn(v, a.params + s, vb - b0, __ldg(pre + s + 1) - b0);
    } else {
      const SimView v = a.views[s];
      fn(v, a.params + s, vb - b0, __ldg(pre + s + 1) - b0);
    }
    if (SYNC) __syncthreads();
  }
}

__host__ __device__ __forceinline__ int solid_pad_of(int S) { return ((S * GL + 31) / 32) * 32; }
__host__ __device__ __forceinline__ int bond_pad_of(int C, int NT) { return ((C + NT + 31) / 32) * 32; }

#define UPBD_BODY [&](const SimView& v, const DevParams* P, uint32_t vb, uint32_t nblk)

template <bool INTEGRATE, bool COUNT>
__global__ void __launch_bounds__(256) kb_integrate_count(BatchArgs a) {
  batch_loop<D_N, false, true>(a, UPBD_BODY { b_integrate_count<INTEGRATE, COUNT>(v, P, vb); });
}
__global__ void __launch_bounds__(SCAN_THREADS) kb_scan(BatchArgs a) {
  batch_loop<D_TILES, true, true>(a, UPBD_BODY { b_scan(v, vb); });
}
__global__ void __launch_bounds__(256) kb_scatter(BatchArgs a) {
  batch_loop<D_SCATTER, false>(a, UPBD_BODY { b_scatter(v, vb); });
}
__global__ void __launch_bounds__(256) kb_rankfix(BatchArgs a) {
  batch_loop<D_N, false, true>(a, UPBD_BODY { b_rankfix(v, vb); });
}
// density and the solve are latency-bound: at most 40 registers (6 CTAs of
// 256 per SM) hides more of it than the few spilled values cost
__global__ void __launch_bounds__(256, 6) kb_density(BatchArgs a) {
  batch_loop<D_FGL, false, true>(a, UPBD_BODY { b_density(v, P, vb); });
}
template <bool APPLY>
__global__ void __launch_bounds__(256) kb_disp(BatchArgs a) {
  batch_loop<D_DISP, false>(a, UPBD_BODY { b_disp<APPLY>(v, P, vb); });
}
__global__ void __launch_bounds__(256) kb_apply_fluid(BatchArgs a) {
  batch_loop<D_F, false>(a, UPBD_BODY { b_apply_fluid(v, P, vb); });
}
template <bool APPLY_FLUID, int OUT>
__global__ void __launch_bounds__(256, 6) kb_solid_solve(BatchArgs a, int it) {
  batch_loop<APPLY_FLUID ? D_SOLVE0 : D_SOLVE, false, true>(
      a, UPBD_BODY { b_solid_solve<APPLY_FLUID, OUT>(v, P, solid_pad_of(v.S), it, vb); });
}
template <bool MARK>
__global__ void __launch_bounds__(256) kb_apply_solid(BatchArgs a) {
  batch_loop<MARK ? D_SGL : D_S, false>(a, UPBD_BODY { b_apply_solid<MARK>(v, P, vb); });
}
__global__ void __launch_bounds__(256) kb_contact_mark(BatchArgs a) {
  batch_loop<D_SGL, false>(a, UPBD_BODY { b_contact_mark(v, P, vb); });
}
__global__ void __launch_bounds__(256) kb_collect_contacts(BatchArgs a) {
  batch_loop<D_S, false>(a, UPBD_BODY { b_collect_contacts(v, P, vb); });
}
__global__ void __launch_bounds__(256) kb_solid_contacts(BatchArgs a) {
  batch_loop<D_S, false>(a, UPBD_BODY { b_solid_contacts(v, P, vb); });
}
__global__ void __launch_bounds__(256) kb_apply_solid_contacts(BatchArgs a) {
  batch_loop<D_S, false>(a, UPBD_BODY { b_apply_solid_contacts(v, P, vb); });
}
__global__ void __launch_bounds__(256) kb_solve_tets(BatchArgs a) {
  batch_loop<D_S, false>(a, UPBD_BODY { b_solve_tets(v, P, vb); });
}
__global__ void __launch_bounds__(256) kb_bond_contacts(BatchArgs a, int tets) {
  batch_loop<D_BC, false>(a, UPBD_BODY {
    const int nt = tets ? v.NT : 0;
    b_bond_contacts(v, P, v.C, nt, bond_pad_of(v.C, nt), v.N, vb);
  });
}
__global__ void __launch_bounds__(256) kb_apply_bounds_vel(BatchArgs a) {
  batch_loop<D_N, false>(a, UPBD_BODY { b_apply_bounds_vel(v, P, 3, vb); });
}
__global__ void __launch_bounds__(256) kb_solid_visc(BatchArgs a) {
  batch_loop<D_S, false>(a, UPBD_BODY {
    if (P->solid_viscosity > 0.f) b_solid_visc(v, P, vb);
  });
}
__global__ void __launch_bounds__(256) kb_solid_visc_apply(BatchArgs a) {
  batch_loop<D_S, false>(a, UPBD_BODY {
    if (P->solid_viscosity > 0.f) b_solid_visc_apply(v, vb);
  });
}
__global__ void __launch_bounds__(256) kb_xsph(BatchArgs a) {
  batch_loop<D_FGL, false>(a, UPBD_BODY { b_xsph<true>(v, P, vb); });
}
__global__ void __launch_bounds__(256) kb_count_active(BatchArgs a) {
  batch_loop<D_F, true>(a, UPBD_BODY { b_count_active(v, vb, nblk); });
}

#undef UPBD_BODY

inline uint32_t ceil_div(long long n, int bs) {
  const long long b = (n + bs - 1) / bs;
  return (uint32_t)(b < 1 ? 1 : b);
}

// Virtual blocks of one scene in every domain (block size bt; the scan's
// blocks are SCAN_THREADS wide and cover SCAN_TILE buckets each).
void scene_blocks(const SimView& v, bool tets, int bt, uint32_t out[NUM_DOMAINS]) {
  const int sp = solid_pad_of(v.S);
  const int nt = tets ? v.NT : 0;
  out[D_N] = ceil_div(v.N, bt);
  out[D_TILES] = (uint32_t)std::max(v.num_tiles, 1);
  out[D_SCATTER] = ceil_div(std::max(v.N, tile_words(v.num_tiles)), bt);
  out[D_FGL] = ceil_div((long long)v.N * GLF, bt);
  out[D_DISP] = ceil_div((long long)v.N * DL, bt);
  out[D_F] = ceil_div(v.F, bt);
  out[D_SOLVE0] = ceil_div((long long)sp + v.F, bt);
  out[D_SOLVE] = ceil_div(sp, bt);
  out[D_SGL] = ceil_div((long long)v.S * GL, bt);
  out[D_S] = ceil_div(v.S, bt);
  out[D_BC] = ceil_div((long long)bond_pad_of(v.C, nt) + (long long)v.N * GL, bt);
}

// First-fit allocator over device chunks (256-byte granules), coalescing on
// free. Chunks are allocated on demand and kept until the batch is destroyed.
class DevicePool {
 public:
  static constexpr size_t kAlign = 256;
  static constexpr size_t kChunk = size_t(1) << 30;

  ~DevicePool() { release(); }

  void release() {
    for (auto& c : chunks_) cudaFree(c.base);
    chunks_.clear();
    reserved_ = 0;
  }

  // nullptr when no chunk has room and a new chunk cannot be allocated
  char* alloc(size_t bytes) {
    bytes = round(bytes);
    for (auto& c : chunks_)
      if (char* p = take(c, bytes)) return p;
    const size_t sz = std::max(kChunk, bytes);
    void* mem = nullptr;
    if (cudaMalloc(&mem, sz) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    chunks_.push_back(Chunk{(char*)mem, sz, {{0, sz}}});
    reserved_ += sz;
    return take(chunks_.back(), bytes);
  }

  void free(char* p, size_t bytes) {
    bytes = round(bytes);
    for (auto& c : chunks_) {
      if (p < c.base || p >= c.base + c.size) continue;
      size_t off = (size_t)(p - c.base);
      auto next = c.free.lower_bound(off);
      if (next != c.free.end() && next->first == off + bytes) {
        bytes += next->second;
        next = c.free.erase(next);
      }
      if (next != c.free.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == off) {
          prev->second += bytes;
          return;
        }
      }
      c.free.emplace(off, bytes);
      return;
    }
  }

  size_t reserved() const { return reserved_; }

 private:
  struct Chunk {
    char* base;
    size_t size;
    std::map<size_t, size_t> free;  // offset -> bytes
  };
  static size_t round(size_t b) { return ((b + kAlign - 1) / kAlign) * kAlign; }
  static char* take(Chunk& c, size_t bytes) {
    for (auto it = c.free.begin(); it != c.free.end(); ++it) {
      if (it->second < bytes) continue;
      const size_t off = it->first, rest = it->second - bytes;
      c.free.erase(it);
      if (rest) c.free.emplace(off + bytes, rest);
      return c.base + off;
    }
    return nullptr;
  }
  std::vector<Chunk> chunks_;
  size_t reserved_ = 0;
};

struct BScene {
  int32_t id = 0;
  int hm_slot = 0;
  upbd_scene_desc desc{};
  upbd_params prm{};
  SimView v{};
  DevParams hp{};
  char* mem = nullptr;
  size_t bytes = 0;
  std::vector<uint4> init_cons;  // endpoints, for write_constraints checks
};

struct ProfRec {
  int kind;
  cudaEvent_t a, b;
};

thread_local std::string g_batch_error;

}  // namespace

struct upbd_batch {
  upbd_batch_desc desc{};
  int device = 0, num_sms = 0;
  int bt = 256, cps = 8;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::map<int32_t, BScene> scenes;  // id order = table order
  int32_t next_id = 1;
  std::vector<int> free_hm;
  uint32_t* hmapped = nullptr;  // pinned, device-mapped: HM_WORDS per scene slot
  uint32_t* dmapped = nullptr;
  // device table: [meta][prefix NUM_DOMAINS x stride][views max][params max]
  char* d_tab = nullptr;
  char* h_tab = nullptr;  // pinned staging of the same layout
  size_t off_prefix = 0, off_views = 0, off_params = 0, tab_bytes = 0;
  uint32_t stride = 0;
  cudaEvent_t tab_ev = nullptr;
  bool dirty = true;
  float cur_h = -1.f;
  DevicePool pool;
  size_t in_use = 0;
  int64_t particles = 0, solids = 0;
  struct Graph {
    cudaGraphExec_t exec;
    uint64_t kernels;
  };
  std::map<uint64_t, Graph> graphs;
  uint64_t launches = 0, frames = 0;
  std::string err;
  bool prof_on = false;
  std::vector<ProfRec> prof;
  std::vector<cudaEvent_t> prof_pool;
  size_t prof_used = 0;
};

namespace {

int bfail(upbd_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  g_batch_error = msg;
  return code;
}

#define BCK(b, call)                                                                  \
  do {                                                                                \
    cudaError_t _e = (call);                                                          \
    if (_e != cudaSuccess)                                                            \
      return bfail((b), UPBD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

cudaEvent_t prof_event(upbd_batch* b) {
  if (b->prof_used == b->prof_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    b->prof_pool.push_back(e);
  }
  return b->prof_pool[b->prof_used++];
}

#define BLAUNCH(b, kind, ...)                              \
  do {                                                     \
    if ((b)->prof_on) {                                    \
      ProfRec r_{kind, prof_event(b), prof_event(b)};      \
      cudaEventRecord(r_.a, (b)->stream);                  \
      __VA_ARGS__;                                         \
      cudaEventRecord(r_.b, (b)->stream);                  \
      (b)->prof.push_back(r_);                             \
    } else {                                               \
      __VA_ARGS__;                                         \
    }                                                      \
    (b)->launches++;                                       \
  } while (0)

BatchArgs batch_args(const upbd_batch* b) {
  BatchArgs a;
  a.views = (const SimView*)(b->d_tab + b->off_views);
  a.params = (const DevParams*)(b->d_tab + b->off_params);
  a.prefix = (const uint32_t*)(b->d_tab + b->off_prefix);
  a.meta = (const uint32_t*)b->d_tab;
  a.stride = b->stride;
  return a;
}

// Rewrites the table for the live scenes (id order) and enqueues its upload.
int upload_table(upbd_batch* b) {
  BCK(b, cudaEventSynchronize(b->tab_ev));  // the previous upload has left the staging buffer
  const bool tets = (b->desc.features & UPBD_FEAT_TETS) != 0;
  uint32_t* meta = (uint32_t*)b->h_tab;
  uint32_t* pre = (uint32_t*)(b->h_tab + b->off_prefix);
  SimView* views = (SimView*)(b->h_tab + b->off_views);
  DevParams* params = (DevParams*)(b->h_tab + b->off_params);
  std::memset(meta, 0, kMetaWords * 4);
  const uint32_t n = (uint32_t)b->scenes.size();
  meta[0] = n;
  for (int d = 0; d < NUM_DOMAINS; d++) pre[(size_t)d * b->stride] = 0;
  uint32_t k = 0;
  for (auto& kv : b->scenes) {
    BScene& sc = kv.second;
    uint32_t blk[NUM_DOMAINS];
    scene_blocks(sc.v, tets, b->bt, blk);
    for (int d = 0; d < NUM_DOMAINS; d++) {
      uint32_t* row = pre + (size_t)d * b->stride;
      row[k + 1] = row[k] + blk[d];
    }
    views[k] = sc.v;
    sc.hp.h = b->cur_h;
    params[k] = sc.hp;
    k++;
  }
  BCK(b, cudaMemcpyAsync(b->d_tab, b->h_tab, b->off_views + (size_t)n * sizeof(SimView), cudaMemcpyHostToDevice,
                         b->stream));
  if (n > 0)
    BCK(b, cudaMemcpyAsync(b->d_tab + b->off_params, b->h_tab + b->off_params, (size_t)n * sizeof(DevParams),
                           cudaMemcpyHostToDevice, b->stream));
  BCK(b, cudaEventRecord(b->tab_ev, b->stream));
  b->dirty = false;
  return UPBD_OK;
}

// The frame's launch sequence (GpuSim.encode's pass order, src/gpu/sim.js:
// 354-391), each pass one persistent launch over every scene.
int launch_batch_frame(upbd_batch* b, int nsub, bool visc) {
  const BatchArgs a = batch_args(b);
  const unsigned G = (unsigned)(b->cps * b->num_sms);
  const unsigned BT = (unsigned)b->bt;
  cudaStream_t st = b->stream;
  const bool tets = (b->desc.features & UPBD_FEAT_TETS) != 0;
  const bool scc = (b->desc.features & UPBD_FEAT_SOLID_CONTACTS) != 0;
  const int iters = b->desc.solid_iters;
  const bool mark_in_apply = iters > 0 && !tets && !scc;
  const bool fold = iters >= 2 && !tets && !scc;  // solve + apply in one launch per iteration
  for (int k = 0; k < nsub; k++) {
    BLAUNCH(b, K_INTEGRATE, kb_integrate_count<true, true><<<G, BT, 0, st>>>(a));
    BLAUNCH(b, K_SCAN, kb_scan<<<G, SCAN_THREADS, 0, st>>>(a));
    BLAUNCH(b, K_SCATTER, kb_scatter<<<G, BT, 0, st>>>(a));
    BLAUNCH(b, K_RANKFIX, kb_rankfix<<<G, BT, 0, st>>>(a));
    BLAUNCH(b, K_DENSITY, kb_density<<<G, BT, 0, st>>>(a));
    if (fold)  // the displacement pass applies the fluid's move (b_disp<true>)
      BLAUNCH(b, K_DISP, kb_disp<true><<<G, BT, 0, st>>>(a));
    else
      BLAUNCH(b, K_DISP, kb_disp<false><<<G, BT, 0, st>>>(a));
    if (iters == 0) BLAUNCH(b, K_APPLY_FLUID, kb_apply_fluid<<<G, BT, 0, st>>>(a));
    if (scc) BLAUNCH(b, K_COLLECT, kb_collect_contacts<<<G, BT, 0, st>>>(a));
    for (int it = 0; it < iters && fold; it++) {  // each iteration one launch (b_solid_solve's OUT)
      if (it < iters - 1) BLAUNCH(b, K_SOLID_SOLVE, (kb_solid_solve<false, SOLVE_STEP><<<G, BT, 0, st>>>(a, it)));
      else BLAUNCH(b, K_SOLID_SOLVE, (kb_solid_solve<false, SOLVE_LAST><<<G, BT, 0, st>>>(a, it)));
    }
    for (int it = 0; it < iters && !fold; it++) {
      if (it == 0) BLAUNCH(b, K_SOLID_SOLVE, (kb_solid_solve<true, SOLVE_DELTA><<<G, BT, 0, st>>>(a, it)));
      else BLAUNCH(b, K_SOLID_SOLVE, (kb_solid_solve<false, SOLVE_DELTA><<<G, BT, 0, st>>>(a, it)));
      if (mark_in_apply && it == iters - 1) BLAUNCH(b, K_APPLY_SOLID, kb_apply_solid<true><<<G, BT, 0, st>>>(a));
      else BLAUNCH(b, K_APPLY_SOLID, kb_apply_solid<false><<<G, BT, 0, st>>>(a));
      if (tets) {
        BLAUNCH(b, K_SOLVE_TETS, kb_solve_tets<<<G, BT, 0, st>>>(a));
        BLAUNCH(b, K_APPLY_SOLID_CONTACTS, kb_apply_solid_contacts<<<G, BT, 0, st>>>(a));
      }
      if (scc) {
        BLAUNCH(b, K_SOLID_CONTACTS, kb_solid_contacts<<<G, BT, 0, st>>>(a));
        BLAUNCH(b, K_APPLY_SOLID_CONTACTS, kb_apply_solid_contacts<<<G, BT, 0, st>>>(a));
      }
    }
    if (!mark_in_apply) BLAUNCH(b, K_APPLY_SOLID, kb_contact_mark<<<G, BT, 0, st>>>(a));
    BLAUNCH(b, K_BOND_CONTACTS, kb_bond_contacts<<<G, BT, 0, st>>>(a, tets ? 1 : 0));
    BLAUNCH(b, K_APPLY_BOUNDS_VEL, kb_apply_bounds_vel<<<G, BT, 0, st>>>(a));
    if (visc) {
      BLAUNCH(b, K_SOLID_VISC, kb_solid_visc<<<G, BT, 0, st>>>(a));
      BLAUNCH(b, K_SOLID_VISC, kb_solid_visc_apply<<<G, BT, 0, st>>>(a));
    }
    BLAUNCH(b, K_XSPH, kb_xsph<<<G, BT, 0, st>>>(a));  // writes the blended velocity itself
  }
  BLAUNCH(b, K_COUNT_ACTIVE, kb_count_active<<<G, BT, 0, st>>>(a));
  const cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) return bfail(b, UPBD_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return UPBD_OK;
}

uint64_t graph_kernels(cudaGraph_t g) {
  size_t n = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return 0;
  std::vector<cudaGraphNode_t> nodes(n);
  cudaGraphGetNodes(g, nodes.data(), &n);
  uint64_t k = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) k++;
  }
  return k;
}

int enqueue_batch_frame(upbd_batch* b, double dt, int nsub, bool profile) {
  if (nsub < 1 || nsub > 1000) return bfail(b, UPBD_ERR_INVALID, "substeps out of range [1, 1000]");
  const double h = dt / nsub;
  if (!(h > 0) || !std::isfinite(h)) return bfail(b, UPBD_ERR_INVALID, "frame length must be > 0");
  if ((float)h != b->cur_h) {
    b->cur_h = (float)h;
    b->dirty = true;
  }
  if (b->dirty) {
    const int rc = upload_table(b);
    if (rc) return rc;
  }
  bool visc = false;
  for (auto& kv : b->scenes) visc = visc || kv.second.prm.solid_viscosity > 0;
  if (!profile) {
    const uint64_t key = (uint64_t)nsub | ((uint64_t)b->bt << 16) | ((uint64_t)b->cps << 32) | ((uint64_t)visc << 48);
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
      cudaGraph_t g;
      BCK(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      const uint64_t before = b->launches;
      const int rc = launch_batch_frame(b, nsub, visc);
      cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
      b->launches = before;
      if (rc) return rc;
      if (ce != cudaSuccess) return bfail(b, UPBD_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
      cudaGraphExec_t ge;
      ce = cudaGraphInstantiate(&ge, g, 0);
      const uint64_t nk = graph_kernels(g);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess) return bfail(b, UPBD_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(ce));
      it = b->graphs.emplace(key, upbd_batch::Graph{ge, nk}).first;
    }
    BCK(b, cudaGraphLaunch(it->second.exec, b->stream));
    b->launches += it->second.kernels;
  } else {
    b->prof_on = true;
    const int rc = launch_batch_frame(b, nsub, visc);
    b->prof_on = false;
    if (rc) return rc;
  }
  b->frames++;
  return UPBD_OK;
}

BScene* find(upbd_batch* b, int32_t id) {
  auto it = b->scenes.find(id);
  return it == b->scenes.end() ? nullptr : &it->second;
}

}  // namespace

namespace upbd {

size_t prepared_bytes(const PreparedScene& ps) {
  SimView v;
  return layout_scene(ps.desc, *ps.lat, v).bytes;
}

int batch_add_prepared(upbd_batch* b, const PreparedScene& ps, int32_t* id) {
  if (!b || !id || !ps.lat) return bfail(b, UPBD_ERR_INVALID, "null argument");
  const upbd_scene_desc& d = ps.desc;
  if (d.solid_iters != b->desc.solid_iters || d.features != b->desc.features)
    return bfail(b, UPBD_ERR_INVALID, "scene solid_iters/features differ from the batch's");
  if (b->free_hm.empty()) return bfail(b, UPBD_ERR_CAPACITY, "scene table is full");
  cudaSetDevice(b->device);
  BScene sc;
  const SceneLayout L = layout_scene(d, *ps.lat, sc.v);
  if (b->desc.hbm_budget && b->in_use + L.bytes > b->desc.hbm_budget)
    return bfail(b, UPBD_ERR_CAPACITY, "scene does not fit the HBM budget");
  sc.mem = b->pool.alloc(L.bytes);
  if (!sc.mem) return bfail(b, UPBD_ERR_OOM, "device memory for the scene is not available");
  sc.bytes = L.bytes;
  DevParams* unused = nullptr;
  bind_scene(L, sc.mem, sc.v, &unused);
  sc.hm_slot = b->free_hm.back();
  sc.v.host_mapped = b->dmapped + (size_t)sc.hm_slot * HM_WORDS;
  cudaStream_t st = b->stream;
  cudaError_t e = cudaMemsetAsync(sc.mem, 0, sc.bytes, st);
  if (e == cudaSuccess) e = upload_prepared(ps, sc.v, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    b->pool.free(sc.mem, sc.bytes);
    return bfail(b, UPBD_ERR_CUDA, std::string("scene upload: ") + cudaGetErrorString(e));
  }
  b->free_hm.pop_back();
  std::memset(b->hmapped + (size_t)sc.hm_slot * HM_WORDS, 0, HM_WORDS * 4);
  sc.id = b->next_id++;
  sc.desc = d;
  sc.prm = ps.prm;
  fill_dev_params(ps.prm, d, sc.hp);
  sc.hp.grab_lattice = 0xffff;
  sc.init_cons = ps.lat->cons;
  b->in_use += sc.bytes;
  b->particles += sc.v.N;
  b->solids += sc.v.S;
  *id = sc.id;
  b->scenes.emplace(sc.id, std::move(sc));
  b->dirty = true;
  return UPBD_OK;
}

cudaStream_t batch_stream(upbd_batch* b) { return b ? b->stream : nullptr; }

bool batch_scene_counters(upbd_batch* b, int32_t id, uint32_t* active, uint32_t* health, int32_t* solids) {
  BScene* sc = find(b, id);
  if (!sc) return false;
  const volatile uint32_t* hm = b->hmapped + (size_t)sc->hm_slot * HM_WORDS;
  if (active) *active = hm[HM_ACTIVE];
  if (health) *health = hm[HM_HEALTH];
  if (solids) *solids = sc->v.S;
  return true;
}

}  // namespace upbd

extern "C" {

int upbd_batch_default_desc(upbd_batch_desc* d) {
  if (!d) return UPBD_ERR_INVALID;
  std::memset(d, 0, sizeof(*d));
  d->device = 0;
  d->solid_iters = 3;
  d->features = 0;
  d->max_scenes = 1024;
  d->block_threads = 256;
  d->ctas_per_sm = 8;
  d->hbm_budget = 0;
  return UPBD_OK;
}

const char* upbd_batch_last_error(upbd_batch* b) { return b ? b->err.c_str() : g_batch_error.c_str(); }

int upbd_batch_scene_bytes(const upbd_scene_desc* d, uint64_t* bytes) {
  if (!d || !bytes) return UPBD_ERR_INVALID;
  upbd_params p;
  upbd_default_params(&p);
  if (const char* why = check_desc(d, &p)) return bfail(nullptr, UPBD_ERR_INVALID, why);
  SimView v;
  *bytes = layout_scene(*d, *lattice_of(*d), v).bytes;
  return UPBD_OK;
}

int upbd_batch_create(const upbd_batch_desc* d, upbd_batch** out) {
  if (!out || !d) return bfail(nullptr, UPBD_ERR_INVALID, "null argument");
  *out = nullptr;
  if (d->max_scenes < 1 || d->max_scenes > 65536) return bfail(nullptr, UPBD_ERR_INVALID, "max_scenes out of range");
  if (d->block_threads != 64 && d->block_threads != 128 && d->block_threads != 256)
    return bfail(nullptr, UPBD_ERR_INVALID, "block_threads must be 64, 128 or 256");
  if (d->ctas_per_sm < 1 || d->ctas_per_sm > 256) return bfail(nullptr, UPBD_ERR_INVALID, "ctas_per_sm out of range");
  if (d->solid_iters < 0 || d->solid_iters > 1000) return bfail(nullptr, UPBD_ERR_INVALID, "solid_iters out of range");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return bfail(nullptr, UPBD_ERR_NO_DEVICE, "no CUDA device");
  if (d->device < 0 || d->device >= ndev) return bfail(nullptr, UPBD_ERR_INVALID, "bad device ordinal");
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, d->device) != cudaSuccess || prop.major < 10)
    return bfail(nullptr, UPBD_ERR_NO_DEVICE, "libupbd is built for sm_100a (B200); device is older");
  if (cudaSetDevice(d->device) != cudaSuccess) return bfail(nullptr, UPBD_ERR_CUDA, "cudaSetDevice failed");
  upbd_batch* b = new upbd_batch();
  b->desc = *d;
  b->device = d->device;
  b->num_sms = prop.multiProcessorCount;
  b->bt = d->block_threads;
  b->cps = d->ctas_per_sm;
  const size_t M = (size_t)d->max_scenes;
  b->stride = (uint32_t)(M + 1);
  auto al = [](size_t x) { return ((x + 255) / 256) * 256; };
  b->off_prefix = al(kMetaWords * 4);
  b->off_views = b->off_prefix + al((size_t)NUM_DOMAINS * b->stride * 4);
  b->off_params = b->off_views + al(M * sizeof(SimView));
  b->tab_bytes = b->off_params + al(M * sizeof(DevParams));
  auto bail = [&](int code, const char* msg) {
    upbd_batch_destroy(b);
    return bfail(nullptr, code, msg);
  };
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(UPBD_ERR_CUDA, "stream creation failed");
  b->own_stream = true;
  if (cudaMalloc((void**)&b->d_tab, b->tab_bytes) != cudaSuccess) return bail(UPBD_ERR_OOM, "table allocation failed");
  if (cudaMemset(b->d_tab, 0, b->tab_bytes) != cudaSuccess) return bail(UPBD_ERR_CUDA, "table clear failed");
  if (cudaHostAlloc((void**)&b->h_tab, b->tab_bytes, cudaHostAllocDefault) != cudaSuccess)
    return bail(UPBD_ERR_OOM, "pinned table allocation failed");
  std::memset(b->h_tab, 0, b->tab_bytes);
  if (cudaHostAlloc((void**)&b->hmapped, M * HM_WORDS * 4, cudaHostAllocMapped) != cudaSuccess)
    return bail(UPBD_ERR_OOM, "mapped host allocation failed");
  std::memset(b->hmapped, 0, M * HM_WORDS * 4);
  if (cudaHostGetDevicePointer((void**)&b->dmapped, b->hmapped, 0) != cudaSuccess)
    return bail(UPBD_ERR_CUDA, "mapped host pointer failed");
  if (cudaEventCreateWithFlags(&b->tab_ev, cudaEventDisableTiming) != cudaSuccess)
    return bail(UPBD_ERR_CUDA, "event creation failed");
  for (int k = (int)M - 1; k >= 0; k--) b->free_hm.push_back(k);
  *out = b;
  return UPBD_OK;
}

int upbd_batch_destroy(upbd_batch* b) {
  if (!b) return UPBD_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second.exec);
  for (cudaEvent_t e : b->prof_pool) cudaEventDestroy(e);
  if (b->tab_ev) cudaEventDestroy(b->tab_ev);
  b->pool.release();
  if (b->d_tab) cudaFree(b->d_tab);
  if (b->h_tab) cudaFreeHost(b->h_tab);
  if (b->hmapped) cudaFreeHost(b->hmapped);
  if (b->stream && b->own_stream) cudaStreamDestroy(b->stream);
  delete b;
  return UPBD_OK;
}

int upbd_batch_get_info(upbd_batch* b, upbd_batch_info* info) {
  if (!b || !info) return UPBD_ERR_INVALID;
  std::memset(info, 0, sizeof(*info));
  info->scenes = (int32_t)b->scenes.size();
  info->max_scenes = b->desc.max_scenes;
  info->particles = b->particles;
  info->solids = b->solids;
  info->bytes_in_use = b->in_use;
  info->bytes_reserved = b->pool.reserved();
  info->hbm_budget = b->desc.hbm_budget;
  info->frames = b->frames;
  info->launches = b->launches;
  info->block_threads = b->bt;
  info->ctas_per_sm = b->cps;
  info->num_sms = b->num_sms;
  return UPBD_OK;
}

int upbd_batch_add_scene(upbd_batch* b, const upbd_scene_desc* d, const upbd_params* p, int32_t n_fluid,
                         const float* fluid_pos3, const float* fluid_vel3, double fluid_mass, int32_t* id) {
  if (!b || !d || !p || !id) return bfail(b, UPBD_ERR_INVALID, "null argument");
  if (n_fluid < 0 || n_fluid > d->max_fluid) return bfail(b, UPBD_ERR_CAPACITY, "n_fluid exceeds max_fluid");
  PreparedScene ps;
  if (const char* why = prepare_scene(*d, *p, n_fluid, fluid_pos3, fluid_vel3, fluid_mass, ps))
    return bfail(b, UPBD_ERR_INVALID, why);
  return batch_add_prepared(b, ps, id);
}

int upbd_batch_remove_scene(upbd_batch* b, int32_t id) {
  if (!b) return UPBD_ERR_INVALID;
  BScene* sc = find(b, id);
  if (!sc) return bfail(b, UPBD_ERR_INVALID, "no such scene");
  b->pool.free(sc->mem, sc->bytes);
  b->free_hm.push_back(sc->hm_slot);
  b->in_use -= sc->bytes;
  b->particles -= sc->v.N;
  b->solids -= sc->v.S;
  b->scenes.erase(id);
  b->dirty = true;
  return UPBD_OK;
}

int upbd_batch_set_params(upbd_batch* b, int32_t id, const upbd_params* p) {
  if (!b || !p) return UPBD_ERR_INVALID;
  BScene* sc = find(b, id);
  if (!sc) return bfail(b, UPBD_ERR_INVALID, "no such scene");
  if (const char* why = check_desc(&sc->desc, p)) return bfail(b, UPBD_ERR_INVALID, why);
  sc->prm = *p;
  fill_dev_params(*p, sc->desc, sc->hp);
  sc->hp.grab_lattice = 0xffff;
  b->dirty = true;
  return UPBD_OK;
}

int upbd_batch_step(upbd_batch* b, double dt, int32_t substeps) {
  if (!b) return UPBD_ERR_INVALID;
  cudaSetDevice(b->device);
  return enqueue_batch_frame(b, dt, substeps, false);
}

int upbd_batch_sync(upbd_batch* b) {
  if (!b) return UPBD_ERR_INVALID;
  cudaSetDevice(b->device);
  BCK(b, cudaStreamSynchronize(b->stream));
  for (auto& kv : b->scenes) {
    const uint32_t hb = ((volatile uint32_t*)b->hmapped)[(size_t)kv.second.hm_slot * HM_WORDS + HM_HEALTH];
    if (hb & UPBD_HEALTH_NAN)
      return bfail(b, UPBD_ERR_NAN, "non-finite velocity detected in scene " + std::to_string(kv.first));
    if (hb & UPBD_HEALTH_BOUNDS)
      return bfail(b, UPBD_ERR_INTERNAL,
                   "an index out of range was skipped in scene " + std::to_string(kv.first) + " (checked build)");
  }
  return UPBD_OK;
}

int upbd_batch_set_stream(upbd_batch* b, void* stream) {
  if (!b) return UPBD_ERR_INVALID;
  cudaSetDevice(b->device);
  BCK(b, cudaStreamSynchronize(b->stream));
  if (b->own_stream) cudaStreamDestroy(b->stream);
  b->own_stream = false;
  b->stream = (cudaStream_t)stream;
  if (!stream) {
    BCK(b, cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->own_stream = true;
  }
  return UPBD_OK;
}

int upbd_batch_set_tuning(upbd_batch* b, int32_t block_threads, int32_t ctas_per_sm) {
  if (!b) return UPBD_ERR_INVALID;
  if (block_threads != 64 && block_threads != 128 && block_threads != 256)
    return bfail(b, UPBD_ERR_INVALID, "block_threads must be 64, 128 or 256");
  if (ctas_per_sm < 1 || ctas_per_sm > 256) return bfail(b, UPBD_ERR_INVALID, "ctas_per_sm out of range");
  if (block_threads != b->bt) b->dirty = true;  // tile counts change with the block size
  b->bt = block_threads;
  b->cps = ctas_per_sm;
  return UPBD_OK;
}

int upbd_batch_read_state(upbd_batch* b, int32_t id, float* pos4, float* prev4, float* vel4, float* density2,
                          uint32_t* flags) {
  if (!b) return UPBD_ERR_INVALID;
  BScene* sc = find(b, id);
  if (!sc) return bfail(b, UPBD_ERR_INVALID, "no such scene");
  cudaSetDevice(b->device);
  const size_t N = (size_t)sc->v.N;
  if (pos4) BCK(b, cudaMemcpyAsync(pos4, sc->v.pos, N * 16, cudaMemcpyDeviceToHost, b->stream));
  if (prev4) BCK(b, cudaMemcpyAsync(prev4, sc->v.prev, N * 16, cudaMemcpyDeviceToHost, b->stream));
  if (vel4) BCK(b, cudaMemcpyAsync(vel4, sc->v.vel, N * 16, cudaMemcpyDeviceToHost, b->stream));
  if (density2) BCK(b, cudaMemcpyAsync(density2, sc->v.density, N * 8, cudaMemcpyDeviceToHost, b->stream));
  if (flags) BCK(b, cudaMemcpyAsync(flags, sc->v.flags, N * 4, cudaMemcpyDeviceToHost, b->stream));
  BCK(b, cudaStreamSynchronize(b->stream));
  return UPBD_OK;
}

int upbd_batch_write_state(upbd_batch* b, int32_t id, const float* pos4, const float* prev4, const float* vel4,
                           const float* density2, const uint32_t* flags) {
  if (!b) return UPBD_ERR_INVALID;
  BScene* sc = find(b, id);
  if (!sc) return bfail(b, UPBD_ERR_INVALID, "no such scene");
  cudaSetDevice(b->device);
  const size_t N = (size_t)sc->v.N;
  cudaStream_t st = b->stream;
  if (pos4) BCK(b, cudaMemcpyAsync(sc->v.pos, pos4, N * 16, cudaMemcpyHostToDevice, st));
  if (prev4) BCK(b, cudaMemcpyAsync(sc->v.prev, prev4, N * 16, cudaMemcpyHostToDevice, st));
  if (vel4) BCK(b, cudaMemcpyAsync(sc->v.vel, vel4, N * 16, cudaMemcpyHostToDevice, st));
  if (density2) BCK(b, cudaMemcpyAsync(sc->v.density, density2, N * 8, cudaMemcpyHostToDevice, st));
  if (flags) BCK(b, cudaMemcpyAsync(sc->v.flags, flags, N * 4, cudaMemcpyHostToDevice, st));
  BCK(b, cudaStreamSynchronize(st));
  return UPBD_OK;
}

int upbd_batch_read_constraints(upbd_batch* b, int32_t id, uint32_t* cons4) {
  if (!b || !cons4) return UPBD_ERR_INVALID;
  BScene* sc = find(b, id);
  if (!sc) return bfail(b, UPBD_ERR_INVALID, "no such scene");
  cudaSetDevice(b->device);
  if (sc->v.C > 0)
    BCK(b, cudaMemcpyAsync(cons4, sc->v.cons, (size_t)sc->v.C * 16, cudaMemcpyDeviceToHost, b->stream));
  BCK(b, cudaStreamSynchronize(b->stream));
  return UPBD_OK;
}

int upbd_batch_write_constraints(upbd_batch* b, int32_t id, const uint32_t* cons4) {
  if (!b || !cons4) return UPBD_ERR_INVALID;
  BScene* sc = find(b, id);
  if (!sc) return bfail(b, UPBD_ERR_INVALID, "no such scene");
  for (int c = 0; c < sc->v.C; c++)
    if (cons4[4 * c] != sc->init_cons[c].x || cons4[4 * c + 1] != sc->init_cons[c].y)
      return bfail(b, UPBD_ERR_INVALID, "constraint endpoints must match the scene's");
  cudaSetDevice(b->device);
  if (sc->v.C > 0)
    BCK(b, cudaMemcpyAsync(sc->v.cons, cons4, (size_t)sc->v.C * 16, cudaMemcpyHostToDevice, b->stream));
  BCK(b, cudaStreamSynchronize(b->stream));
  return UPBD_OK;
}

int upbd_batch_scene_info(upbd_batch* b, int32_t id, upbd_info* info) {
  if (!b || !info) return UPBD_ERR_INVALID;
  BScene* sc = find(b, id);
  if (!sc) return bfail(b, UPBD_ERR_INVALID, "no such scene");
  std::memset(info, 0, sizeof(*info));
  info->solid_n = sc->v.S;
  info->n1 = sc->v.N1;
  info->dim1 = sc->v.dim1;
  info->dim2 = sc->v.dim2;
  info->max_fluid = sc->v.F;
  info->total = sc->v.N;
  info->num_cons = sc->v.C;
  info->num_tets = sc->v.NT;
  info->table_size = sc->v.T;
  info->substeps = sc->desc.substeps;
  info->solid_iters = sc->desc.solid_iters;
  info->features = sc->desc.features;
  info->frames = (int64_t)b->frames;
  info->device_bytes = sc->bytes;
  info->param_bytes = (uint32_t)sizeof(DevParams);
  return UPBD_OK;
}

int upbd_batch_active_count(upbd_batch* b, int32_t id, uint32_t* count) {
  if (!b || !count) return UPBD_ERR_INVALID;
  BScene* sc = find(b, id);
  if (!sc) return bfail(b, UPBD_ERR_INVALID, "no such scene");
  cudaSetDevice(b->device);
  BCK(b, cudaStreamSynchronize(b->stream));
  *count = ((volatile uint32_t*)b->hmapped)[(size_t)sc->hm_slot * HM_WORDS + HM_ACTIVE];
  return UPBD_OK;
}

int upbd_batch_profile_frame(upbd_batch* b, double dt, int32_t substeps, double* ms, uint32_t* launches) {
  if (!b || !ms || !launches || substeps < 1) return UPBD_ERR_INVALID;
  cudaSetDevice(b->device);
  b->prof.clear();
  b->prof_used = 0;
  int rc = enqueue_batch_frame(b, dt, substeps, true);
  if (rc) return rc;
  BCK(b, cudaStreamSynchronize(b->stream));
  for (int k = 0; k < UPBD_KERNEL_KINDS; k++) {
    ms[k] = 0;
    launches[k] = 0;
  }
  for (const ProfRec& r : b->prof) {
    float t = 0;
    BCK(b, cudaEventElapsedTime(&t, r.a, r.b));
    ms[r.kind] += t;
    launches[r.kind]++;
  }
  b->prof.clear();
  b->prof_used = 0;
  return UPBD_OK;
}

}  // extern "C"
