// Host runtime and C ABI of libupbd.so (declared in include/upbd.h).
//
// One upbd_sim owns one scene resident in device memory (one arena
// allocation). A frame is a fixed launch sequence (per-substep pass chain of
// GpuSim.encode, src/gpu/sim.js:333-398); it is captured once per shape into
// a CUDA graph and replayed. The frame's uniforms live in a device buffer that
// is refreshed from pinned host memory before each replay, so graphs never
// need re-instantiation when tools change values.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/upbd.h"
#include "upbd_groups.cuh"
#include "upbd_kernels.cuh"
#include "upbd_kinds.h"
#include "upbd_scene.h"

using namespace upbd;

namespace upbd {
const char* const kKernelNames[K_NUM_KINDS] = {
  "integrate_count", "scan", "scatter", "rankfix", "density", "disp", "apply_fluid",
  "collect_contacts", "solid_solve", "apply_solid", "solve_tets", "solid_contacts",
  "apply_solid_contacts", "bond_contacts", "apply_bounds_vel", "solid_visc", "xsph",
  "xsph_apply", "emit", "cut", "count_active"};
}  // namespace upbd

namespace {

thread_local std::string g_last_error;

constexpr int kStageRing = 8;

inline unsigned blocks_for(long long n, int bs = 256) {
  long long b = (n + bs - 1) / bs;
  return (unsigned)(b < 1 ? 1 : b);
}

struct CutReq {
  double o[3], d1[3], d2[3];
};

struct ProfRec {
  int kind;
  cudaEvent_t a, b;
};

}  // namespace

struct upbd_sim {
  upbd_scene_desc desc{};
  upbd_params prm{};
  int device = 0;
  SimView v{};
  DevParams hp{};              // host mirror of the device uniforms
  DevParams* dparams = nullptr;
  DevParams* stage = nullptr;  // pinned ring
  cudaEvent_t stage_ev[kStageRing] = {};
  int stage_next = 0;
  uint32_t* hmapped = nullptr;  // pinned, device-mapped
  void* arena = nullptr;
  size_t arena_bytes = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // second stream of the substep: the solid solve's first iterations run
  // there beside the grid build and the fluid gathers (fork / join events)
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, grid_ev = nullptr, join_ev = nullptr;
  // asynchronous readback: device staging copy, copy stream, events
  void* rb_stage = nullptr;  // float4 pos[N] then uint32 flags[N]
  cudaStream_t rb_stream = nullptr;
  cudaEvent_t rb_ready = nullptr, rb_done = nullptr;
  // host copies for reset
  std::vector<float4> init_pos;
  std::vector<uint4> init_cons;
  std::vector<uint32_t> adj_host;
  std::vector<float> init_tet_vol;
  // pending tool state (GpuSim.pending, src/gpu/sim.js:92)
  bool emit_pending = false;
  uint32_t emit_count = 0, emit_start = 0;
  float4 emit_pos{}, emit_dir{}, emit_side{}, emit_up{};
  std::deque<CutReq> cuts;
  double grab_delta[3] = {0, 0, 0};
  int fluid_next = 0;
  int frames = 0;
  bool use_graphs = true;
  struct Graph {
    cudaGraphExec_t exec;
    uint64_t kernels;
  };
  std::map<uint64_t, Graph> graphs;
  uint64_t launches = 0;  // kernels enqueued (graph replays count their nodes)
  std::string err;
  // per-kernel timing of an eager frame
  bool prof_on = false;
  std::vector<ProfRec> prof;
  std::vector<cudaEvent_t> prof_pool;
  size_t prof_used = 0;
};

namespace {

int fail(upbd_sim* s, int code, const std::string& msg) {
  if (s) s->err = msg;
  g_last_error = msg;
  return code;
}

#define UPBD_CK(s, call)                                                              \
  do {                                                                                \
    cudaError_t _e = (call);                                                          \
    if (_e != cudaSuccess)                                                            \
      return fail((s), UPBD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

#define UPBD_KCK(s)                                                                  \
  do {                                                                               \
    cudaError_t _e = cudaPeekAtLastError();                                          \
    if (_e != cudaSuccess)                                                           \
      return fail((s), UPBD_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(_e)); \
  } while (0)

cudaEvent_t prof_event(upbd_sim* s) {
  if (s->prof_used == s->prof_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    s->prof_pool.push_back(e);
  }
  return s->prof_pool[s->prof_used++];
}

// Event pair around one launch while a profiled frame is being recorded.
#define PROF(s, kind, ...)                                  \
  do {                                                      \
    if ((s)->prof_on) {                                     \
      ProfRec r_{kind, prof_event(s), prof_event(s)};       \
      cudaEventRecord(r_.a, (s)->stream);                   \
      __VA_ARGS__;                                          \
      cudaEventRecord(r_.b, (s)->stream);                   \
      (s)->prof.push_back(r_);                              \
    } else {                                                \
      __VA_ARGS__;                                          \
    }                                                       \
  } while (0)

void fill_static_params(upbd_sim* s) { fill_dev_params(s->prm, s->desc, s->hp); }

int upload_params(upbd_sim* s) {
  const int k = s->stage_next;
  s->stage_next = (k + 1) % kStageRing;
  UPBD_CK(s, cudaEventSynchronize(s->stage_ev[k]));
  s->stage[k] = s->hp;
  UPBD_CK(s, cudaMemcpyAsync(s->dparams, &s->stage[k], sizeof(DevParams), cudaMemcpyHostToDevice,
                             s->stream));
  UPBD_CK(s, cudaEventRecord(s->stage_ev[k], s->stream));
  return UPBD_OK;
}

// Launch sequence of one substep (GpuSim.encode loop body,
// src/gpu/sim.js:354-385), stopping after `last` (UPBD_PASS_*).
int launch_substep(upbd_sim* s, int last) {
  const SimView& v = s->v;
  const DevParams* P = s->dparams;
  cudaStream_t st = s->stream;
  const bool tets = (s->desc.features & UPBD_FEAT_TETS) != 0;
  const bool scc = (s->desc.features & UPBD_FEAT_SOLID_CONTACTS) != 0;
  const int iters = s->desc.solid_iters;
  uint64_t& L = s->launches;
  if (last < UPBD_PASS_INTEGRATE) return UPBD_OK;
  if (last < UPBD_PASS_GRID) {
    PROF(s, K_INTEGRATE, k_integrate_count<true, false><<<blocks_for(v.N), 256, 0, st>>>(v, P));
    L++;
    UPBD_KCK(s);
    return UPBD_OK;
  }
  // With two or more plain Jacobi iterations (no tets, no solid contacts)
  // each iteration is one launch that also applies (b_solid_solve's OUT), and
  // the displacement pass applies the fluid's move itself. The iterations
  // before the last read and write solid positions only (pos, sbuf), which no
  // pass of the grid build or the fluid gathers writes, so they run on the
  // side stream meanwhile; the last one also writes the solids' slot copies,
  // so it waits for the grid build, and still runs beside density and
  // displacement (they read fluid slots only), followed there by the contact
  // marks, which read the fluid's grid positions with a reach widened by the
  // displacement limit (the pass that applies the displacement marks the
  // particles that change cell). Eager per-kernel timing keeps one stream
  // and marks from the displaced fluid after the solve.
  const bool fold = iters >= 2 && !tets && !scc && last >= UPBD_PASS_SOLID;
  const bool overlap = fold && !s->prof_on && s->side;
  const int solid_pad = ((v.S * GL + 31) / 32) * 32;  // lane threads of the solve, whole warps
  PROF(s, K_INTEGRATE, k_integrate_count<true, true><<<blocks_for(v.N), 256, 0, st>>>(v, P));
  if (overlap) {
    UPBD_CK(s, cudaEventRecord(s->fork_ev, st));
    UPBD_CK(s, cudaStreamWaitEvent(s->side, s->fork_ev, 0));
    for (int it = 0; it < iters - 1; it++) {
      k_solid_solve<false, SOLVE_STEP><<<blocks_for(solid_pad), 256, 0, s->side>>>(v, P, solid_pad, it);
      L++;
    }
  }
  PROF(s, K_SCAN, k_scan<<<v.num_tiles, SCAN_THREADS, 0, st>>>(v));
  PROF(s, K_SCATTER, k_scatter<<<blocks_for(std::max(v.N, tile_words(v.num_tiles))), 256, 0, st>>>(v));
  PROF(s, K_RANKFIX, k_rankfix<<<blocks_for(v.N), 256, 0, st>>>(v));
  L += 4;
  UPBD_KCK(s);
  if (overlap) {
    UPBD_CK(s, cudaEventRecord(s->grid_ev, st));
    UPBD_CK(s, cudaStreamWaitEvent(s->side, s->grid_ev, 0));
    k_solid_solve<false, SOLVE_FINAL><<<blocks_for(solid_pad), 256, 0, s->side>>>(v, P, solid_pad, iters - 1);
    L++;
    // the contact marks from the solids' final positions and the fluid's
    // grid positions (reach widened by the displacement limit), so they run
    // here beside density and displacement rather than after them
    if (v.S > 0) {
      k_contact_mark<32, true><<<blocks_for((long long)v.S * 32), 256, 0, s->side>>>(v, P);
      L++;
    }
    UPBD_CK(s, cudaEventRecord(s->join_ev, s->side));
  }
  if (last < UPBD_PASS_DENSITY) return UPBD_OK;
  const long long fl = (long long)v.N * GLF;  // lane-parallel fluid gathers over the slots
  PROF(s, K_DENSITY, k_density<<<blocks_for(fl), 256, 0, st>>>(v, P));
  L++;
  if (last < UPBD_PASS_DISP) return UPBD_OK;
  if (fold)  // DL threads per slot
    PROF(s, K_DISP, k_disp<true><<<blocks_for((long long)v.N * DL), 256, 0, st>>>(v, P));
  else
    PROF(s, K_DISP, k_disp<false><<<blocks_for((long long)v.N * DL), 256, 0, st>>>(v, P));
  L++;
  UPBD_KCK(s);
  if (last < UPBD_PASS_APPLY_FLUID) return UPBD_OK;
  if (!fold && (last < UPBD_PASS_SOLID || iters == 0)) {
    PROF(s, K_APPLY_FLUID, k_apply_fluid<<<blocks_for(v.F), 256, 0, st>>>(v, P));
    L++;
    if (last < UPBD_PASS_SOLID) return UPBD_OK;
  }
  if (scc) {
    PROF(s, K_COLLECT, k_collect_contacts<<<blocks_for(v.S), 256, 0, st>>>(v, P));
    L++;
  }
  // the contact marks ride on the last applyDeltaSolid when that is the last
  // position update of the solve; otherwise they get their own launch
  const bool mark_in_apply = iters > 0 && !tets && !scc;
  if (fold) {
    if (overlap) {
      UPBD_CK(s, cudaStreamWaitEvent(st, s->join_ev, 0));  // the solve and the marks
    } else {
      for (int it = 0; it < iters - 1; it++) {
        PROF(s, K_SOLID_SOLVE, k_solid_solve<false, SOLVE_STEP><<<blocks_for(solid_pad), 256, 0, st>>>(v, P, solid_pad, it));
        L++;
      }
      PROF(s, K_SOLID_SOLVE,
           k_solid_solve<false, SOLVE_LAST><<<blocks_for(solid_pad), 256, 0, st>>>(v, P, solid_pad, iters - 1));
      L++;
    }
  }
  for (int it = 0; it < iters && !fold; it++) {
    if (it == 0)
      PROF(s, K_SOLID_SOLVE, k_solid_solve<true, SOLVE_DELTA>
           <<<blocks_for((long long)solid_pad + v.F), 256, 0, st>>>(v, P, solid_pad, it));
    else
      PROF(s, K_SOLID_SOLVE, k_solid_solve<false, SOLVE_DELTA><<<blocks_for(solid_pad), 256, 0, st>>>(v, P, solid_pad, it));
    if (mark_in_apply && it == iters - 1)
      PROF(s, K_APPLY_SOLID, k_apply_solid<true><<<blocks_for((long long)v.S * GL), 256, 0, st>>>(v, P));
    else
      PROF(s, K_APPLY_SOLID, k_apply_solid<false><<<blocks_for(v.S), 256, 0, st>>>(v, P));
    L += 2;
    if (tets) {
      PROF(s, K_SOLVE_TETS, k_solve_tets<<<blocks_for(v.S), 256, 0, st>>>(v, P));
      PROF(s, K_APPLY_SOLID_CONTACTS, k_apply_solid_contacts<<<blocks_for(v.S), 256, 0, st>>>(v, P));
      L += 2;
    }
    if (scc) {
      PROF(s, K_SOLID_CONTACTS, k_solid_contacts<<<blocks_for(v.S), 256, 0, st>>>(v, P));
      PROF(s, K_APPLY_SOLID_CONTACTS, k_apply_solid_contacts<<<blocks_for(v.S), 256, 0, st>>>(v, P));
      L += 2;
    }
  }
  if (!mark_in_apply && v.S > 0) {
    PROF(s, K_APPLY_SOLID, k_contact_mark<32><<<blocks_for((long long)v.S * 32), 256, 0, st>>>(v, P));
    L++;
  }
  UPBD_KCK(s);
  if (last < UPBD_PASS_BONDS) return UPBD_OK;
  {
    const int nb = v.C, nt = tets ? v.NT : 0;
    const int nb_pad = ((nb + nt + 31) / 32) * 32;
    const int nc = (last < UPBD_PASS_CONTACTS) ? 0 : v.N;
    const long long threads = (long long)nb_pad + (long long)nc * GL;
    PROF(s, K_BOND_CONTACTS,
         k_bond_contacts<<<blocks_for(threads), 256, 0, st>>>(v, P, nb, nt, nb_pad, nc));
    L++;
  }
  if (last < UPBD_PASS_APPLY_ALL) return UPBD_OK;
  {
    const int stage = (last < UPBD_PASS_BOUNDS) ? 1 : (last < UPBD_PASS_VELOCITY) ? 2 : 3;
    PROF(s, K_APPLY_BOUNDS_VEL, k_apply_bounds_vel<<<blocks_for(v.N), 256, 0, st>>>(v, P, stage));
    L++;
  }
  UPBD_KCK(s);
  if (last < UPBD_PASS_SOLID_VISC) return UPBD_OK;
  if (s->prm.solid_viscosity > 0) {
    PROF(s, K_SOLID_VISC, k_solid_visc<<<blocks_for(v.S), 256, 0, st>>>(v, P));
    PROF(s, K_SOLID_VISC, k_solid_visc_apply<<<blocks_for(v.S), 256, 0, st>>>(v));
    L += 2;
  }
  if (last < UPBD_PASS_XSPH) return UPBD_OK;
  if (last < UPBD_PASS_XSPH_APPLY) {  // stop with the result in delta, as the reference's xsph pass leaves it
    PROF(s, K_XSPH, k_xsph<false><<<blocks_for((long long)v.N * GLF), 256, 0, st>>>(v, P));
    L++;
    return UPBD_OK;
  }
  if (!s->prof_on && s->side) {
    // xsph as two launches side by side: the groups that walk on the side
    // stream (its launch first, so its long warps start early) and those that
    // read their lists on the main stream, each launch with the registers its
    // own form needs. Eager per-kernel timing keeps the one launch of both
    // forms.
    UPBD_CK(s, cudaEventRecord(s->fork_ev, st));
    UPBD_CK(s, cudaStreamWaitEvent(s->side, s->fork_ev, 0));
    k_xsph<true, 2><<<blocks_for((long long)v.N * GLF), 256, 0, s->side>>>(v, P);
    UPBD_CK(s, cudaEventRecord(s->join_ev, s->side));
    k_xsph<true, 1><<<blocks_for((long long)v.N * GLF), 256, 0, st>>>(v, P);
    UPBD_CK(s, cudaStreamWaitEvent(st, s->join_ev, 0));
    L += 2;
    UPBD_KCK(s);
    return UPBD_OK;
  }
  PROF(s, K_XSPH, k_xsph<true><<<blocks_for((long long)v.N * GLF), 256, 0, st>>>(v, P));
  L++;
  UPBD_KCK(s);
  return UPBD_OK;
}

int launch_frame(upbd_sim* s, int nsub, uint32_t emit_blocks, bool cut) {
  const SimView& v = s->v;
  const DevParams* P = s->dparams;
  cudaStream_t st = s->stream;
  if (emit_blocks) {
    PROF(s, K_EMIT, k_emit<<<emit_blocks, 64, 0, st>>>(v, P));
    s->launches++;
  }
  for (int k = 0; k < nsub; k++) {
    int rc = launch_substep(s, 1000);
    if (rc) return rc;
  }
  if (cut) {
    PROF(s, K_CUT, k_cut<<<blocks_for(v.C), 256, 0, st>>>(v, P));
    s->launches++;
    if ((s->desc.features & UPBD_FEAT_TETS) && v.NT > 0) {
      PROF(s, K_CUT, k_cut_tets<<<blocks_for(v.NT), 256, 0, st>>>(v, P));
      s->launches++;
    }
  }
  PROF(s, K_COUNT_ACTIVE, k_count_active<<<blocks_for(v.F), 256, 0, st>>>(v));
  s->launches++;
  UPBD_KCK(s);
  return UPBD_OK;
}

uint64_t count_graph_kernels(cudaGraph_t g) {
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

// One frame on the stream: GpuSim.encode (src/gpu/sim.js:333-398).
int enqueue_frame(upbd_sim* s, double h, int nsub, bool profile = false) {
  if (nsub < 1 || nsub > 1000) return fail(s, UPBD_ERR_INVALID, "substeps out of range [1, 1000]");
  if (!(h > 0) || !std::isfinite(h)) return fail(s, UPBD_ERR_INVALID, "substep length must be > 0");
  bool cut = false;
  if (!s->cuts.empty()) {
    const CutReq c = s->cuts.front();
    s->cuts.pop_front();
    for (int k = 0; k < 3; k++) {
      s->hp.cut_o[k] = c.o[k];
      s->hp.cut_d1[k] = c.d1[k];
      s->hp.cut_d2[k] = c.d2[k];
    }
    cut = true;
  }
  s->hp.h = (float)h;
  // grabDelta / substeps, src/gpu/sim.js:321-322 (JS double, f32 uniform)
  s->hp.grab_delta = make_float4((float)(s->grab_delta[0] / nsub), (float)(s->grab_delta[1] / nsub),
                                 (float)(s->grab_delta[2] / nsub), 0.f);
  uint32_t emit_blocks = 0;
  if (s->emit_pending && s->emit_count > 0) {
    s->hp.emit_count = s->emit_count;
    s->hp.emit_start = s->emit_start;
    s->hp.emit_pos = s->emit_pos;
    s->hp.emit_dir = s->emit_dir;
    s->hp.emit_side = s->emit_side;
    s->hp.emit_up = s->emit_up;
    // graph shape depends on the grid only: round up to a power of two
    uint32_t b = 1;
    while (b * 64 < s->emit_count) b <<= 1;
    emit_blocks = b;
  }
  int rc = upload_params(s);
  if (rc) return rc;
  if (s->use_graphs && !profile) {
    const bool visc = s->prm.solid_viscosity > 0;
    const uint64_t key = (uint64_t)nsub | ((uint64_t)emit_blocks << 16) | ((uint64_t)cut << 40) |
                         ((uint64_t)visc << 41);
    auto it = s->graphs.find(key);
    if (it == s->graphs.end()) {
      cudaGraph_t g;
      UPBD_CK(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
      const uint64_t before = s->launches;
      rc = launch_frame(s, nsub, emit_blocks, cut);
      cudaError_t ce = cudaStreamEndCapture(s->stream, &g);
      s->launches = before;
      if (rc) return rc;
      if (ce != cudaSuccess) return fail(s, UPBD_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
      cudaGraphExec_t ge;
      ce = cudaGraphInstantiate(&ge, g, 0);
      const uint64_t nk = count_graph_kernels(g);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess) return fail(s, UPBD_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(ce));
      it = s->graphs.emplace(key, upbd_sim::Graph{ge, nk}).first;
    }
    UPBD_CK(s, cudaGraphLaunch(it->second.exec, s->stream));
    s->launches += it->second.kernels;
  } else {
    s->prof_on = profile;
    rc = launch_frame(s, nsub, emit_blocks, cut);
    s->prof_on = false;
    if (rc) return rc;
  }
  if (s->emit_pending) {
    s->fluid_next = (int)(((long long)s->fluid_next + s->emit_count) % s->v.F);
    s->emit_pending = false;
  }
  s->grab_delta[0] = s->grab_delta[1] = s->grab_delta[2] = 0;
  s->frames++;
  return UPBD_OK;
}

}  // namespace

// =========================================================== C ABI
extern "C" {

int upbd_default_desc(upbd_scene_desc* d) {
  if (!d) return UPBD_ERR_INVALID;
  std::memset(d, 0, sizeof(*d));
  // GpuSim DEFAULTS, src/gpu/sim.js:20-33
  d->solid_dim = 20;
  d->solid_dim2 = 0;
  d->max_fluid = 65536;
  d->table_size = 1 << 18;
  d->substeps = 5;
  d->solid_iters = 8;
  d->features = 0;
  d->device = 0;
  d->spacing = 0.065;
  d->solid_mass = 0.004;
  d->fluid_mass = 0.0015;
  d->cube_center[0] = 0; d->cube_center[1] = 1.8; d->cube_center[2] = 0;
  d->cube2_center[0] = 1.1; d->cube2_center[1] = 0.5; d->cube2_center[2] = 0.7;
  return UPBD_OK;
}

int upbd_default_params(upbd_params* p) {
  if (!p) return UPBD_ERR_INVALID;
  std::memset(p, 0, sizeof(*p));
  // GpuSim DEFAULTS.params, src/gpu/sim.js:34-63
  p->h = 1.0 / 300; p->gravity = -10; p->solid_radius = 0.034; p->fluid_radius = 0.05;
  p->cell_size = 0.13; p->fluid_h = 0.13; p->rest_density = 3.0; p->stiffness = 0.0015;
  p->near_stiffness = 0.006; p->viscosity = 0.3; p->compliance = 5e-4; p->omega = 1.5;
  p->plastic_threshold = 0.38; p->plastic_rate = 0.04; p->tear_gap = 1.3; p->max_speed = 14;
  p->wall_x = 3.5; p->wall_z = 3.5; p->wall_h = 0.92; p->wall_t = 0.07; p->cull_r = 7.0;
  p->damp_solid = 1.2; p->damp_fluid = 0.6; p->friction_solid = 0.4; p->friction_fluid = 0.04;
  p->grab_k = 0.6; p->sleep_speed = 0; p->solid_viscosity = 0;
  p->break_strain = 2.6;   // src/solver.js:21
  p->contact_scale = 0.5;  // src/gpu/wgsl.js:641
  p->tear_mode = 0;
  p->plastic_clamp = 1;
  return UPBD_OK;
}

int upbd_create(const upbd_scene_desc* desc, const upbd_params* params, upbd_sim** out) {
  if (!out) return fail(nullptr, UPBD_ERR_INVALID, "null out");
  *out = nullptr;
  if (const char* why = check_desc(desc, params)) return fail(nullptr, UPBD_ERR_INVALID, why);
  int rc = UPBD_OK;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(nullptr, UPBD_ERR_NO_DEVICE, "no CUDA device");
  if (desc->device < 0 || desc->device >= ndev) return fail(nullptr, UPBD_ERR_INVALID, "bad device ordinal");
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, desc->device) != cudaSuccess || prop.major < 10)
    return fail(nullptr, UPBD_ERR_NO_DEVICE, "libupbd is built for sm_100a (B200); device is older");
  if (cudaSetDevice(desc->device) != cudaSuccess) return fail(nullptr, UPBD_ERR_CUDA, "cudaSetDevice failed");

  upbd_sim* s = new upbd_sim();
  s->desc = *desc;
  s->prm = *params;
  s->device = desc->device;
  HostScene hs;
  build_scene(*desc, hs);
  SimView& v = s->v;
  const SceneLayout L = layout_scene(*desc, hs, v);
  s->arena_bytes = L.bytes;
  if (cudaMalloc(&s->arena, s->arena_bytes) != cudaSuccess) {
    delete s;
    return fail(nullptr, UPBD_ERR_OOM, "device arena allocation failed");
  }
  bind_scene(L, (char*)s->arena, v, &s->dparams);

  auto cleanup_fail = [&](int code, const char* msg) {
    upbd_destroy(s);
    return fail(nullptr, code, msg);
  };
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup_fail(UPBD_ERR_CUDA, "stream creation failed");
  s->own_stream = true;
  if (cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->grid_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&s->join_ev, cudaEventDisableTiming) != cudaSuccess)
    return cleanup_fail(UPBD_ERR_CUDA, "side stream creation failed");
  if (cudaHostAlloc((void**)&s->stage, sizeof(DevParams) * kStageRing, cudaHostAllocDefault) != cudaSuccess)
    return cleanup_fail(UPBD_ERR_OOM, "pinned staging allocation failed");
  if (cudaHostAlloc((void**)&s->hmapped, sizeof(uint32_t) * HM_WORDS, cudaHostAllocMapped) != cudaSuccess)
    return cleanup_fail(UPBD_ERR_OOM, "mapped host allocation failed");
  std::memset(s->hmapped, 0, sizeof(uint32_t) * HM_WORDS);
  uint32_t* dmapped = nullptr;
  if (cudaHostGetDevicePointer((void**)&dmapped, s->hmapped, 0) != cudaSuccess)
    return cleanup_fail(UPBD_ERR_CUDA, "mapped host pointer failed");
  v.host_mapped = dmapped;
  for (int k = 0; k < kStageRing; k++)
    if (cudaEventCreateWithFlags(&s->stage_ev[k], cudaEventDisableTiming) != cudaSuccess)
      return cleanup_fail(UPBD_ERR_CUDA, "event creation failed");

  // uploads
  cudaStream_t st = s->stream;
  bool ok = cudaMemsetAsync(s->arena, 0, s->arena_bytes, st) == cudaSuccess;
  ok = ok && upload_scene(hs, v, st) == cudaSuccess;
  if (!ok) return cleanup_fail(UPBD_ERR_CUDA, "initial upload failed");
  s->init_pos = std::move(hs.pos);
  s->init_cons = std::move(hs.cons);
  s->init_tet_vol = std::move(hs.tet_vol);
  s->adj_host = std::move(hs.adj);
  fill_static_params(s);
  s->hp.grab_lattice = 0xffff;
  if (upload_params(s)) return cleanup_fail(UPBD_ERR_CUDA, "param upload failed");
  rc = upbd_reset_solid(s);
  if (rc) {
    upbd_destroy(s);
    return rc;
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) return cleanup_fail(UPBD_ERR_CUDA, "initial sync failed");
  *out = s;
  return UPBD_OK;
}

int upbd_destroy(upbd_sim* s) {
  if (!s) return UPBD_OK;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second.exec);
  for (cudaEvent_t e : s->prof_pool) cudaEventDestroy(e);
  for (int k = 0; k < kStageRing; k++)
    if (s->stage_ev[k]) cudaEventDestroy(s->stage_ev[k]);
  if (s->stage) cudaFreeHost(s->stage);
  if (s->hmapped) cudaFreeHost(s->hmapped);
  if (s->arena) cudaFree(s->arena);
  if (s->stream && s->own_stream) cudaStreamDestroy(s->stream);
  if (s->side) {
    cudaStreamSynchronize(s->side);
    cudaStreamDestroy(s->side);
  }
  if (s->rb_stream) {
    cudaStreamSynchronize(s->rb_stream);
    cudaStreamDestroy(s->rb_stream);
  }
  if (s->rb_ready) cudaEventDestroy(s->rb_ready);
  if (s->rb_done) cudaEventDestroy(s->rb_done);
  if (s->rb_stage) cudaFree(s->rb_stage);
  if (s->fork_ev) cudaEventDestroy(s->fork_ev);
  if (s->grid_ev) cudaEventDestroy(s->grid_ev);
  if (s->join_ev) cudaEventDestroy(s->join_ev);
  delete s;
  return UPBD_OK;
}

int upbd_get_info(upbd_sim* s, upbd_info* info) {
  if (!s || !info) return UPBD_ERR_INVALID;
  std::memset(info, 0, sizeof(*info));
  info->solid_n = s->v.S;
  info->n1 = s->v.N1;
  info->dim1 = s->v.dim1;
  info->dim2 = s->v.dim2;
  info->max_fluid = s->v.F;
  info->total = s->v.N;
  info->num_cons = s->v.C;
  info->num_tets = s->v.NT;
  info->table_size = s->v.T;
  info->substeps = s->desc.substeps;
  info->solid_iters = s->desc.solid_iters;
  info->fluid_next = s->fluid_next;
  info->features = s->desc.features;
  info->frames = s->frames;
  info->device_bytes = s->arena_bytes;
  info->param_bytes = (uint32_t)sizeof(DevParams);
  return UPBD_OK;
}

int upbd_set_params(upbd_sim* s, const upbd_params* p) {
  if (!s || !p) return UPBD_ERR_INVALID;
  if (!(p->cell_size > 0)) return fail(s, UPBD_ERR_INVALID, "cell_size must be > 0");
  cudaSetDevice(s->device);
  s->prm = *p;
  fill_static_params(s);
  return upload_params(s);
}

int upbd_get_params(upbd_sim* s, upbd_params* p) {
  if (!s || !p) return UPBD_ERR_INVALID;
  *p = s->prm;
  return UPBD_OK;
}

int upbd_set_stream(upbd_sim* s, void* stream) {
  if (!s) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  if (s->own_stream) cudaStreamDestroy(s->stream);
  s->own_stream = false;
  s->stream = (cudaStream_t)stream;
  if (!stream) {
    UPBD_CK(s, cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->own_stream = true;
  }
  return UPBD_OK;
}

int upbd_get_device_ptrs(upbd_sim* s, upbd_device_ptrs* o) {
  if (!s || !o) return UPBD_ERR_INVALID;
  o->pos = s->v.pos;
  o->prev = s->v.prev;
  o->vel = s->v.vel;
  o->density = s->v.density;
  o->flags = s->v.flags;
  o->cons = s->v.cons;
  o->stream = s->stream;
  return UPBD_OK;
}

const char* upbd_last_error(upbd_sim* s) {
  if (s) return s->err.c_str();
  return g_last_error.c_str();
}

int upbd_step(upbd_sim* s, double dt, int32_t substeps) {
  if (!s) return UPBD_ERR_INVALID;
  if (substeps < 1) return fail(s, UPBD_ERR_INVALID, "substeps must be >= 1");
  cudaSetDevice(s->device);
  return enqueue_frame(s, dt / substeps, substeps);
}

int upbd_frame(upbd_sim* s) {
  if (!s) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  return enqueue_frame(s, s->prm.h, s->desc.substeps);
}

int upbd_sync(upbd_sim* s) {
  if (!s) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  const uint32_t hb = ((volatile uint32_t*)s->hmapped)[HM_HEALTH];
  if (hb & UPBD_HEALTH_TIMEOUT) return fail(s, UPBD_ERR_TIMEOUT, "a bounded device wait gave up");
  if (hb & UPBD_HEALTH_NAN) return fail(s, UPBD_ERR_NAN, "non-finite velocity detected");
  if (hb & UPBD_HEALTH_BOUNDS)
    return fail(s, UPBD_ERR_INTERNAL, "an index out of range was skipped (checked build)");
  return UPBD_OK;
}

int upbd_health(upbd_sim* s, uint32_t* bits) {
  if (!s || !bits) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  uint32_t h = 0;
  UPBD_CK(s, cudaMemcpy(&h, &s->v.scratch[SCR_HEALTH], 4, cudaMemcpyDeviceToHost));
  *bits = h;
  return UPBD_OK;
}

int upbd_clear_health(upbd_sim* s) {
  if (!s) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  UPBD_CK(s, cudaMemsetAsync(&s->v.scratch[SCR_HEALTH], 0, 4, s->stream));
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  ((volatile uint32_t*)s->hmapped)[HM_HEALTH] = 0;
  return UPBD_OK;
}

int upbd_set_graphs(upbd_sim* s, int32_t enabled) {
  if (!s) return UPBD_ERR_INVALID;
  s->use_graphs = enabled != 0;
  return UPBD_OK;
}

int upbd_reset_solid(upbd_sim* s) {
  if (!s) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  const SimView& v = s->v;
  cudaStream_t st = s->stream;
  // GpuSim.resetSolid, src/gpu/sim.js:283-292: the whole pos/prev buffers
  // (fluid slots included) back to the initial data, every velocity zeroed,
  // solids' flags and density reset, constraints and tets pristine.
  UPBD_CK(s, state_to_device((real*)v.pos, (const float*)s->init_pos.data(), (size_t)v.N, 4, v, st));
  UPBD_CK(s, state_to_device((real*)v.prev, (const float*)s->init_pos.data(), (size_t)v.N, 4, v, st));
  UPBD_CK(s, cudaMemsetAsync(v.vel, 0, (size_t)v.N * sizeof(real4), st));
  if (v.S > 0) {
    UPBD_CK(s, cudaMemsetAsync(v.density, 0, (size_t)v.S * sizeof(real2), st));
    std::vector<uint32_t> f(v.S, F_ACTIVE);
    UPBD_CK(s, cudaMemcpyAsync(v.flags, f.data(), (size_t)v.S * 4, cudaMemcpyHostToDevice, st));
    UPBD_CK(s, cudaStreamSynchronize(st));
  }
  if (v.C > 0)
    UPBD_CK(s, cudaMemcpyAsync(v.cons, s->init_cons.data(), (size_t)v.C * 16, cudaMemcpyHostToDevice, st));
  if (v.NT > 0)
    UPBD_CK(s, cudaMemcpyAsync(v.tet_vol, s->init_tet_vol.data(), (size_t)v.NT * 4, cudaMemcpyHostToDevice, st));
  UPBD_CK(s, cudaStreamSynchronize(st));
  return UPBD_OK;
}

int upbd_drain(upbd_sim* s) {
  if (!s) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  if (s->v.F > 0) {
    k_drain<<<blocks_for(s->v.F), 256, 0, s->stream>>>(s->v);
    s->launches++;
    UPBD_KCK(s);
  }
  return UPBD_OK;
}

int upbd_active_count(upbd_sim* s, uint32_t* count) {
  if (!s || !count) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  k_count_active<<<blocks_for(s->v.F), 256, 0, s->stream>>>(s->v);
  s->launches++;
  UPBD_KCK(s);
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  *count = ((volatile uint32_t*)s->hmapped)[HM_ACTIVE];
  return UPBD_OK;
}

int upbd_emit(upbd_sim* s, int32_t count, const float pos[3], const float dir[3], const float side[3],
              const float up[3], float speed, float phase) {
  if (!s || !pos || !dir || !side || !up) return UPBD_ERR_INVALID;
  if (count < 0 || count > s->v.F) return fail(s, UPBD_ERR_CAPACITY, "emit count exceeds max_fluid");
  // GpuSim.emit, src/gpu/sim.js:400-407
  s->emit_pending = true;
  s->emit_count = (uint32_t)count;
  s->emit_start = (uint32_t)s->fluid_next;
  s->emit_pos = make_float4(pos[0], pos[1], pos[2], speed);
  s->emit_dir = make_float4(dir[0], dir[1], dir[2], phase);
  s->emit_side = make_float4(side[0], side[1], side[2], 0.f);
  s->emit_up = make_float4(up[0], up[1], up[2], 0.f);
  return UPBD_OK;
}

int upbd_emit_particles(upbd_sim* s, int32_t n, const float* pos3, const float* vel3, double mass) {
  if (!s || (n > 0 && (!pos3 || !vel3))) return UPBD_ERR_INVALID;
  if (n < 0 || n > s->v.F) return fail(s, UPBD_ERR_CAPACITY, "emit count exceeds max_fluid");
  if (!(mass > 0)) return fail(s, UPBD_ERR_INVALID, "mass must be > 0");
  if (n == 0) return UPBD_OK;
  cudaSetDevice(s->device);
  float* dbuf = nullptr;
  UPBD_CK(s, cudaMallocAsync((void**)&dbuf, (size_t)n * 24, s->stream));
  UPBD_CK(s, cudaMemcpyAsync(dbuf, pos3, (size_t)n * 12, cudaMemcpyHostToDevice, s->stream));
  UPBD_CK(s, cudaMemcpyAsync(dbuf + 3 * (size_t)n, vel3, (size_t)n * 12, cudaMemcpyHostToDevice, s->stream));
  k_emit_particles<<<blocks_for(n), 256, 0, s->stream>>>(s->v, dbuf, dbuf + 3 * (size_t)n, n, s->fluid_next,
                                                         (float)(1 / mass));
  s->launches++;
  UPBD_KCK(s);
  UPBD_CK(s, cudaFreeAsync(dbuf, s->stream));
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  s->fluid_next = (int)(((long long)s->fluid_next + n) % s->v.F);
  return UPBD_OK;
}

int upbd_slice(upbd_sim* s, const double o[3], const double d1[3], const double d2[3]) {
  if (!s || !o || !d1 || !d2) return UPBD_ERR_INVALID;
  CutReq c;
  std::memcpy(c.o, o, 24);
  std::memcpy(c.d1, d1, 24);
  std::memcpy(c.d2, d2, 24);
  s->cuts.push_back(c);
  return UPBD_OK;
}

int upbd_slice_now(upbd_sim* s, const double o[3], const double d1[3], const double d2[3],
                   uint32_t* cut_count) {
  if (!s || !o || !d1 || !d2) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  for (int k = 0; k < 3; k++) {
    s->hp.cut_o[k] = o[k];
    s->hp.cut_d1[k] = d1[k];
    s->hp.cut_d2[k] = d2[k];
  }
  int rc = upload_params(s);
  if (rc) return rc;
  UPBD_CK(s, cudaMemsetAsync(&s->v.scratch[SCR_CUT], 0, 4, s->stream));
  if (s->v.C > 0) {
    k_cut<<<blocks_for(s->v.C), 256, 0, s->stream>>>(s->v, s->dparams);
    s->launches++;
  }
  if ((s->desc.features & UPBD_FEAT_TETS) && s->v.NT > 0) {
    k_cut_tets<<<blocks_for(s->v.NT), 256, 0, s->stream>>>(s->v, s->dparams);
    s->launches++;
  }
  UPBD_KCK(s);
  uint32_t n = 0;
  UPBD_CK(s, cudaMemcpyAsync(&n, &s->v.scratch[SCR_CUT], 4, cudaMemcpyDeviceToHost, s->stream));
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  if (cut_count) *cut_count = n;
  return UPBD_OK;
}

int upbd_pick(upbd_sim* s, const double ro[3], const double rd[3], double max_perp, int32_t* id, double* t) {
  if (!s || !ro || !rd || !id) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  for (int k = 0; k < 3; k++) {
    s->hp.pick_o[k] = ro[k];
    s->hp.pick_d[k] = rd[k];
  }
  s->hp.pick_o[3] = max_perp;
  int rc = upload_params(s);
  if (rc) return rc;
  UPBD_CK(s, cudaMemsetAsync(&s->v.scratch[SCR_PICK_T], 0xff, 12, s->stream));
  if (s->v.S > 0) {
    k_pick_min_t<<<blocks_for(s->v.S), 256, 0, s->stream>>>(s->v, s->dparams);
    k_pick_min_i<<<blocks_for(s->v.S), 256, 0, s->stream>>>(s->v, s->dparams);
    s->launches += 2;
    UPBD_KCK(s);
  }
  uint32_t res[3];
  UPBD_CK(s, cudaMemcpyAsync(res, &s->v.scratch[SCR_PICK_T], 12, cudaMemcpyDeviceToHost, s->stream));
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  uint64_t bits = (uint64_t)res[0] | ((uint64_t)res[1] << 32);
  if (bits == ~0ull || res[2] == 0xffffffffu) {
    *id = -1;
    if (t) *t = INFINITY;
    return UPBD_OK;
  }
  *id = (int32_t)res[2];
  if (t) std::memcpy(t, &bits, 8);
  return UPBD_OK;
}

int upbd_grab_select(upbd_sim* s, const float center[3], float radius, uint32_t lattice) {
  if (!s || !center) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  s->hp.grab_c = make_float4(center[0], center[1], center[2], radius);
  s->hp.grab_lattice = lattice;
  int rc = upload_params(s);
  if (rc) return rc;
  if (s->v.S > 0) {
    k_grab_select<<<blocks_for(s->v.S), 256, 0, s->stream>>>(s->v, s->dparams);
    s->launches++;
    UPBD_KCK(s);
  }
  return UPBD_OK;
}

int upbd_grab_indices(upbd_sim* s, const uint32_t* idx, int32_t n, const float* weight, const float* targets3) {
  if (!s || (n > 0 && !idx) || n < 0) return UPBD_ERR_INVALID;
  if (n == 0) return UPBD_OK;
  for (int k = 0; k < n; k++)
    if (idx[k] >= (uint32_t)s->v.S) return fail(s, UPBD_ERR_INVALID, "grab index is not a solid");
  {
    std::vector<uint32_t> sorted(idx, idx + n);
    std::sort(sorted.begin(), sorted.end());
    if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
      return fail(s, UPBD_ERR_INVALID, "duplicate grab index");
  }
  cudaSetDevice(s->device);
  char* d = nullptr;
  const size_t bytes = (size_t)n * 20;
  UPBD_CK(s, cudaMallocAsync((void**)&d, bytes, s->stream));
  float* dw = (float*)(d + (size_t)n * 4);
  float* dt = (float*)(d + (size_t)n * 8);
  UPBD_CK(s, cudaMemcpyAsync(d, idx, (size_t)n * 4, cudaMemcpyHostToDevice, s->stream));
  if (weight) UPBD_CK(s, cudaMemcpyAsync(dw, weight, (size_t)n * 4, cudaMemcpyHostToDevice, s->stream));
  if (targets3) UPBD_CK(s, cudaMemcpyAsync(dt, targets3, (size_t)n * 12, cudaMemcpyHostToDevice, s->stream));
  k_grab_indices<<<blocks_for(n), 256, 0, s->stream>>>(s->v, (const uint32_t*)d, weight ? dw : nullptr,
                                                       targets3 ? dt : nullptr, n);
  s->launches++;
  UPBD_KCK(s);
  UPBD_CK(s, cudaFreeAsync(d, s->stream));
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  return UPBD_OK;
}

int upbd_grab_move(upbd_sim* s, const float delta[3]) {
  if (!s || !delta) return UPBD_ERR_INVALID;
  s->grab_delta[0] += delta[0];
  s->grab_delta[1] += delta[1];
  s->grab_delta[2] += delta[2];
  return UPBD_OK;
}

int upbd_release(upbd_sim* s) {
  if (!s) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  s->grab_delta[0] = s->grab_delta[1] = s->grab_delta[2] = 0;
  if (s->v.S > 0) {
    k_grab_release<<<blocks_for(s->v.S), 256, 0, s->stream>>>(s->v);
    s->launches++;
    UPBD_KCK(s);
  }
  return UPBD_OK;
}

int upbd_read_state(upbd_sim* s, float* pos4, float* prev4, float* vel4, float* density2, uint32_t* flags) {
  if (!s) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  const size_t N = (size_t)s->v.N;
  cudaStream_t st = s->stream;
  const SimView& v = s->v;
  if (pos4) UPBD_CK(s, state_to_host(pos4, (const real*)v.pos, N, 4, v, st));
  if (prev4) UPBD_CK(s, state_to_host(prev4, (const real*)v.prev, N, 4, v, st));
  if (vel4) UPBD_CK(s, state_to_host(vel4, (const real*)v.vel, N, 4, v, st));
  if (density2) UPBD_CK(s, state_to_host(density2, (const real*)v.density, N, 2, v, st));
  if (flags) UPBD_CK(s, cudaMemcpyAsync(flags, s->v.flags, N * 4, cudaMemcpyDeviceToHost, st));
  UPBD_CK(s, cudaStreamSynchronize(st));
  return UPBD_OK;
}

int upbd_read_state_async(upbd_sim* s, float* pos4, uint32_t* flags) {
  if (!s) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  const size_t N = (size_t)s->v.N;
  if (!s->rb_stage) {  // first use: staging copy, copy stream and its events
    if (!s->rb_stream) UPBD_CK(s, cudaStreamCreateWithFlags(&s->rb_stream, cudaStreamNonBlocking));
    if (!s->rb_ready) UPBD_CK(s, cudaEventCreateWithFlags(&s->rb_ready, cudaEventDisableTiming));
    if (!s->rb_done) UPBD_CK(s, cudaEventCreateWithFlags(&s->rb_done, cudaEventDisableTiming));
    UPBD_CK(s, cudaEventRecord(s->rb_done, s->rb_stream));
    UPBD_CK(s, cudaMalloc(&s->rb_stage, N * 20));  // last: its presence means all are ready
  }
  float4* spos = (float4*)s->rb_stage;
  uint32_t* sflags = (uint32_t*)(spos + N);
  cudaStream_t st = s->stream;
  // the staging copy may still be on its way to the host from the last call
  UPBD_CK(s, cudaStreamWaitEvent(st, s->rb_done, 0));
  if (pos4) UPBD_CK(s, state_to_f32((float*)spos, (const real*)s->v.pos, N, 4, st));
  if (flags) UPBD_CK(s, cudaMemcpyAsync(sflags, s->v.flags, N * 4, cudaMemcpyDeviceToDevice, st));
  UPBD_CK(s, cudaEventRecord(s->rb_ready, st));
  UPBD_CK(s, cudaStreamWaitEvent(s->rb_stream, s->rb_ready, 0));
  if (pos4) UPBD_CK(s, cudaMemcpyAsync(pos4, spos, N * 16, cudaMemcpyDeviceToHost, s->rb_stream));
  if (flags) UPBD_CK(s, cudaMemcpyAsync(flags, sflags, N * 4, cudaMemcpyDeviceToHost, s->rb_stream));
  UPBD_CK(s, cudaEventRecord(s->rb_done, s->rb_stream));
  return UPBD_OK;
}

int upbd_read_wait(upbd_sim* s) {
  if (!s) return UPBD_ERR_INVALID;
  if (!s->rb_done) return UPBD_OK;
  cudaSetDevice(s->device);
  UPBD_CK(s, cudaEventSynchronize(s->rb_done));
  return UPBD_OK;
}

int upbd_write_state(upbd_sim* s, const float* pos4, const float* prev4, const float* vel4,
                     const float* density2, const uint32_t* flags) {
  if (!s) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  const size_t N = (size_t)s->v.N;
  cudaStream_t st = s->stream;
  const SimView& v = s->v;
  if (pos4) UPBD_CK(s, state_to_device((real*)v.pos, pos4, N, 4, v, st));
  if (prev4) UPBD_CK(s, state_to_device((real*)v.prev, prev4, N, 4, v, st));
  if (vel4) UPBD_CK(s, state_to_device((real*)v.vel, vel4, N, 4, v, st));
  if (density2) UPBD_CK(s, state_to_device((real*)v.density, density2, N, 2, v, st));
  if (flags) UPBD_CK(s, cudaMemcpyAsync(s->v.flags, flags, N * 4, cudaMemcpyHostToDevice, st));
  UPBD_CK(s, cudaStreamSynchronize(st));
  return UPBD_OK;
}

int upbd_read_constraints(upbd_sim* s, uint32_t* cons4) {
  if (!s || !cons4) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  if (s->v.C > 0)
    UPBD_CK(s, cudaMemcpyAsync(cons4, s->v.cons, (size_t)s->v.C * 16, cudaMemcpyDeviceToHost, s->stream));
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  return UPBD_OK;
}

int upbd_write_constraints(upbd_sim* s, const uint32_t* cons4) {
  if (!s || !cons4) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  for (int c = 0; c < s->v.C; c++) {
    const uint4 ic = s->init_cons[c];
    if (cons4[4 * c] != ic.x || cons4[4 * c + 1] != ic.y)
      return fail(s, UPBD_ERR_INVALID, "constraint endpoints must match the scene's");
  }
  if (s->v.C > 0)
    UPBD_CK(s, cudaMemcpyAsync(s->v.cons, cons4, (size_t)s->v.C * 16, cudaMemcpyHostToDevice, s->stream));
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  return UPBD_OK;
}

int upbd_read_adjacency(upbd_sim* s, uint32_t* adj) {
  if (!s || !adj) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  UPBD_CK(s, cudaMemcpyAsync(adj, s->v.adj, s->adj_host.size() * 4, cudaMemcpyDeviceToHost, s->stream));
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  return UPBD_OK;
}

int upbd_read_grid(upbd_sim* s, uint32_t* counts, uint32_t* offsets, uint32_t* entries, uint32_t* n_entries) {
  if (!s) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  const size_t T = (size_t)s->v.T;
  std::vector<uint32_t> off(T + 1);
  UPBD_CK(s, cudaMemcpyAsync(off.data(), s->v.start, (T + 1) * 4, cudaMemcpyDeviceToHost, s->stream));
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  const uint32_t n = off[T];
  if (n > (uint32_t)s->v.N) return fail(s, UPBD_ERR_INVALID, "grid not built");
  if (offsets) std::memcpy(offsets, off.data(), (T + 1) * 4);
  if (counts)
    for (size_t h = 0; h < T; h++) counts[h] = off[h + 1] - off[h];
  if (entries && n > 0) {
    UPBD_CK(s, cudaMemcpyAsync(entries, s->v.entries, (size_t)n * 4, cudaMemcpyDeviceToHost, s->stream));
    UPBD_CK(s, cudaStreamSynchronize(s->stream));
  }
  if (n_entries) *n_entries = n;
  return UPBD_OK;
}

int upbd_rebuild_grid(upbd_sim* s) {
  if (!s) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  const SimView& v = s->v;
  cudaStream_t st = s->stream;
  k_integrate_count<false, true><<<blocks_for(v.N), 256, 0, st>>>(v, s->dparams);
  k_scan<<<v.num_tiles, SCAN_THREADS, 0, st>>>(v);
  k_scatter<<<blocks_for(std::max(v.N, tile_words(v.num_tiles))), 256, 0, st>>>(v);
  k_rankfix<<<blocks_for(v.N), 256, 0, st>>>(v);
  s->launches += 4;
  UPBD_KCK(s);
  UPBD_CK(s, cudaStreamSynchronize(st));
  return UPBD_OK;
}

int upbd_substep_partial(upbd_sim* s, double h, int32_t last_pass) {
  if (!s) return UPBD_ERR_INVALID;
  if (!(h > 0)) return fail(s, UPBD_ERR_INVALID, "h must be > 0");
  cudaSetDevice(s->device);
  s->hp.h = (float)h;
  s->hp.grab_delta = make_float4(0, 0, 0, 0);
  int rc = upload_params(s);
  if (rc) return rc;
  rc = launch_substep(s, last_pass);
  if (rc) return rc;
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  return UPBD_OK;
}

int upbd_read_tets(upbd_sim* s, uint32_t* tets5) {
  if (!s || !tets5) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  const int NT = s->v.NT;
  if (NT == 0) return UPBD_OK;
  std::vector<uint32_t> idx(4 * (size_t)NT);
  std::vector<float> vol(NT);
  UPBD_CK(s, cudaMemcpyAsync(idx.data(), s->v.tet_idx, idx.size() * 4, cudaMemcpyDeviceToHost, s->stream));
  UPBD_CK(s, cudaMemcpyAsync(vol.data(), s->v.tet_vol, vol.size() * 4, cudaMemcpyDeviceToHost, s->stream));
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  for (int t = 0; t < NT; t++) {
    for (int q = 0; q < 4; q++) tets5[5 * t + q] = idx[4 * t + q];
    std::memcpy(&tets5[5 * t + 4], &vol[t], 4);
  }
  return UPBD_OK;
}

int upbd_write_tets(upbd_sim* s, const uint32_t* tets5) {
  if (!s || !tets5) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  const int NT = s->v.NT;
  if (NT == 0) return UPBD_OK;
  std::vector<uint32_t> idx(4 * (size_t)NT);
  std::vector<float> vol(NT);
  UPBD_CK(s, cudaMemcpyAsync(idx.data(), s->v.tet_idx, idx.size() * 4, cudaMemcpyDeviceToHost, s->stream));
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  for (int t = 0; t < NT; t++) {
    for (int q = 0; q < 4; q++)
      if (tets5[5 * t + q] != idx[4 * t + q]) return fail(s, UPBD_ERR_INVALID, "tet vertices must match the scene's");
    std::memcpy(&vol[t], &tets5[5 * t + 4], 4);
  }
  UPBD_CK(s, cudaMemcpyAsync(s->v.tet_vol, vol.data(), vol.size() * 4, cudaMemcpyHostToDevice, s->stream));
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  return UPBD_OK;
}

int upbd_set_fluid_next(upbd_sim* s, int32_t next) {
  if (!s) return UPBD_ERR_INVALID;
  if (next < 0 || (s->v.F > 0 && next >= s->v.F) || (s->v.F == 0 && next != 0))
    return fail(s, UPBD_ERR_INVALID, "fluid_next out of range [0, max_fluid)");
  s->fluid_next = next;
  return UPBD_OK;
}

// Solver._recomputeGroups, src/solver.js:488-499 — union-find with path
// halving over alive constraints in constraint order, on the host over the
// downloaded alive flags (the same sequential algorithm, so root ids match).
int upbd_groups_device(upbd_sim* s, int32_t* d_group) {
  if (!s) return UPBD_ERR_INVALID;
  const int S = s->v.S, C = s->v.C;
  if (S == 0) return UPBD_OK;
  if (!d_group) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  cudaStream_t st = s->stream;
  int32_t* par = reinterpret_cast<int32_t*>(s->v.tmp);  // the grid's scatter buffer, N >= S words
  if (S <= GROUPS_SMEM_MAX) {
    const size_t smem = (size_t)S * sizeof(int32_t);
    if (smem > 48 * 1024)
      UPBD_CK(s, cudaFuncSetAttribute(k_groups_replay<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    k_groups_replay<true><<<1, 32, smem, st>>>(s->v.cons, C, S, par);
  } else {
    k_groups_replay<false><<<1, 32, 0, st>>>(s->v.cons, C, S, par);
  }
  UPBD_KCK(s);
  k_groups_label<<<blocks_for(S), 256, 0, st>>>(par, S, d_group);
  UPBD_KCK(s);
  return UPBD_OK;
}

int upbd_groups(upbd_sim* s, int32_t* group) {
  if (!s || (!group && s->v.S > 0)) return UPBD_ERR_INVALID;
  const int S = s->v.S;
  if (S == 0) return UPBD_OK;
  // labels land in the grid's ticket buffer (N >= S words, free between
  // substeps) and come back in one copy
  int32_t* d = reinterpret_cast<int32_t*>(s->v.ticket);
  if (int rc = upbd_groups_device(s, d)) return rc;
  UPBD_CK(s, cudaMemcpyAsync(group, d, (size_t)S * sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  return UPBD_OK;
}

// ---------------------------------------------------- stateless grid build
namespace {
struct GridPool {
  std::mutex mu;
  struct Dev {
    void* mem = nullptr;
    size_t n_cap = 0, t_cap = 0;
  } dev[64];
};
GridPool g_pool;

// counts[h] = offsets[h+1] - offsets[h] (the scan clears its own counts)
__global__ void k_counts_from_offsets(const uint32_t* __restrict__ offsets, uint32_t* __restrict__ counts, int T) {
  const int h = UPBD_TID;
  if (h < T) counts[h] = offsets[h + 1] - offsets[h];
}

}  // namespace

int upbd_grid_build(const void* pos4, const void* flags, int32_t n, int32_t table_size, double cell_size,
                    void* counts, void* offsets, void* entries, void* stream) {
#ifdef UPBD_FP64_BUILD
  return fail(nullptr, UPBD_ERR_INVALID, "the stateless grid build reads float rows: not in the FP64 build");
#endif
  if (n < 0 || (n > 0 && (!pos4 || !flags || !entries)) || !offsets)
    return fail(nullptr, UPBD_ERR_INVALID, "bad grid_build arguments");
  if (table_size < 1 || (table_size & (table_size - 1)) || table_size > (1 << 28))
    return fail(nullptr, UPBD_ERR_INVALID, "table_size must be a power of two <= 2^28");
  if (!(cell_size > 0)) return fail(nullptr, UPBD_ERR_INVALID, "cell_size must be > 0");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev >= 64) return fail(nullptr, UPBD_ERR_NO_DEVICE, "no device");
  cudaStream_t st = (cudaStream_t)stream;
  const int tiles = (table_size + SCAN_TILE - 1) / SCAN_TILE;
  std::lock_guard<std::mutex> lk(g_pool.mu);
  GridPool::Dev& pd = g_pool.dev[dev];
  if ((size_t)n > pd.n_cap || (size_t)table_size > pd.t_cap) {
    if (pd.mem) {
      cudaDeviceSynchronize();
      cudaFree(pd.mem);
      pd.mem = nullptr;
      pd.n_cap = pd.t_cap = 0;
    }
    const size_t nc = std::max<size_t>((size_t)n, pd.n_cap), tc = std::max<size_t>((size_t)table_size, pd.t_cap);
    const size_t bytes = grid_scratch_layout(nc, tc, sizeof(DevParams)).words * 4;
    if (cudaMalloc(&pd.mem, bytes) != cudaSuccess) return fail(nullptr, UPBD_ERR_OOM, "grid scratch allocation failed");
    // cleared in the caller's stream order: the count kernel below runs on
    // that stream, which may be a non-blocking one
    if (cudaMemsetAsync(pd.mem, 0, bytes, st) != cudaSuccess)
      return fail(nullptr, UPBD_ERR_CUDA, "grid scratch clear failed");
    pd.n_cap = nc;
    pd.t_cap = tc;
  }
  const GridScratchLayout lay = grid_scratch_layout(pd.n_cap, pd.t_cap, sizeof(DevParams));
  uint32_t* w = (uint32_t*)pd.mem;
  SimView v{};
  v.pos = (real4*)pos4;
  v.flags = (uint32_t*)flags;
  v.N = n;
  v.T = table_size;
  v.num_tiles = tiles;
  v.counts = w + lay.counts;
  v.ticket = w + lay.ticket;
  v.cell = w + lay.cell;
  v.tmp = w + lay.tmp;
  v.tile_sum = w + lay.tiles;
  v.start = (uint32_t*)offsets;
  v.entries = (uint32_t*)entries;
  // the count kernel reads 1/cell_size (a double) from a params block at the
  // pool's tail, on a 256-byte boundary
  DevParams* dp = (DevParams*)(w + lay.params);
  if ((reinterpret_cast<uintptr_t>(dp) & 15u) != 0)
    return fail(nullptr, UPBD_ERR_INTERNAL, "grid scratch params block is not 16-byte aligned");
  DevParams hp{};
  hp.inv_cell = 1.0 / cell_size;
  if (cudaMemcpyAsync(dp, &hp, sizeof(DevParams), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return fail(nullptr, UPBD_ERR_CUDA, "params upload failed");
  k_integrate_count<false, true><<<blocks_for(n), 256, 0, st>>>(v, dp);
  k_scan<<<tiles, SCAN_THREADS, 0, st>>>(v);
  k_scatter<<<blocks_for(std::max(n, tile_words(tiles))), 256, 0, st>>>(v);
  k_rankfix<<<blocks_for(n), 256, 0, st>>>(v);
  // counts[h] = offsets[h+1] - offsets[h] (the scan cleared its own counts)
  if (counts) k_counts_from_offsets<<<blocks_for(table_size), 256, 0, st>>>(v.start, (uint32_t*)counts, table_size);
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) return fail(nullptr, UPBD_ERR_CUDA, cudaGetErrorString(e));
  return UPBD_OK;
}

// Kernels launched on this handle so far (captured frames count their nodes).
uint64_t upbd_launch_count(upbd_sim* s) { return s ? s->launches : 0; }

const char* upbd_kernel_name(int32_t kind) {
  return (kind >= 0 && kind < K_NUM_KINDS) ? kKernelNames[kind] : nullptr;
}

int upbd_profile_frame(upbd_sim* s, double dt, int32_t substeps, double* ms, uint32_t* launches) {
  if (!s || !ms || !launches || substeps < 1) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  s->prof.clear();
  s->prof_used = 0;
  int rc = enqueue_frame(s, dt / substeps, substeps, true);
  if (rc) return rc;
  UPBD_CK(s, cudaStreamSynchronize(s->stream));
  for (int k = 0; k < UPBD_KERNEL_KINDS; k++) {
    ms[k] = 0;
    launches[k] = 0;
  }
  for (const ProfRec& r : s->prof) {
    float t = 0;
    UPBD_CK(s, cudaEventElapsedTime(&t, r.a, r.b));
    ms[r.kind] += t;
    launches[r.kind]++;
  }
  s->prof.clear();
  s->prof_used = 0;
  return UPBD_OK;
}

// The launch floor of a frame graph: the frame is captured as upbd_step
// captures it, then every kernel node of a copy is given an empty kernel with
// the node's own grid and block, so the copy keeps the graph's shape (nodes,
// dependencies, the side-stream branches, the memset nodes) and does no work.
// Its replay time is what the frame pays for launching and ordering its
// kernels. Nothing in the simulation's state changes.
int upbd_profile_graph_floor(upbd_sim* s, double dt, int32_t substeps, int32_t reps, double* floor_ms,
                             uint32_t* kernel_nodes) {
  if (!s || !floor_ms || !kernel_nodes || substeps < 1 || substeps > 1000 || reps < 1) return UPBD_ERR_INVALID;
  cudaSetDevice(s->device);
  cudaGraph_t g = nullptr;
  UPBD_CK(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  const uint64_t before = s->launches;
  int rc = launch_frame(s, substeps, 0u, false);
  cudaError_t ce = cudaStreamEndCapture(s->stream, &g);
  s->launches = before;
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (ce != cudaSuccess) return fail(s, UPBD_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
  size_t n = 0;
  cudaGraphGetNodes(g, nullptr, &n);
  std::vector<cudaGraphNode_t> nodes(n);
  cudaGraphGetNodes(g, nodes.data(), &n);
  uint32_t nk = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nd, &t) != cudaSuccess || t != cudaGraphNodeTypeKernel) continue;
    cudaKernelNodeParams kp;
    ce = cudaGraphKernelNodeGetParams(nd, &kp);
    if (ce == cudaSuccess) {
      kp.func = (void*)k_empty;
      kp.sharedMemBytes = 0;
      kp.kernelParams = nullptr;
      kp.extra = nullptr;
      ce = cudaGraphKernelNodeSetParams(nd, &kp);
    }
    if (ce != cudaSuccess) {
      cudaGraphDestroy(g);
      return fail(s, UPBD_ERR_CUDA, std::string("kernel node: ") + cudaGetErrorString(ce));
    }
    nk++;
  }
  cudaGraphExec_t ge;
  ce = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) return fail(s, UPBD_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(ce));
  cudaEvent_t a = nullptr, b = nullptr;
  ce = cudaEventCreate(&a);
  if (ce == cudaSuccess) ce = cudaEventCreate(&b);
  for (int k = 0; k < 3 && ce == cudaSuccess; k++) ce = cudaGraphLaunch(ge, s->stream);
  if (ce == cudaSuccess) ce = cudaEventRecord(a, s->stream);
  for (int k = 0; k < reps && ce == cudaSuccess; k++) ce = cudaGraphLaunch(ge, s->stream);
  if (ce == cudaSuccess) ce = cudaEventRecord(b, s->stream);
  if (ce == cudaSuccess) ce = cudaEventSynchronize(b);
  float t = 0.f;
  if (ce == cudaSuccess) ce = cudaEventElapsedTime(&t, a, b);
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  cudaGraphExecDestroy(ge);
  if (ce != cudaSuccess) return fail(s, UPBD_ERR_CUDA, std::string("floor timing: ") + cudaGetErrorString(ce));
  *floor_ms = (double)t / reps;
  *kernel_nodes = nk;
  return UPBD_OK;
}

}  // extern "C"

// ===================================================== allocation-free grid build
// upbd_grid_build takes its scratch (bucket counts, arrival tickets, bucket of
// each particle, the unordered scatter, scan tile totals) from a pool that it
// grows with cudaMalloc. Some callers cannot allocate device memory at all: a
// host that embeds this library in a runtime which owns the device-memory
// budget and refuses allocations it did not make, or a frame loop that must
// never stall on an allocation. For them, upbd_grid_build_noalloc keeps the
// same scratch in this file-scope array, which lives in the library image:
// every GPU that loads the library holds its 4 MiB until the process exits.
namespace {

constexpr int kNoAllocMaxN = 1 << 18;  // particles per call
constexpr int kNoAllocMaxT = 1 << 18;  // hash buckets per call
// word offsets inside the array (params on a 256-byte boundary)
constexpr GridScratchLayout kNa = grid_scratch_layout(kNoAllocMaxN, kNoAllocMaxT, sizeof(DevParams));
static_assert(kNa.params % 64 == 0, "params block must start on a 256-byte boundary");
constexpr size_t kNaWords = kNa.words;

__device__ __align__(256) uint32_t g_grid_scratch[kNaWords];

std::mutex g_noalloc_mu;
uint32_t* g_noalloc_ptr[64] = {};  // device address of g_grid_scratch, per device

// The hash reads 1/cell_size from a params block: set it on the device from
// a kernel argument (no host-to-device copy, no staging buffer).
__global__ void k_noalloc_params(DevParams* p, double inv_cell) { p->inv_cell = inv_cell; }

}  // namespace

extern "C" int upbd_grid_build_noalloc(const void* pos4, const void* flags, int32_t n, int32_t table_size,
                                       double cell_size, void* counts, void* offsets, void* entries,
                                       void* stream) {
#ifdef UPBD_FP64_BUILD
  return fail(nullptr, UPBD_ERR_INVALID, "the stateless grid build reads float rows: not in the FP64 build");
#endif
  if (n < 0 || (n > 0 && (!pos4 || !flags || !entries)) || !offsets)
    return fail(nullptr, UPBD_ERR_INVALID, "bad grid_build_noalloc arguments");
  if (table_size < 1 || (table_size & (table_size - 1)))
    return fail(nullptr, UPBD_ERR_INVALID, "table_size must be a power of two");
  if (n > kNoAllocMaxN || table_size > kNoAllocMaxT)
    return fail(nullptr, UPBD_ERR_CAPACITY,
                "grid_build_noalloc handles at most 262144 particles and 262144 buckets per call "
                "(its scratch is a fixed array in the library)");
  if (!(cell_size > 0)) return fail(nullptr, UPBD_ERR_INVALID, "cell_size must be > 0");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return fail(nullptr, UPBD_ERR_NO_DEVICE, "no current CUDA device");
  uint32_t* w = nullptr;
  {
    // set-up, once per device and with that device current: the array's name
    // is a host-side stand-in, the kernels need its device address
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_grid_scratch);
      if (e != cudaSuccess)
        return fail(nullptr, UPBD_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_noalloc_ptr[dev] = (uint32_t*)p;
    }
    w = g_noalloc_ptr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int tiles = (table_size + SCAN_TILE - 1) / SCAN_TILE;
  SimView v{};
  v.pos = (real4*)pos4;
  v.flags = (uint32_t*)flags;
  v.N = n;
  v.T = table_size;
  v.num_tiles = tiles;
  v.counts = w + kNa.counts;
  v.ticket = w + kNa.ticket;
  v.cell = w + kNa.cell;
  v.tmp = w + kNa.tmp;
  v.tile_sum = w + kNa.tiles;
  v.start = (uint32_t*)offsets;
  v.entries = (uint32_t*)entries;
  DevParams* dp = (DevParams*)(w + kNa.params);
  // the array keeps the previous call's contents: counts and tile totals
  // must start at zero
  cudaError_t e = cudaMemsetAsync(v.counts, 0, (size_t)table_size * 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(v.tile_sum, 0, (size_t)tile_words(tiles) * 4, st);
  if (e != cudaSuccess) return fail(nullptr, UPBD_ERR_CUDA, std::string("scratch clear: ") + cudaGetErrorString(e));
  k_noalloc_params<<<1, 1, 0, st>>>(dp, 1.0 / cell_size);
  k_integrate_count<false, true><<<blocks_for(n), 256, 0, st>>>(v, dp);
  k_scan<<<tiles, SCAN_THREADS, 0, st>>>(v);
  k_scatter<<<blocks_for(std::max(n, tile_words(tiles))), 256, 0, st>>>(v);
  k_rankfix<<<blocks_for(n), 256, 0, st>>>(v);
  if (counts) k_counts_from_offsets<<<blocks_for(table_size), 256, 0, st>>>(v.start, (uint32_t*)counts, table_size);
  e = cudaPeekAtLastError();
  if (e != cudaSuccess) return fail(nullptr, UPBD_ERR_CUDA, cudaGetErrorString(e));
  return UPBD_OK;
}
