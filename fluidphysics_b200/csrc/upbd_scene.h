// Host-side scene construction shared by the single-scene handle (upbd.cu)
// and the batch of scenes (upbd_batch.cu): the host data of
// _buildHostData (src/gpu/sim.js:98-214), the layout of one scene's arrays
// inside its device arena, the static uploads, and the f32 uniform block.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <memory>
#include <vector>

#include "../../include/upbd.h"
#include "upbd_device.cuh"

namespace upbd {

struct HostScene {
  std::vector<float4> pos;
  std::vector<uint4> cons;
  std::vector<uint32_t> adj;
  std::vector<uint32_t> adj_other;
  std::vector<float> adj_scale;
  std::vector<uint32_t> tet_idx;
  std::vector<float> tet_vol;
  std::vector<uint32_t> tet_adj;
  int S = 0, N1 = 0, N = 0;
};

// Lattices, 26-neighbour constraints, CSR adjacency, tets with rest volumes
// and their CSR (_buildHostData, src/gpu/sim.js:98-214).
void build_scene(const upbd_scene_desc& d, HostScene& out);

// Byte offsets of one scene's arrays inside its arena (each 256-byte aligned).
struct SceneLayout {
  size_t pos, prev, vel, delta, dens, flags, cons, adj, counts, start, entries, tmp, ticket, cell, tiles;
  size_t tidx, tvol, tadj, mark, spos, sdens, svel, slot, fend, nbr, ncount, aoth, ascl, ccount, clist;
  size_t sbuf, sfp, smove, bmove, scr, par, conv;
  size_t bytes;
};

// Fills the sizes of v from the descriptor and host scene (full or
// lattice-only: N = S + d.max_fluid) and returns the arena layout;
// bind_scene then points v's arrays (and *params, the scene's uniform block)
// into an arena that starts at base.
SceneLayout layout_scene(const upbd_scene_desc& d, const HostScene& hs, SimView& v);
void bind_scene(const SceneLayout& L, char* base, SimView& v, DevParams** params);

// Copies of particle-state rows (comps = 4 for pos/prev/vel/delta, 2 for
// density) between host float rows and device rows of the scalar type
// `real`, asynchronous on st. In the FP32 builds they are plain copies; in
// the FP64 build the rows pass through v.conv and a conversion kernel (so
// calls on one stream must not overlap the caller's use of v.conv).
// state_to_f32 writes float rows to device memory (the readback staging).
cudaError_t state_to_device(real* dst, const float* src_host, size_t rows, int comps, const SimView& v,
                            cudaStream_t st);
cudaError_t state_to_host(float* dst_host, const real* src, size_t rows, int comps, const SimView& v,
                          cudaStream_t st);
cudaError_t state_to_f32(float* dst_dev, const real* src, size_t rows, int comps, cudaStream_t st);

// Uploads into a zeroed arena: the static CSR data and tets, then the
// initial state of GpuSim's constructor and resetSolid (src/gpu/sim.js:174,
// 283-292): pos and prev from the host scene (fluid slots inactive with
// their inverse mass), solids active, constraints and tets pristine.
cudaError_t upload_scene(const HostScene& hs, const SimView& v, cudaStream_t st);

// The lattice part of a scene: build_scene of the descriptor with no fluid
// slots (N = S). Scenes whose bodies agree (dims, spacing, solid mass,
// centres) share one entry; the cache is thread-safe and bounded.
std::shared_ptr<const HostScene> lattice_of(const upbd_scene_desc& d);

// Host data of one scene ready for upload into a fresh arena: the shared
// lattice plus its own fluid slots, laid out as upbd_create followed by
// upbd_emit_particles leaves them (placed slots: pos (x, y, z, 1/mass),
// prev (x, y, z, 0), active; the other slots: (0, 0, 0, 1/fluid_mass)).
struct PreparedScene {
  upbd_scene_desc desc{};
  upbd_params prm{};
  std::shared_ptr<const HostScene> lat;
  std::vector<float4> fluid_pos;   // max_fluid slots
  std::vector<float4> fluid_prev;  // max_fluid slots
  std::vector<float4> fluid_vel;   // n_fluid slots, empty = at rest
  int n_fluid = 0;
};

// nullptr on success, else the reason (then `out` is unspecified).
const char* prepare_scene(const upbd_scene_desc& d, const upbd_params& p, int n_fluid, const float* pos3,
                          const float* vel3, double mass, PreparedScene& out);
// Enqueues the uploads of a prepared scene into a zeroed arena bound to v.
// The copies are from pageable memory: keep `ps` alive until the stream
// has passed them.
cudaError_t upload_prepared(const PreparedScene& ps, const SimView& v, cudaStream_t st);

// nullptr when the descriptor and parameters are valid, else the reason.
const char* check_desc(const upbd_scene_desc* d, const upbd_params* p);

// _writeParams, src/gpu/sim.js:300-330: JS numbers rounded into the f32
// uniform block (the per-frame fields are left to the caller).
void fill_dev_params(const upbd_params& p, const upbd_scene_desc& d, DevParams& out);

}  // namespace upbd
