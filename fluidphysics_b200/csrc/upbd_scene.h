// Host-side scene construction shared by the single-scene handle (upbd.cu)
// and the batch of scenes (upbd_batch.cu): the host data of
// _buildHostData (src/gpu/sim.js:98-214), the layout of one scene's arrays
// inside its device arena, the static uploads, and the f32 uniform block.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
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
  size_t scr, par;
  size_t bytes;
};

// Fills the sizes of v from the descriptor and host scene and returns the
// arena layout; bind_scene then points v's arrays (and *params, the scene's
// uniform block) into an arena that starts at base.
SceneLayout layout_scene(const upbd_scene_desc& d, const HostScene& hs, SimView& v);
void bind_scene(const SceneLayout& L, char* base, SimView& v, DevParams** params);

// Uploads into a zeroed arena: the static CSR data and tets, then the
// initial state of GpuSim's constructor and resetSolid (src/gpu/sim.js:174,
// 283-292): pos and prev from the host scene (fluid slots inactive with
// their inverse mass), solids active, constraints and tets pristine.
cudaError_t upload_scene(const HostScene& hs, const SimView& v, cudaStream_t st);

// nullptr when the descriptor and parameters are valid, else the reason.
const char* check_desc(const upbd_scene_desc* d, const upbd_params* p);

// _writeParams, src/gpu/sim.js:300-330: JS numbers rounded into the f32
// uniform block (the per-frame fields are left to the caller).
void fill_dev_params(const upbd_params& p, const upbd_scene_desc& d, DevParams& out);

}  // namespace upbd
