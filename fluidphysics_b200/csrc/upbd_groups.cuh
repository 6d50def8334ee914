// Solver._recomputeGroups (src/solver.js:488-499) on the GPU, bit for bit.
//
// The reference runs a union-find over the alive constraints in index order:
// ra = find(a), rb = find(b), and when they differ parent[ra] = rb; then
// group[i] = find(i). Its labels are the roots that this exact sequence of
// unions leaves, which depend on the order (a component's root is not its
// smallest index), so a label-propagation pass would not reproduce them.
// Path halving inside find changes only the shape of the trees, never which
// node is a root, so the labels are fixed by the unions alone.
//
// k_groups_replay: one warp replays the unions 32 constraints at a time.
// Each lane finds the roots of its constraint's two ends in the forest left
// by the earlier batches (the finds run in parallel; their halving writes
// point nodes at ancestors, which no concurrent find can mistake for a
// root). Only a lane whose roots differ can unite: those lanes then take
// their turns in lane (constraint) order, and after each union ja -> jb
// every later lane holding root ja now holds jb. The roots each lane sees at
// its turn are those the sequential loop would find at that constraint, so
// the unions, and the final forest's roots, are the reference's.
// k_groups_label: group[i] = root of i, one thread per solid.
//
// The parent array sits in shared memory when it fits (S * 4 bytes), in the
// scene's grid scatter buffer (free between substeps) otherwise, read and
// written through L2 there so the warp's lanes see each other's writes.
#pragma once
#include "upbd_device.cuh"

namespace upbd {

constexpr int GROUPS_SMEM_MAX = 200 * 1024 / 4;  // solids whose parents fit in shared memory

template <bool SMEM>
__device__ __forceinline__ int32_t uf_ld(const int32_t* p, int32_t i) {
  if (SMEM) return p[i];
  return __ldcg(p + i);
}
template <bool SMEM>
__device__ __forceinline__ void uf_st(int32_t* p, int32_t i, int32_t x) {
  if (SMEM)
    p[i] = x;
  else
    __stcg(p + i, x);
}

// find with path halving (parent[x] = parent[parent[x]]; x = parent[x]),
// src/solver.js:492. The parents always form a forest, so the walk ends
// within S steps; the bound only guards the loop.
template <bool SMEM>
__device__ __forceinline__ int32_t uf_find(int32_t* par, int32_t x, int32_t S) {
  int32_t p = uf_ld<SMEM>(par, x);
  for (int32_t it = 0; p != x && it < S; it++) {
    const int32_t g = uf_ld<SMEM>(par, p);
    uf_st<SMEM>(par, x, g);
    x = g;
    p = uf_ld<SMEM>(par, x);
  }
  return x;
}

// One warp. gpar: S words of global memory; with SMEM the replay runs in
// shared memory (S words of dynamic shared memory) and copies the final
// parents to gpar.
template <bool SMEM>
__global__ void __launch_bounds__(32) k_groups_replay(const uint4* __restrict__ cons, int C, int S,
                                                      int32_t* __restrict__ gpar) {
  extern __shared__ int32_t s_par[];
  const unsigned FULL = 0xffffffffu;
  const int lane = (int)threadIdx.x;
  int32_t* par = SMEM ? s_par : gpar;
  for (int i = lane; i < S; i += 32) uf_st<SMEM>(par, i, i);
  __syncwarp();
  for (int base = 0; base < C; base += 32) {
    const int c = base + lane;
    const uint4 k = (c < C) ? cons[c] : make_uint4(0u, 0u, 0u, 0u);
    const bool alive = c < C && k.w != 0u && k.x < (uint32_t)S && k.y < (uint32_t)S;
    int32_t ra = 0, rb = 0;
    if (alive) {
      ra = uf_find<SMEM>(par, (int32_t)k.x, S);
      rb = uf_find<SMEM>(par, (int32_t)k.y, S);
    }
    __syncwarp();
    // a lane whose two roots agree now never unites: the remapping below
    // moves both of its roots together
    unsigned todo = __ballot_sync(FULL, alive && ra != rb);
    while (todo) {
      const int j = __ffs(todo) - 1;
      todo &= todo - 1u;
      const int32_t ja = __shfl_sync(FULL, ra, j), jb = __shfl_sync(FULL, rb, j);
      if (ja != jb) {  // the same on every lane
        if (lane == j) uf_st<SMEM>(par, ja, jb);
        if (lane > j) {
          if (ra == ja) ra = jb;
          if (rb == ja) rb = jb;
        }
      }
    }
    __syncwarp();  // this batch's unions land before the next batch's finds
  }
  if (SMEM)
    for (int i = lane; i < S; i += 32) gpar[i] = s_par[i];
}

// group[i] = find(i) over the final parents (read-only: no halving).
__global__ void k_groups_label(const int32_t* __restrict__ par, int S, int32_t* __restrict__ group) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= S) return;
  int32_t x = i, p = par[x];
  for (int32_t it = 0; p != x && it < S; it++) {
    x = p;
    p = par[x];
  }
  group[i] = x;
}

}  // namespace upbd
