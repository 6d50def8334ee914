// Word layout of the hash-grid build's scratch memory (scan tiles, tile
// counters, and the pooled / fixed scratch of the stateless grid builds).
// Plain constexpr arithmetic with no CUDA types, so host code, device code and
// a CPU test compiled with g++ all see the same offsets.
#pragma once
#include <cstddef>
#include <cstdint>

#if defined(__CUDACC__)
#define UPBD_HD __host__ __device__
#else
#define UPBD_HD
#endif

namespace upbd {

constexpr int SCAN_TILE = 2048;  // counts scanned per block

// The count pass adds every arrival to its scan tile's total. With 2^18
// buckets there are only 128 tiles, so one counter per tile took ~600 atomics
// at one L2 address per substep and the kernel's drain dominated its time.
// Each tile therefore has `tile_reps` counters, a warp adding to counter
// (warp index mod reps): tile_sum[r * num_tiles + t]. The scan sums them back;
// reps * num_tiles stays <= 2048 words up to 2^22 buckets, so that sum is at
// most 8 independent loads per scan thread.
UPBD_HD constexpr int tile_reps(int num_tiles) {
  int r = 16;
  while (r > 1 && r * num_tiles > 2048) r >>= 1;
  return r;
}
UPBD_HD constexpr int tile_words(int num_tiles) { return tile_reps(num_tiles) * num_tiles; }

// Scratch of one stateless grid build sized for up to n_cap particles and
// t_cap buckets, in 32-bit words from a 256-byte aligned base: bucket counts
// [t_cap], arrival tickets, bucket of each particle and the unordered scatter
// [n_cap each], the scan tile counters, then a params block of params_bytes.
// The params block holds a double (1 / cell size), so it starts on a 64-word
// (256-byte) boundary whatever n_cap is; tile_words() does not decrease with
// the tile count, so the layout for the capacity covers every smaller call.
struct GridScratchLayout {
  size_t counts, ticket, cell, tmp, tiles, params, words;
};

constexpr GridScratchLayout grid_scratch_layout(size_t n_cap, size_t t_cap, size_t params_bytes) {
  GridScratchLayout L{};
  L.counts = 0;
  L.ticket = L.counts + t_cap;
  L.cell = L.ticket + n_cap;
  L.tmp = L.cell + n_cap;
  L.tiles = L.tmp + n_cap;
  const size_t tiles = (t_cap + (size_t)SCAN_TILE - 1) / (size_t)SCAN_TILE;
  L.params = ((L.tiles + (size_t)tile_words((int)tiles) + 63) / 64) * 64;
  L.words = L.params + (params_bytes + 3) / 4;
  return L;
}

}  // namespace upbd
