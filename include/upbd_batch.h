/* Scene batch of libupbd.so: many independent scenes of uneven size stepped
 * together, one launch per pass for all of them.
 *
 * No reference counterpart: the reference steps one scene per GpuSim
 * (src/gpu/sim.js:76-584, encode at :333-398) and one per Solver
 * (src/solver.js:192-237). A batch runs the same passes, in the same order,
 * over every live scene at once: each pass is a persistent kernel whose CTAs
 * walk a per-scene offset table (tiles of scene 0, then scene 1, ...), so a
 * scene's arithmetic is the one of upbd_step and its results match a
 * single-scene handle's. The table lives in device memory and the frame is
 * a captured CUDA graph, so scenes join and leave between frames without a
 * new capture.
 *
 * Conventions are those of upbd.h: every call returns an int status
 * (UPBD_OK or a negative UPBD_ERR_*), host buffers are caller-owned and
 * copied, device state is owned by the batch. A batch is not internally
 * synchronized: one host thread drives it (the server in upbd_server.h
 * wraps one batch behind its own lock).
 */
#ifndef UPBD_BATCH_H
#define UPBD_BATCH_H

#include "upbd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct upbd_batch upbd_batch;

typedef struct upbd_batch_desc {
  int32_t device;
  int32_t solid_iters;    /* Jacobi iterations of every scene (scene desc must agree) */
  uint32_t features;      /* UPBD_FEAT_* of every scene (scene desc must agree) */
  int32_t max_scenes;     /* capacity of the scene table, 1..65536 */
  int32_t block_threads;  /* threads per CTA of the per-particle passes: 64, 128 or 256 */
  int32_t ctas_per_sm;    /* persistent grid of every pass: CTAs per SM, 1..256 */
  uint64_t hbm_budget;    /* device bytes of scene state the batch may hold; 0 = no limit */
  int32_t reserved[8];
} upbd_batch_desc;

typedef struct upbd_batch_info {
  int32_t scenes;          /* live scenes */
  int32_t max_scenes;
  int64_t particles;       /* sum of particle slots (N) over live scenes */
  int64_t solids;          /* sum of body particles over live scenes */
  uint64_t bytes_in_use;   /* device bytes of the live scenes' arenas */
  uint64_t bytes_reserved; /* device bytes the scene pool holds (live + free) */
  uint64_t hbm_budget;
  uint64_t frames;
  uint64_t launches;       /* kernels enqueued (graph replays count their nodes) */
  int32_t block_threads, ctas_per_sm, num_sms, reserved0;
  int32_t reserved[8];
} upbd_batch_info;

int upbd_batch_default_desc(upbd_batch_desc* d);
int upbd_batch_create(const upbd_batch_desc* d, upbd_batch** out);
int upbd_batch_destroy(upbd_batch* b);
/* Message of the last failed call on b (or of the last failed create). */
const char* upbd_batch_last_error(upbd_batch* b);
int upbd_batch_get_info(upbd_batch* b, upbd_batch_info* info);
/* Device bytes one scene of this descriptor occupies in a batch (its arena). */
int upbd_batch_scene_bytes(const upbd_scene_desc* d, uint64_t* bytes);

/* Adds a scene: the lattices of d (as upbd_create builds them) and n_fluid
 * fluid particles at slots S.. with the given positions and velocities
 * (xyz, n_fluid x 3 floats each; vel3 may be NULL for rest) and inverse mass
 * 1/fluid_mass, as upbd_emit_particles places them. Fails with
 * UPBD_ERR_CAPACITY when the scene table is full or the scene does not fit
 * the HBM budget, leaving the batch unchanged. The scene joins at the next
 * upbd_batch_step. *id identifies it until upbd_batch_remove_scene. */
int upbd_batch_add_scene(upbd_batch* b, const upbd_scene_desc* d, const upbd_params* p, int32_t n_fluid,
                         const float* fluid_pos3, const float* fluid_vel3, double fluid_mass, int32_t* id);
/* Removes a scene at the next frame boundary; its memory returns to the pool
 * (stream-ordered: work already enqueued still sees it). */
int upbd_batch_remove_scene(upbd_batch* b, int32_t id);
/* Replaces a scene's constants (cell_size included) from the next frame. */
int upbd_batch_set_params(upbd_batch* b, int32_t id, const upbd_params* p);

/* One frame (substeps substeps of dt/substeps) of every live scene, enqueued
 * on the batch's stream; returns without waiting. */
int upbd_batch_step(upbd_batch* b, double dt, int32_t substeps);
/* Waits for the stream; UPBD_ERR_NAN when a scene saw a non-finite velocity
 * (the message names the scene). */
int upbd_batch_sync(upbd_batch* b);
int upbd_batch_set_stream(upbd_batch* b, void* stream);
/* Persistent-grid shape of every pass from the next frame on. */
int upbd_batch_set_tuning(upbd_batch* b, int32_t block_threads, int32_t ctas_per_sm);

/* Synchronous readbacks / writes of one scene (NULL pointers skip). */
int upbd_batch_read_state(upbd_batch* b, int32_t id, float* pos4, float* prev4, float* vel4, float* density2,
                          uint32_t* flags);
int upbd_batch_write_state(upbd_batch* b, int32_t id, const float* pos4, const float* prev4, const float* vel4,
                           const float* density2, const uint32_t* flags);
int upbd_batch_read_constraints(upbd_batch* b, int32_t id, uint32_t* cons4);
int upbd_batch_write_constraints(upbd_batch* b, int32_t id, const uint32_t* cons4);
/* Particle counts of a scene: slots, body particles, constraints. */
int upbd_batch_scene_info(upbd_batch* b, int32_t id, upbd_info* info);
/* Active fluid particles of a scene after the last completed frame. */
int upbd_batch_active_count(upbd_batch* b, int32_t id, uint32_t* count);

/* One eager frame with an event pair around every launch: per kernel class
 * (upbd_kernel_name) the summed device milliseconds and the launch count. */
int upbd_batch_profile_frame(upbd_batch* b, double dt, int32_t substeps, double* ms, uint32_t* launches);

#ifdef __cplusplus
}
#endif

#endif /* UPBD_BATCH_H */
