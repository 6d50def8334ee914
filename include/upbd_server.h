/* Frame server of libupbd.so: continuous batching of scene requests on one
 * GPU.
 *
 * No reference counterpart: the reference runs one interactive scene per
 * page (src/gpu/main.js). A request here is a scene plus a number of frames
 * to step. Requests are prepared on host builder threads once they arrive,
 * admitted in arrival order while the HBM budget and the scene table have
 * room, kept resident on the device between frames, and stepped together:
 * every frame of the server is one batched frame (upbd_batch.h) of all live
 * requests, and a request leaves the batch, freeing its memory for the next
 * ones, after its last frame. Requests that arrive while others are on the
 * GPU join at the next frame boundary, so their work overlaps.
 *
 * Latency of a frame: completion time of that frame minus the time it could
 * first run (the request's arrival for its first frame, the completion of
 * its previous frame after that), on the server clock (steady clock, zero at
 * the first upbd_server_run).
 *
 * upbd_server_submit may be called from any thread, also while another
 * thread is inside upbd_server_run; every other call comes from one thread.
 */
#ifndef UPBD_SERVER_H
#define UPBD_SERVER_H

#include "upbd_batch.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct upbd_server upbd_server;

typedef struct upbd_server_desc {
  upbd_batch_desc batch;  /* device, solid_iters, features, max_scenes, grid shape, hbm_budget */
  double dt;              /* frame length in seconds */
  int32_t substeps;       /* substeps per frame */
  int32_t builders;       /* host threads preparing arrived requests, 1..64 */
  int32_t keep_results;   /* keep each finished request's final pos/flags for upbd_server_result */
  int32_t reserved[9];
} upbd_server_desc;

typedef struct upbd_request {
  upbd_scene_desc desc;   /* solid_iters and features must match the server's */
  upbd_params params;
  int32_t frames;         /* frames to step, >= 1 */
  int32_t n_fluid;        /* fluid particles placed at slots S.. (<= desc.max_fluid) */
  double fluid_mass;
  double arrival_s;       /* server-clock time from which the request may be admitted */
  const float* fluid_pos3;  /* n_fluid x 3, copied by submit */
  const float* fluid_vel3;  /* n_fluid x 3 or NULL (at rest), copied by submit */
  int32_t reserved[8];
} upbd_request;

enum {
  UPBD_REQ_QUEUED = 0,
  UPBD_REQ_PREPARING = 1,
  UPBD_REQ_READY = 2,
  UPBD_REQ_RUNNING = 3,
  UPBD_REQ_DONE = 4,
  UPBD_REQ_REJECTED = 5
};

typedef struct upbd_request_result {
  int32_t state;          /* UPBD_REQ_* */
  int32_t status;         /* UPBD_OK, or why it was rejected / stopped (UPBD_ERR_NAN, ...) */
  int32_t frames_done;
  int32_t slots;          /* particle slots N of the scene */
  double arrival_s, admit_s, done_s;
  double frame_ms_max;    /* its slowest frame */
  int32_t reserved[8];
} upbd_request_result;

typedef struct upbd_server_stats {
  int64_t submitted, admitted, completed, rejected;
  int64_t scene_frames;       /* frames stepped, summed over requests */
  int64_t batch_frames;       /* batched frames launched */
  double particle_substeps;   /* sum over stepped scene-frames of (body + active fluid) x substeps */
  double wall_s;              /* server clock at the end of the last run */
  double device_s;            /* device time of the batched frames (CUDA events) */
  double frame_ms_p50, frame_ms_p90, frame_ms_p99, frame_ms_max, frame_ms_mean;
  double wait_ms_p50, wait_ms_p99;    /* arrival -> admission */
  double batch_ms_p50, batch_ms_p99;  /* device time of one batched frame */
  double mean_scenes;         /* live requests per batched frame */
  int32_t peak_scenes, reserved0;
  uint64_t peak_bytes;        /* most device bytes the live requests held at once */
  double reserved[8];
} upbd_server_stats;

int upbd_server_default_desc(upbd_server_desc* d);
int upbd_server_create(const upbd_server_desc* d, upbd_server** out);
/* Stops the builder threads; requests still queued or running are dropped. */
int upbd_server_destroy(upbd_server* s);
const char* upbd_server_last_error(upbd_server* s);
/* Queues a request; *id names it for upbd_server_result. */
int upbd_server_submit(upbd_server* s, const upbd_request* r, int64_t* id);
/* Serves until every submitted request is done or rejected, or max_seconds
 * of server clock have passed in this call (then returns UPBD_ERR_TIMEOUT
 * with the work kept for the next call). */
int upbd_server_run(upbd_server* s, double max_seconds);
int upbd_server_get_stats(upbd_server* s, upbd_server_stats* out);
/* State of a request; for a finished request of a server that keeps results,
 * also its final positions (N x 4) and flags (N) when the pointers are set. */
int upbd_server_result(upbd_server* s, int64_t id, upbd_request_result* res, float* pos4, uint32_t* flags);

#ifdef __cplusplus
}
#endif

#endif /* UPBD_SERVER_H */
