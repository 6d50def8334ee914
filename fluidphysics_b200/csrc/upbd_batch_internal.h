// C++ entry points of the scene batch for the frame server (same library):
// admission of a scene prepared off the driving thread, and the per-scene
// counters the server reads between frames.
#pragma once
#include <cuda_runtime.h>

#include "../../include/upbd_batch.h"
#include "upbd_scene.h"

namespace upbd {

// upbd_batch_add_scene after prepare_scene: checks, pool allocation and
// uploads (synchronous on the batch's stream).
int batch_add_prepared(upbd_batch* b, const PreparedScene& ps, int32_t* id);
cudaStream_t batch_stream(upbd_batch* b);
// Active fluid count and health bits the last completed frame published for
// a scene (mapped host memory: valid once that frame's stream work is done).
bool batch_scene_counters(upbd_batch* b, int32_t id, uint32_t* active, uint32_t* health, int32_t* solids);
// Device bytes a prepared scene occupies (its arena).
size_t prepared_bytes(const PreparedScene& ps);

}  // namespace upbd
