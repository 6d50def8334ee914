/*
 * upbd.h — C ABI of the B200-native unified-particle step (libupbd.so).
 *
 * One handle (upbd_sim) owns one scene: a soft-body lattice (or two) held
 * together by 26-neighbour XPBD distance constraints, plus a ring buffer of
 * fluid particles, all resident in device memory. Every substep runs the
 * reference's pass chain as sm_100a CUDA kernels:
 *
 *   integrate → hash-grid count/scan/stable scatter → fluid density →
 *   fluid displacement → I × (XPBD Jacobi solve + apply) → bond update
 *   (plasticity, tearing) → solid↔fluid contacts → apply + bounds +
 *   velocity → XSPH
 *
 * plus the per-frame tools (hose emit, queued slice wedge, pick, grab, drain).
 *
 * Reference surfaces this ABI replaces (paths inside fuugus/fluidphysics):
 *   - GPU solver class GpuSim            src/gpu/sim.js:76-584
 *   - CPU solver class Solver            src/solver.js:8-516
 *   - the WGSL kernels they encode       src/gpu/wgsl.js:121-879
 * Each entry point below names the reference method it stands in for.
 *
 * Conventions
 *   - Every call returns int status: UPBD_OK (0) or a negative UPBD_ERR_*.
 *     The message of the last failure is in upbd_last_error(sim) (or
 *     upbd_last_error(NULL) for failures before a handle exists).
 *   - Host buffers are caller-owned and copied; device state is owned by the
 *     handle. Calls on one handle must come from one thread at a time;
 *     different handles are independent.
 *   - Work is enqueued on the handle's CUDA stream. upbd_step returns before
 *     the GPU finishes; readbacks synchronise the stream.
 *   - Arrays indexed by particle have upbd_info.total entries: solids occupy
 *     [0, solid_n), fluid slots [solid_n, total) (src/gpu/wgsl.js:256).
 *   - Particle state layout (src/gpu/wgsl.js:92-98): pos = xyz + inverse mass,
 *     prev = xyz + grab target x, vel = xyz + grab target y,
 *     density = (rho, rho_near) or, for grabbed solids, (grab target z, grip).
 *     flags bit0 = ACTIVE, bit1 = GRABBED.
 *   - Constraints: uint32 {a, b, rest (float bits), alive} per constraint.
 */
#ifndef UPBD_H
#define UPBD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UPBD_ABI_VERSION 1

/* ---- status codes ---- */
#define UPBD_OK              0
#define UPBD_ERR_INVALID    -1  /* bad argument or descriptor */
#define UPBD_ERR_OOM        -2  /* device or pinned allocation failed */
#define UPBD_ERR_CUDA       -3  /* a CUDA runtime call failed */
#define UPBD_ERR_TIMEOUT    -4  /* a bounded device-side wait gave up */
#define UPBD_ERR_NAN        -5  /* non-finite velocity seen by the step */
#define UPBD_ERR_BUSY       -6  /* resource in use (e.g. server full) */
#define UPBD_ERR_NO_DEVICE  -7  /* no CUDA device / wrong architecture */
#define UPBD_ERR_CAPACITY   -8  /* request exceeds a fixed capacity */
#define UPBD_ERR_INTERNAL   -9  /* an internal invariant does not hold (a library bug) */

/* ---- particle flags (src/gpu/wgsl.js:33-34) ---- */
#define UPBD_F_ACTIVE  1u
#define UPBD_F_GRABBED 2u

/* ---- optional passes of the GPU reference schedule (src/gpu/sim.js:365-383) ---- */
#define UPBD_FEAT_TETS            (1u << 0) /* solveTets/tetUpdate/cutTets */
#define UPBD_FEAT_SOLID_CONTACTS  (1u << 1) /* collectContacts/solidContacts cache */

/* ---- health bits returned by upbd_health ---- */
#define UPBD_HEALTH_NAN      1u
#define UPBD_HEALTH_TIMEOUT  2u
#define UPBD_HEALTH_OVERFLOW 4u
#define UPBD_HEALTH_BOUNDS   8u  /* checked build only: an index out of range was skipped */

/* Scene layout: GpuSim DEFAULTS (src/gpu/sim.js:20-33) and
 * _buildHostData (src/gpu/sim.js:98-214). */
typedef struct upbd_scene_desc {
  int32_t solid_dim;       /* SOLID_DIM: body lattice edge (0 = no body)            */
  int32_t solid_dim2;      /* SOLID_DIM2: companion lattice edge (0 = none)         */
  int32_t max_fluid;       /* MAX_FLUID: fluid ring-buffer capacity                 */
  int32_t table_size;      /* TABLE: hash buckets, power of two                     */
  int32_t substeps;        /* substeps per upbd_frame()                             */
  int32_t solid_iters;     /* XPBD Jacobi iterations per substep                    */
  uint32_t features;       /* UPBD_FEAT_* bits                                      */
  int32_t device;          /* CUDA device ordinal                                   */
  double spacing;          /* lattice spacing                                       */
  double solid_mass;       /* mass per body particle                                */
  double fluid_mass;       /* mass per fluid particle                               */
  double cube_center[3];   /* centre of lattice 1                                   */
  double cube2_center[3];  /* centre of lattice 2 (sim.js:171 places it at
                              [1.1, (n2-1)*spacing/2 + 0.5, 0.7])                   */
  uint32_t reserved[8];
} upbd_scene_desc;

/* Physical constants: GpuSim params (src/gpu/sim.js:34-63), Params struct
 * (src/gpu/wgsl.js:36-90). Doubles, as JavaScript numbers are; the device
 * copy is rounded to float like _writeParams (src/gpu/sim.js:300-330), except
 * 1/cell_size, which hashes in double exactly like Solver._hashPos
 * (src/solver.js:166-172). */
typedef struct upbd_params {
  double h;                 /* substep used by upbd_frame()                         */
  double gravity;
  double solid_radius;
  double fluid_radius;
  double cell_size;
  double fluid_h;           /* double-density interaction radius H                  */
  double rest_density;
  double stiffness;
  double near_stiffness;
  double viscosity;         /* XSPH blend                                           */
  double compliance;        /* XPBD compliance (alpha = compliance / h^2)           */
  double omega;             /* Jacobi relaxation of the solid solve                 */
  double plastic_threshold;
  double plastic_rate;
  double tear_gap;          /* gap rule: tear when d > rest + tear_gap*2*solid_radius */
  double max_speed;
  double wall_x, wall_z, wall_h, wall_t;
  double cull_r;
  double damp_solid, damp_fluid;
  double friction_solid, friction_fluid;
  double grab_k;
  double sleep_speed;       /* kept for layout parity; unused (as in the reference) */
  double solid_viscosity;   /* bonded-velocity XSPH; 0 disables the pass            */
  double break_strain;      /* strain rule: tear when d > rest*break_strain         */
  double contact_scale;     /* solid↔fluid pair scale (0.5 in the GPU reference)    */
  int32_t tear_mode;        /* 0 = gap rule (wgsl.js:392), 1 = strain rule (solver.js:370) */
  int32_t plastic_clamp;    /* 1 = clamp rest to [0.9,1.25]·lattice rest (wgsl.js:402) */
  uint32_t reserved[6];
} upbd_params;

/* Sizes of a created scene. */
typedef struct upbd_info {
  int32_t solid_n;      /* SOLID_N                                 */
  int32_t n1;           /* particles of lattice 1                  */
  int32_t dim1, dim2;
  int32_t max_fluid;
  int32_t total;        /* TOTAL = SOLID_N + MAX_FLUID             */
  int32_t num_cons;
  int32_t num_tets;
  int32_t table_size;
  int32_t substeps;
  int32_t solid_iters;
  int32_t fluid_next;   /* ring-buffer cursor                      */
  uint32_t features;
  int32_t frames;       /* frames stepped since create/reset       */
  uint64_t device_bytes;/* device memory held by the handle        */
  uint32_t param_bytes; /* uniform block uploaded per frame (H2D)  */
  uint32_t reserved;
} upbd_info;

/* Device pointers of the resident state, for a zero-copy consumer on the
 * same device (replaces the renderer's direct use of sim.buf.pos/flags,
 * src/gpu/render.js:142-151). Valid until upbd_destroy. (In the test-only
 * FP64 build, libupbd_fp64.so, the float4/float2 rows are double4/double2.) */
typedef struct upbd_device_ptrs {
  void* pos;      /* float4[total] */
  void* prev;     /* float4[total] */
  void* vel;      /* float4[total] */
  void* density;  /* float2[total] */
  void* flags;    /* uint32[total] */
  void* cons;     /* uint4[num_cons] */
  void* stream;   /* cudaStream_t the handle enqueues on */
} upbd_device_ptrs;

typedef struct upbd_sim upbd_sim;

/* ---------------- lifetime ---------------- */

/* Fills desc/params with the GpuSim defaults (src/gpu/sim.js:20-63) and the
 * defaults of the GPU rules: tear_mode 0, plastic_clamp 1, break_strain 2.6,
 * contact_scale 0.5. */
int upbd_default_desc(upbd_scene_desc* desc);
int upbd_default_params(upbd_params* params);

/* new GpuSim(device, opts) — src/gpu/sim.js:77-95 (+ _buildHostData, _buildGpu).
 * Builds lattices, constraints, CSR adjacency (and tets) on the host, uploads
 * them, and leaves every fluid slot inactive. */
int upbd_create(const upbd_scene_desc* desc, const upbd_params* params, upbd_sim** out);
/* GpuSim.dispose — src/gpu/sim.js:549-552 */
int upbd_destroy(upbd_sim* sim);
int upbd_get_info(upbd_sim* sim, upbd_info* info);
/* sim.o.params = ... / window.__sim.setParam — src/gpu/main.js:540 */
int upbd_set_params(upbd_sim* sim, const upbd_params* params);
int upbd_get_params(upbd_sim* sim, upbd_params* params);
/* Use an external CUDA stream (cudaStream_t) instead of the handle's own. */
int upbd_set_stream(upbd_sim* sim, void* stream);
int upbd_get_device_ptrs(upbd_sim* sim, upbd_device_ptrs* out);
/* Message of the last failure on this handle (NULL: of the last create). */
const char* upbd_last_error(upbd_sim* sim);

/* ---------------- stepping ---------------- */

/* Solver.step(dt, substeps) — src/solver.js:187-242 — run with the GPU pass
 * chain of GpuSim.encode (src/gpu/sim.js:333-398): h = dt / substeps.
 * Pending emit runs first, one queued slice after the substeps. Async. */
int upbd_step(upbd_sim* sim, double dt, int32_t substeps);
/* GpuSim.encode(encoder) — one frame of desc.substeps substeps of params.h. */
int upbd_frame(upbd_sim* sim);
/* Waits for the handle's stream. Returns UPBD_ERR_NAN / UPBD_ERR_TIMEOUT when
 * a device-side check fired since the last upbd_clear_health. */
int upbd_sync(upbd_sim* sim);
int upbd_health(upbd_sim* sim, uint32_t* bits);
int upbd_clear_health(upbd_sim* sim);
/* Use (1) or bypass (0) captured CUDA graphs for frames (default 1). */
int upbd_set_graphs(upbd_sim* sim, int32_t enabled);

/* ---------------- tools ---------------- */

/* GpuSim.resetSolid — src/gpu/sim.js:283-292 (also Solver.resetSolid,
 * src/solver.js:125-137): pristine lattice, constraints and tets; solids
 * at rest, grabs released. Fluid slots keep their state. */
int upbd_reset_solid(upbd_sim* sim);
/* GpuSim.clearFluid — src/gpu/sim.js:294-297; Solver.clearFluid —
 * src/solver.js:151-153. Every fluid slot becomes inactive. */
int upbd_drain(upbd_sim* sim);
/* GpuSim.readActiveCount — src/gpu/sim.js:466-479 (exact, synchronous);
 * Solver.fluidCount — src/solver.js:155-159. */
int upbd_active_count(upbd_sim* sim, uint32_t* count);

/* GpuSim.emit(count, pos, dir, side, up, speed, phase) — src/gpu/sim.js:400-407,
 * kernel src/gpu/wgsl.js:781-801. Queued: runs at the start of the next frame
 * into ring slots fluid_next.., and a later call before that frame replaces it.
 * count <= max_fluid. */
int upbd_emit(upbd_sim* sim, int32_t count, const float pos[3], const float dir[3],
              const float side[3], const float up[3], float speed, float phase);
/* Solver.emitFluid(x,y,z,vx,vy,vz,mass) for n particles at once —
 * src/solver.js:139-149. Immediate ring-buffer writes (pos = prev = p,
 * vel = v, inverse mass = 1/mass, ACTIVE). pos3/vel3 are n*3 floats. */
int upbd_emit_particles(upbd_sim* sim, int32_t n, const float* pos3, const float* vel3,
                        double mass);

/* GpuSim.queueCut(o, d1, d2) — src/gpu/sim.js:409-411. One queued wedge is
 * applied per frame, after its substeps (src/gpu/sim.js:336-340,387-390). */
int upbd_slice(upbd_sim* sim, const double o[3], const double d1[3], const double d2[3]);
/* Solver.cut(o, d1, d2) — src/solver.js:458-486: immediate, in double
 * precision; *cut_count = constraints killed. */
int upbd_slice_now(upbd_sim* sim, const double o[3], const double d1[3], const double d2[3],
                   uint32_t* cut_count);

/* Solver.pickSolid(o, d, maxPerp) — src/solver.js:502-515 (GpuSim.pick,
 * src/gpu/sim.js:414-438, without its millimetre quantisation): nearest
 * solid along the ray, lowest index on ties. *id = -1 when nothing is hit. */
int upbd_pick(upbd_sim* sim, const double ro[3], const double rd[3], double max_perp,
              int32_t* id, double* t);
/* GpuSim.grabAt(center, radius, lattice) — src/gpu/sim.js:440-452, kernel
 * src/gpu/wgsl.js:843-865. lattice 0xffff = any. */
int upbd_grab_select(upbd_sim* sim, const float center[3], float radius, uint32_t lattice);
/* Grabs an explicit set of solids — the list form of Solver.grabs
 * (src/solver.js:35,205-210) — with the GPU spring of integrate
 * (src/gpu/wgsl.js:129-155): weight[k] = grip (NULL = 1.0), targets3[3k..]
 * = spring target (NULL = the particle's current position). Indices must be
 * distinct solids. */
int upbd_grab_indices(upbd_sim* sim, const uint32_t* idx, int32_t n, const float* weight,
                      const float* targets3);
/* Per-frame mouse motion of grabbed targets — pending.grabDelta
 * (src/gpu/sim.js:321-322,342): spread over the next frame's substeps. */
int upbd_grab_move(upbd_sim* sim, const float delta[3]);
/* GpuSim.release — src/gpu/sim.js:454-464, kernel src/gpu/wgsl.js:867-871. */
int upbd_release(upbd_sim* sim);

/* ---------------- readback / state ---------------- */

/* GpuSim.readState — src/gpu/sim.js:568-583 (any pointer may be NULL). */
int upbd_read_state(upbd_sim* sim, float* pos4, float* prev4, float* vel4, float* density2,
                    uint32_t* flags);
/* GpuSim._readBuffer — src/gpu/sim.js:481-490 (copyBufferToBuffer into a
 * staging buffer, then mapAsync): the positions and flags as they stand
 * after the work enqueued so far are copied on the device into a staging
 * copy, in the simulation's stream order, and from there into pos4[total*4]
 * and flags[total] (either may be NULL) on a copy stream, so the host copy
 * overlaps the frames stepped after it. The host buffers must be pinned for
 * the copy to run asynchronously, and must not be read (or passed to another
 * readback) before upbd_read_wait returns. */
int upbd_read_state_async(upbd_sim* sim, float* pos4, uint32_t* flags);
/* Waits until the readbacks started so far have landed in host memory. */
int upbd_read_wait(upbd_sim* sim);
/* Writes the particle state (any pointer may be NULL) — restore's buffer
 * writes, src/gpu/sim.js:526-547. */
int upbd_write_state(upbd_sim* sim, const float* pos4, const float* prev4, const float* vel4,
                     const float* density2, const uint32_t* flags);
/* cons[num_cons*4] = {a, b, rest bits, alive}; GpuSim.readConsAlive —
 * src/gpu/sim.js:555-565 reads the same buffer. */
int upbd_read_constraints(upbd_sim* sim, uint32_t* cons4);
int upbd_write_constraints(upbd_sim* sim, const uint32_t* cons4);
/* CSR adjacency [solid_n+1 offsets][2*num_cons constraint ids] — the adj
 * buffer of src/gpu/sim.js:205-211. */
int upbd_read_adjacency(upbd_sim* sim, uint32_t* adj);
/* Hash grid of the last grid build: counts[T], offsets[T+1] (exclusive scan,
 * offsets[T] = total), entries[total] (particle ids, descending inside a
 * bucket as Solver._buildGrid leaves them, src/solver.js:174-184). Any
 * pointer may be NULL. *n_entries = offsets[T]. */
int upbd_read_grid(upbd_sim* sim, uint32_t* counts, uint32_t* offsets, uint32_t* entries,
                   uint32_t* n_entries);
/* Rebuilds the hash grid from the current positions (no integrate). */
int upbd_rebuild_grid(upbd_sim* sim);
/* Runs one substep of length h, stopping after pass `last_pass`
 * (UPBD_PASS_*), for per-pass comparisons. */
int upbd_substep_partial(upbd_sim* sim, double h, int32_t last_pass);
/* Tets: tets5[num_tets*5] = {a, b, c, d, rest volume bits (negative = dead)}. */
int upbd_read_tets(upbd_sim* sim, uint32_t* tets5);
/* The tet part of GpuSim.restore (src/gpu/sim.js:528-535): writes the rest
 * volumes (sign = alive) of tets5 back; the vertex indices must be the
 * scene's own. */
int upbd_write_tets(upbd_sim* sim, const uint32_t* tets5);
/* GpuSim.restore's fluidNext (src/gpu/sim.js:544): the next emit slot of the
 * hose ring buffer, 0 <= next < max_fluid. */
int upbd_set_fluid_next(upbd_sim* sim, int32_t next);
/* Solver._recomputeGroups — src/solver.js:488-499: union-find over alive
 * constraints in index order; group[solid_n] = the root id the reference's
 * sequence of unions leaves (bit for bit). Computed on the GPU
 * (upbd_groups_device) and copied back; returns after the copy. */
int upbd_groups(upbd_sim* sim, int32_t* group);
/* The same labels written to device memory d_group[solid_n] on the sim's
 * stream, without a host synchronisation (capturable in a CUDA graph).
 * Uses the grid build's scratch, which is free between substeps. */
int upbd_groups_device(upbd_sim* sim, int32_t* d_group);

/* Pass ids for upbd_substep_partial (order of src/gpu/sim.js:354-385). */
#define UPBD_PASS_INTEGRATE      1
#define UPBD_PASS_GRID           2
#define UPBD_PASS_DENSITY        3
#define UPBD_PASS_DISP           4
#define UPBD_PASS_APPLY_FLUID    5
#define UPBD_PASS_SOLID          7
#define UPBD_PASS_BONDS          8
#define UPBD_PASS_CONTACTS       9
#define UPBD_PASS_APPLY_ALL     10
#define UPBD_PASS_BOUNDS        11
#define UPBD_PASS_VELOCITY      12
#define UPBD_PASS_SOLID_VISC    13
#define UPBD_PASS_XSPH          14
#define UPBD_PASS_XSPH_APPLY    15

/* ---------------- stateless kernel entry points ---------------- */

/* Hash-grid build over caller-owned device arrays — the count / scan /
 * scatter of src/gpu/wgsl.js:163-245 with Solver._buildGrid's membership
 * order (src/solver.js:174-184). pos4: float4[n] device, flags: uint32[n]
 * device (bit0 = active), counts[T], offsets[T+1], entries[n] device
 * outputs (counts may be NULL). stream = cudaStream_t (NULL = default
 * stream). Scratch comes from one per-device pool that the library allocates
 * on first use and grows when a call needs more: growing it calls
 * cudaDeviceSynchronize, cudaFree and cudaMalloc, so a call that grows the
 * pool must not be captured into a CUDA graph (make one call of the largest
 * size first). Every call on a device shares that pool: calls whose work
 * overlaps on the GPU (different streams or threads) race on it, so order
 * them on one stream or with events. All work, including the counts, is
 * enqueued on `stream`; the call does not wait for it. */
int upbd_grid_build(const void* pos4, const void* flags, int32_t n, int32_t table_size,
                    double cell_size, void* counts, void* offsets, void* entries,
                    void* stream);

/* The same hash-grid build for callers that cannot allocate device memory
 * (this entry point has no counterpart in the reference). A host that embeds
 * the library in a runtime owning the device-memory budget, which refuses
 * allocations it did not make, or a frame loop that must not stall on an
 * allocation, cannot use upbd_grid_build's cudaMalloc-grown scratch pool.
 * This variant calls no cudaMalloc/cudaFree: its scratch is a fixed 4 MiB
 * array inside the library, held by every GPU that loads the library until
 * the process exits. Limits: n <= 262144 particles and table_size <= 262144
 * buckets per call; larger sizes return UPBD_ERR_CAPACITY. Arguments and
 * outputs are those of upbd_grid_build (counts may be NULL).
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress, with that device current); make that first call
 * before any stream capture. Every call shares the one array: calls whose
 * work overlaps on the GPU (other streams, other threads) race and corrupt
 * each other's results, so order them on one stream or with events. Each call
 * clears the parts of the array that must start at zero. The device address
 * is looked up once per device and kept: after cudaDeviceReset on a device,
 * unload and reload the library before calling this entry point there again. */
int upbd_grid_build_noalloc(const void* pos4, const void* flags, int32_t n, int32_t table_size,
                            double cell_size, void* counts, void* offsets, void* entries,
                            void* stream);

/* Kernels this handle has launched so far (each replay of a captured frame
 * counts its kernel nodes). Instrumentation for benchmarks. */
uint64_t upbd_launch_count(upbd_sim* sim);

/* Per-kernel timing: runs one frame like upbd_step, launched without a graph
 * and with a CUDA event pair around every kernel, then fills
 * ms[UPBD_KERNEL_KINDS] (summed device time per kernel class) and
 * launches[UPBD_KERNEL_KINDS]. Synchronous. upbd_kernel_name(kind) names a
 * class (NULL past the last). */
#define UPBD_KERNEL_KINDS 32
int upbd_profile_frame(upbd_sim* sim, double dt, int32_t substeps, double* ms, uint32_t* launches);
const char* upbd_kernel_name(int32_t kind);

/* Launch floor of the frame graph: captures one frame of `substeps` substeps
 * the way upbd_step does, replaces every kernel node's kernel by an empty one
 * with the node's own grid and block (the graph's nodes and dependencies are
 * kept), and times `reps` replays of that copy with CUDA events on the
 * simulation's stream. *floor_ms = device time per replay, *kernel_nodes =
 * kernel nodes in the frame. The simulation's state is not touched.
 * Synchronous. Instrumentation for benchmarks; no counterpart in the
 * reference (WebGPU gives no such measurement). */
int upbd_profile_graph_floor(upbd_sim* sim, double dt, int32_t substeps, int32_t reps, double* floor_ms,
                             uint32_t* kernel_nodes);

#ifdef __cplusplus
}
#endif
#endif /* UPBD_H */
