/*
 * mpm_b200.h — C ABI of the B200 MLS-MPM fluid + diffuse library.
 *
 * This is the drop-in boundary for the compute side of the reference's
 * fluid-gpu.js (class FluidGPU) and diffuse-gpu.js (class DiffuseGPU).  A
 * JavaScript host keeps its classes and packs the same uniform bytes it
 * would pass to queue.writeBuffer; each entry point below replaces one
 * WebGPU-facing member (cited as file:line).  Plain pointers and sizes only.
 *
 * Conventions
 *  - Every call returns mpm_status; mpm_last_error() describes the last
 *    failure on the calling thread.
 *  - A scene owns one CUDA stream; calls that enqueue GPU work return without
 *    waiting (like a WebGPU submit).  mpm_download/mpm_sync wait.
 *  - One scene is not thread-safe; different scenes may be driven from
 *    different threads.
 *  - Device buffers keep the reference layouts: pos/vel vec4<f32> (16 B per
 *    particle), affine 9 x f32 row-major, mass/density f32, cell_mv 3 x i32
 *    per cell, cell_mass i32, cell_mv_f32 3 x f32, cell_mass_f32 f32, the
 *    diffuse pool 48 B per slot with a u32 free list and an i32 top.
 */
#ifndef MPM_B200_H
#define MPM_B200_H

#include <stddef.h>
#include <stdint.h>

#include "mpm_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define MPM_ABI_VERSION 1

typedef enum mpm_status {
    MPM_OK = 0,
    MPM_ERR_INVALID_ARG = 1,
    MPM_ERR_OOM = 2,
    MPM_ERR_DEVICE = 3,
    MPM_ERR_TIMEOUT = 4,
    MPM_ERR_NAN = 5,
    MPM_ERR_NO_DEVICE = 6,
    MPM_ERR_BUSY = 7,
    MPM_ERR_UNSUPPORTED = 8,
    MPM_ERR_CAPACITY = 9
} mpm_status;

/* Buffers exposed by mpm_get_buffer / mpm_download / mpm_upload, named after
 * the reference's GPUBuffer members (fluid-gpu.js:208-219, diffuse-gpu.js:52-55). */
typedef enum mpm_buffer {
    MPM_BUF_POS = 0,            /* particlePosBuffer     N x vec4<f32> */
    MPM_BUF_VEL = 1,            /* particleVelBuffer     N x vec4<f32> */
    MPM_BUF_AFFINE = 2,         /* particleAffineBuffer  N x 9 f32     */
    MPM_BUF_MASS = 3,           /* particleMassBuffer    N x f32       */
    MPM_BUF_DENSITY = 4,        /* particleDensityBuffer N x f32       */
    MPM_BUF_CELL_MV = 5,        /* cellMvBuffer          G x 3 i32     */
    MPM_BUF_CELL_MASS = 6,      /* cellMassBuffer        G x i32       */
    MPM_BUF_CELL_MV_F32 = 7,    /* cellMvF32Buffer       G x 3 f32     */
    MPM_BUF_CELL_MASS_F32 = 8,  /* cellMassF32Buffer     G x f32       */
    MPM_BUF_DIFFUSE = 9,        /* DiffuseGPU.particleBuffer  M x 48 B */
    MPM_BUF_FREE_LIST = 10,     /* DiffuseGPU.freeListBuffer  M x u32  */
    MPM_BUF_FREE_TOP = 11       /* DiffuseGPU.freeListTopBuffer i32    */
} mpm_buffer;

/* mpm_desc.flags: run the plain engine (one kernel per reference pass on
 * reference-layout buffers) instead of the binned engine.  Both give the
 * same bits; the plain engine exists as a cross-check and for debugging. */
#define MPM_FLAG_PLAIN 1u

/* Scene creation descriptor (FluidGPU constructor, fluid-gpu.js:10-17). */
typedef struct mpm_desc {
    uint32_t grid_X, grid_Y, grid_Z;  /* cells */
    uint32_t particle_capacity;       /* particleNum: buffer capacity */
    int32_t device;                   /* CUDA device ordinal */
    uint32_t flags;                   /* MPM_FLAG_* */
} mpm_desc;

typedef struct mpm_scene mpm_scene;

/* ABI version (MPM_ABI_VERSION). */
int mpm_abi_version(void);

/* Text of the last error on this thread ("" if none). */
const char* mpm_last_error(void);

/* Number of visible CUDA devices (0 is not an error). */
mpm_status mpm_device_count(int* count);

/* Cap on the device memory this library holds at once, over every scene,
 * batch and server of the process (no counterpart in the reference, where
 * the browser's WebGPU device enforces its own limits).  0 (the default)
 * means no cap.  An allocation that would pass it fails the way an
 * exhausted device does: the call returns MPM_ERR_OOM and leaves its object
 * as it was.  Lowering the cap frees nothing.  Use it to keep the library
 * inside a share of the GPU, or to exercise out-of-memory paths. */
mpm_status mpm_set_device_memory_limit(uint64_t bytes);

/* Device bytes this library holds now (what the cap counts). */
mpm_status mpm_device_memory_in_use(uint64_t* bytes);

/* Grid sizing of the FluidGPU constructor (fluid-gpu.js:10-16):
 * grid_* = ceil(aspect_* / (4 * particle_radius)). */
mpm_status mpm_desc_from_aspect(double aspect_x, double aspect_y, double aspect_z, double particle_radius,
                                uint32_t particle_num, mpm_desc* out);

/* Constructor defaults of FluidGPU (fluid-gpu.js:24-45) for this grid with
 * dt = DT / SUBSTEPS and particle_num = 0 (fluid-gpu.js:297-313 layout). */
mpm_status mpm_default_params(const mpm_desc* desc, mpm_params* out);

/* Diffuse defaults (diffuse-gpu.js:20-31, 70-94): seed = 1. */
mpm_status mpm_default_diffuse_params(uint32_t max_count, mpm_gen_params* gen, mpm_advect_params* adv);

/* FluidGPU.initGPU -> _createBuffers (fluid-gpu.js:183-293): allocate the
 * device buffers (zero-filled) and the scene's stream. */
mpm_status mpm_create(const mpm_desc* desc, mpm_scene** out);

/* Release every device allocation of the scene. */
mpm_status mpm_destroy(mpm_scene* scene);

/* Initial particle upload, fluid-gpu.js:278-281 (writeBuffer of pos/vel in
 * vec4 layout, affine, mass).  Host arrays; n <= capacity becomes
 * active_particle_num.  vel4/affine9 may be NULL (zeros). */
mpm_status mpm_upload_particles(mpm_scene* scene, const float* pos4, const float* vel4, const float* affine9,
                                const float* mass, uint32_t n);

/* _writeParamsBuffer (fluid-gpu.js:295-328): the 80-byte Params uniform.
 * grid dims must equal the scene's; particle_num <= capacity. */
mpm_status mpm_set_params(mpm_scene* scene, const mpm_params* params);

/* _writeWallParams upload (fluid-gpu.js:337-413): the 336-byte WallParams. */
mpm_status mpm_set_walls(mpm_scene* scene, const mpm_wall_params* walls);

/* updateHand (fluid-gpu.js:479-527): the 80-byte HandParams plus the
 * dispatch box (_handBBoxDim*); APPLY_HAND runs iff active and all dims > 0. */
mpm_status mpm_set_hand(mpm_scene* scene, const mpm_hand_params* hand, int active, const int32_t bbox_dims[3]);

/* DiffuseGPU constructor + initGPU (diffuse-gpu.js:16-94): pool of max_count
 * slots, free list [0..max-1], top = max, GenParams/AdvectParams uniforms.
 * adv->diffuse_max is replaced by max_count. */
mpm_status mpm_diffuse_enable(mpm_scene* scene, uint32_t max_count, const mpm_gen_params* gen,
                              const mpm_advect_params* adv);

/* _writeGenParams (diffuse-gpu.js:84-94): replaces the whole GenParams
 * (thresholds and seed).  DiffuseGPU.step only rewrites the seed, so other
 * fields changed on the host take effect only through this call. */
mpm_status mpm_diffuse_set_gen_params(mpm_scene* scene, const mpm_gen_params* gen);

/* FluidGPU.simFrame (fluid-gpu.js:648-684): runs `substeps` substeps of
 * CLEAR..G2P (+ APPLY_HAND when active) and, when diffuse is enabled,
 * DiffuseGPU.step (diffuse-gpu.js:148-166: seed+1, GENERATE, ADVECT) after
 * each.  Enqueues work and returns. */
mpm_status mpm_step(mpm_scene* scene, int substeps);

/* Wait for all work enqueued on the scene's stream, and for queued
 * alive-count readbacks.  Returns MPM_ERR_NAN when the scene's particle state
 * holds a NaN or an infinity (MPM_HEALTH_NONFINITE below). */
mpm_status mpm_sync(mpm_scene* scene);

/* mpm_sync with a limit (no counterpart in the reference, whose frame loop
 * never waits): waits at most timeout_s seconds (0: only looks) and returns
 * MPM_ERR_TIMEOUT while the scene's work is still running, for a host loop
 * that must not block, e.g. a renderer that skips a frame instead. */
mpm_status mpm_wait(mpm_scene* scene, double timeout_s);

/* Health of a scene (no counterpart in the reference, which reports
 * nothing): bits kept on the device, set by the kernels and sticky until
 * read with clear != 0.  Binned engine only (the plain engine reports 0).
 *  MPM_HEALTH_NONFINITE: a particle position was NaN or infinite at the
 *    start of a substep (P2G_MASS).  A NaN position survives every clamp of
 *    the reference's passes, so it never heals (velocities cannot stay
 *    non-finite: the next P2G clamps them); mpm_sync and mpm_wait return
 *    MPM_ERR_NAN.
 *  MPM_HEALTH_SATURATED: encode's clamp of +-20000 (shaders.js:17-24) could
 *    engage, so the fixed-point grid may no longer hold the true sum, the
 *    usual sign of a simulation that has blown up.  Set for a particle whose
 *    bound on its P2G contributions passes about 45,000: every real clamp is
 *    flagged, and near misses too.  Results still follow the reference bit
 *    for bit; no call fails on it. */
#define MPM_HEALTH_NONFINITE 1u
#define MPM_HEALTH_SATURATED 2u
mpm_status mpm_get_health(mpm_scene* scene, uint32_t* flags, int clear);

/* Device pointer and byte size of a buffer in its reference layout, for a
 * zero-copy consumer such as a renderer's vertex inputs
 * (fluid-renderer.js:315-328).  The pointer stays valid for the scene's life.
 * Contents, in stream order (read after mpm_sync, or order work after the
 * scene's stream):
 *  - MPM_BUF_POS, MPM_BUF_VEL, MPM_BUF_DENSITY: the first such call makes
 *    every later substep write these three in place (a renderer reads them
 *    every frame), so they follow each step with no further call;
 *  - MPM_BUF_AFFINE, MPM_BUF_MASS: as of this call, until the next mpm_step;
 *  - grid and diffuse buffers: always current.  The diffuse pool is for
 *    reading: write it with mpm_upload (ADVECT keeps an index of live slots). */
mpm_status mpm_get_buffer(mpm_scene* scene, mpm_buffer which, void** dev_ptr, size_t* bytes);

/* Zero-copy export of a buffer (reference layout) to another process on the
 * same node, e.g. a renderer reading the particle positions, velocities and
 * densities as vertex inputs (fluid-renderer.js:315-328) or the diffuse pool
 * (850-856): `handle` receives the MPM_IPC_HANDLE_BYTES-byte CUDA IPC handle
 * (cudaIpcMemHandle_t) of the device allocation that holds the buffer, and
 * `offset` the buffer's byte offset in it.  The consumer opens the handle
 * with cudaIpcOpenMemHandle.  Contents follow the same rules as
 * mpm_get_buffer; order the consumer's reads after mpm_sync. */
#define MPM_IPC_HANDLE_BYTES 64
mpm_status mpm_get_ipc_handle(mpm_scene* scene, mpm_buffer which, void* handle, size_t* offset, size_t* bytes);

/* Copy a buffer (reference layout) to host memory; waits for the stream.
 * `bytes` may be smaller than the buffer (a prefix is copied). */
mpm_status mpm_download(mpm_scene* scene, mpm_buffer which, void* host_dst, size_t bytes);

/* Overwrite a buffer (reference layout) from host memory (a prefix of
 * `bytes`); used for restoring saved state. */
mpm_status mpm_upload(mpm_scene* scene, mpm_buffer which, const void* host_src, size_t bytes);

/* DiffuseGPU.requestDebugReadback + pollDebug (diffuse-gpu.js:172-188):
 * alive = maxCount - freeListTop.  Waits for the stream. */
mpm_status mpm_diffuse_alive_count(mpm_scene* scene, int32_t* alive);

/* DiffuseGPU.requestDebugReadback (diffuse-gpu.js:172-176), asynchronous: a
 * 4-byte copy of freeListTop as of the work already enqueued, into a ring of
 * 4 pinned slots.  With every slot still in flight it first waits for the
 * oldest one (so the host never runs more than 4 readbacks ahead of the
 * device).  After a step the copy reads the value the last kill pass recorded
 * on the device and runs on a side stream, so later steps do not wait for it;
 * after top was uploaded or exported it copies top itself, in stream order. */
mpm_status mpm_diffuse_request_alive(mpm_scene* scene);

/* DiffuseGPU.pollDebug (diffuse-gpu.js:178-188), non-blocking: reads every
 * completed readback in order; *alive = maxCount - top of the newest one read
 * so far (0 before the first), *ready = 1 if this call read at least one. */
mpm_status mpm_diffuse_poll_alive(mpm_scene* scene, int32_t* alive, int32_t* ready);

/* The scene's CUDA stream (cudaStream_t), for callers that order their own
 * work after a step. */
mpm_status mpm_get_stream(mpm_scene* scene, void** stream);

/* ---- particle editing: deleteNear / raycastFluid / spawnParticles ---- */

/* FluidGPU.deleteNear + pollDelete (fluid-gpu.js:544-592): removes the active
 * particles within `radius` of the line through `origin` along `dir` (the
 * COMPACT pass, shaders.js:521-546), keeping the survivors in index order;
 * the affine buffer is not compacted (shaders.js:516-520).  Waits for the
 * stream and returns the new active count in *new_count. */
mpm_status mpm_delete_near(mpm_scene* scene, const double origin[3], const double dir[3], double radius,
                           uint32_t* new_count);

/* FluidGPU.raycastFluid + pollRaycast (fluid-gpu.js:594-628): the smallest t
 * > 0 along the ray among active particles within `radius` of it (the
 * RAYCAST pass, shaders.js:563-576).  *hit = 0 when none; else *t_out = t
 * and hit_pos = origin + t * dir (in double, as the JS side computes it).
 * Waits for the stream. */
mpm_status mpm_raycast_fluid(mpm_scene* scene, const double origin[3], const double dir[3], double radius,
                             int* hit, float* t_out, double hit_pos[3]);

/* The buffer writes of FluidGPU.spawnParticles (fluid-gpu.js:145-179):
 * appends min(count, capacity - active) particles (pos4/vel4 vec4<f32>,
 * mass f32; vel4 may be NULL for zero velocity) after the active ones and
 * raises the active count; *appended gets the number written.  The sphere
 * sampling stays on the host side. */
mpm_status mpm_append_particles(mpm_scene* scene, const float* pos4, const float* vel4, const float* mass,
                                uint32_t count, uint32_t* appended);

/* The COMPACT pass over caller-owned device buffers (shaders.js:521-546 with
 * bindings 0-8 as arguments): survivors of pos_in/vel_in/mass_in (n
 * particles) go to the front of pos_out/vel_out/mass_out in index order and
 * *count_dev (device memory) receives their number.  Enqueued on `stream`
 * (a cudaStream_t on the current device; NULL = legacy default stream); the
 * per-block scratch is a stream-ordered allocation freed on that stream.
 * Inputs and outputs must not overlap. */
mpm_status mpm_compact(const mpm_ray_params* del, uint32_t n, const float* pos_in, const float* vel_in,
                       const float* mass_in, float* pos_out, float* vel_out, float* mass_out, uint32_t* count_dev,
                       void* stream);

/* The RAYCAST pass over a caller-owned device buffer (shaders.js:563-576):
 * *hit_dev (device memory) = the smallest f32 bit pattern of t among hits,
 * 0xFFFFFFFF when none (the sentinel is written by this call). */
mpm_status mpm_raycast(const mpm_ray_params* ray, uint32_t n, const float* pos_in, uint32_t* hit_dev,
                       void* stream);

/* Largest n mpm_compact_noalloc accepts (its scratch is a fixed array of
 * 8,193 32-bit words, about 32 KB, one survivor count per 2,048 particles). */
#define MPM_COMPACT_NOALLOC_MAX_N (1u << 24)

/* No counterpart in the reference (whose COMPACT needs no scratch beyond its
 * atomic counter).  mpm_compact with the same arguments and results, but the
 * call allocates nothing: for hosts that must not allocate device memory
 * while they run (a real-time frame loop with a fixed memory plan, a caller
 * whose allocator is someone else's, code running inside a stream capture),
 * the per-block scratch is a fixed device array of this library instead of a
 * stream-ordered allocation.  Runs on the current device.
 * n > MPM_COMPACT_NOALLOC_MAX_N fails with MPM_ERR_CAPACITY before any work
 * is enqueued; n = 0 only sets *count_dev to 0.  The first call on a device
 * (and the first after its context was re-created, e.g. by cudaDeviceReset)
 * looks up the array's address, so make it outside any stream capture.
 * Calls on one device share the scratch: calls that can overlap in time
 * (different streams, unordered threads) race. */
mpm_status mpm_compact_noalloc(const mpm_ray_params* del, uint32_t n, const float* pos_in, const float* vel_in,
                               const float* mass_in, float* pos_out, float* vel_out, float* mass_out,
                               uint32_t* count_dev, void* stream);

/* ---- tracing (no counterpart in the reference, whose only timers are
 * render-pass timestamps, fluid-renderer.js:34-41) ---- */

/* Phases of a substep timed by the profiler. */
typedef enum mpm_phase {
    MPM_PHASE_CLEAR = 0,        /* CLEAR (shaders.js:196-210)                */
    MPM_PHASE_P2G_MASS = 1,     /* COMPUTE_WEIGHTS + P2G_MASS (216-274)      */
    MPM_PHASE_DECODE_MASS = 2,  /* DECODE_MASS (373-384)                     */
    MPM_PHASE_P2G_MOM = 3,      /* P2G_MOM (276-371)                         */
    MPM_PHASE_UPDATE_GRID = 4,  /* UPDATE_GRID (435-513)                     */
    MPM_PHASE_APPLY_HAND = 5,   /* APPLY_HAND (394-433)                      */
    MPM_PHASE_G2P = 6,          /* G2P (579-705)                             */
    MPM_PHASE_DIFFUSE_GEN = 7,  /* DIFFUSE_GENERATE + slot ranking (721-856) */
    MPM_PHASE_DIFFUSE_ADV = 8,  /* DIFFUSE_ADVECT + free-list push (858-997) */
    MPM_PHASE_SORT = 9,         /* particle binning (no reference pass)      */
    MPM_PHASE_COUNT = 10
} mpm_phase;

/* Name of a phase ("p2g_mom", ...), or "" for an unknown index. */
const char* mpm_phase_name(int phase);

/* Turn per-phase CUDA-event timing on the scene's stream on or off
 * (off by default; events add a few microseconds per substep). */
mpm_status mpm_profile_enable(mpm_scene* scene, int on);

/* Accumulated per-phase GPU time (ms) and sample counts since the last
 * reset; waits for the stream.  Arrays hold MPM_PHASE_COUNT entries. */
mpm_status mpm_profile_read(mpm_scene* scene, double* ms, uint64_t* count, int reset);

/* Number of kernels this scene has launched (CUDA kernels only). */
mpm_status mpm_launch_count(mpm_scene* scene, uint64_t* launches);

/* ---- batching: many independent scenes advanced together (no counterpart
 * in the reference, which runs one FluidGPU per page).  Every kernel of a
 * substep runs once for all scenes of the batch over a device table of
 * per-scene grid dims, Params, WallParams and HandParams; results per scene
 * are bit-identical to the same scene run alone.  No diffuse in batches. ---- */

typedef struct mpm_batch mpm_batch;

/* mpm_batch_desc.flags: step without CUDA graphs (one launch per kernel). */
#define MPM_BATCH_NO_GRAPH 1u
/* mpm_batch_desc.flags: time the first substeps of each workload under
 * several launch shapes and keep the fastest (results do not depend on it). */
#define MPM_BATCH_AUTOTUNE 2u

typedef struct mpm_batch_desc {
    uint32_t particle_capacity;   /* particles over all scenes at once */
    uint32_t scene_capacity;      /* scenes at once */
    uint64_t cell_capacity;       /* grid cells over all scenes at once */
    int32_t device;               /* CUDA device ordinal */
    uint32_t flags;               /* MPM_BATCH_* */
} mpm_batch_desc;

typedef struct mpm_batch_info {
    uint32_t scenes;              /* live scenes */
    uint32_t particles;           /* particles over live scenes */
    uint64_t cells;               /* cells over live scenes */
    uint64_t launches;            /* kernels launched so far */
    uint64_t substeps;            /* batch substeps run so far */
    uint64_t device_bytes;        /* device memory held by the batch */
    uint32_t item_blocks, grid_blocks;   /* launch shape in use */
} mpm_batch_info;

/* Device bytes mpm_batch_create would allocate for these capacities (for
 * admission against an HBM budget). */
mpm_status mpm_batch_footprint(uint32_t particle_capacity, uint64_t cell_capacity, uint32_t scene_capacity,
                               uint64_t* bytes);

mpm_status mpm_batch_create(const mpm_batch_desc* desc, mpm_batch** out);
mpm_status mpm_batch_destroy(mpm_batch* batch);

/* Adds a scene: `params` as mpm_set_params gives them (grid_X/Y/Z set the
 * scene's grid, at least 5 per axis; particle_num is replaced by n), walls
 * may be NULL (none), host particle arrays as mpm_upload_particles takes
 * them.  *scene receives the scene id.  MPM_ERR_CAPACITY when particles,
 * cells or scene slots are exhausted; MPM_ERR_BUSY when the particle layout
 * still holds removed scenes' slots (step once, then add).  The arrays are
 * copied in stream order through a device staging buffer the batch keeps and
 * grows to its largest scene (76 B per particle, shared with particle
 * downloads; outgrown buffers are released by mpm_batch_destroy).  From page-locked memory the copy is
 * asynchronous: keep such arrays unchanged until the batch's stream has
 * passed the add (any later mpm_batch_download, or a stream synchronize). */
mpm_status mpm_batch_add(mpm_batch* batch, const mpm_params* params, const mpm_wall_params* walls,
                         const float* pos4, const float* vel4, const float* affine9, const float* mass, uint32_t n,
                         int32_t* scene);

/* Removes a scene and frees its particles, cells and id range. */
mpm_status mpm_batch_remove(mpm_batch* batch, int32_t scene);

/* Per-scene uniforms, as mpm_set_params / mpm_set_walls / mpm_set_hand
 * (grid dims must equal the scene's; particle_num is ignored). */
mpm_status mpm_batch_set_params(mpm_batch* batch, int32_t scene, const mpm_params* params);
mpm_status mpm_batch_set_walls(mpm_batch* batch, int32_t scene, const mpm_wall_params* walls);
mpm_status mpm_batch_set_hand(mpm_batch* batch, int32_t scene, const mpm_hand_params* hand, int active,
                              const int32_t bbox_dims[3]);

/* Advances every scene by `substeps` substeps; enqueues and returns. */
mpm_status mpm_batch_step(mpm_batch* batch, int substeps);

/* Waits for the batch's stream; MPM_ERR_NAN when a live scene's state holds
 * a NaN or an infinity (mpm_batch_get_health tells which). */
mpm_status mpm_batch_sync(mpm_batch* batch);

/* A scene's MPM_HEALTH_* bits, as mpm_get_health (waits for the stream). */
mpm_status mpm_batch_get_health(mpm_batch* batch, int32_t scene, uint32_t* flags, int clear);

/* Copies one buffer of one scene (reference layout, the scene's own particle
 * ids and grid) to host memory; waits. */
mpm_status mpm_batch_download(mpm_batch* batch, int32_t scene, mpm_buffer which, void* host_dst, size_t bytes);

mpm_status mpm_batch_get_stream(mpm_batch* batch, void** stream);
mpm_status mpm_batch_get_info(mpm_batch* batch, mpm_batch_info* info);

/* ---- serving: a request loop over a batch (no counterpart in the
 * reference).  Jobs (a scene + a substep count + an arrival time) are queued
 * with mpm_server_submit; mpm_server_run admits arrived jobs in FIFO order
 * while they fit the device memory the server was sized for, keeps every
 * admitted scene resident, advances all active scenes together every
 * substep, and retires each job after its last substep.  Job latency =
 * completion (taken in stream order on the device's timeline) - arrival. ---- */

typedef struct mpm_server mpm_server;

/* mpm_server_desc.flags: keep each job's final particle state (pos, vel,
 * density) on the host for mpm_server_download (costs a synchronous copy per
 * job; meant for checking results). */
#define MPM_SERVER_KEEP_STATE 0x100u

typedef struct mpm_server_desc {
    uint64_t hbm_budget_bytes;     /* device bytes the server's batch may hold */
    double cells_per_particle;     /* split of the budget between cells and particles (e.g. 2.0) */
    uint32_t scene_capacity;       /* concurrent scenes */
    int32_t device;
    uint32_t flags;                /* MPM_BATCH_* | MPM_SERVER_KEEP_STATE */
    uint32_t max_inflight;         /* substeps the host may run ahead of the device (0: 2) */
} mpm_server_desc;

typedef struct mpm_server_stats {
    uint64_t jobs;                 /* jobs finished */
    uint64_t substeps;             /* batch substeps run */
    uint64_t particle_updates;     /* sum over jobs of n * substeps */
    double wall_s;                 /* from the start of mpm_server_run to the last completion */
    double p50_latency_s, p99_latency_s, mean_latency_s, max_latency_s;
    double mean_active, max_active;   /* scenes per batch substep */
    uint64_t particle_capacity, cell_capacity;   /* what the budget bought */
    uint64_t launches;             /* kernels launched */
} mpm_server_stats;

typedef struct mpm_job_result {
    double arrival_s, admit_s, finish_s;   /* server clock: seconds since mpm_server_run started */
    uint32_t n, substeps;
    int32_t done;
    int32_t health;                        /* MPM_HEALTH_* bits of the job's scene at its last substep */
} mpm_job_result;

mpm_status mpm_server_create(const mpm_server_desc* desc, mpm_server** out);
mpm_status mpm_server_destroy(mpm_server* server);

/* Queues a job.  params: grid dims and uniforms as mpm_set_params takes them
 * (particle_num replaced by n); host arrays are copied into page-locked host
 * memory (pageable if page-locking fails), held until the mpm_server_run
 * that admits the job returns, so admission uploads are asynchronous.
 * MPM_ERR_CAPACITY if the job can never fit the server. */
mpm_status mpm_server_submit(mpm_server* server, const mpm_params* params, const float* pos4, const float* vel4,
                             const float* mass, uint32_t n, uint32_t substeps, double arrival_s, int64_t* job);

/* Runs until every job submitted since the last run has finished (the clock
 * restarts at 0 for each run); fills *stats for those jobs. */
mpm_status mpm_server_run(mpm_server* server, mpm_server_stats* stats);

mpm_status mpm_server_job(mpm_server* server, int64_t job, mpm_job_result* out);

/* A finished job's final state (MPM_SERVER_KEEP_STATE): MPM_BUF_POS, VEL or
 * DENSITY in the reference layout. */
mpm_status mpm_server_download(mpm_server* server, int64_t job, mpm_buffer which, void* host_dst, size_t bytes);

#ifdef __cplusplus
}
#endif

#endif /* MPM_B200_H */
