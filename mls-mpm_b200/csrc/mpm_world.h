// mpm_world.h — the binned, item-major engine over a world of scenes.
//
// A world holds any number of independent scenes (each its own grid, params
// and walls) in shared device arrays: every scene owns a range of global
// cells, a range of global tiles and a range of particle ids; particles of
// all scenes share one position space, one chunk list and one
// launch per kernel per substep.  A single scene is a world of one.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/mpm_types.h"

namespace mpm {

// Grid tile (cells) used by the sparse grid passes and the binning.
constexpr int kTileX = 16, kTileY = 8, kTileZ = 8;
constexpr int kTileCells = kTileX * kTileY * kTileZ;   // 1024: one thread per cell in k_bin_cells

// Particles are sorted by (tile, cell); each tile's particles are cut into
// chunks of at most kChunk consecutive particles.  A chunk is one block's work
// in the particle kernels: its cells form a box inside one tile, and the P2G
// sums of the box plus a one-cell halo are accumulated in shared memory and
// flushed to the grid once.
#ifndef MPM_CHUNK
#define MPM_CHUNK 512
#endif
#ifndef MPM_CHUNK_THREADS
#define MPM_CHUNK_THREADS 256
#endif
constexpr uint32_t kChunk = MPM_CHUNK;
constexpr int kChunkThreads = MPM_CHUNK_THREADS;
static_assert(kChunk % kChunkThreads == 0, "a chunk is a whole number of passes of the block");
// Small worlds, whose kChunk-particle chunks would not fill the chunk
// kernels' grid, are cut into chunks of one pass instead (shorter blocks on
// more SMs); the size is chosen per substep.
constexpr uint32_t kChunkSmall = kChunkThreads;
static_assert(kChunkSmall <= kChunk, "the small chunk is one pass");
// Largest halo box (a whole tile plus one cell on every side).
constexpr int kHaloCells = (kTileX + 2) * (kTileY + 2) * (kTileZ + 2);
// Positions of the layout beyond the particle count: none (the layout is
// dense); the slack only rounds the position space.
constexpr uint32_t kPosSlack = 256u;
constexpr uint32_t kHole = 0xFFFFFFFFu;   // key / id of a position without a particle

// Device scene table entry (read by the kernels).
struct alignas(16) SceneDesc {
    uint32_t X, Y, Z, G;
    uint32_t cell_base, tile_base, ntx, nty;
    uint32_t ntz, id_base, n, flags;
    int32_t hand_box[6];        // cells APPLY_HAND may write this substep (x0 > x1: none)
    uint32_t pad[2];
    mpm_params P;
    mpm_wall_params W;
    mpm_hand_params H;          // APPLY_HAND uniform, applied inside UPDATE_GRID over hand_box
};
static_assert(sizeof(SceneDesc) == 576, "bench.py SCENE_DESC_BYTES counts this block per uniform upload");

// Small device-side control block.  The first kCtrlZeroBytes (per-substep
// counters) start at zero and are cleared again by G2P, which runs after
// their last use in the substep.
struct Ctrl {
    uint32_t n_occ, n_grid, bins_done, pad1;   // bins_done: k_bin_cells blocks finished
    // persistent
    uint32_t total_chunks;      // chunks of the current layout
    uint32_t total_pos;         // positions of the current layout
    uint32_t prev_total_pos;    // positions of the previous layout (read through perm)
    uint32_t pad2;
};
constexpr size_t kCtrlZeroBytes = 16;

// Everything the device kernels need (passed by value).
struct WorldView {
    uint32_t npos;             // capacity of the position space
    uint32_t ntiles;           // tiles in use (end of the allocated tile range)
    uint32_t ngroups;          // ceil(ntiles / 1024): groups of the two-level tile scan
    uint32_t chunk_cap;        // capacity of the chunk list
    uint32_t chunk;            // particles per chunk this substep (kChunk or kChunkSmall)
    const SceneDesc* scenes;
    const uint32_t* tile_scene;    // scene of each global tile (kHole: free)
    uint32_t* cell_count;      // total cells + 1, zero outside binning
    uint32_t* cell_start;      // per cell: first position of its particles (local to the tile until finished)
    uint32_t* key;             // npos: binning cell (global) of each position of the current state, or kHole
    uint32_t* rank;            // npos: rank within the cell
    uint32_t* perm;            // npos: position -> position of the previous layout
    uint32_t* tile_flags;      // per tile
    uint32_t* tile_occ;        // per tile: 1 if the tile holds particles this substep
    uint32_t* tile_cnt;        // per tile: particles (occupied tiles)
    uint32_t* tile_pstart;     // per tile: exclusive scan of tile_cnt inside its 1024-tile group
    uint32_t* tile_cstart;     // per tile: exclusive scan of the chunk counts inside its group
    uint32_t* group_pstart;    // per group: exclusive scan of the group particle totals
    uint32_t* group_cstart;    // per group: exclusive scan of the group chunk totals
    uint4* chunk_info;         // per chunk: (tile, first position, end position, first local cell)
    uint32_t* chunk_last;      // per chunk: last local cell
    uint4* chunk_hdr;          // per chunk, 2 words: the packed ChunkHdr (written by P2G_MASS)
    uint4* chunk_geo;          // per chunk: (scene, tile x, tile y, tile z) of its tile
    uint32_t* tile_occ_list;
    uint32_t* tile_grid_list;
    Ctrl* ctrl;
    float* dens;               // npos, layout of the last substep
    uint32_t* health;          // per scene slot: MPM_HEALTH_* bits (sticky until read with clear)
};

// Diffuse spawn staging for the one scene of a world that has diffuse on.
struct DiffuseView {
    int enabled;
    uint32_t scene;
    const mpm_gen_params* gen;       // device copy; seed bumped on the device each substep
    mpm_diffuse_particle* staging;   // by particle id
    uint32_t* spawn_bits;            // by particle id
    uint32_t* group_counts;          // spawners per group of kGroupIds ids
};

// Reference-layout particle buffers (by particle id) that the substep keeps
// current for the one scene of a single-scene world whose consumer reads them
// every frame (a renderer's vertex inputs): G2P writes pos/vel, P2G_MOM
// writes density.  Disabled: nothing written.
struct RefOut {
    int enabled;
    uint32_t scene;
    float4* pos;
    float4* vel;
    float* dens;
};

// Host record of a scene in a world.
struct SceneRec {
    bool live = false;
    uint32_t X = 0, Y = 0, Z = 0;
    uint32_t cell_base = 0, G = 0, tile_base = 0, ntiles = 0, id_base = 0, n = 0, id_cap = 0;
    mpm_params P{};
    mpm_wall_params W{};
    int32_t hand_box[6] = {1, 1, 1, 0, 0, 0};
    mpm_hand_params H{};
};

// First-fit range allocator (host side) for cells, tiles and ids.
struct RangeAlloc {
    uint64_t cap = 0;
    std::vector<std::pair<uint64_t, uint64_t>> free_;   // (start, len), sorted
    void reset(uint64_t c) { cap = c; free_.assign(1, {0, c}); }
    bool alloc(uint64_t len, uint64_t& start);
    void release(uint64_t start, uint64_t len);
    uint64_t high_water() const;   // end of the last allocated range
};

struct World {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t pcap = 0, npos = 0;            // particle capacity, position capacity
    uint64_t cell_cap = 0;
    uint32_t tile_cap = 0, id_cap = 0, scene_cap = 0;
    uint32_t sms = 0;
    uint32_t item_blocks = 0, grid_blocks = 0, bin_blocks = 0, pos_blocks = 0;   // item_blocks: blocks of the chunk kernels
    uint64_t device_bytes = 0;              // device memory of the arrays below
    std::vector<SceneRec> scenes;           // by scene slot
    RangeAlloc cells, tiles, ids;
    uint32_t n_total = 0;                   // particles in all scenes
    uint32_t pos_bound = 0;                 // host bound on the layout end (device ctrl->total_pos)
    int cur = 0;                            // particle state copy holding the latest state
    int gbuf = 0;                           // i32 grid buffer the next substep accumulates into
    bool dens_valid = false;
    bool table_dirty = true;
    // true when the last substep's G2P left every position's rank within its
    // binning cell in rank/cell_count; adding or removing a scene clears it
    // and the next substep recounts (k_count)
    bool counted = false;
    uint64_t launches = 0;
    uint64_t generation = 1;                // bumps whenever the captured launch arguments change

    // device arrays
    // the device scene table, one copy per buffer parity: a substep of
    // parity c, and every kernel launched while cur == c, reads copy c
    // (d_scenes + c * scene_cap), so a copy can be rewritten while the
    // substep of the other parity runs
    SceneDesc* d_scenes = nullptr;          // 2 * scene_cap entries
    bool tbl_dirty[2] = {true, true};       // copy c is behind h_scenes
    bool tbl_outside[2] = {false, false};   // copy c was read outside a substep since its last in-order upload
    cudaStream_t tbl_side = nullptr;        // table uploads beside the running substep
    cudaEvent_t sub_done[2] = {nullptr, nullptr};   // after the last substep of each parity
    cudaEvent_t tbl_ev = nullptr;           // the last upload on tbl_side
    SceneDesc* scenes_dev(int c) const { return d_scenes + (size_t)c * scene_cap; }
    std::vector<SceneDesc> h_scenes;        // host copy of the table
    // pinned staging copies of the table for asynchronous uploads (a copy from
    // pageable memory would wait for the stream); each is reused only after
    // the upload that last read it has completed (stage_ev)
    SceneDesc* h_stage[2] = {nullptr, nullptr};
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    int stage_i = 0;
    uint32_t* tile_scene = nullptr;
    std::vector<uint32_t> h_tile_scene;
    float4* posm[2] = {nullptr, nullptr};   // (x, y, z, mass)
    float4* velid[2] = {nullptr, nullptr};  // (vx, vy, vz, id bits)
    float* aff[2] = {nullptr, nullptr};     // 9 planes of npos floats
    float* dens = nullptr;
    uint32_t* cell_count = nullptr;
    uint32_t* cell_start = nullptr;
    uint32_t* key = nullptr;
    uint32_t* rank = nullptr;
    uint32_t* perm = nullptr;
    uint32_t* tile_flags = nullptr;
    uint32_t* tile_occ = nullptr;
    uint32_t* tile_cnt = nullptr;
    uint32_t* tile_pstart = nullptr;
    uint32_t* tile_cstart = nullptr;
    uint32_t* group_pstart = nullptr;
    uint32_t* group_cstart = nullptr;
    uint4* chunk_info = nullptr;
    uint32_t* chunk_last = nullptr;
    uint4* chunk_hdr = nullptr;
    uint4* chunk_geo = nullptr;
    uint32_t chunk_cap = 0;
    uint32_t chunk = kChunk;   // chunk size of the substep being enqueued
    uint32_t* tile_occ_list = nullptr;
    uint32_t* tile_grid_list = nullptr;
    Ctrl* ctrl = nullptr;
    int32_t* grid_i32[2] = {nullptr, nullptr};   // each [cm: cells][mv: 3 cells]
    int32_t* cm_current = nullptr;               // buffer holding the last substep's P2G sums
    float* cmf = nullptr;                        // cells
    float* mvf = nullptr;                        // 3 cells
    float4* vel4 = nullptr;                      // cells: (vx, vy, vz, 0), the same velocities 16-byte aligned
    uint32_t* health = nullptr;                  // scene_cap words: MPM_HEALTH_* bits per scene slot

    // CUDA graphs of one substep, one per buffer parity and per whether a
    // deferred diffuse tail runs inside it (index 2 * parity + tail), valid
    // for `generation`
    static constexpr int kGraphs = 4;
    cudaGraphExec_t graph[kGraphs] = {};
    uint64_t graph_gen[kGraphs] = {};
    uint64_t graph_kernels[kGraphs] = {};    // kernels in each graph (launch accounting)
    bool graph_diffuse[kGraphs] = {};        // the graph includes the diffuse update of its scene
    bool graph_mirror[kGraphs] = {};         // the graph writes the owner's reference-layout mirrors

    WorldView view() const;
};

cudaError_t world_alloc(World& w, int device, cudaStream_t stream, uint32_t particle_cap, uint64_t cell_cap,
                        uint32_t scene_cap);
void world_free(World& w);
// Device bytes world_alloc takes for these capacities.
uint64_t world_footprint(uint32_t particle_cap, uint64_t cell_cap, uint32_t scene_cap);
// Grid sizes of the item kernels and the tile passes (results do not depend on them).
void world_set_launch_shape(World& w, uint32_t item_blocks, uint32_t grid_blocks);
// Adds a scene (grid dims, params, walls) with particles from reference-layout
// device buffers (pos4, vel4 or null, affine9 or null, mass); returns its slot.
cudaError_t world_add_scene(World& w, uint32_t X, uint32_t Y, uint32_t Z, const mpm_params& P,
                            const mpm_wall_params& W, const float4* pos, const float4* vel, const float* aff,
                            const float* mass, uint32_t n, int* slot);
cudaError_t world_remove_scene(World& w, int slot);
// Writes a scene's particles (reference layouts, by local id) to device buffers.
cudaError_t world_export_scene(World& w, int slot, float4* pos, float4* vel, float* aff, float* mass, float* dens);
// Grid buffers of a scene (reference layouts) inside the world arrays.
void world_scene_grid(const World& w, int slot, int32_t** cm, int32_t** mv, float** cmf, float** mvf);
// A scene's MPM_HEALTH_* bits as of the work enqueued so far (waits for the
// world's stream); clear: reset them afterwards (in stream order).
cudaError_t world_read_health(World& w, int slot, uint32_t* flags, bool clear);
cudaError_t world_upload_table(World& w);
// Sets a scene's uniforms (Params, WallParams, HandParams + dispatch dims;
// hand_dims null or active == 0: no APPLY_HAND).  Takes effect at the next substep.
void world_set_uniforms(World& w, int slot, const mpm_params& P, const mpm_wall_params& W,
                        const mpm_hand_params* H, int hand_active, const int32_t* hand_dims);

struct Scene;
// One substep of every scene.  owner: the single-scene wrapper of a world of
// one scene (its diffuse pool and reference-layout mirrors follow that scene;
// null for batches).  use_graph: replay a captured CUDA graph of the substep
// (captured on first use and whenever the scene set changes).
cudaError_t world_substep(World& w, Scene* owner, bool use_graph);
// Runs the owner's deferred diffuse tail now, in stream order (no-op when
// none is pending).
cudaError_t world_flush_diffuse(Scene& owner);

}  // namespace mpm
