// mpm_scene.h — host-side scene object behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mpm_b200.h"
#include "mpm_world.h"

namespace mpm {

// Deterministic free-list ranking: one bit per particle id (spawns) or pool
// slot (kills), popcounts per group of kGroupIds ids, one exclusive scan over
// the groups, then each set bit's rank = group offset + popcount before it.
constexpr uint32_t kGroupIds = 256;                 // ids per group (8 words, one 256-thread block)

struct DiffuseState {
    bool enabled = false;
    uint32_t max_count = 0;
    mpm_gen_params gen{};       // last _writeGenParams contents
    mpm_advect_params adv{};
    uint32_t seed = 1;          // DiffuseGPU._seed (diffuse-gpu.js:31)
    mpm_diffuse_particle* pool = nullptr;   // M x 48 B
    uint32_t* free_list = nullptr;          // M
    int32_t* top = nullptr;                 // 1 (device)
    // ranking scratch
    uint32_t* spawn_bits = nullptr;         // ceil(N/32) words, one bit per fluid particle id
    uint32_t* kill_bits = nullptr;          // ceil(M/32) words, one bit per slot
    // one bit per pool slot, set exactly when the slot's record is alive: the
    // spawn pass sets the bits of the slots it fills, ADVECT clears the bits
    // of the slots it kills, and an upload of the pool rebuilds it; ADVECT
    // reads only the records of set bits
    uint32_t* alive_mask = nullptr;         // ceil(M/32) words
    uint32_t* block_counts = nullptr;       // spawners per group of kGroupIds fluid ids
    uint32_t* kill_counts = nullptr;        // kills per group of kGroupIds slots
    int32_t* rank_state = nullptr;          // [0] top before the pass, [1] total, [2] applied, [3] ticket, [4] kill passes
    mpm_diffuse_particle* staging = nullptr;  // N x 48 B spawn records indexed by particle id
    int32_t* host_top = nullptr;            // pinned 4 B for alive-count readback
    // asynchronous alive-count readbacks (requestDebugReadback / pollDebug):
    // a ring of pinned slots, each with the event recorded after its copy
    static constexpr uint32_t kAliveRing = 4;
    int32_t* alive_ring = nullptr;          // pinned kAliveRing x 4 B
    cudaEvent_t alive_ev[kAliveRing] = {};
    uint32_t alive_head = 0, alive_tail = 0;   // next slot to fill / oldest unread
    int32_t alive_last = 0;                 // latest value read back
    uint64_t alive_pass[kAliveRing] = {};   // kill pass whose top each slot reads
    // top after each kill pass, kept on the device so a readback copies it on
    // a side stream and the scene stream never waits for that copy
    static constexpr uint32_t kTopHist = 256;
    int32_t* top_hist = nullptr;            // kTopHist entries, written by the kill pass
    uint64_t passes = 0;                    // kill passes enqueued (host mirror of rank_state[4])
    bool top_written = false;               // top changed outside a kill pass since the last one
    bool top_exported = false;              // a caller holds top's device address
    cudaStream_t rb_stream = nullptr;       // readback side stream
    cudaEvent_t rb_after = nullptr;         // scene-stream point a readback copies after
    mpm_gen_params* gen_dev = nullptr;      // device GenParams (binned engine: seed bumped on the device)
    mpm_advect_params* adv_dev = nullptr;   // device copy of adv (binned engine)
    // Binned engine: DiffuseGPU.step of the last substep (spawn pass, ADVECT,
    // kill pass) is deferred and runs on a side stream beside the next
    // substep's binning, P2G_MASS, DECODE_MASS and P2G_MOM, joining before its
    // UPDATE_GRID (the first pass that writes what the tail reads).  Any call
    // that observes or changes the scene runs a pending tail first (flush).
    bool tail_pending = false;
    cudaStream_t side = nullptr;            // the tail's stream
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    // the uniforms of the substep the pending tail belongs to (copied on the
    // device after its G2P, so later uploads of the scene table do not reach it)
    mpm_params* tail_P = nullptr;
    mpm_wall_params* tail_W = nullptr;
    // readbacks requested while the kill pass they read was still deferred:
    // issued once that pass is enqueued
    bool alive_issued[kAliveRing] = {true, true, true, true};
};

// Engines: the binned item-major substep (default) and the plain per-pass
// substep (MPM_FLAG_PLAIN), which mirrors the reference's dispatch list.
enum Engine { kEngineBinned = 0, kEnginePlain = 1 };

struct Scene {
    int device = 0;
    int engine = kEngineBinned;
    cudaStream_t stream = nullptr;
    uint32_t X = 0, Y = 0, Z = 0;
    uint64_t G = 0;
    uint32_t capacity = 0;
    uint32_t n_active = 0;

    mpm_params params{};
    mpm_wall_params walls{};
    mpm_hand_params hand{};
    int hand_active = 0;
    int32_t hand_dims[3] = {0, 0, 0};

    // particle buffers, reference layout
    float4* pos = nullptr;
    float4* vel = nullptr;
    float* aff = nullptr;
    float* mass = nullptr;
    float* dens = nullptr;
    // grid buffers, reference layout; cm and mv share one allocation
    int32_t* grid_i32 = nullptr;   // [cm: G][mv: 3G]
    int32_t* cm = nullptr;
    int32_t* mv = nullptr;
    float* cmf = nullptr;
    float* mvf = nullptr;
    const float4* vel4 = nullptr;   // binned engine: the grid velocities as float4 (null: read mvf)

    DiffuseState diffuse;
    World world;              // binned engine: a world holding this one scene
    int world_slot = -1;
    // binned engine: which copy of the particle state is newer
    bool ref_stale = false;    // reference-layout buffers behind the binned state
    bool fast_stale = false;   // binned state behind the reference-layout buffers
    // binned engine: pos, vel and density in the reference layout are written
    // by every substep (turned on by the first mpm_get_buffer of one of them,
    // the sign of a consumer that reads them every frame)
    bool mirror = false;
    uint64_t substeps_done = 0;
    uint64_t launches = 0;

    // deleteNear / raycastFluid scratch, allocated on first use (the
    // reference's particle*Scratch and counter buffers, fluid-gpu.js:230-240)
    float4* edit_pos = nullptr;
    float4* edit_vel = nullptr;
    float* edit_mass = nullptr;
    uint32_t* edit_blocks = nullptr;   // compact_scratch_words(capacity)
    uint32_t* edit_word = nullptr;     // device: survivor count / hit bits
    uint32_t* edit_host = nullptr;     // pinned readback of edit_word

    // per-phase CUDA-event profiler (mpm_profile_enable)
    struct Pending { int phase; cudaEvent_t a, b; };
    bool profile = false;
    std::vector<cudaEvent_t> event_pool;
    std::vector<Pending> pending;
    double prof_ms[MPM_PHASE_COUNT] = {};
    uint64_t prof_n[MPM_PHASE_COUNT] = {};

    cudaEvent_t take_event();
    void begin_phase(int phase, cudaEvent_t* a);
    void end_phase(int phase, cudaEvent_t a);
    cudaError_t drain_profile();
};

void set_error(const std::string& msg);

// RAII phase marker: records a start/end event pair when profiling is on.
struct Phase {
    Scene* s;
    int ph;
    cudaEvent_t a = nullptr;
    Phase(Scene& sc, int p) : s(&sc), ph(p) { s->begin_phase(ph, &a); }
    Phase(Scene* sc, int p) : s(sc), ph(p) {   // null: not profiled
        if (s) s->begin_phase(ph, &a);
    }
    ~Phase() {
        if (s) s->end_phase(ph, a);
    }
};

}  // namespace mpm

struct mpm_scene {
    mpm::Scene s;
};
