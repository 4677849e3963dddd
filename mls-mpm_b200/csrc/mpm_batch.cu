// mpm_batch.cu — the batch C ABI (include/mpm_b200.h, mpm_batch_*): many
// independent scenes in one world, advanced together, plus the online
// launch-shape autotuner.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "../../include/mpm_b200.h"
#include "mpm_alloc.h"
#include "mpm_world.h"

namespace mpm {

void set_error(const std::string& msg);

namespace {

mpm_status bfail(mpm_status st, const std::string& msg) {
    set_error(msg);
    return st;
}

mpm_status bcuda(cudaError_t e, const char* what) {
    const mpm_status st = (e == cudaErrorMemoryAllocation) ? MPM_ERR_OOM : MPM_ERR_DEVICE;
    return bfail(st, std::string(what) + ": " + cudaGetErrorString(e));
}

#define BATCH_TRY(expr, what)                      \
    do {                                           \
        cudaError_t _e = (expr);                   \
        if (_e != cudaSuccess) return bcuda(_e, what); \
    } while (0)

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DevGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// Online autotuner: for each workload class (log2 of the particle count, log2
// of the scene count) the first substeps cycle through candidate launch
// shapes, each timed with CUDA events over kTrialSubsteps substeps after one
// warm-up substep (which also absorbs the graph capture); the fastest shape
// is kept for the class.  Results do not depend on the shape.
struct Tuner {
    static constexpr int kTrialSubsteps = 2;
    struct Shape { uint32_t item_mult, grid_mult; };
    std::vector<Shape> cands{{8, 8}, {4, 8}, {16, 8}, {2, 8}, {8, 4}, {8, 16}};
    std::map<int, Shape> best;
    int key = -1;
    int cand = 0, sub = 0;
    std::vector<float> ms;
    cudaEvent_t ev[2] = {nullptr, nullptr};
};

}  // namespace
}  // namespace mpm

using namespace mpm;

struct mpm_batch {
    World w;
    int device = 0;
    uint32_t flags = 0;
    uint64_t substeps = 0;
    Tuner tune;
    // device staging of an added scene's reference-layout arrays, kept
    // between adds and grown to the largest scene.  Allocating it per add
    // (stream-ordered pool) blocked the host for up to 0.16 s while the pool
    // re-mapped memory, and freeing an outgrown buffer (cudaFree) for up to
    // 0.45 s next to a large world, so outgrown buffers are kept until the
    // batch is destroyed.
    void* stage = nullptr;
    size_t stage_bytes = 0;
    std::vector<void*> stage_old;
};

namespace mpm {
// Staging for a scene of n particles (76 bytes each: an add uses 72, a
// particle download 76), allocated before it is needed (the serving loop
// reserves for its largest job before it starts).
// Device address of a scene's health word (MPM_HEALTH_* bits).
uint32_t* batch_health_word(mpm_batch* b, int32_t scene) { return b->w.health + scene; }

cudaError_t batch_reserve_stage(mpm_batch* b, uint32_t n) {
    const size_t need = (size_t)(n ? n : 1) * 76;
    if (need <= b->stage_bytes) return cudaSuccess;
    const size_t bytes = std::max(need, (size_t)64 << 20);
    void* p = nullptr;
    const cudaError_t e = dmalloc(&p, bytes);
    if (e != cudaSuccess) return e;
    if (b->stage) b->stage_old.push_back(b->stage);   // a queued import may still read it
    b->stage = p;
    b->stage_bytes = bytes;
    return cudaSuccess;
}
}  // namespace mpm

namespace {

int workload_key(const World& w) {
    uint32_t scenes = 0;
    for (const SceneRec& r : w.scenes) scenes += r.live ? 1u : 0u;
    const int lp = w.n_total ? (int)std::floor(std::log2((double)w.n_total)) : 0;
    const int ls = scenes ? (int)std::floor(std::log2((double)scenes)) : 0;
    return lp * 64 + ls;
}

void apply_shape(World& w, const Tuner::Shape& s) {
    world_set_launch_shape(w, w.sms * s.item_mult, w.sms * s.grid_mult);
}

// One batch substep, with the tuner's bookkeeping around it.
cudaError_t batch_substep(mpm_batch& b) {
    World& w = b.w;
    const bool graph = !(b.flags & MPM_BATCH_NO_GRAPH);
    Tuner& t = b.tune;
    if (!(b.flags & MPM_BATCH_AUTOTUNE)) return world_substep(w, nullptr, graph);
    const int key = workload_key(w);
    auto it = t.best.find(key);
    if (it != t.best.end()) {
        apply_shape(w, it->second);
        return world_substep(w, nullptr, graph);
    }
    if (t.key != key) {   // start (or restart) trials for this class
        t.key = key;
        t.cand = 0;
        t.sub = 0;
        t.ms.assign(t.cands.size(), 0.0f);
    }
    if (!t.ev[0]) {
        cudaError_t e = cudaEventCreate(&t.ev[0]);
        if (e == cudaSuccess) e = cudaEventCreate(&t.ev[1]);
        if (e != cudaSuccess) return e;
    }
    apply_shape(w, t.cands[t.cand]);
    cudaError_t e = cudaSuccess;
    if (t.sub == 1) e = cudaEventRecord(t.ev[0], w.stream);
    if (e == cudaSuccess) e = world_substep(w, nullptr, graph);
    if (e != cudaSuccess) return e;
    if (t.sub == Tuner::kTrialSubsteps) {
        e = cudaEventRecord(t.ev[1], w.stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(t.ev[1]);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t.ev[0], t.ev[1]);
        if (e != cudaSuccess) return e;
        t.ms[t.cand] = ms;
        t.sub = 0;
        if (++t.cand == (int)t.cands.size()) {
            const int bi = (int)(std::min_element(t.ms.begin(), t.ms.end()) - t.ms.begin());
            t.best[key] = t.cands[bi];
            apply_shape(w, t.cands[bi]);
            t.key = -1;
        }
        return cudaSuccess;
    }
    t.sub++;
    return cudaSuccess;
}

}  // namespace

extern "C" {

mpm_status mpm_batch_footprint(uint32_t particle_capacity, uint64_t cell_capacity, uint32_t scene_capacity,
                               uint64_t* bytes) {
    if (!bytes) return bfail(MPM_ERR_INVALID_ARG, "NULL argument");
    *bytes = world_footprint(particle_capacity, cell_capacity, scene_capacity);
    return MPM_OK;
}

mpm_status mpm_batch_create(const mpm_batch_desc* d, mpm_batch** out) {
    if (!d || !out) return bfail(MPM_ERR_INVALID_ARG, "NULL argument");
    *out = nullptr;
    if (d->scene_capacity == 0 || d->cell_capacity == 0) return bfail(MPM_ERR_INVALID_ARG, "empty capacity");
    if (d->particle_capacity >= (1u << 31) - kPosSlack)
        return bfail(MPM_ERR_INVALID_ARG, "particle capacity too large");
    if (d->cell_capacity >= (1ull << 31) / 3) return bfail(MPM_ERR_INVALID_ARG, "cell capacity too large for 32-bit cell indexing");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess) {
        cudaGetLastError();
        ndev = 0;
    }
    if (ndev == 0) return bfail(MPM_ERR_NO_DEVICE, "no CUDA device");
    if (d->device < 0 || d->device >= ndev) return bfail(MPM_ERR_INVALID_ARG, "bad device ordinal");
    DevGuard g(d->device);
    mpm_batch* b = new (std::nothrow) mpm_batch();
    if (!b) return bfail(MPM_ERR_OOM, "host allocation");
    b->device = d->device;
    b->flags = d->flags;
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = world_alloc(b->w, d->device, st, d->particle_capacity, d->cell_capacity, d->scene_capacity);
    if (e != cudaSuccess) {
        world_free(b->w);
        if (st) cudaStreamDestroy(st);
        delete b;
        return bcuda(e, "mpm_batch_create");
    }
    *out = b;
    return MPM_OK;
}

mpm_status mpm_batch_destroy(mpm_batch* b) {
    if (!b) return MPM_OK;
    DevGuard g(b->device);
    cudaStream_t st = b->w.stream;
    world_free(b->w);   // waits for the stream
    dfree(b->stage);
    for (void* p : b->stage_old) dfree(p);
    for (cudaEvent_t& e : b->tune.ev)
        if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
    delete b;
    return MPM_OK;
}

static bool scene_ok(const mpm_batch* b, int32_t scene) {
    return b && scene >= 0 && scene < (int32_t)b->w.scene_cap && b->w.scenes[scene].live;
}

mpm_status mpm_batch_add(mpm_batch* b, const mpm_params* P, const mpm_wall_params* W, const float* pos4,
                         const float* vel4, const float* aff9, const float* mass, uint32_t n, int32_t* scene) {
    if (!b || !P || !scene || (n && (!pos4 || !mass))) return bfail(MPM_ERR_INVALID_ARG, "NULL argument");
    *scene = -1;
    if (P->grid_X < 5 || P->grid_Y < 5 || P->grid_Z < 5)
        return bfail(MPM_ERR_INVALID_ARG, "grid must be at least 5 cells per axis");
    World& w = b->w;
    const uint64_t G = (uint64_t)P->grid_X * P->grid_Y * P->grid_Z;
    uint32_t live = 0;
    for (const SceneRec& r : w.scenes) live += r.live ? 1u : 0u;
    if (live == w.scene_cap) return bfail(MPM_ERR_CAPACITY, "scene capacity reached");
    if ((uint64_t)w.n_total + n > w.pcap) return bfail(MPM_ERR_CAPACITY, "particle capacity reached");
    if ((uint64_t)w.pos_bound + n > w.npos)
        return bfail(MPM_ERR_BUSY, "particle layout still holds removed scenes; step once, then add");
    if (G > w.cell_cap) return bfail(MPM_ERR_CAPACITY, "grid larger than the batch's cell capacity");
    DevGuard g(b->device);
    cudaStream_t st = w.stream;
    // stage the host arrays in the reference layouts on the device (pos 16,
    // vel 16, affine 36, mass 4 bytes per particle; the last add's import
    // reads it earlier in stream order)
    const size_t N = n ? n : 1;
    BATCH_TRY(batch_reserve_stage(b, n), "stage allocation");
    float4* dpos = reinterpret_cast<float4*>(b->stage);
    float4* dvel = dpos + N;
    float* daff = reinterpret_cast<float*>(dvel + N);
    float* dmass = daff + 9 * N;
    cudaError_t e = cudaSuccess;
    if (n) {
        e = cudaMemcpyAsync(dpos, pos4, (size_t)n * 16, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = vel4 ? cudaMemcpyAsync(dvel, vel4, (size_t)n * 16, cudaMemcpyHostToDevice, st)
                     : cudaMemsetAsync(dvel, 0, (size_t)n * 16, st);
        if (e == cudaSuccess)
            e = aff9 ? cudaMemcpyAsync(daff, aff9, (size_t)n * 36, cudaMemcpyHostToDevice, st)
                     : cudaMemsetAsync(daff, 0, (size_t)n * 36, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dmass, mass, (size_t)n * 4, cudaMemcpyHostToDevice, st);
    }
    mpm_wall_params none;
    std::memset(&none, 0, sizeof none);
    int slot = -1;
    if (e == cudaSuccess)
        e = world_add_scene(w, P->grid_X, P->grid_Y, P->grid_Z, *P, W ? *W : none, dpos, dvel, daff, dmass, n, &slot);
    if (e == cudaErrorMemoryAllocation) return bfail(MPM_ERR_CAPACITY, "no free cell, tile or id range for the scene");
    if (e == cudaErrorNotReady) return bfail(MPM_ERR_BUSY, "particle layout full; step once, then add");
    BATCH_TRY(e, "mpm_batch_add");
    *scene = slot;
    return MPM_OK;
}

mpm_status mpm_batch_remove(mpm_batch* b, int32_t scene) {
    if (!scene_ok(b, scene)) return bfail(MPM_ERR_INVALID_ARG, "unknown scene");
    DevGuard g(b->device);
    BATCH_TRY(world_remove_scene(b->w, scene), "mpm_batch_remove");
    return MPM_OK;
}

static bool dims_match(const SceneRec& r, const mpm_params* P) {
    return P->grid_X == r.X && P->grid_Y == r.Y && P->grid_Z == r.Z;
}

mpm_status mpm_batch_set_params(mpm_batch* b, int32_t scene, const mpm_params* P) {
    if (!scene_ok(b, scene) || !P) return bfail(MPM_ERR_INVALID_ARG, "unknown scene or NULL params");
    SceneRec& r = b->w.scenes[scene];
    if (!dims_match(r, P)) return bfail(MPM_ERR_INVALID_ARG, "params grid dims differ from the scene's");
    const mpm_wall_params W = r.W;
    const mpm_hand_params H = r.H;
    int32_t box[6];
    std::memcpy(box, r.hand_box, sizeof box);
    world_set_uniforms(b->w, scene, *P, W, nullptr, 0, nullptr);
    r.H = H;   // the hand stays as mpm_batch_set_hand left it
    std::memcpy(r.hand_box, box, sizeof box);
    return MPM_OK;
}

mpm_status mpm_batch_set_walls(mpm_batch* b, int32_t scene, const mpm_wall_params* W) {
    if (!scene_ok(b, scene) || !W) return bfail(MPM_ERR_INVALID_ARG, "unknown scene or NULL walls");
    SceneRec& r = b->w.scenes[scene];
    const mpm_params P = r.P;
    const mpm_hand_params H = r.H;
    int32_t box[6];
    std::memcpy(box, r.hand_box, sizeof box);
    world_set_uniforms(b->w, scene, P, *W, nullptr, 0, nullptr);
    r.H = H;
    std::memcpy(r.hand_box, box, sizeof box);
    return MPM_OK;
}

mpm_status mpm_batch_set_hand(mpm_batch* b, int32_t scene, const mpm_hand_params* H, int active,
                              const int32_t dims[3]) {
    if (!scene_ok(b, scene) || !H) return bfail(MPM_ERR_INVALID_ARG, "unknown scene or NULL hand");
    SceneRec& r = b->w.scenes[scene];
    const mpm_params P = r.P;
    const mpm_wall_params W = r.W;
    world_set_uniforms(b->w, scene, P, W, H, active, dims);
    return MPM_OK;
}

mpm_status mpm_batch_step(mpm_batch* b, int substeps) {
    if (!b || substeps < 0) return bfail(MPM_ERR_INVALID_ARG, "bad argument");
    DevGuard g(b->device);
    for (int i = 0; i < substeps; ++i) {
        BATCH_TRY(batch_substep(*b), "mpm_batch_step");
        b->substeps++;
    }
    return MPM_OK;
}

mpm_status mpm_batch_sync(mpm_batch* b) {
    if (!b) return bfail(MPM_ERR_INVALID_ARG, "NULL argument");
    DevGuard g(b->device);
    World& w = b->w;
    BATCH_TRY(cudaStreamSynchronize(w.stream), "mpm_batch_sync");
    // health of every live scene: one copy of the health words
    std::vector<uint32_t> h(w.scene_cap ? w.scene_cap : 1, 0u);
    BATCH_TRY(cudaMemcpy(h.data(), w.health, h.size() * 4, cudaMemcpyDeviceToHost), "health readback");
    for (uint32_t i = 0; i < w.scene_cap; ++i)
        if (w.scenes[i].live && (h[i] & MPM_HEALTH_NONFINITE))
            return bfail(MPM_ERR_NAN, "scene " + std::to_string(i) +
                                          " holds a NaN or an infinity (MPM_HEALTH_NONFINITE)");
    return MPM_OK;
}

mpm_status mpm_batch_get_health(mpm_batch* b, int32_t scene, uint32_t* flags, int clear) {
    if (!scene_ok(b, scene) || !flags) return bfail(MPM_ERR_INVALID_ARG, "unknown scene or NULL argument");
    DevGuard g(b->device);
    BATCH_TRY(world_read_health(b->w, scene, flags, clear != 0), "mpm_batch_get_health");
    return MPM_OK;
}

mpm_status mpm_batch_download(mpm_batch* b, int32_t scene, mpm_buffer which, void* host, size_t bytes) {
    if (!scene_ok(b, scene) || (!host && bytes)) return bfail(MPM_ERR_INVALID_ARG, "unknown scene or NULL buffer");
    World& w = b->w;
    const SceneRec& r = w.scenes[scene];
    DevGuard g(b->device);
    cudaStream_t st = w.stream;
    const size_t n = r.n, G = r.G;
    size_t size = 0;
    const void* src = nullptr;
    int32_t *cm, *mv;
    float *cmf, *mvf;
    world_scene_grid(w, scene, &cm, &mv, &cmf, &mvf);
    switch (which) {
        case MPM_BUF_CELL_MASS: src = cm; size = G * 4; break;
        case MPM_BUF_CELL_MV: src = mv; size = G * 12; break;
        case MPM_BUF_CELL_MASS_F32: src = cmf; size = G * 4; break;
        case MPM_BUF_CELL_MV_F32: src = mvf; size = G * 12; break;
        case MPM_BUF_POS: case MPM_BUF_VEL: case MPM_BUF_AFFINE: case MPM_BUF_MASS: case MPM_BUF_DENSITY: {
            // the batch's staging buffer (queued imports read it earlier in
            // stream order; this download waits for its copy before returning)
            const size_t N = n ? n : 1;
            BATCH_TRY(batch_reserve_stage(b, (uint32_t)n), "download staging");
            char* base = (char*)b->stage;
            float4* pos = (float4*)base;
            float4* vel = (float4*)(base + N * 16);
            float* aff = (float*)(base + N * 32);
            float* mass = (float*)(base + N * 68);
            float* dens = (float*)(base + N * 72);
            cudaError_t e = cudaMemsetAsync(dens, 0, N * 4, st);
            if (e == cudaSuccess) e = world_export_scene(w, scene, pos, vel, aff, mass, dens);
            if (e != cudaSuccess) return bcuda(e, "export");
            if (which == MPM_BUF_POS) { src = pos; size = n * 16; }
            if (which == MPM_BUF_VEL) { src = vel; size = n * 16; }
            if (which == MPM_BUF_AFFINE) { src = aff; size = n * 36; }
            if (which == MPM_BUF_MASS) { src = mass; size = n * 4; }
            if (which == MPM_BUF_DENSITY) { src = dens; size = n * 4; }
            break;
        }
        default: return bfail(MPM_ERR_INVALID_ARG, "buffer not available per batch scene");
    }
    cudaError_t e = bytes > size ? cudaErrorInvalidValue : cudaSuccess;
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(host, src, bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaErrorInvalidValue) return bfail(MPM_ERR_INVALID_ARG, "bytes exceeds buffer size");
    BATCH_TRY(e, "download");
    BATCH_TRY(cudaStreamSynchronize(st), "download sync");
    return MPM_OK;
}

mpm_status mpm_batch_get_stream(mpm_batch* b, void** stream) {
    if (!b || !stream) return bfail(MPM_ERR_INVALID_ARG, "NULL argument");
    *stream = (void*)b->w.stream;
    return MPM_OK;
}

mpm_status mpm_batch_get_info(mpm_batch* b, mpm_batch_info* info) {
    if (!b || !info) return bfail(MPM_ERR_INVALID_ARG, "NULL argument");
    std::memset(info, 0, sizeof *info);
    for (const SceneRec& r : b->w.scenes) {
        if (!r.live) continue;
        info->scenes++;
        info->particles += r.n;
        info->cells += r.G;
    }
    info->launches = b->w.launches;
    info->substeps = b->substeps;
    info->device_bytes = b->w.device_bytes;
    info->item_blocks = b->w.item_blocks;
    info->grid_blocks = b->w.grid_blocks;
    return MPM_OK;
}

}  // extern "C"
