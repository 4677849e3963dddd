// mpm_capi.cu — the C ABI (include/mpm_b200.h): scene lifetime, uploads,
// uniforms, stepping and buffer export.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mpm_b200.h"
#include "mpm_alloc.h"
#include "mpm_edit.h"
#include "mpm_kernels.h"
#include "mpm_scene.h"

static_assert(sizeof(mpm_params) == 80, "Params is 80 B (shaders.js:27-49)");
static_assert(sizeof(mpm_wall) == 80, "Wall is 80 B (shaders.js:123-129)");
static_assert(sizeof(mpm_wall_params) == 336, "WallParams is 16 + 4*80 B");
static_assert(sizeof(mpm_hand_params) == 80, "HandParams is 80 B");
static_assert(sizeof(mpm_gen_params) == 32, "GenParams is 32 B");
static_assert(sizeof(mpm_advect_params) == 16, "AdvectParams is 16 B");
static_assert(sizeof(mpm_diffuse_particle) == 48, "DiffuseParticle is 48 B");
static_assert(sizeof(mpm_ray_params) == 32, "RayParams is 32 B");

namespace mpm {

static thread_local std::string g_err;

void set_error(const std::string& msg) { g_err = msg; }

static mpm_status fail(mpm_status st, const std::string& msg) {
    set_error(msg);
    return st;
}

static mpm_status cuda_fail(cudaError_t e, const char* what) {
    const mpm_status st = (e == cudaErrorMemoryAllocation) ? MPM_ERR_OOM
                          : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? MPM_ERR_NO_DEVICE
                                                                                         : MPM_ERR_DEVICE;
    return fail(st, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CUDA_TRY(expr, what)                          \
    do {                                              \
        cudaError_t _e = (expr);                      \
        if (_e != cudaSuccess) return cuda_fail(_e, what); \
    } while (0)

template <class T> static cudaError_t dalloc(T** p, size_t bytes) { return dmalloc(p, bytes); }

cudaEvent_t Scene::take_event() {
    if (!event_pool.empty()) {
        cudaEvent_t e = event_pool.back();
        event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

void Scene::begin_phase(int phase, cudaEvent_t* a) {
    (void)phase;
    *a = nullptr;
    if (!profile) return;
    *a = take_event();
    if (*a) cudaEventRecord(*a, stream);
}

void Scene::end_phase(int phase, cudaEvent_t a) {
    if (!profile || !a) return;
    cudaEvent_t b = take_event();
    if (!b) { event_pool.push_back(a); return; }
    cudaEventRecord(b, stream);
    pending.push_back(Pending{phase, a, b});
}

cudaError_t Scene::drain_profile() {
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    for (const Pending& p : pending) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            prof_ms[p.phase] += ms;
            prof_n[p.phase] += 1;
        }
        event_pool.push_back(p.a);
        event_pool.push_back(p.b);
    }
    pending.clear();
    return cudaSuccess;
}

static void free_scene(Scene& s) {
    if (s.stream) cudaStreamSynchronize(s.stream);
    for (const Scene::Pending& p : s.pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    for (cudaEvent_t e : s.event_pool) cudaEventDestroy(e);
    s.pending.clear();
    s.event_pool.clear();
    if (s.engine == kEngineBinned) {
        world_free(s.world);   // owns cmf/mvf of the binned engine
        s.cmf = nullptr;
        s.mvf = nullptr;
        s.vel4 = nullptr;
    }
    void* ptrs[] = {s.pos, s.vel, s.aff, s.mass, s.dens, s.grid_i32, s.cmf, s.mvf,
                    s.diffuse.pool, s.diffuse.free_list, s.diffuse.top, s.diffuse.spawn_bits,
                    s.diffuse.kill_bits, s.diffuse.alive_mask, s.diffuse.block_counts, s.diffuse.kill_counts,
                    s.diffuse.rank_state,
                    s.diffuse.staging,
                    s.diffuse.top_hist, s.diffuse.tail_P, s.diffuse.tail_W,
                    s.edit_pos, s.edit_vel, s.edit_mass, s.edit_blocks, s.edit_word, s.diffuse.gen_dev,
                    s.diffuse.adv_dev};
    for (void* p : ptrs) dfree(p);
    if (s.diffuse.host_top) cudaFreeHost(s.diffuse.host_top);
    if (s.diffuse.alive_ring) cudaFreeHost(s.diffuse.alive_ring);
    for (cudaEvent_t& ev : s.diffuse.alive_ev)
        if (ev) cudaEventDestroy(ev);
    if (s.diffuse.rb_after) cudaEventDestroy(s.diffuse.rb_after);
    if (s.diffuse.rb_stream) cudaStreamDestroy(s.diffuse.rb_stream);
    if (s.diffuse.fork_ev) cudaEventDestroy(s.diffuse.fork_ev);
    if (s.diffuse.join_ev) cudaEventDestroy(s.diffuse.join_ev);
    if (s.diffuse.side) cudaStreamDestroy(s.diffuse.side);
    if (s.edit_host) cudaFreeHost(s.edit_host);
    if (s.stream) cudaStreamDestroy(s.stream);
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

static bool buffer_info(Scene& s, mpm_buffer which, void** ptr, size_t* bytes) {
    const size_t N = s.capacity, G = s.G, M = s.diffuse.max_count;
    switch (which) {
        case MPM_BUF_POS: *ptr = s.pos; *bytes = N * 16; return true;
        case MPM_BUF_VEL: *ptr = s.vel; *bytes = N * 16; return true;
        case MPM_BUF_AFFINE: *ptr = s.aff; *bytes = N * 36; return true;
        case MPM_BUF_MASS: *ptr = s.mass; *bytes = N * 4; return true;
        case MPM_BUF_DENSITY: *ptr = s.dens; *bytes = N * 4; return true;
        case MPM_BUF_CELL_MV:
        case MPM_BUF_CELL_MASS: {
            int32_t* cm = s.cm;
            int32_t* mv = s.mv;
            if (s.engine == kEngineBinned) world_scene_grid(s.world, s.world_slot, &cm, &mv, nullptr, nullptr);
            *ptr = which == MPM_BUF_CELL_MV ? (void*)mv : (void*)cm;
            *bytes = which == MPM_BUF_CELL_MV ? G * 12 : G * 4;
            return true;
        }
        case MPM_BUF_CELL_MV_F32: *ptr = s.mvf; *bytes = G * 12; return true;
        case MPM_BUF_CELL_MASS_F32: *ptr = s.cmf; *bytes = G * 4; return true;
        case MPM_BUF_DIFFUSE:
            if (!s.diffuse.enabled) return false;
            *ptr = s.diffuse.pool; *bytes = M * 48; return true;
        case MPM_BUF_FREE_LIST:
            if (!s.diffuse.enabled) return false;
            *ptr = s.diffuse.free_list; *bytes = M * 4; return true;
        case MPM_BUF_FREE_TOP:
            if (!s.diffuse.enabled) return false;
            *ptr = s.diffuse.top; *bytes = 4; return true;
    }
    return false;
}

// The buffers the deferred diffuse tail writes (the pool, its free list and top).
static bool is_diffuse_buffer(mpm_buffer w) {
    return w == MPM_BUF_DIFFUSE || w == MPM_BUF_FREE_LIST || w == MPM_BUF_FREE_TOP;
}

static bool is_particle_buffer(mpm_buffer w) {
    return w == MPM_BUF_POS || w == MPM_BUF_VEL || w == MPM_BUF_AFFINE || w == MPM_BUF_MASS || w == MPM_BUF_DENSITY;
}

// Binned engine: bring the reference-layout particle buffers up to date.
static cudaError_t sync_reference_buffers(Scene& s) {
    if (s.engine != kEngineBinned || !s.ref_stale) return cudaSuccess;
    cudaError_t e = world_export_scene(s.world, s.world_slot, s.pos, s.vel, s.aff, s.mass, s.dens);
    if (e == cudaSuccess) s.ref_stale = false;
    return e;
}

// The buffers a renderer reads every frame (fluid-renderer.js:315-328).
static bool render_buffer(mpm_buffer w) { return w == MPM_BUF_POS || w == MPM_BUF_VEL || w == MPM_BUF_DENSITY; }

// Binned engine: make one reference-layout particle buffer current.  Once the
// substeps mirror pos/vel/density (Scene::mirror), those three need nothing.
static cudaError_t ensure_reference(Scene& s, mpm_buffer which) {
    if (s.engine != kEngineBinned || !is_particle_buffer(which)) return cudaSuccess;
    if (s.mirror && render_buffer(which)) return cudaSuccess;
    return sync_reference_buffers(s);
}

// Binned engine: (re)load the working state from the reference-layout buffers.
static cudaError_t import_state(Scene& s) {
    // drop the scene from its world and add it back with the buffers' particles
    // (this also zeroes its grids, as a fresh load does)
    cudaError_t e = cudaSuccess;
    if (s.world_slot >= 0) e = world_remove_scene(s.world, s.world_slot);
    s.world_slot = -1;
    if (e == cudaSuccess)
        e = world_add_scene(s.world, s.X, s.Y, s.Z, s.params, s.walls, s.pos, s.vel, s.aff, s.mass,
                            s.params.particle_num, &s.world_slot);
    if (e == cudaSuccess) s.fast_stale = false;
    return e;
}

// A readback still copying from top_hist must finish before the kill pass
// kTopHist passes later overwrites its entry: the scene stream waits for it.
static cudaError_t guard_top_history(Scene& s) {
    DiffuseState& d = s.diffuse;
    if (!d.enabled) return cudaSuccess;
    constexpr uint32_t R = DiffuseState::kAliveRing;
    for (uint32_t i = d.alive_tail; i != d.alive_head; ++i) {
        const uint32_t t = i % R;
        if (d.alive_issued[t] && d.alive_pass[t] != UINT64_MAX &&
            d.alive_pass[t] + DiffuseState::kTopHist <= d.passes) {
            const cudaError_t e = cudaStreamWaitEvent(s.stream, d.alive_ev[t], 0);
            if (e != cudaSuccess) return e;
            d.alive_pass[t] = UINT64_MAX;
        }
    }
    return cudaSuccess;
}

// Binned engine: the alive readbacks requested while the kill pass they read
// was deferred, once that pass has been enqueued: copy its top_hist entry on
// the readback stream after the point the scene stream has reached.
static cudaError_t issue_readbacks(Scene& s) {
    DiffuseState& d = s.diffuse;
    if (!d.enabled) return cudaSuccess;
    constexpr uint32_t R = DiffuseState::kAliveRing;
    bool ordered = false;
    for (uint32_t i = d.alive_tail; i != d.alive_head; ++i) {
        const uint32_t h = i % R;
        if (d.alive_issued[h] || d.alive_pass[h] >= d.passes) continue;
        cudaError_t e = cudaSuccess;
        if (!ordered) {
            e = cudaEventRecord(d.rb_after, s.stream);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(d.rb_stream, d.rb_after, 0);
            ordered = true;
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d.alive_ring + h, d.top_hist + d.alive_pass[h] % DiffuseState::kTopHist, 4,
                                cudaMemcpyDeviceToHost, d.rb_stream);
        if (e == cudaSuccess) e = cudaEventRecord(d.alive_ev[h], d.rb_stream);
        if (e != cudaSuccess) return e;
        d.alive_issued[h] = true;
    }
    return cudaSuccess;
}

// Binned engine: run a deferred diffuse tail now (every call that observes or
// changes the scene does, so it sees the state the reference would after the
// last step).
static cudaError_t flush_tail(Scene& s) {
    if (s.engine != kEngineBinned || !s.diffuse.tail_pending) return cudaSuccess;
    cudaError_t e = world_flush_diffuse(s);
    if (e == cudaSuccess) e = issue_readbacks(s);
    return e;
}

static cudaError_t launch_substep(Scene& s) {
    s.substeps_done++;
    const cudaError_t ge = guard_top_history(s);
    if (ge != cudaSuccess) return ge;
    if (s.engine == kEnginePlain) return launch_substep_plain(s);
    s.ref_stale = true;
    world_set_uniforms(s.world, s.world_slot, s.params, s.walls, &s.hand, s.hand_active, s.hand_dims);
    return world_substep(s.world, &s, true);
}

}  // namespace mpm

using namespace mpm;

extern "C" {

int mpm_abi_version(void) { return MPM_ABI_VERSION; }

const char* mpm_last_error(void) { return g_err.c_str(); }

mpm_status mpm_device_count(int* count) {
    if (!count) return fail(MPM_ERR_INVALID_ARG, "count is NULL");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    *count = n;
    return MPM_OK;
}

mpm_status mpm_desc_from_aspect(double ax, double ay, double az, double r, uint32_t particle_num, mpm_desc* out) {
    if (!out || !(r > 0.0) || !(ax > 0.0) || !(ay > 0.0) || !(az > 0.0))
        return fail(MPM_ERR_INVALID_ARG, "aspect and radius must be positive");
    const double normToGrid = 1.0 / (r * 4.0);   // fluid-gpu.js:11
    std::memset(out, 0, sizeof *out);
    out->grid_X = (uint32_t)std::ceil(ax * normToGrid);
    out->grid_Y = (uint32_t)std::ceil(ay * normToGrid);
    out->grid_Z = (uint32_t)std::ceil(az * normToGrid);
    out->particle_capacity = particle_num;
    return MPM_OK;
}

mpm_status mpm_default_params(const mpm_desc* d, mpm_params* o) {
    if (!d || !o) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    std::memset(o, 0, sizeof *o);
    o->grid_X = d->grid_X; o->grid_Y = d->grid_Y; o->grid_Z = d->grid_Z;
    o->particle_num = 0;
    o->dt = (float)(0.3 / 1.0);     // DT / SUBSTEPS (fluid-gpu.js:24,30,649)
    o->gravity = -0.98f;
    o->rest_density = 8.0f;
    o->stiffness = 100.0f;
    o->eos_power = 1.0f;
    o->viscosity = 0.01f;
    o->hard_min = 2.0f;             // fluid-gpu.js:41-45
    o->hard_max_x = (float)(d->grid_X - 2);
    o->hard_max_y = (float)(d->grid_Y - 2);
    o->hard_max_z = (float)(d->grid_Z - 2);
    o->wall_min = 3.0f;             // fluid-gpu.js:37-39
    o->wall_stiffness = 1.0f;
    o->lookahead_k = 2.0f;
    return MPM_OK;
}

mpm_status mpm_default_diffuse_params(uint32_t max_count, mpm_gen_params* g, mpm_advect_params* a) {
    if (!g || !a) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    g->ke_threshold = 0.5f;          // diffuse-gpu.js:20-28
    g->spawn_rate_k = 3.0f;
    g->density_spray_max = 1.5f;
    g->density_bubble_min = 6.0f;
    g->lifetime_foam = 3.0f;
    g->pressure_threshold = 1.0f;
    g->crest_dot_threshold = 0.3f;
    g->seed = 1u;                    // diffuse-gpu.js:31
    a->diffuse_max = max_count;
    a->buoyancy = 1.2f;
    a->drag = 4.0f;
    a->_pad = 0.0f;
    return MPM_OK;
}

mpm_status mpm_create(const mpm_desc* d, mpm_scene** out) {
    if (!d || !out) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    *out = nullptr;
    if (d->grid_X < 5 || d->grid_Y < 5 || d->grid_Z < 5)
        return fail(MPM_ERR_INVALID_ARG, "grid must be at least 5 cells per axis");
    const uint64_t G = (uint64_t)d->grid_X * d->grid_Y * d->grid_Z;
    if (G >= (1ull << 31) / 3) return fail(MPM_ERR_INVALID_ARG, "grid too large for 32-bit cell indexing");
    if (d->particle_capacity >= (1u << 31)) return fail(MPM_ERR_INVALID_ARG, "particle capacity too large");
    int ndev = 0;
    mpm_device_count(&ndev);
    if (ndev == 0) return fail(MPM_ERR_NO_DEVICE, "no CUDA device");
    if (d->device < 0 || d->device >= ndev) return fail(MPM_ERR_INVALID_ARG, "bad device ordinal");
    DeviceGuard guard(d->device);
    mpm_scene* sc = new (std::nothrow) mpm_scene();
    if (!sc) return fail(MPM_ERR_OOM, "host allocation");
    Scene& s = sc->s;
    s.device = d->device;
    s.X = d->grid_X; s.Y = d->grid_Y; s.Z = d->grid_Z; s.G = G;
    s.capacity = d->particle_capacity;
    s.engine = (d->flags & MPM_FLAG_PLAIN) ? kEnginePlain : kEngineBinned;
    mpm_desc dd = *d;
    mpm_default_params(&dd, &s.params);
    cudaError_t e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
    const size_t N = s.capacity;
    if (e == cudaSuccess) e = dalloc(&s.pos, N * 16);
    if (e == cudaSuccess) e = dalloc(&s.vel, N * 16);
    if (e == cudaSuccess) e = dalloc(&s.aff, N * 36);
    if (e == cudaSuccess) e = dalloc(&s.mass, N * 4);
    if (e == cudaSuccess) e = dalloc(&s.dens, N * 4);
    if (e == cudaSuccess && s.engine == kEnginePlain) e = dalloc(&s.grid_i32, G * 16);
    if (e == cudaSuccess && s.engine == kEngineBinned) e = world_alloc(s.world, s.device, s.stream, s.capacity, G, 1);
    if (e == cudaSuccess && s.engine == kEnginePlain) e = dalloc(&s.cmf, G * 4);
    if (e == cudaSuccess && s.engine == kEnginePlain) e = dalloc(&s.mvf, G * 12);
    if (e == cudaSuccess && s.engine == kEngineBinned) {
        s.cmf = s.world.cmf;
        s.mvf = s.world.mvf;
        s.vel4 = s.world.vel4;
    }
    if (e != cudaSuccess) {
        free_scene(s);
        delete sc;
        return cuda_fail(e, "mpm_create allocation");
    }
    if (s.grid_i32) {
        s.cm = s.grid_i32;
        s.mv = s.grid_i32 + G;
    }
    // WebGPU zero-fills new buffers (fluid-gpu.js:226-227)
    cudaMemsetAsync(s.pos, 0, N * 16, s.stream);
    cudaMemsetAsync(s.vel, 0, N * 16, s.stream);
    cudaMemsetAsync(s.aff, 0, N * 36, s.stream);
    cudaMemsetAsync(s.mass, 0, N * 4, s.stream);
    cudaMemsetAsync(s.dens, 0, N * 4, s.stream);
    if (s.grid_i32) cudaMemsetAsync(s.grid_i32, 0, G * 16, s.stream);
    if (s.engine == kEngineBinned) {
        e = import_state(s);
        if (e != cudaSuccess) {
            free_scene(s);
            delete sc;
            return cuda_fail(e, "mpm_create world");
        }
    }
    cudaMemsetAsync(s.cmf, 0, G * 4, s.stream);
    cudaMemsetAsync(s.mvf, 0, G * 12, s.stream);
    e = cudaStreamSynchronize(s.stream);
    if (e != cudaSuccess) {
        free_scene(s);
        delete sc;
        return cuda_fail(e, "mpm_create init");
    }
    *out = sc;
    return MPM_OK;
}

mpm_status mpm_destroy(mpm_scene* sc) {
    if (!sc) return MPM_OK;
    DeviceGuard guard(sc->s.device);
    if (sc->s.stream) cudaStreamSynchronize(sc->s.stream);
    free_scene(sc->s);
    delete sc;
    return MPM_OK;
}

// The plain engine indexes P2G_MOM's and G2P's stencils unchecked, as the
// reference does (shaders.js:303-304, 598-599): every position must keep its
// 3x3x3 stencil inside the grid, i.e. lie in [1, dim - 1) on each axis and be
// finite.  The binned engine guards every stencil and takes any input.
static mpm_status plain_positions_ok(const Scene& s, const float* pos4, uint32_t n) {
    if (s.engine != kEnginePlain) return MPM_OK;
    const float hi[3] = {(float)s.X - 1.0f, (float)s.Y - 1.0f, (float)s.Z - 1.0f};
    for (uint32_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            const float x = pos4[4 * (size_t)i + a];
            if (!(x >= 1.0f && x < hi[a]))
                return fail(MPM_ERR_INVALID_ARG, "plain engine: particle " + std::to_string(i) +
                                                     " lies outside [1, dim - 1) or is not finite");
        }
    return MPM_OK;
}

mpm_status mpm_upload_particles(mpm_scene* sc, const float* pos4, const float* vel4, const float* aff9,
                                const float* mass, uint32_t n) {
    if (!sc || (!pos4 && n) || (!mass && n)) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    Scene& s = sc->s;
    if (n > s.capacity) return fail(MPM_ERR_CAPACITY, "n exceeds particle capacity");
    if (const mpm_status bad = plain_positions_ok(s, pos4, n)) return bad;
    DeviceGuard guard(s.device);
    CUDA_TRY(flush_tail(s), "diffuse");
    cudaStream_t st = s.stream;
    CUDA_TRY(cudaMemcpyAsync(s.pos, pos4, (size_t)n * 16, cudaMemcpyHostToDevice, st), "upload pos");
    if (vel4) CUDA_TRY(cudaMemcpyAsync(s.vel, vel4, (size_t)n * 16, cudaMemcpyHostToDevice, st), "upload vel");
    else CUDA_TRY(cudaMemsetAsync(s.vel, 0, (size_t)n * 16, st), "zero vel");
    if (aff9) CUDA_TRY(cudaMemcpyAsync(s.aff, aff9, (size_t)n * 36, cudaMemcpyHostToDevice, st), "upload affine");
    else CUDA_TRY(cudaMemsetAsync(s.aff, 0, (size_t)n * 36, st), "zero affine");
    CUDA_TRY(cudaMemcpyAsync(s.mass, mass, (size_t)n * 4, cudaMemcpyHostToDevice, st), "upload mass");
    s.n_active = n;
    s.params.particle_num = n;
    if (s.engine == kEngineBinned) {
        s.ref_stale = false;
        CUDA_TRY(import_state(s), "import");
    }
    CUDA_TRY(cudaStreamSynchronize(st), "upload sync");
    return MPM_OK;
}

mpm_status mpm_set_params(mpm_scene* sc, const mpm_params* p) {
    if (!sc || !p) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    Scene& s = sc->s;
    if (p->grid_X != s.X || p->grid_Y != s.Y || p->grid_Z != s.Z)
        return fail(MPM_ERR_INVALID_ARG, "params grid dims differ from the scene's");
    if (p->particle_num > s.capacity) return fail(MPM_ERR_CAPACITY, "particle_num exceeds capacity");
    if (s.engine == kEngineBinned && s.world_slot >= 0 && p->particle_num != s.world.scenes[s.world_slot].n) {
        // active count changed (spawn / delete): reload the working state next step
        DeviceGuard guard(s.device);
        CUDA_TRY(flush_tail(s), "diffuse");
        CUDA_TRY(sync_reference_buffers(s), "export");
        s.fast_stale = true;
    }
    s.params = *p;
    s.n_active = p->particle_num;
    return MPM_OK;
}

mpm_status mpm_set_walls(mpm_scene* sc, const mpm_wall_params* w) {
    if (!sc || !w) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    sc->s.walls = *w;
    return MPM_OK;
}

mpm_status mpm_set_hand(mpm_scene* sc, const mpm_hand_params* h, int active, const int32_t dims[3]) {
    if (!sc || !h) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    Scene& s = sc->s;
    s.hand = *h;
    s.hand_active = active ? 1 : 0;
    for (int i = 0; i < 3; ++i) s.hand_dims[i] = dims ? dims[i] : 0;
    return MPM_OK;
}

mpm_status mpm_diffuse_enable(mpm_scene* sc, uint32_t max_count, const mpm_gen_params* gen,
                              const mpm_advect_params* adv) {
    if (!sc || !gen || !adv) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    if (max_count == 0 || max_count >= (1u << 30)) return fail(MPM_ERR_INVALID_ARG, "bad diffuse max_count");
    Scene& s = sc->s;
    DeviceGuard guard(s.device);
    DiffuseState& d = s.diffuse;
    if (d.enabled) return fail(MPM_ERR_BUSY, "diffuse already enabled");
    const size_t M = max_count, N = s.capacity;
    const size_t nwN = (N + 31) / 32, nwM = (M + 31) / 32;
    const size_t nb = std::max((N + kGroupIds - 1) / kGroupIds, (M + kGroupIds - 1) / kGroupIds) + 1;
    cudaError_t e = dalloc(&d.pool, M * 48);
    if (e == cudaSuccess) e = dalloc(&d.free_list, M * 4);
    if (e == cudaSuccess) e = dalloc(&d.top, 16);
    if (e == cudaSuccess) e = dalloc(&d.spawn_bits, nwN * 4);
    if (e == cudaSuccess) e = dalloc(&d.kill_bits, nwM * 4);
    if (e == cudaSuccess) e = dalloc(&d.alive_mask, nwM * 4);
    if (e == cudaSuccess) e = dalloc(&d.block_counts, nb * 4);
    if (e == cudaSuccess) e = dalloc(&d.kill_counts, nb * 4);
    if (e == cudaSuccess) e = dalloc(&d.rank_state, 32);
    if (e == cudaSuccess) e = dalloc(&d.top_hist, DiffuseState::kTopHist * 4);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&d.rb_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&d.rb_after, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&d.side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&d.fork_ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&d.join_ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = dalloc(&d.tail_P, sizeof(mpm_params));
    if (e == cudaSuccess) e = dalloc(&d.tail_W, sizeof(mpm_wall_params));
    if (e == cudaSuccess) e = dalloc(&d.staging, N * 48);
    if (e == cudaSuccess) e = dalloc(&d.gen_dev, sizeof(mpm_gen_params));
    if (e == cudaSuccess) e = dalloc(&d.adv_dev, sizeof(mpm_advect_params));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&d.host_top, 16);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&d.alive_ring, DiffuseState::kAliveRing * 4);
    for (uint32_t i = 0; i < DiffuseState::kAliveRing && e == cudaSuccess; ++i)
        e = cudaEventCreateWithFlags(&d.alive_ev[i], cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(e, "mpm_diffuse_enable allocation");
    // diffuse-gpu.js:60-68: free list [0..M-1], top = M, all slots dead
    std::vector<uint32_t> fl(M);
    for (size_t i = 0; i < M; ++i) fl[i] = (uint32_t)i;
    const int32_t top = (int32_t)M;
    CUDA_TRY(cudaMemcpyAsync(d.free_list, fl.data(), M * 4, cudaMemcpyHostToDevice, s.stream), "free list");
    CUDA_TRY(cudaMemcpyAsync(d.top, &top, 4, cudaMemcpyHostToDevice, s.stream), "top");
    CUDA_TRY(cudaMemsetAsync(d.pool, 0, M * 48, s.stream), "pool");
    CUDA_TRY(cudaMemsetAsync(d.alive_mask, 0, nwM * 4, s.stream), "alive mask");
    CUDA_TRY(cudaMemsetAsync(d.rank_state, 0, 32, s.stream), "free-list pass state");
    // the spawn bits and counts start clear; each kill pass clears them again
    CUDA_TRY(cudaMemsetAsync(d.spawn_bits, 0, nwN * 4, s.stream), "spawn bits");
    CUDA_TRY(cudaMemsetAsync(d.block_counts, 0, nb * 4, s.stream), "spawn counts");
    CUDA_TRY(cudaStreamSynchronize(s.stream), "diffuse init sync");
    d.max_count = (uint32_t)M;
    d.gen = *gen;
    d.adv = *adv;
    d.adv.diffuse_max = (uint32_t)M;
    d.seed = gen->seed;
    CUDA_TRY(cudaMemcpyAsync(d.gen_dev, &d.gen, sizeof(mpm_gen_params), cudaMemcpyHostToDevice, s.stream),
             "gen params");
    CUDA_TRY(cudaMemcpyAsync(d.adv_dev, &d.adv, sizeof(mpm_advect_params), cudaMemcpyHostToDevice, s.stream),
             "advect params");
    d.enabled = true;
    return MPM_OK;
}

mpm_status mpm_diffuse_set_gen_params(mpm_scene* sc, const mpm_gen_params* gen) {
    if (!sc || !gen) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    if (!sc->s.diffuse.enabled) return fail(MPM_ERR_INVALID_ARG, "diffuse not enabled");
    DiffuseState& d = sc->s.diffuse;
    d.gen = *gen;
    d.seed = gen->seed;
    DeviceGuard guard(sc->s.device);
    CUDA_TRY(cudaMemcpyAsync(d.gen_dev, gen, sizeof(mpm_gen_params), cudaMemcpyHostToDevice, sc->s.stream),
             "gen params");
    return MPM_OK;
}

mpm_status mpm_step(mpm_scene* sc, int substeps) {
    if (!sc || substeps < 0) return fail(MPM_ERR_INVALID_ARG, "bad argument");
    Scene& s = sc->s;
    DeviceGuard guard(s.device);
    if (s.engine == kEngineBinned && s.fast_stale) {
        CUDA_TRY(flush_tail(s), "diffuse");
        cudaError_t e = import_state(s);
        if (e != cudaSuccess) return cuda_fail(e, "import");
    }
    for (int i = 0; i < substeps; ++i) {
        cudaError_t e = launch_substep(s);
        if (e != cudaSuccess) return cuda_fail(e, "mpm_step launch");
    }
    if (s.engine == kEngineBinned) CUDA_TRY(issue_readbacks(s), "alive readbacks");
    return MPM_OK;
}

// After the scene's stream has drained: MPM_ERR_NAN when its state went
// non-finite (binned engine; the flag stays until mpm_get_health clears it).
static mpm_status health_status(Scene& s) {
    if (s.engine != kEngineBinned || s.world_slot < 0) return MPM_OK;
    uint32_t flags = 0;
    CUDA_TRY(world_read_health(s.world, s.world_slot, &flags, false), "health readback");
    if (flags & MPM_HEALTH_NONFINITE)
        return fail(MPM_ERR_NAN, "the scene's particle state holds a NaN or an infinity (MPM_HEALTH_NONFINITE)");
    return MPM_OK;
}

mpm_status mpm_sync(mpm_scene* sc) {
    if (!sc) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    DeviceGuard guard(sc->s.device);
    CUDA_TRY(flush_tail(sc->s), "diffuse");
    CUDA_TRY(cudaStreamSynchronize(sc->s.stream), "mpm_sync");
    // queued alive-count readbacks have landed too
    if (sc->s.diffuse.rb_stream) CUDA_TRY(cudaStreamSynchronize(sc->s.diffuse.rb_stream), "mpm_sync readbacks");
    return health_status(sc->s);
}

mpm_status mpm_wait(mpm_scene* sc, double timeout_s) {
    if (!sc || !(timeout_s >= 0.0)) return fail(MPM_ERR_INVALID_ARG, "NULL scene or negative timeout");
    DeviceGuard guard(sc->s.device);
    CUDA_TRY(flush_tail(sc->s), "diffuse");
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaStreamQuery(sc->s.stream);
        if (e == cudaSuccess && sc->s.diffuse.rb_stream) e = cudaStreamQuery(sc->s.diffuse.rb_stream);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) return cuda_fail(e, "mpm_wait");
        const double waited = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (waited >= timeout_s) return fail(MPM_ERR_TIMEOUT, "mpm_wait: the scene's work is still running");
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    return health_status(sc->s);
}

mpm_status mpm_get_health(mpm_scene* sc, uint32_t* flags, int clear) {
    if (!sc || !flags) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    *flags = 0;
    if (sc->s.engine != kEngineBinned || sc->s.world_slot < 0) return MPM_OK;
    DeviceGuard guard(sc->s.device);
    CUDA_TRY(world_read_health(sc->s.world, sc->s.world_slot, flags, clear != 0), "mpm_get_health");
    return MPM_OK;
}

mpm_status mpm_get_buffer(mpm_scene* sc, mpm_buffer which, void** dev_ptr, size_t* bytes) {
    if (!sc || !dev_ptr || !bytes) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    if (!buffer_info(sc->s, which, dev_ptr, bytes)) return fail(MPM_ERR_INVALID_ARG, "unknown or disabled buffer");
    if (which == MPM_BUF_FREE_TOP) sc->s.diffuse.top_exported = true;
    if (is_diffuse_buffer(which)) {
        DeviceGuard guard(sc->s.device);
        CUDA_TRY(flush_tail(sc->s), "diffuse");
    }
    if (is_particle_buffer(which)) {
        Scene& s = sc->s;
        DeviceGuard guard(s.device);
        CUDA_TRY(ensure_reference(s, which), "export");
        // a consumer that takes the pos/vel/density pointer reads it every
        // frame: from now on every substep writes those three in place
        if (s.engine == kEngineBinned && render_buffer(which) && !s.mirror) {
            CUDA_TRY(sync_reference_buffers(s), "export");
            s.mirror = true;
        }
    }
    return MPM_OK;
}

// Base address of the device allocation that holds p (driver entry point
// looked up at run time, so the library needs no link-time libcuda).
static cudaError_t allocation_base(const void* p, CUdeviceptr* base, size_t* size) {
    using RangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
    static RangeFn fn = nullptr;
    if (!fn) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        const cudaError_t e = cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q);
        if (e != cudaSuccess) return e;
        if (q != cudaDriverEntryPointSuccess || !f) return cudaErrorSymbolNotFound;
        fn = reinterpret_cast<RangeFn>(f);
    }
    return fn(base, size, reinterpret_cast<CUdeviceptr>(p)) == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

mpm_status mpm_get_ipc_handle(mpm_scene* sc, mpm_buffer which, void* handle, size_t* offset, size_t* bytes) {
    if (!sc || !handle || !offset || !bytes) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    void* p;
    size_t sz;
    if (!buffer_info(sc->s, which, &p, &sz)) return fail(MPM_ERR_INVALID_ARG, "unknown or disabled buffer");
    if (which == MPM_BUF_FREE_TOP) sc->s.diffuse.top_exported = true;
    DeviceGuard guard(sc->s.device);
    if (is_diffuse_buffer(which)) CUDA_TRY(flush_tail(sc->s), "diffuse");
    if (is_particle_buffer(which)) {
        Scene& s = sc->s;
        CUDA_TRY(ensure_reference(s, which), "export");
        if (s.engine == kEngineBinned && render_buffer(which) && !s.mirror) {   // as mpm_get_buffer
            CUDA_TRY(sync_reference_buffers(s), "export");
            s.mirror = true;
        }
    }
    CUdeviceptr base = 0;
    size_t alloc = 0;
    CUDA_TRY(allocation_base(p, &base, &alloc), "allocation range");
    static_assert(sizeof(cudaIpcMemHandle_t) == MPM_IPC_HANDLE_BYTES, "IPC handle size");
    cudaIpcMemHandle_t h;
    CUDA_TRY(cudaIpcGetMemHandle(&h, reinterpret_cast<void*>(base)), "cudaIpcGetMemHandle");
    std::memcpy(handle, &h, sizeof h);
    *offset = (size_t)(reinterpret_cast<CUdeviceptr>(p) - base);
    *bytes = sz;
    return MPM_OK;
}

mpm_status mpm_download(mpm_scene* sc, mpm_buffer which, void* host_dst, size_t bytes) {
    if (!sc || (!host_dst && bytes)) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    void* p;
    size_t sz;
    if (!buffer_info(sc->s, which, &p, &sz)) return fail(MPM_ERR_INVALID_ARG, "unknown or disabled buffer");
    if (bytes > sz) return fail(MPM_ERR_INVALID_ARG, "bytes exceeds buffer size");
    DeviceGuard guard(sc->s.device);
    if (is_diffuse_buffer(which)) CUDA_TRY(flush_tail(sc->s), "diffuse");
    CUDA_TRY(ensure_reference(sc->s, which), "export");
    CUDA_TRY(cudaMemcpyAsync(host_dst, p, bytes, cudaMemcpyDeviceToHost, sc->s.stream), "download");
    CUDA_TRY(cudaStreamSynchronize(sc->s.stream), "download sync");
    return MPM_OK;
}

mpm_status mpm_upload(mpm_scene* sc, mpm_buffer which, const void* host_src, size_t bytes) {
    if (!sc || (!host_src && bytes)) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    void* p;
    size_t sz;
    if (!buffer_info(sc->s, which, &p, &sz)) return fail(MPM_ERR_INVALID_ARG, "unknown or disabled buffer");
    if (bytes > sz) return fail(MPM_ERR_INVALID_ARG, "bytes exceeds buffer size");
    if (which == MPM_BUF_POS && sc->s.engine == kEnginePlain) {
        if (bytes % 16) return fail(MPM_ERR_INVALID_ARG, "plain engine: positions are uploaded as whole vec4 records");
        if (const mpm_status bad = plain_positions_ok(sc->s, static_cast<const float*>(host_src), (uint32_t)(bytes / 16)))
            return bad;
    }
    DeviceGuard guard(sc->s.device);
    CUDA_TRY(flush_tail(sc->s), "diffuse");   // before the upload replaces what the tail would write
    if (which == MPM_BUF_FREE_TOP) sc->s.diffuse.top_written = true;
    if (is_particle_buffer(which)) {
        CUDA_TRY(sync_reference_buffers(sc->s), "export");
        if (sc->s.engine == kEngineBinned) sc->s.fast_stale = true;
    }
    CUDA_TRY(cudaMemcpyAsync(p, host_src, bytes, cudaMemcpyHostToDevice, sc->s.stream), "upload");
    // ADVECT reads only the slots the alive mask names: rebuild it from the new pool
    if (which == MPM_BUF_DIFFUSE) CUDA_TRY(launch_alive_mask_build(sc->s), "alive mask");
    CUDA_TRY(cudaStreamSynchronize(sc->s.stream), "upload sync");
    return MPM_OK;
}

mpm_status mpm_diffuse_alive_count(mpm_scene* sc, int32_t* alive) {
    if (!sc || !alive) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    DiffuseState& d = sc->s.diffuse;
    if (!d.enabled) return fail(MPM_ERR_INVALID_ARG, "diffuse not enabled");
    DeviceGuard guard(sc->s.device);
    CUDA_TRY(flush_tail(sc->s), "diffuse");
    CUDA_TRY(cudaMemcpyAsync(d.host_top, d.top, 4, cudaMemcpyDeviceToHost, sc->s.stream), "top readback");
    CUDA_TRY(cudaStreamSynchronize(sc->s.stream), "top sync");
    *alive = (int32_t)d.max_count - *d.host_top;
    return MPM_OK;
}

mpm_status mpm_diffuse_request_alive(mpm_scene* sc) {
    if (!sc) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    Scene& s = sc->s;
    DiffuseState& d = s.diffuse;
    if (!d.enabled) return fail(MPM_ERR_INVALID_ARG, "diffuse not enabled");
    DeviceGuard guard(s.device);
    constexpr uint32_t R = DiffuseState::kAliveRing;
    if (d.alive_head - d.alive_tail == R) {   // every slot in flight: take the oldest
        const uint32_t t = d.alive_tail % R;
        if (!d.alive_issued[t]) CUDA_TRY(flush_tail(s), "diffuse");   // its kill pass is still deferred
        CUDA_TRY(cudaEventSynchronize(d.alive_ev[t]), "alive readback wait");
        d.alive_last = (int32_t)d.max_count - d.alive_ring[t];
        ++d.alive_tail;
    }
    const uint32_t h = d.alive_head % R;
    if (d.top_written || d.top_exported || (d.passes == 0 && !d.tail_pending)) {
        // top may differ from the last kill pass's: copy it in stream order,
        // after the deferred tail
        CUDA_TRY(flush_tail(s), "diffuse");
        CUDA_TRY(cudaMemcpyAsync(d.alive_ring + h, d.top, 4, cudaMemcpyDeviceToHost, s.stream), "alive readback");
        CUDA_TRY(cudaEventRecord(d.alive_ev[h], s.stream), "alive readback event");
        d.alive_pass[h] = UINT64_MAX;
        d.alive_issued[h] = true;
    } else if (d.tail_pending) {
        // the top this readback reads is what the deferred kill pass (the
        // passes-th) records in top_hist: the copy is issued once that pass is
        // enqueued (the next step or a flush)
        d.alive_pass[h] = d.passes;
        d.alive_issued[h] = false;
    } else {
        // top is what the latest kill pass left in top_hist: copy that entry on
        // the side stream once the scene stream gets here, without holding the
        // scene stream back
        const uint64_t k = d.passes - 1;
        CUDA_TRY(cudaEventRecord(d.rb_after, s.stream), "alive readback point");
        CUDA_TRY(cudaStreamWaitEvent(d.rb_stream, d.rb_after, 0), "alive readback order");
        CUDA_TRY(cudaMemcpyAsync(d.alive_ring + h, d.top_hist + k % DiffuseState::kTopHist, 4, cudaMemcpyDeviceToHost,
                                 d.rb_stream), "alive readback");
        CUDA_TRY(cudaEventRecord(d.alive_ev[h], d.rb_stream), "alive readback event");
        d.alive_pass[h] = k;
        d.alive_issued[h] = true;
    }
    ++d.alive_head;
    return MPM_OK;
}

mpm_status mpm_diffuse_poll_alive(mpm_scene* sc, int32_t* alive, int32_t* ready) {
    if (!sc || !alive || !ready) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    DiffuseState& d = sc->s.diffuse;
    if (!d.enabled) return fail(MPM_ERR_INVALID_ARG, "diffuse not enabled");
    DeviceGuard guard(sc->s.device);
    constexpr uint32_t R = DiffuseState::kAliveRing;
    int32_t got = 0;
    while (d.alive_tail != d.alive_head) {
        const uint32_t t = d.alive_tail % R;
        if (!d.alive_issued[t]) break;   // its copy waits for a deferred kill pass
        const cudaError_t q = cudaEventQuery(d.alive_ev[t]);
        if (q == cudaErrorNotReady) break;
        if (q != cudaSuccess) return cuda_fail(q, "alive readback query");
        d.alive_last = (int32_t)d.max_count - d.alive_ring[t];
        ++d.alive_tail;
        got = 1;
    }
    *alive = d.alive_last;
    *ready = got;
    return MPM_OK;
}

mpm_status mpm_get_stream(mpm_scene* sc, void** stream) {
    if (!sc || !stream) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    *stream = (void*)sc->s.stream;
    return MPM_OK;
}

// fluid-gpu.js:547-550 / 597-600: the RayParams uniform (f32) from JS numbers.
static mpm_ray_params pack_ray(const double o[3], const double d[3], double radius) {
    mpm_ray_params r;
    r.ox = (float)o[0]; r.oy = (float)o[1]; r.oz = (float)o[2];
    r.radius = (float)radius;
    r.dx = (float)d[0]; r.dy = (float)d[1]; r.dz = (float)d[2];
    r._pad = 0.0f;
    return r;
}

static cudaError_t ensure_edit_scratch(Scene& s, bool compact) {
    cudaError_t e = cudaSuccess;
    if (!s.edit_word) e = dalloc(&s.edit_word, 16);
    if (e == cudaSuccess && !s.edit_host) e = cudaMallocHost((void**)&s.edit_host, 16);
    if (!compact || e != cudaSuccess || s.edit_pos) return e;
    const size_t N = s.capacity;
    e = dalloc(&s.edit_pos, N * 16);
    if (e == cudaSuccess) e = dalloc(&s.edit_vel, N * 16);
    if (e == cudaSuccess) e = dalloc(&s.edit_mass, N * 4);
    if (e == cudaSuccess) e = dalloc(&s.edit_blocks, compact_scratch_words(N) * 4);
    if (e != cudaSuccess) {
        dfree(s.edit_pos); dfree(s.edit_vel); dfree(s.edit_mass); dfree(s.edit_blocks);
        s.edit_pos = nullptr; s.edit_vel = nullptr; s.edit_mass = nullptr; s.edit_blocks = nullptr;
    }
    return e;
}

mpm_status mpm_delete_near(mpm_scene* sc, const double origin[3], const double dir[3], double radius,
                           uint32_t* new_count) {
    if (!sc || !origin || !dir || !new_count) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    Scene& s = sc->s;
    DeviceGuard guard(s.device);
    CUDA_TRY(ensure_edit_scratch(s, true), "deleteNear scratch");
    CUDA_TRY(flush_tail(s), "diffuse");
    CUDA_TRY(sync_reference_buffers(s), "export");
    const mpm_ray_params del = pack_ray(origin, dir, radius);
    const uint32_t n = s.params.particle_num;
    cudaStream_t st = s.stream;
    CUDA_TRY(launch_compact(del, n, s.pos, s.vel, s.mass, s.edit_pos, s.edit_vel, s.edit_mass, s.edit_blocks,
                            s.edit_word, st),
             "compact");
    s.launches += n ? 3 : 0;
    CUDA_TRY(cudaMemcpyAsync(s.edit_host, s.edit_word, 4, cudaMemcpyDeviceToHost, st), "count readback");
    CUDA_TRY(cudaStreamSynchronize(st), "compact sync");
    const uint32_t m = *s.edit_host;
    // survivors back into the main buffers (fluid-gpu.js:566-568)
    CUDA_TRY(cudaMemcpyAsync(s.pos, s.edit_pos, (size_t)m * 16, cudaMemcpyDeviceToDevice, st), "copy pos");
    CUDA_TRY(cudaMemcpyAsync(s.vel, s.edit_vel, (size_t)m * 16, cudaMemcpyDeviceToDevice, st), "copy vel");
    CUDA_TRY(cudaMemcpyAsync(s.mass, s.edit_mass, (size_t)m * 4, cudaMemcpyDeviceToDevice, st), "copy mass");
    s.params.particle_num = m;
    s.n_active = m;
    if (s.engine == kEngineBinned) s.fast_stale = true;
    *new_count = m;
    return MPM_OK;
}

mpm_status mpm_raycast_fluid(mpm_scene* sc, const double origin[3], const double dir[3], double radius, int* hit,
                             float* t_out, double hit_pos[3]) {
    if (!sc || !origin || !dir || !hit) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    Scene& s = sc->s;
    DeviceGuard guard(s.device);
    CUDA_TRY(ensure_edit_scratch(s, false), "raycast scratch");
    CUDA_TRY(flush_tail(s), "diffuse");
    CUDA_TRY(sync_reference_buffers(s), "export");
    const mpm_ray_params ray = pack_ray(origin, dir, radius);
    CUDA_TRY(launch_raycast(ray, s.params.particle_num, s.pos, s.edit_word, s.stream), "raycast");
    s.launches += s.params.particle_num ? 1 : 0;
    CUDA_TRY(cudaMemcpyAsync(s.edit_host, s.edit_word, 4, cudaMemcpyDeviceToHost, s.stream), "hit readback");
    CUDA_TRY(cudaStreamSynchronize(s.stream), "raycast sync");
    const uint32_t bits = *s.edit_host;
    // pollRaycast (fluid-gpu.js:617-627)
    *hit = bits != 0xFFFFFFFFu;
    if (*hit) {
        float t;
        std::memcpy(&t, &bits, 4);
        if (t_out) *t_out = t;
        if (hit_pos)
            for (int i = 0; i < 3; ++i) hit_pos[i] = origin[i] + (double)t * dir[i];
    }
    return MPM_OK;
}

mpm_status mpm_append_particles(mpm_scene* sc, const float* pos4, const float* vel4, const float* mass,
                                uint32_t count, uint32_t* appended) {
    if (!sc || !appended || (count && (!pos4 || !mass))) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    Scene& s = sc->s;
    const uint32_t start = s.params.particle_num;
    const uint32_t n = std::min<uint32_t>(count, s.capacity - start);   // fluid-gpu.js:147-149
    *appended = 0;
    if (n == 0) return MPM_OK;
    if (const mpm_status bad = plain_positions_ok(s, pos4, n)) return bad;
    DeviceGuard guard(s.device);
    cudaStream_t st = s.stream;
    CUDA_TRY(flush_tail(s), "diffuse");
    CUDA_TRY(sync_reference_buffers(s), "export");
    CUDA_TRY(cudaMemcpyAsync(s.pos + start, pos4, (size_t)n * 16, cudaMemcpyHostToDevice, st), "append pos");
    if (vel4) CUDA_TRY(cudaMemcpyAsync(s.vel + start, vel4, (size_t)n * 16, cudaMemcpyHostToDevice, st), "append vel");
    else CUDA_TRY(cudaMemsetAsync(s.vel + start, 0, (size_t)n * 16, st), "append vel");
    CUDA_TRY(cudaMemcpyAsync(s.mass + start, mass, (size_t)n * 4, cudaMemcpyHostToDevice, st), "append mass");
    CUDA_TRY(cudaStreamSynchronize(st), "append sync");
    s.params.particle_num = start + n;
    s.n_active = start + n;
    if (s.engine == kEngineBinned) s.fast_stale = true;
    *appended = n;
    return MPM_OK;
}

mpm_status mpm_compact(const mpm_ray_params* del, uint32_t n, const float* pos_in, const float* vel_in,
                       const float* mass_in, float* pos_out, float* vel_out, float* mass_out, uint32_t* count_dev,
                       void* stream) {
    if (!del || !count_dev || (n && (!pos_in || !vel_in || !mass_in || !pos_out || !vel_out || !mass_out)))
        return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t* scratch = nullptr;
    CUDA_TRY(cudaMallocAsync((void**)&scratch, compact_scratch_words(n) * 4, st), "compact scratch");
    const cudaError_t e = launch_compact(*del, n, (const float4*)pos_in, (const float4*)vel_in, mass_in,
                                         (float4*)pos_out, (float4*)vel_out, mass_out, scratch, count_dev, st);
    const cudaError_t e2 = cudaFreeAsync(scratch, st);
    CUDA_TRY(e, "compact");
    CUDA_TRY(e2, "compact scratch free");
    return MPM_OK;
}

mpm_status mpm_raycast(const mpm_ray_params* ray, uint32_t n, const float* pos_in, uint32_t* hit_dev, void* stream) {
    if (!ray || !hit_dev || (n && !pos_in)) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    CUDA_TRY(launch_raycast(*ray, n, (const float4*)pos_in, hit_dev, (cudaStream_t)stream), "raycast");
    return MPM_OK;
}

static const char* const kPhaseNames[MPM_PHASE_COUNT] = {
    "clear", "p2g_mass", "decode_mass", "p2g_mom", "update_grid", "apply_hand", "g2p",
    "diffuse_generate", "diffuse_advect", "sort"};

const char* mpm_phase_name(int phase) {
    if (phase < 0 || phase >= MPM_PHASE_COUNT) return "";
    return kPhaseNames[phase];
}

mpm_status mpm_profile_enable(mpm_scene* sc, int on) {
    if (!sc) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    DeviceGuard guard(sc->s.device);
    CUDA_TRY(flush_tail(sc->s), "diffuse");
    sc->s.profile = on != 0;
    return MPM_OK;
}

mpm_status mpm_profile_read(mpm_scene* sc, double* ms, uint64_t* count, int reset) {
    if (!sc) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    Scene& s = sc->s;
    DeviceGuard guard(s.device);
    CUDA_TRY(flush_tail(s), "diffuse");
    CUDA_TRY(s.drain_profile(), "mpm_profile_read");
    for (int i = 0; i < MPM_PHASE_COUNT; ++i) {
        if (ms) ms[i] = s.prof_ms[i];
        if (count) count[i] = s.prof_n[i];
        if (reset) { s.prof_ms[i] = 0.0; s.prof_n[i] = 0; }
    }
    return MPM_OK;
}

mpm_status mpm_launch_count(mpm_scene* sc, uint64_t* launches) {
    if (!sc || !launches) return fail(MPM_ERR_INVALID_ARG, "NULL argument");
    *launches = sc->s.launches + sc->s.world.launches;
    return MPM_OK;
}

}  // extern "C"
