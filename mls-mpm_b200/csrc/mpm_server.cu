// mpm_server.cu — the serving loop (include/mpm_b200.h, mpm_server_*): jobs
// admitted by device-memory budget into one batch, all resident scenes
// advanced together every substep, latency stamped in stream order.
//
// Built on the batch C ABI: the server owns one mpm_batch sized from the
// budget, admits with mpm_batch_add (FIFO by arrival; the head of the queue
// waits when it does not fit, so admission order is arrival order), steps
// with mpm_batch_step, and retires with mpm_batch_remove right after a job's
// last substep is enqueued.  A host function enqueued behind that substep
// stamps the completion time when the device reaches it, so the host can run
// ahead of the device (at most max_inflight substeps) without blurring
// latencies.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mpm_b200.h"
#include "mpm_world.h"

namespace mpm {
void set_error(const std::string& msg);
// Device staging of a batch (mpm_batch.cu) large enough to add a scene of n
// particles without allocating then.
cudaError_t batch_reserve_stage(mpm_batch* b, uint32_t n);
uint32_t* batch_health_word(mpm_batch* b, int32_t scene);
}

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
    mpm_params P{};
    std::vector<float> pos, vel, mass;   // page-locked while the job waits (pinned = true)
    bool pinned = false;
    uint32_t n = 0, substeps = 0, left = 0;
    double arrival = 0.0, admit = -1.0;
    volatile double finish = -1.0;   // written by the stream-ordered host function
    int32_t sid = -1;
    int state = 0;                   // 0 queued, 1 active, 2 done
    std::vector<float> out_pos, out_vel, out_dens;
    const Clock::time_point* t0 = nullptr;
    // the scene's health bits, copied at retirement into a pinned slot and
    // from there into `health` by the stream-ordered host function
    const volatile uint32_t* health_slot = nullptr;
    volatile uint32_t health = 0;
};

void CUDART_CB stamp_finish(void* p) {
    Job* j = static_cast<Job*>(p);
    j->finish = std::chrono::duration<double>(Clock::now() - *j->t0).count();
    if (j->health_slot) j->health = *j->health_slot;
}

mpm_status sfail(mpm_status st, const std::string& msg) {
    mpm::set_error(msg);
    return st;
}

// A job's input arrays are page-locked when it is submitted, so its upload at
// admission is an asynchronous copy: the serving loop never blocks on it
// while the device runs out of queued substeps.  Without page-locking the
// upload still works, as a copy from pageable memory.
void pin_inputs(Job& j) {
    bool ok = true;
    for (std::vector<float>* v : {&j.pos, &j.vel, &j.mass}) {
        if (v->empty()) continue;
        if (cudaHostRegister(v->data(), v->size() * sizeof(float), cudaHostRegisterDefault) != cudaSuccess) {
            cudaGetLastError();   // clear the error: the pageable path still works
            ok = false;
        }
    }
    if (ok) {
        j.pinned = true;
        return;
    }
    for (std::vector<float>* v : {&j.pos, &j.vel, &j.mass})
        if (!v->empty() && cudaHostUnregister(v->data()) != cudaSuccess) cudaGetLastError();
}

// Release the inputs of an admitted job (only once no copy from them can be
// in flight: after a stream synchronisation).
void release_inputs(Job& j) {
    if (j.pinned) {
        for (std::vector<float>* v : {&j.pos, &j.vel, &j.mass})
            if (!v->empty()) cudaHostUnregister(v->data());
        j.pinned = false;
    }
    std::vector<float>().swap(j.pos);
    std::vector<float>().swap(j.vel);
    std::vector<float>().swap(j.mass);
}

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace

struct mpm_server {
    mpm_batch* batch = nullptr;
    int device = 0;
    uint32_t flags = 0;
    uint32_t max_inflight = 2;
    uint64_t pcap = 0, ccap = 0;
    uint32_t scap = 0;
    std::vector<std::unique_ptr<Job>> jobs;
    Clock::time_point t0;
    // pinned ring of health words copied at job retirement; a slot is reused
    // only after ring_size later retirements, by which time the host function
    // that read it has run (the host stays at most max_inflight substeps
    // ahead, each retiring at most scene_capacity jobs)
    uint32_t* health_ring = nullptr;
    uint32_t ring_size = 0, ring_next = 0;
};

extern "C" {

mpm_status mpm_server_create(const mpm_server_desc* d, mpm_server** out) {
    if (!d || !out) return sfail(MPM_ERR_INVALID_ARG, "NULL argument");
    *out = nullptr;
    if (d->scene_capacity == 0 || !(d->cells_per_particle > 0.0))
        return sfail(MPM_ERR_INVALID_ARG, "scene_capacity and cells_per_particle must be positive");
    // split the budget: footprint = base + particles * pb + cells * cb
    const uint32_t S = d->scene_capacity;
    const double base = (double)mpm::world_footprint(0, 1, S);
    const double pb = ((double)mpm::world_footprint(1u << 20, 1, S) - base) / (double)(1u << 20);
    const double cb = ((double)mpm::world_footprint(0, 1 + (1u << 20), S) - base) / (double)(1u << 20);
    const double avail = (double)d->hbm_budget_bytes - base;
    if (avail <= 0.0) return sfail(MPM_ERR_INVALID_ARG, "budget below the fixed footprint");
    const double cell_limit = (double)((1ull << 31) / 3 - 1);
    const double part_limit = (double)((1u << 31) - mpm::kPosSlack - 1);
    double p = avail / (pb + d->cells_per_particle * cb);
    double c = p * d->cells_per_particle;
    if (c > cell_limit) {
        c = cell_limit;
        p = (avail - c * cb) / pb;
    }
    p = std::min(p, part_limit);
    if (p < 1.0 || c < 125.0) return sfail(MPM_ERR_INVALID_ARG, "budget too small");
    mpm_server* s = new (std::nothrow) mpm_server();
    if (!s) return sfail(MPM_ERR_OOM, "host allocation");
    s->device = d->device;
    s->flags = d->flags;
    s->max_inflight = d->max_inflight ? d->max_inflight : 2;
    s->pcap = (uint64_t)p;
    s->ccap = (uint64_t)c;
    s->scap = S;
    mpm_batch_desc bd;
    std::memset(&bd, 0, sizeof bd);
    bd.particle_capacity = (uint32_t)s->pcap;
    bd.scene_capacity = S;
    bd.cell_capacity = s->ccap;
    bd.device = d->device;
    bd.flags = d->flags & (MPM_BATCH_NO_GRAPH | MPM_BATCH_AUTOTUNE);
    const mpm_status st = mpm_batch_create(&bd, &s->batch);
    if (st != MPM_OK) {
        delete s;
        return st;
    }
    s->ring_size = std::max<uint32_t>(4096u, S * (s->max_inflight + 2u));
    if (cudaMallocHost((void**)&s->health_ring, (size_t)s->ring_size * 4) != cudaSuccess) {
        cudaGetLastError();
        mpm_batch_destroy(s->batch);
        delete s;
        return sfail(MPM_ERR_OOM, "pinned health ring");
    }
    std::memset(s->health_ring, 0, (size_t)s->ring_size * 4);
    *out = s;
    return MPM_OK;
}

mpm_status mpm_server_destroy(mpm_server* s) {
    if (!s) return MPM_OK;
    mpm_batch_destroy(s->batch);   // waits for the batch's stream
    for (auto& j : s->jobs) release_inputs(*j);
    if (s->health_ring) cudaFreeHost(s->health_ring);
    delete s;
    return MPM_OK;
}

mpm_status mpm_server_submit(mpm_server* s, const mpm_params* P, const float* pos4, const float* vel4,
                             const float* mass, uint32_t n, uint32_t substeps, double arrival_s, int64_t* job) {
    if (!s || !P || !job || (n && (!pos4 || !mass))) return sfail(MPM_ERR_INVALID_ARG, "NULL argument");
    if (substeps == 0) return sfail(MPM_ERR_INVALID_ARG, "a job needs at least one substep");
    const uint64_t G = (uint64_t)P->grid_X * P->grid_Y * P->grid_Z;
    if (n > s->pcap || G > s->ccap) return sfail(MPM_ERR_CAPACITY, "job larger than the server's budget");
    if (P->grid_X < 5 || P->grid_Y < 5 || P->grid_Z < 5)
        return sfail(MPM_ERR_INVALID_ARG, "grid must be at least 5 cells per axis");
    std::unique_ptr<Job> j(new (std::nothrow) Job());
    if (!j) return sfail(MPM_ERR_OOM, "host allocation");
    j->P = *P;
    j->n = n;
    j->substeps = j->left = substeps;
    j->arrival = arrival_s;
    j->pos.assign(pos4, pos4 + (size_t)n * 4);
    if (vel4) j->vel.assign(vel4, vel4 + (size_t)n * 4);
    j->mass.assign(mass, mass + n);
    {
        int prev = -1;
        cudaGetDevice(&prev);
        cudaSetDevice(s->device);
        pin_inputs(*j);
        if (prev >= 0) cudaSetDevice(prev);
    }
    j->t0 = &s->t0;
    *job = (int64_t)s->jobs.size();
    s->jobs.push_back(std::move(j));
    return MPM_OK;
}

mpm_status mpm_server_run(mpm_server* s, mpm_server_stats* stats) {
    if (!s) return sfail(MPM_ERR_INVALID_ARG, "NULL argument");
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    struct Restore {
        int dev;
        ~Restore() {
            if (dev >= 0) cudaSetDevice(dev);
        }
    } restore{prev};
    void* sp = nullptr;
    mpm_batch_get_stream(s->batch, &sp);
    cudaStream_t stream = (cudaStream_t)sp;
    std::deque<Job*> queue;
    for (auto& j : s->jobs)
        if (j->state == 0) queue.push_back(j.get());
    const std::vector<Job*> this_run(queue.begin(), queue.end());   // stats cover the jobs of this call
    std::stable_sort(queue.begin(), queue.end(), [](const Job* a, const Job* b) { return a->arrival < b->arrival; });
    const size_t R = s->max_inflight + 1;
    std::vector<cudaEvent_t> ev(R, nullptr);
    for (auto& e : ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            return sfail(MPM_ERR_DEVICE, "event creation");
    struct Events {
        std::vector<cudaEvent_t>& v;
        ~Events() {
            for (auto e : v)
                if (e) cudaEventDestroy(e);
        }
    } events{ev};
    mpm_batch_info i0;
    mpm_batch_get_info(s->batch, &i0);
    // staging for the largest queued job, allocated before the clock starts
    {
        uint32_t nmax = 0;
        for (const Job* j : queue) nmax = std::max(nmax, j->n);
        if (mpm::batch_reserve_stage(s->batch, nmax) != cudaSuccess) return sfail(MPM_ERR_OOM, "staging allocation");
    }
    std::vector<Job*> active;
    uint64_t k = 0, updates = 0, active_sum = 0, active_max = 0;
    const bool keep = (s->flags & MPM_SERVER_KEEP_STATE) != 0;
    s->t0 = Clock::now();
    auto now = [&]() { return std::chrono::duration<double>(Clock::now() - s->t0).count(); };
    for (;;) {
        // admit arrived jobs in arrival order while they fit
        const double t = now();
        while (!queue.empty() && queue.front()->arrival <= t) {
            Job* j = queue.front();
            int32_t sid = -1;
            const mpm_status st = mpm_batch_add(s->batch, &j->P, nullptr, j->pos.data(),
                                                j->vel.empty() ? nullptr : j->vel.data(), nullptr, j->mass.data(),
                                                j->n, &sid);
            if ((st == MPM_ERR_BUSY || st == MPM_ERR_CAPACITY) && !active.empty()) break;   // wait for retirements
            if (st != MPM_OK) return st;   // an empty batch that cannot take the job never will
            j->sid = sid;
            j->admit = t;
            j->state = 1;   // its inputs are released after the final synchronisation
            queue.pop_front();
            active.push_back(j);
        }
        if (active.empty()) {
            if (queue.empty()) break;
            const double wait = queue.front()->arrival - now();
            if (wait > 0.0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.01)));
            continue;
        }
        // one substep of every active scene, at most max_inflight ahead of the device
        cudaEvent_t& slot = ev[k % R];
        if (k >= R && cudaEventSynchronize(slot) != cudaSuccess) return sfail(MPM_ERR_DEVICE, "event wait");
        mpm_status st = mpm_batch_step(s->batch, 1);
        if (st != MPM_OK) return st;
        if (cudaEventRecord(slot, stream) != cudaSuccess) return sfail(MPM_ERR_DEVICE, "event record");
        ++k;
        active_sum += active.size();
        active_max = std::max<uint64_t>(active_max, active.size());
        // retire jobs whose last substep was just enqueued
        size_t w = 0;
        for (size_t r = 0; r < active.size(); ++r) {
            Job* j = active[r];
            if (--j->left > 0) {
                active[w++] = j;
                continue;
            }
            uint32_t* slot_h = s->health_ring + (s->ring_next++ % s->ring_size);
            if (cudaMemcpyAsync(slot_h, mpm::batch_health_word(s->batch, j->sid), 4, cudaMemcpyDeviceToHost,
                                stream) != cudaSuccess)
                return sfail(MPM_ERR_DEVICE, "health copy");
            j->health_slot = slot_h;
            if (cudaLaunchHostFunc(stream, stamp_finish, j) != cudaSuccess) return sfail(MPM_ERR_DEVICE, "host func");
            if (keep) {
                j->out_pos.resize((size_t)j->n * 4);
                j->out_vel.resize((size_t)j->n * 4);
                j->out_dens.resize(j->n);
                st = mpm_batch_download(s->batch, j->sid, MPM_BUF_POS, j->out_pos.data(), (size_t)j->n * 16);
                if (st == MPM_OK)
                    st = mpm_batch_download(s->batch, j->sid, MPM_BUF_VEL, j->out_vel.data(), (size_t)j->n * 16);
                if (st == MPM_OK)
                    st = mpm_batch_download(s->batch, j->sid, MPM_BUF_DENSITY, j->out_dens.data(), (size_t)j->n * 4);
                if (st != MPM_OK) return st;
            }
            st = mpm_batch_remove(s->batch, j->sid);
            if (st != MPM_OK) return st;
            j->state = 2;
            updates += (uint64_t)j->n * j->substeps;
        }
        active.resize(w);
    }
    if (cudaStreamSynchronize(stream) != cudaSuccess) return sfail(MPM_ERR_DEVICE, "final sync");
    for (Job* j : this_run)
        if (j->state != 0) release_inputs(*j);
    if (stats) {
        std::memset(stats, 0, sizeof *stats);
        std::vector<double> lat;
        double last = 0.0;
        for (Job* j : this_run) {
            if (j->state != 2) continue;
            lat.push_back(j->finish - j->arrival);
            last = std::max(last, (double)j->finish);
        }
        mpm_batch_info i1;
        mpm_batch_get_info(s->batch, &i1);
        stats->jobs = lat.size();
        stats->substeps = k;
        stats->particle_updates = updates;
        stats->wall_s = last;
        stats->p50_latency_s = percentile(lat, 0.50);
        stats->p99_latency_s = percentile(lat, 0.99);
        double sum = 0.0, mx = 0.0;
        for (double x : lat) {
            sum += x;
            mx = std::max(mx, x);
        }
        stats->mean_latency_s = lat.empty() ? 0.0 : sum / (double)lat.size();
        stats->max_latency_s = mx;
        stats->mean_active = k ? (double)active_sum / (double)k : 0.0;
        stats->max_active = (double)active_max;
        stats->particle_capacity = s->pcap;
        stats->cell_capacity = s->ccap;
        stats->launches = i1.launches - i0.launches;
    }
    return MPM_OK;
}

mpm_status mpm_server_job(mpm_server* s, int64_t job, mpm_job_result* out) {
    if (!s || !out || job < 0 || job >= (int64_t)s->jobs.size()) return sfail(MPM_ERR_INVALID_ARG, "unknown job");
    const Job& j = *s->jobs[(size_t)job];
    out->arrival_s = j.arrival;
    out->admit_s = j.admit;
    out->finish_s = j.finish;
    out->n = j.n;
    out->substeps = j.substeps;
    out->done = j.state == 2;
    out->health = j.state == 2 ? (int32_t)j.health : 0;
    return MPM_OK;
}

mpm_status mpm_server_download(mpm_server* s, int64_t job, mpm_buffer which, void* host, size_t bytes) {
    if (!s || job < 0 || job >= (int64_t)s->jobs.size() || (!host && bytes))
        return sfail(MPM_ERR_INVALID_ARG, "unknown job or NULL buffer");
    const Job& j = *s->jobs[(size_t)job];
    if (j.state != 2 || !(s->flags & MPM_SERVER_KEEP_STATE))
        return sfail(MPM_ERR_INVALID_ARG, "job not finished or state not kept");
    const std::vector<float>* v = which == MPM_BUF_POS ? &j.out_pos
                                  : which == MPM_BUF_VEL ? &j.out_vel
                                  : which == MPM_BUF_DENSITY ? &j.out_dens
                                                             : nullptr;
    if (!v) return sfail(MPM_ERR_INVALID_ARG, "only pos, vel and density are kept");
    if (bytes > v->size() * 4) return sfail(MPM_ERR_INVALID_ARG, "bytes exceeds buffer size");
    std::memcpy(host, v->data(), bytes);
    return MPM_OK;
}

}  // extern "C"
