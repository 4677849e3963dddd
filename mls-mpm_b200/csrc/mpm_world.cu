// mpm_world.cu — the binned, item-major MLS-MPM substep over a world of scenes.
//
// Same arithmetic as mpm_kernels.cu (and so the same bits), organised for
// the B200:
//   * Work item = up to kMaxL particles of one cell.  One thread owns an
//     item: the 27 neighbour masses (P2G_MOM) or velocities (G2P) are loaded
//     once per item, and P2G contributions are summed as i32 (the same
//     wrapping sums the reference's atomics produce), flushed with one
//     atomic per (cell, component) per item.
//   * Items are bucketed by length, and particles are stored warp-interleaved:
//     the k-th particle of the item held by lane l of warp w of bucket b sits
//     at position pos_off[b] + w*32*b + k*32 + l.  All 32 lanes of a warp run
//     the same trip count and every per-particle load/store is coalesced.
//   * Within a bucket, items are ordered by (tile, cell) — a deterministic
//     layout that changes little from one substep to the next, so reading a
//     particle through the permutation (new position -> previous position)
//     stays nearly coalesced.  Cells holding more than kMaxL particles are
//     split into several items placed after the ordered ones.
//   * Scenes: cells, tiles and particle ids of every scene are ranges of the
//     world's arrays; an item carries its scene, a tile maps to its scene,
//     and each kernel reads the scene's grid dims, params and walls from the
//     device scene table.  All scenes advance in one launch per kernel.
//   * The grid is processed per tile (16x8x8 cells) and only for tiles a
//     particle stencil touches now or touched last substep (cells elsewhere
//     are zero, as the reference's CLEAR/DECODE/UPDATE would leave them).
//     The i32 grid is double-buffered: UPDATE_GRID of substep s reads
//     buffer s%2 and zeroes buffer (s+1)%2, which is the CLEAR of s+1.
//   * The diffuse spawn decision runs in the G2P epilogue (post-G2P pos/vel,
//     this substep's density), staging records by particle id.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "mpm_device.cuh"
#include "mpm_kernels.h"
#include "mpm_scene.h"
#include "mpm_world.h"

namespace mpm {

// ---------------------------------------------------------------------------
// Host: range allocator
// ---------------------------------------------------------------------------
bool RangeAlloc::alloc(uint64_t len, uint64_t& start) {
    if (len == 0) len = 1;
    for (size_t i = 0; i < free_.size(); ++i) {
        if (free_[i].second >= len) {
            start = free_[i].first;
            free_[i].first += len;
            free_[i].second -= len;
            if (free_[i].second == 0) free_.erase(free_.begin() + (long)i);
            return true;
        }
    }
    return false;
}

void RangeAlloc::release(uint64_t start, uint64_t len) {
    if (len == 0) len = 1;
    auto it = std::lower_bound(free_.begin(), free_.end(), std::make_pair(start, (uint64_t)0));
    it = free_.insert(it, {start, len});
    // merge with neighbours
    size_t i = (size_t)(it - free_.begin());
    if (i + 1 < free_.size() && free_[i].first + free_[i].second == free_[i + 1].first) {
        free_[i].second += free_[i + 1].second;
        free_.erase(free_.begin() + (long)i + 1);
    }
    if (i > 0 && free_[i - 1].first + free_[i - 1].second == free_[i].first) {
        free_[i - 1].second += free_[i].second;
        free_.erase(free_.begin() + (long)i);
    }
}

uint64_t RangeAlloc::high_water() const {
    if (free_.empty()) return cap;
    const auto& last = free_.back();
    return (last.first + last.second == cap) ? last.first : cap;
}

WorldView World::view() const {
    WorldView v;
    v.npos = npos;
    v.ntiles = (uint32_t)tiles.high_water();
    v.nchunks = (v.ntiles + 1023u) / 1024u;
    if (v.nchunks == 0) v.nchunks = 1;
    for (int b = 0; b < kMaxL + 2; ++b) v.cap_off[b] = cap_off[b];
    v.scenes = d_scenes;
    v.tile_scene = tile_scene;
    v.cell_count = cell_count; v.cell_info = cell_info; v.bucket_items = bucket_items;
    v.key = key; v.rank = rank; v.perm = perm;
    v.tile_flags = tile_flags; v.tile_occ = tile_occ; v.tile_hist = tile_hist; v.tile_base_ = tile_base;
    v.tile_occ_list = tile_occ_list; v.tile_grid_list = tile_grid_list; v.tile_chunk = tile_chunk;
    v.ctrl = ctrl; v.dens = dens;
    return v;
}

namespace {

constexpr int kItemThreads = 128;

// Register-pressure strategies of the item kernels (compile-time; defaults
// are the measured best: see the profiles for the A/B).
#ifndef MPM_MOM_LB
#define MPM_MOM_LB 1
#endif
#ifndef MPM_G2P_LB
#define MPM_G2P_LB 3
#endif

__device__ __forceinline__ int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ uint32_t local_cell(const SceneDesc& sd, int32_t x, int32_t y, int32_t z) {
    return ((uint32_t)z * sd.Y + (uint32_t)y) * sd.X + (uint32_t)x;
}

__device__ __forceinline__ uint32_t tile_of(const SceneDesc& sd, int32_t cx, int32_t cy, int32_t cz) {
    return sd.tile_base +
           ((uint32_t)(cz / kTileZ) * sd.nty + (uint32_t)(cy / kTileY)) * sd.ntx + (uint32_t)(cx / kTileX);
}

// Mark a tile as holding particles for the next substep (bit 0).
__device__ __forceinline__ void mark_occupied(const WorldView& v, uint32_t t) {
    if ((v.tile_flags[t] & 1u) == 0u) atomicOr(&v.tile_flags[t], 1u);
}

// Binning cell of a position (clamped into the scene's grid; binning only).
__device__ __forceinline__ void bin_cell(const SceneDesc& sd, float px, float py, float pz, int32_t& cx, int32_t& cy,
                                         int32_t& cz) {
    cx = clampi(__float2int_rz(floorf(px)), 0, (int32_t)sd.X - 1);
    cy = clampi(__float2int_rz(floorf(py)), 0, (int32_t)sd.Y - 1);
    cz = clampi(__float2int_rz(floorf(pz)), 0, (int32_t)sd.Z - 1);
}

// ---------------------------------------------------------------------------
// Scene import / removal / export
// ---------------------------------------------------------------------------

// Appends a scene's particles at positions [pos0, pos0 + n) with their keys.
__global__ void k_import(WorldView v, uint32_t scene, uint32_t pos0, const float4* __restrict__ pos,
                         const float4* __restrict__ vel, const float* __restrict__ aff,
                         const float* __restrict__ mass, float4* __restrict__ posm, float4* __restrict__ velid,
                         float* __restrict__ aff_out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const SceneDesc& sd = v.scenes[scene];
    const uint32_t p = pos0 + i;
    const size_t plane = v.npos;
    const float4 q = pos[i];
    const float4 vv = vel ? vel[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    posm[p] = make_float4(q.x, q.y, q.z, mass[i]);
    velid[p] = make_float4(vv.x, vv.y, vv.z, __uint_as_float(sd.id_base + i));
#pragma unroll
    for (int e = 0; e < 9; ++e) aff_out[e * plane + p] = aff ? aff[9ull * i + e] : 0.0f;
    int32_t cx, cy, cz;
    bin_cell(sd, q.x, q.y, q.z, cx, cy, cz);
    v.key[p] = sd.cell_base + local_cell(sd, cx, cy, cz);
    mark_occupied(v, tile_of(sd, cx, cy, cz));
}

// Drops a scene's particles: their positions become holes.
__global__ void k_remove(WorldView v, const float4* __restrict__ velid, uint32_t id0, uint32_t n) {
    const uint32_t total = min(v.ctrl->total_pos, v.npos);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += gridDim.x * blockDim.x) {
        if (v.key[p] == kHole) continue;
        const uint32_t id = __float_as_uint(velid[p].w);
        if (id - id0 < n) v.key[p] = kHole;
    }
}

// Marks positions [total_pos, end) as holes and sets the layout size to end:
// scenes appended at `end` leave no stale keys between the old layout and them.
__global__ void k_extend(WorldView v, uint32_t end) {
    const uint32_t start = v.ctrl->total_pos;
    for (uint32_t p = start + blockIdx.x * blockDim.x + threadIdx.x; p < end; p += gridDim.x * blockDim.x)
        v.key[p] = kHole;
}

// Writes a scene's particles to reference-layout buffers by local id.
__global__ void k_export(WorldView v, const float4* __restrict__ posm, const float4* __restrict__ velid,
                         const float* __restrict__ aff, const float* __restrict__ dens, uint32_t id0, uint32_t n,
                         float4* __restrict__ pos, float4* __restrict__ vel, float* __restrict__ aff_out,
                         float* __restrict__ mass, float* __restrict__ dens_out) {
    const uint32_t total = min(v.ctrl->total_pos, v.npos);
    const size_t plane = v.npos;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < total; j += gridDim.x * blockDim.x) {
        if (v.key[j] == kHole) continue;
        const float4 vv = velid[j];
        const uint32_t id = __float_as_uint(vv.w) - id0;
        if (id >= n) continue;
        const float4 p = posm[j];
        pos[id] = make_float4(p.x, p.y, p.z, 0.0f);
        vel[id] = make_float4(vv.x, vv.y, vv.z, 0.0f);
        mass[id] = p.w;
        if (dens_out) dens_out[id] = dens[j];
#pragma unroll
        for (int e = 0; e < 9; ++e) aff_out[9ull * id + e] = aff[e * plane + j];
    }
}

// Sets the layout size after imports/removals done outside a substep.
__global__ void k_set_total(Ctrl* ctrl, uint32_t total) {
    ctrl->total_pos = total;
    ctrl->prev_total_pos = total;
}

// ---------------------------------------------------------------------------
// Binning
// ---------------------------------------------------------------------------

// Rank of every particle of the current state within its binning cell.
__global__ void k_count(WorldView v) {
    const uint32_t total = v.ctrl->total_pos;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const uint32_t c = v.key[i];
        if (c != kHole) v.rank[i] = atomicAdd(&v.cell_count[c], 1u);
    }
}

// Occupied-tile list for the binning and the occupancy used by the scans.
// tile_flags bits: 0 occupied (set by G2P / import), 1 stencil now (set by the
// binning), 2 stencil last substep.
__global__ void k_tiles_occ(WorldView v) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= v.ntiles) return;
    const uint32_t occ = v.tile_flags[t] & 1u;
    v.tile_occ[t] = occ;
    if (occ) v.tile_occ_list[atomicAdd(&v.ctrl->n_occ, 1u)] = t;
}

// One block per occupied tile, one thread per cell.  A cell with 1..kMaxL
// particles becomes one item in bucket `count`, ranked within the tile by
// cell index (match + warp prefix); the tile's per-bucket totals go to
// tile_hist.  Larger cells are split into items that take unordered slots
// after the ordered ones.  Also marks every tile the particles' 3x3x3
// stencils touch (bit 1) and clears the counts.
__global__ void __launch_bounds__(kTileCells) k_bin_cells(WorldView v) {
    __shared__ uint32_t wcnt[kTileCells / 32][kMaxL + 1];
    __shared__ uint32_t dirs;
    const uint32_t nocc = v.ctrl->n_occ;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (uint32_t ti = blockIdx.x; ti < nocc; ti += gridDim.x) {
        const uint32_t t = v.tile_occ_list[ti];
        const uint32_t scene = v.tile_scene[t];
        const SceneDesc& sd = v.scenes[scene];
        const uint32_t lt = t - sd.tile_base;
        const uint32_t tx = lt % sd.ntx, ty = (lt / sd.ntx) % sd.nty, tz = lt / (sd.ntx * sd.nty);
        const uint32_t lx = threadIdx.x % kTileX, ly = (threadIdx.x / kTileX) % kTileY,
                       lz = threadIdx.x / (kTileX * kTileY);
        const uint32_t x = tx * kTileX + lx, y = ty * kTileY + ly, z = tz * kTileZ + lz;
        const bool inside = x < sd.X && y < sd.Y && z < sd.Z;
        const uint32_t c = inside ? sd.cell_base + local_cell(sd, x, y, z) : 0u;
        uint32_t cnt = 0;
        if (inside) {
            cnt = v.cell_count[c];
            if (cnt) v.cell_count[c] = 0u;
        }
        if (threadIdx.x == 0) dirs = 0u;
        for (int b = lane; b <= kMaxL; b += 32) wcnt[wid][b] = 0u;
        __syncthreads();
        // neighbour tiles this cell's stencil reaches (3x3x3 direction bits)
        uint32_t m = 0;
        if (cnt) {
            const int dx = lx == 0 ? -1 : (lx == kTileX - 1 ? 1 : 0);
            const int dy = ly == 0 ? -1 : (ly == kTileY - 1 ? 1 : 0);
            const int dz = lz == 0 ? -1 : (lz == kTileZ - 1 ? 1 : 0);
            for (int kz = 0; kz <= (dz != 0); ++kz)
                for (int ky = 0; ky <= (dy != 0); ++ky)
                    for (int kx = 0; kx <= (dx != 0); ++kx)
                        m |= 1u << ((kz * dz + 1) * 9 + (ky * dy + 1) * 3 + (kx * dx + 1));
        }
        const uint32_t wm = __reduce_or_sync(0xffffffffu, m);
        if (lane == 0 && wm) atomicOr(&dirs, wm);
        const uint32_t b = (cnt >= 1 && cnt <= (uint32_t)kMaxL) ? cnt : 0u;
        const uint32_t grp = __match_any_sync(0xffffffffu, b);
        const uint32_t lrank = __popc(grp & ((1u << lane) - 1u));
        if (b && lrank == 0) wcnt[wid][b] = __popc(grp);
        __syncthreads();
        // exclusive prefix over the 32 warps for each length; tile totals
        if (threadIdx.x >= 1 && threadIdx.x <= kMaxL) {
            uint32_t acc = 0;
            for (int w = 0; w < kTileCells / 32; ++w) {
                const uint32_t k = wcnt[w][threadIdx.x];
                wcnt[w][threadIdx.x] = acc;
                acc += k;
            }
            v.tile_hist[(size_t)(threadIdx.x - 1) * v.ntiles + t] = acc;
        }
        if (threadIdx.x < 27 && ((dirs >> threadIdx.x) & 1u)) {
            const int ox = (int)(threadIdx.x % 3) - 1, oy = (int)((threadIdx.x / 3) % 3) - 1,
                      oz = (int)(threadIdx.x / 9) - 1;
            const int nx = (int)tx + ox, ny = (int)ty + oy, nz = (int)tz + oz;
            if (nx >= 0 && ny >= 0 && nz >= 0 && nx < (int)sd.ntx && ny < (int)sd.nty && nz < (int)sd.ntz) {
                const uint32_t nt = sd.tile_base + ((uint32_t)nz * sd.nty + (uint32_t)ny) * sd.ntx + (uint32_t)nx;
                if ((v.tile_flags[nt] & 2u) == 0u) atomicOr(&v.tile_flags[nt], 2u);
            }
        }
        __syncthreads();
        if (b) {
            v.cell_info[c] = make_uint4(b | (b << 8) | (1u << 16), wcnt[wid][b] + lrank, t, scene);
        } else if (cnt) {
            // overpacked cell: q items of length L (the last of Llast), unordered tail slots
            const uint32_t q = (cnt + kMaxL - 1) / kMaxL;
            const uint32_t L = (cnt + q - 1) / q;
            const uint32_t Llast = cnt - (q - 1) * L;
            const uint32_t nL = (Llast == L) ? q : q - 1;
            const uint32_t idxL = atomicAdd(&v.ctrl->tail_cnt[L], nL);
            const uint32_t idxLast = (Llast != L) ? atomicAdd(&v.ctrl->tail_cnt[Llast], 1u) : idxL + q - 1;
            v.cell_info[c] = make_uint4(L | (Llast << 8) | (q << 16) | 0x80000000u, idxL, idxLast, scene);
        }
        __syncthreads();
    }
}

// Grid-tile list (stencil tiles of this substep or the last one, plus the
// hand boxes); shifts the flags for the next substep.
__global__ void k_tiles_grid(WorldView v) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= v.ntiles) return;
    const uint32_t scene = v.tile_scene[t];
    const uint32_t f = v.tile_flags[t];
    if (scene == kHole) {
        if (f) v.tile_flags[t] = 0u;
        return;
    }
    const SceneDesc& sd = v.scenes[scene];
    const uint32_t lt = t - sd.tile_base;
    const uint32_t tx = lt % sd.ntx, ty = (lt / sd.ntx) % sd.nty, tz = lt / (sd.ntx * sd.nty);
    bool hand = false;
    if (sd.hand_box[0] <= sd.hand_box[3]) {
        const int32_t x0 = (int32_t)tx * kTileX, y0 = (int32_t)ty * kTileY, z0 = (int32_t)tz * kTileZ;
        hand = x0 <= sd.hand_box[3] && x0 + kTileX - 1 >= sd.hand_box[0] && y0 <= sd.hand_box[4] &&
               y0 + kTileY - 1 >= sd.hand_box[1] && z0 <= sd.hand_box[5] && z0 + kTileZ - 1 >= sd.hand_box[2];
    }
    const bool now = (f & 2u) != 0 || hand || (v.tile_occ[t] != 0u);
    const bool prev = (f & 4u) != 0;
    if (now || prev) v.tile_grid_list[atomicAdd(&v.ctrl->n_grid, 1u)] = t;
    if (f != (now ? 4u : 0u)) v.tile_flags[t] = now ? 4u : 0u;
}

// Exclusive scan of the ordered item counts of each length bucket over all
// tiles in index order, in two levels.  Level 1, one block per (1024-tile
// chunk, bucket): tile_base = prefix inside the chunk, tile_chunk = chunk total.
__device__ __forceinline__ uint32_t block_exclusive_scan_1024(uint32_t x, uint32_t* ws, uint32_t& total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t sc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, sc, o);
        if (lane >= o) sc += y;
    }
    if (lane == 31) ws[wid] = sc;
    __syncthreads();
    if (wid == 0) {
        const uint32_t w = ws[lane];
        uint32_t ww = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, ww, o);
            if (lane >= o) ww += y;
        }
        ws[lane] = ww - w;
        if (lane == 31) ws[32] = ww;
    }
    __syncthreads();
    const uint32_t r = ws[wid] + sc - x;
    total = ws[32];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(1024) k_tile_scan_local(WorldView v) {
    __shared__ uint32_t ws[33];
    const uint32_t chunk = blockIdx.x, b = blockIdx.y;
    const uint32_t t = chunk * 1024u + threadIdx.x;
    const uint32_t x = (t < v.ntiles && v.tile_occ[t]) ? v.tile_hist[(size_t)b * v.ntiles + t] : 0u;
    uint32_t total;
    const uint32_t r = block_exclusive_scan_1024(x, ws, total);
    if (t < v.ntiles) v.tile_base_[(size_t)b * v.ntiles + t] = r;
    if (threadIdx.x == 0) v.tile_chunk[(size_t)b * v.nchunks + chunk] = total;
}

// Level 2, one block per bucket: exclusive scan of the chunk totals in place;
// the bucket total goes to bucket_reg.
__global__ void __launch_bounds__(1024) k_tile_scan_chunks(WorldView v) {
    __shared__ uint32_t ws[33];
    const uint32_t b = blockIdx.x;
    uint32_t* chunks = v.tile_chunk + (size_t)b * v.nchunks;
    uint32_t carry = 0;
    for (uint32_t c0 = 0; c0 < v.nchunks; c0 += 1024) {
        const uint32_t c = c0 + threadIdx.x;
        const uint32_t x = c < v.nchunks ? chunks[c] : 0u;
        uint32_t total;
        const uint32_t r = block_exclusive_scan_1024(x, ws, total);
        if (c < v.nchunks) chunks[c] = carry + r;
        carry += total;
    }
    if (threadIdx.x == 0) v.ctrl->bucket_reg[b + 1] = carry;
}

// Bucket offsets (one warp): ordered + tail items, padded to whole warps.
// Also advances the diffuse seed (diffuse-gpu.js:149) for this substep.
__global__ void k_bucket_scan(Ctrl* ctrl, mpm_gen_params* gen) {
    const int lane = threadIdx.x;
    const uint32_t b = (uint32_t)lane;
    const uint32_t cnt = (b >= 1 && b <= (uint32_t)kMaxL) ? ctrl->bucket_reg[b] + ctrl->tail_cnt[b] : 0u;
    const uint32_t pad = (cnt + 31u) & ~31u;
    uint32_t si = pad, sp = pad * b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t yi = __shfl_up_sync(0xffffffffu, si, o);
        const uint32_t yp = __shfl_up_sync(0xffffffffu, sp, o);
        if (lane >= o) { si += yi; sp += yp; }
    }
    if (b <= (uint32_t)kMaxL + 1) {
        ctrl->item_off[b] = si - pad;
        ctrl->pos_off[b] = sp - pad * b;
        ctrl->bucket_cnt[b] = cnt;
    }
    const uint32_t ti = __shfl_sync(0xffffffffu, si, kMaxL);
    const uint32_t tp = __shfl_sync(0xffffffffu, sp, kMaxL);
    if (lane == 0) {
        ctrl->total_items = ti;
        ctrl->prev_total_pos = ctrl->total_pos;
        ctrl->total_pos = tp;
        if (gen) gen->seed = gen->seed + 1u;
    }
}

__device__ __forceinline__ uint32_t item_position(const uint32_t* pos_off, uint32_t b, uint32_t idx) {
    return pos_off[b] + (idx >> 5) * 32u * b + (idx & 31u);
}

// perm[new position] = previous position for every particle; the first
// particle of each item also records the item's (cell, scene).
__global__ void k_scatter(WorldView v) {
    __shared__ uint32_t pos_off[kMaxL + 2];
    __shared__ uint32_t reg[kMaxL + 2];
    if (threadIdx.x < kMaxL + 2) {
        pos_off[threadIdx.x] = v.ctrl->pos_off[threadIdx.x];
        reg[threadIdx.x] = v.ctrl->bucket_reg[threadIdx.x];
    }
    __syncthreads();
    const uint32_t total = v.ctrl->prev_total_pos;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const uint32_t c = v.key[i];
        if (c == kHole) continue;
        const uint32_t r = v.rank[i];
        const uint4 info = v.cell_info[c];
        uint32_t b, idx, kk;
        if (!(info.x & 0x80000000u)) {
            b = info.x & 0xFFu;
            const size_t row = (size_t)(b - 1);
            idx = v.tile_base_[row * v.ntiles + info.z] + v.tile_chunk[row * v.nchunks + (info.z >> 10)] + info.y;
            kk = r;
        } else {
            const uint32_t L = info.x & 0xFFu, Llast = (info.x >> 8) & 0xFFu, q = (info.x >> 16) & 0x7FFFu;
            const uint32_t it = r / L;
            kk = r - it * L;
            if (it + 1 < q || Llast == L) { b = L; idx = reg[L] + info.y + it; }
            else { b = Llast; idx = reg[Llast] + info.z; }
        }
        if (b < 1 || b > (uint32_t)kMaxL) continue;
        const uint32_t pos = item_position(pos_off, b, idx) + kk * 32u;
        if (pos >= v.npos) continue;
        v.perm[pos] = i;
        if (kk == 0 && v.cap_off[b] + idx < v.cap_off[b + 1])
            v.bucket_items[v.cap_off[b] + idx] = make_uint2(c, info.w);
    }
}

// Shared copy of the bucket tables for the item kernels.
struct ItemTables {
    uint32_t item_off[kMaxL + 2];
    uint32_t pos_off[kMaxL + 2];
    uint32_t cnt[kMaxL + 2];
};

__device__ __forceinline__ void load_tables(const WorldView& v, ItemTables& t) {
    if (threadIdx.x < kMaxL + 2) {
        t.item_off[threadIdx.x] = v.ctrl->item_off[threadIdx.x];
        t.pos_off[threadIdx.x] = v.ctrl->pos_off[threadIdx.x];
        t.cnt[threadIdx.x] = (threadIdx.x >= 1 && threadIdx.x <= kMaxL) ? v.ctrl->bucket_cnt[threadIdx.x] : 0u;
    }
    __syncthreads();
}

struct ItemRef {
    uint32_t b, idx, cell, scene, pbase;
    bool valid;
};

__device__ __forceinline__ ItemRef item_ref(const WorldView& v, const ItemTables& t, uint32_t g) {
    ItemRef r;
    uint32_t b = 1;
    while (b < (uint32_t)kMaxL && g >= t.item_off[b + 1]) ++b;
    r.b = b;
    r.idx = g - t.item_off[b];
    r.valid = r.idx < t.cnt[b];
    const uint2 e = r.valid ? v.bucket_items[v.cap_off[b] + r.idx] : make_uint2(0u, 0u);
    r.cell = e.x;
    r.scene = e.y;
    r.pbase = item_position(t.pos_off, b, r.idx);
    return r;
}

// ---------------------------------------------------------------------------
// Per-particle helpers
// ---------------------------------------------------------------------------
struct PW {
    int32_t cx, cy, cz;
    float fx, fy, fz;
    float wx[3], wy[3], wz[3];
};

__device__ __forceinline__ PW particle_weights(float px, float py, float pz) {
    PW w;
    cell_frac(px, w.cx, w.fx);
    cell_frac(py, w.cy, w.fy);
    cell_frac(pz, w.cz, w.fz);
    qweights(w.fx, w.wx[0], w.wx[1], w.wx[2]);
    qweights(w.fy, w.wy[0], w.wy[1], w.wy[2]);
    qweights(w.fz, w.wz[0], w.wz[1], w.wz[2]);
    return w;
}

__device__ __forceinline__ void cell_xyz(const SceneDesc& sd, uint32_t gc, int32_t& x, int32_t& y, int32_t& z) {
    const uint32_t c = gc - sd.cell_base;
    x = (int32_t)(c % sd.X);
    y = (int32_t)((c / sd.X) % sd.Y);
    z = (int32_t)(c / (sd.X * sd.Y));
}

// encode() without the clamp, for values already known to lie in +-20000.
__device__ __forceinline__ int32_t encode_unclamped(float v) { return __float2int_rz(v * kFixed); }

// ---------------------------------------------------------------------------
// P2G_MASS (shaders.js:242-274), item-major
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kItemThreads) k_p2g_mass_items(WorldView v, const float4* __restrict__ posm,
                                                                 int32_t* __restrict__ cm) {
    __shared__ ItemTables tabs;
    load_tables(v, tabs);
    const uint32_t nitems = v.ctrl->total_items;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < nitems; g += gridDim.x * blockDim.x) {
        const ItemRef it = item_ref(v, tabs, g);
        if (!it.valid) continue;
        const SceneDesc& sd = v.scenes[it.scene];
        const int32_t X = sd.X, Y = sd.Y, Z = sd.Z;
        int32_t* scm = cm + sd.cell_base;
        int32_t ix, iy, iz;
        cell_xyz(sd, it.cell, ix, iy, iz);
        int32_t acc[27];
#pragma unroll
        for (int q = 0; q < 27; ++q) acc[q] = 0;
        uint32_t slot_n = it.b > 1 ? v.perm[it.pbase + 32u] : 0u;
        float4 p_c = posm[v.perm[it.pbase]];
        for (uint32_t k = 0; k < it.b; ++k) {
            float4 p_n = p_c;
            uint32_t slot_nn = slot_n;
            if (k + 1 < it.b) {
                p_n = posm[slot_n];
                if (k + 2 < it.b) slot_nn = v.perm[it.pbase + (k + 2) * 32u];
            }
            const float4 p = p_c;
            p_c = p_n;
            slot_n = slot_nn;
            const PW w = particle_weights(p.x, p.y, p.z);
            // weight <= 0.4219: for |mass| < 47000 encode's clamp is the identity
            const bool safe = fabsf(p.w) < 47000.0f;
            if (w.cx == ix && w.cy == iy && w.cz == iz) {
                float wxy[9];
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int i = 0; i < 3; ++i) wxy[j * 3 + i] = w.wx[i] * w.wy[j];
                if (safe) {
#pragma unroll
                    for (int kk = 0; kk < 3; ++kk)
#pragma unroll
                        for (int q = 0; q < 9; ++q) acc[kk * 9 + q] += encode_unclamped(wxy[q] * w.wz[kk] * p.w);
                } else {
#pragma unroll
                    for (int kk = 0; kk < 3; ++kk)
#pragma unroll
                        for (int q = 0; q < 9; ++q) acc[kk * 9 + q] += encode(wxy[q] * w.wz[kk] * p.w);
                }
            } else {
                // particle outside its item's cell (positions outside the grid): per-particle path
                for (int kk = 0; kk < 3; ++kk)
                    for (int j = 0; j < 3; ++j)
                        for (int i = 0; i < 3; ++i) {
                            const int32_t xx = w.cx - 1 + i, yy = w.cy - 1 + j, zz = w.cz - 1 + kk;
                            if (xx < 0 || xx >= X || yy < 0 || yy >= Y || zz < 0 || zz >= Z) continue;
                            const float ww = w.wx[i] * w.wy[j] * w.wz[kk];
                            atomicAdd(&scm[(zz * Y + yy) * X + xx], encode(ww * p.w));
                        }
            }
        }
#pragma unroll
        for (int kk = 0; kk < 3; ++kk)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const int32_t xx = ix - 1 + i, yy = iy - 1 + j, zz = iz - 1 + kk;
                    const int32_t a = acc[kk * 9 + j * 3 + i];
                    if (a != 0 && xx >= 0 && xx < X && yy >= 0 && yy < Y && zz >= 0 && zz < Z)
                        atomicAdd(&scm[(zz * Y + yy) * X + xx], a);
                }
    }
}

// ---------------------------------------------------------------------------
// Grid passes over the grid-tile list: DECODE_MASS and UPDATE_GRID (+ clear
// of the other i32 buffer).
// ---------------------------------------------------------------------------
__device__ __forceinline__ const SceneDesc* tile_cell(const WorldView& v, uint32_t t, uint32_t lid, uint32_t& c,
                                                      int32_t& x, int32_t& y, int32_t& z) {
    const uint32_t scene = v.tile_scene[t];
    if (scene == kHole) return nullptr;
    const SceneDesc& sd = v.scenes[scene];
    const uint32_t lt = t - sd.tile_base;
    const uint32_t tx = lt % sd.ntx, ty = (lt / sd.ntx) % sd.nty, tz = lt / (sd.ntx * sd.nty);
    x = (int32_t)(tx * kTileX + lid % kTileX);
    y = (int32_t)(ty * kTileY + (lid / kTileX) % kTileY);
    z = (int32_t)(tz * kTileZ + lid / (kTileX * kTileY));
    if ((uint32_t)x >= sd.X || (uint32_t)y >= sd.Y || (uint32_t)z >= sd.Z) return nullptr;
    c = sd.cell_base + local_cell(sd, x, y, z);
    return &sd;
}

__global__ void __launch_bounds__(256) k_decode_tiles(WorldView v, const int32_t* __restrict__ cm,
                                                      float* __restrict__ cmf) {
    const uint32_t total = v.ctrl->n_grid * kTileCells;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        uint32_t c;
        int32_t x, y, z;
        if (tile_cell(v, v.tile_grid_list[g / kTileCells], g % kTileCells, c, x, y, z)) cmf[c] = decode(cm[c]);
    }
}

// UPDATE_GRID for one cell with mass c > 0 (shaders.js:435-513).
__device__ __forceinline__ void update_cell(const SceneDesc& sd, const int32_t* __restrict__ cm,
                                            const int32_t* __restrict__ mv, uint32_t idx, float c, int32_t cx,
                                            int32_t cy, int32_t cz, float& vx_out, float& vy_out, float& vz_out) {
    {
        float vx = __fdiv_rn(decode(mv[3 * (size_t)idx + 0]), c);
        float vy = __fdiv_rn(decode(mv[3 * (size_t)idx + 1]), c);
        float vz = __fdiv_rn(decode(mv[3 * (size_t)idx + 2]), c);
        vy += sd.P.gravity * sd.P.dt;
        const int32_t X = sd.X, Y = sd.Y, Z = sd.Z;
        if (cx < 2 || cx > X - 3) vx = 0.0f;
        if (cy < 2 && vy < 0.0f) vy = 0.0f;
        if (cy > Y - 3 && vy > 0.0f) vy = 0.0f;
        if (cz < 2 || cz > Z - 3) vz = 0.0f;
        if (cy < 2) { vx *= 0.85f; vz *= 0.9f; }
        const uint32_t nw = wall_count_of(sd.W.count_pad[0]);
        if (nw > 0) {
            const f3 cellPos = mk(__int2float_rn(cx) + 0.5f, __int2float_rn(cy) + 0.5f, __int2float_rn(cz) + 0.5f);
            f3 wv = mk(vx, vy, vz);
            for (uint32_t wi = 0; wi < nw; ++wi) {
                const WallD w = load_wall(sd.W.walls[wi]);
                const f3 lp = wall_to_local(cellPos, w);
                if (lp.x < w.mn.x - 1.0f || lp.y < w.mn.y - 1.0f || lp.z < w.mn.z - 1.0f || lp.x > w.mx.x + 1.0f ||
                    lp.y > w.mx.y + 1.0f || lp.z > w.mx.z + 1.0f)
                    continue;
                const f3 wvel = wall_vel_at(cellPos, w);
                f3 n;
                const float sw = wall_sdf_normal(lp, w.mn, w.mx, n);
                if (sw < 0.0f) {
                    wv = wvel;
                } else if (sw < 1.0f) {
                    const f3 nn = wall_to_world_dir(n, w);
                    const f3 vrel = sub(wv, wvel);
                    const float vn = dot3(vrel, nn);
                    if (vn < 0.0f) wv = mk(wv.x - vn * nn.x, wv.y - vn * nn.y, wv.z - vn * nn.z);
                }
            }
            vx = wv.x; vy = wv.y; vz = wv.z;
        }
        vx_out = vx; vy_out = vy; vz_out = vz;
    }
}

// APPLY_HAND for one cell inside the dispatch box (shaders.js:413-432), on
// the velocity UPDATE_GRID just produced for it.
__device__ __forceinline__ void hand_push(const mpm_hand_params& H, int32_t cx, int32_t cy, int32_t cz, float& vx,
                                          float& vy, float& vz) {
    const f3 cell = mk(__int2float_rn(cx) + 0.5f, __int2float_rn(cy) + 0.5f, __int2float_rn(cz) + 0.5f);
    const f3 hp = mk(H.px, H.py, H.pz);
    const f3 dv = sub(hp, mk(H.ex, H.ey, H.ez));
    const float dl = len3(dv);
    const f3 dir = mk(__fdiv_rn(dv.x, dl), __fdiv_rn(dv.y, dl), __fdiv_rn(dv.z, dl));
    const f3 to_cell = sub(cell, hp);
    const float t0 = dot3(to_cell, dir);
    const f3 perp = mk(to_cell.x - t0 * dir.x, to_cell.y - t0 * dir.y, to_cell.z - t0 * dir.z);
    const float d = len3(perp);
    if (d >= H.radius) return;
    const float t = 1.0f - __fdiv_rn(d, H.radius);
    const float w = t * t * H.strength;
    vx += H.vx * w;
    vy += H.vy * w;
    vz += H.vz * w;
}

__global__ void __launch_bounds__(256) k_update_tiles(WorldView v, const int32_t* __restrict__ cm,
                                                      const int32_t* __restrict__ mv, float* __restrict__ mvf,
                                                      int32_t* __restrict__ cm_next, int32_t* __restrict__ mv_next) {
    const uint32_t total = v.ctrl->n_grid * kTileCells;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
        uint32_t idx;
        int32_t cx, cy, cz;
        const SceneDesc* sdp = tile_cell(v, v.tile_grid_list[g / kTileCells], g % kTileCells, idx, cx, cy, cz);
        if (!sdp) continue;
        const SceneDesc& sd = *sdp;
        cm_next[idx] = 0;
        mv_next[3 * (size_t)idx + 0] = 0; mv_next[3 * (size_t)idx + 1] = 0; mv_next[3 * (size_t)idx + 2] = 0;
        const float c = decode(cm[idx]);
        float* out = mvf + 3 * (size_t)idx;
        float vx = 0.0f, vy = 0.0f, vz = 0.0f;
        if (c > 0.0f) update_cell(sd, cm, mv, idx, c, cx, cy, cz, vx, vy, vz);
        if (cx >= sd.hand_box[0] && cx <= sd.hand_box[3] && cy >= sd.hand_box[1] && cy <= sd.hand_box[4] &&
            cz >= sd.hand_box[2] && cz <= sd.hand_box[5])
            hand_push(sd.H, cx, cy, cz, vx, vy, vz);
        out[0] = vx; out[1] = vy; out[2] = vz;
    }
}

// ---------------------------------------------------------------------------
// P2G_MOM (shaders.js:276-371), item-major
// ---------------------------------------------------------------------------
struct MomIn {
    float vx, vy, vz, m;
    float a00, a01, a02, a10, a11, a12, a20, a21, a22;
};

// Per-thread accumulator slots of k_p2g_mom_items (81 x 4 B per thread).
__shared__ int32_t g_sacc[81][kItemThreads];

// The scatter part of P2G_MOM for one particle whose density is known.
// kDirect: atomics straight into the grid at the particle's own stencil;
// otherwise the 81 encoded contributions are added into the shared slots.
// kClamp: full encode; without it the caller has bounded every value inside
// +-20000, where encode's clamp is the identity.
template <bool kDirect, bool kClamp>
__device__ __forceinline__ void mom_scatter(const PW& w, const MomIn& in, const float* s, float coef, uint32_t X,
                                            uint32_t SLICE, int32_t* mv, uint32_t baseIdx, uint32_t G) {
    const float s00 = s[0], s11 = s[1], s22 = s[2], s01 = s[3], s02 = s[4], s12 = s[5];
    const float dxs[3] = {-w.fx - 1.0f, -w.fx, 1.0f - w.fx};
    const float dys[3] = {-w.fy - 1.0f, -w.fy, 1.0f - w.fy};
    const float dzs[3] = {-w.fz - 1.0f, -w.fz, 1.0f - w.fz};
#pragma unroll 1
    for (int k = 0; k < 3; ++k) {
        const float wzk = k == 0 ? w.wz[0] : (k == 1 ? w.wz[1] : w.wz[2]);
        const float dzk = k == 0 ? dzs[0] : (k == 1 ? dzs[1] : dzs[2]);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float wyzk = w.wy[j] * wzk, dyj = dys[j];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const float ww = w.wx[i] * wyzk;
                const float dxi = dxs[i];
                const float Qx = in.a00 * dxi + in.a01 * dyj + in.a02 * dzk;
                const float Qy = in.a10 * dxi + in.a11 * dyj + in.a12 * dzk;
                const float Qz = in.a20 * dxi + in.a21 * dyj + in.a22 * dzk;
                const float fxf = coef * (s00 * dxi + s01 * dyj + s02 * dzk);
                const float fyf = coef * (s01 * dxi + s11 * dyj + s12 * dzk);
                const float fzf = coef * (s02 * dxi + s12 * dyj + s22 * dzk);
                const float vx = ww * (in.m * (in.vx + Qx) + fxf);
                const float vy = ww * (in.m * (in.vy + Qy) + fyf);
                const float vz = ww * (in.m * (in.vz + Qz) + fzf);
                const int32_t ex = kClamp ? encode(vx) : encode_unclamped(vx);
                const int32_t ey = kClamp ? encode(vy) : encode_unclamped(vy);
                const int32_t ez = kClamp ? encode(vz) : encode_unclamped(vz);
                if (kDirect) {
                    const uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)j * X + (uint32_t)i;
                    if (cidx < G) {
                        atomicAdd(mv + 3ull * cidx + 0, ex);
                        atomicAdd(mv + 3ull * cidx + 1, ey);
                        atomicAdd(mv + 3ull * cidx + 2, ez);
                    }
                } else {
                    const int q = (k * 9 + j * 3 + i) * 3;
                    atomicAdd(&g_sacc[q + 0][threadIdx.x], ex);
                    atomicAdd(&g_sacc[q + 1][threadIdx.x], ey);
                    atomicAdd(&g_sacc[q + 2][threadIdx.x], ez);
                }
            }
        }
    }
}

__global__ void __launch_bounds__(kItemThreads, MPM_MOM_LB) k_p2g_mom_items(WorldView v,
                                                                             const float4* __restrict__ posm,
                                                                             const float4* __restrict__ velid,
                                                                             const float* __restrict__ aff,
                                                                             const float* __restrict__ cmf,
                                                                             int32_t* __restrict__ mv,
                                                                             float* __restrict__ dens) {
    __shared__ ItemTables tabs;
    load_tables(v, tabs);
    const uint32_t nitems = v.ctrl->total_items;
    const size_t plane = v.npos;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < nitems; g += gridDim.x * blockDim.x) {
        const ItemRef it = item_ref(v, tabs, g);
        if (!it.valid) continue;
        const SceneDesc& sd = v.scenes[it.scene];
        const uint32_t X = sd.X, SLICE = sd.X * sd.Y, G = sd.G;
        const float* scmf = cmf + sd.cell_base;
        int32_t* smv = mv + 3ull * sd.cell_base;
        int32_t ix, iy, iz;
        cell_xyz(sd, it.cell, ix, iy, iz);
        const uint32_t ibase = (uint32_t)(((iz - 1) * (int32_t)sd.Y + (iy - 1)) * (int32_t)X + (ix - 1));
        float m27[27];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const uint32_t cidx = ibase + (uint32_t)k * SLICE + (uint32_t)j * X + (uint32_t)i;
                    m27[k * 9 + j * 3 + i] = cidx < G ? scmf[cidx] : 0.0f;
                }
#pragma unroll
        for (int q = 0; q < 81; ++q) g_sacc[q][threadIdx.x] = 0;
        const float rest = sd.P.rest_density, stiff = sd.P.stiffness, eos = sd.P.eos_power, visc = sd.P.viscosity;
        const float dt = sd.P.dt;
        // software pipeline: the next particle's permutation entry and record are
        // loaded while the current one is processed
        uint32_t slot_n = it.b > 1 ? v.perm[it.pbase + 32u] : 0u;
        float4 p_c, v_c;
        float a_c[9];
        {
            const uint32_t slot = v.perm[it.pbase];
            p_c = posm[slot];
            v_c = velid[slot];
#pragma unroll
            for (int e = 0; e < 9; ++e) a_c[e] = aff[e * plane + slot];
        }
        for (uint32_t kk = 0; kk < it.b; ++kk) {
            const uint32_t pos = it.pbase + kk * 32u;
            float4 p_n = p_c, v_n = v_c;
            float a_n[9];
#pragma unroll
            for (int e = 0; e < 9; ++e) a_n[e] = a_c[e];
            uint32_t slot_nn = slot_n;
            if (kk + 1 < it.b) {
                p_n = posm[slot_n];
                v_n = velid[slot_n];
#pragma unroll
                for (int e = 0; e < 9; ++e) a_n[e] = aff[e * plane + slot_n];
                if (kk + 2 < it.b) slot_nn = v.perm[pos + 64u];
            }
            const float4 p = p_c;
            const MomIn in{v_c.x, v_c.y, v_c.z, p.w, a_c[0], a_c[1], a_c[2], a_c[3], a_c[4], a_c[5],
                           a_c[6], a_c[7], a_c[8]};
            p_c = p_n;
            v_c = v_n;
#pragma unroll
            for (int e = 0; e < 9; ++e) a_c[e] = a_n[e];
            slot_n = slot_nn;
            const PW w = particle_weights(p.x, p.y, p.z);
            const bool same = (w.cx == ix && w.cy == iy && w.cz == iz);
            const uint32_t baseIdx = (uint32_t)(((w.cz - 1) * (int32_t)sd.Y + (w.cy - 1)) * (int32_t)X + (w.cx - 1));
            float density = 0.0f;
            if (same) {
#pragma unroll
                for (int k = 0; k < 3; ++k)
#pragma unroll
                    for (int jj = 0; jj < 3; ++jj)
#pragma unroll
                        for (int i = 0; i < 3; ++i) density += w.wx[i] * w.wy[jj] * w.wz[k] * m27[k * 9 + jj * 3 + i];
            } else {
                for (int k = 0; k < 3; ++k)
                    for (int jj = 0; jj < 3; ++jj)
                        for (int i = 0; i < 3; ++i) {
                            const uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)jj * X + (uint32_t)i;
                            const float cmass = cidx < G ? scmf[cidx] : 0.0f;
                            density += w.wx[i] * w.wy[jj] * w.wz[k] * cmass;
                        }
            }
            dens[pos] = density;
            if (density <= 1e-8f) continue;
            // stress (shaders.js:325-338)
            const float vol = __fdiv_rn(in.m, fmaxf(density, rest * 0.15f));
            float pressure = stiff * (eos_pow(__fdiv_rn(density, rest), eos) - 1.0f);
            const float pFloor = density > rest * kCohesionGate ? kCohesionPressure : 0.0f;
            pressure = fmaxf(pressure, pFloor);
            float s[6];
            s[0] = -pressure + visc * (in.a00 + in.a00);
            s[1] = -pressure + visc * (in.a11 + in.a11);
            s[2] = -pressure + visc * (in.a22 + in.a22);
            s[3] = visc * (in.a01 + in.a10);
            s[4] = visc * (in.a02 + in.a20);
            s[5] = visc * (in.a12 + in.a21);
            const float coef = -vol * 4.0f * dt;
            // |value| <= 0.4219 * (|m| (|v| + 1.5 |A row|_1) + |coef| 1.5 |S row|_1): when that bound
            // is well inside +-20000 encode's clamp cannot change any value (NaN/Inf fail the test).
            const float am = fabsf(in.m), ac = fabsf(coef);
            const float bx = am * (fabsf(in.vx) + 1.5f * (fabsf(in.a00) + fabsf(in.a01) + fabsf(in.a02))) +
                             ac * 1.5f * (fabsf(s[0]) + fabsf(s[3]) + fabsf(s[4]));
            const float by = am * (fabsf(in.vy) + 1.5f * (fabsf(in.a10) + fabsf(in.a11) + fabsf(in.a12))) +
                             ac * 1.5f * (fabsf(s[3]) + fabsf(s[1]) + fabsf(s[5]));
            const float bz = am * (fabsf(in.vz) + 1.5f * (fabsf(in.a20) + fabsf(in.a21) + fabsf(in.a22))) +
                             ac * 1.5f * (fabsf(s[4]) + fabsf(s[5]) + fabsf(s[2]));
            const bool safe = fmaxf(bx, fmaxf(by, bz)) * 0.4222f < 19000.0f;
            if (same) {
                if (safe) mom_scatter<false, false>(w, in, s, coef, X, SLICE, smv, baseIdx, G);
                else mom_scatter<false, true>(w, in, s, coef, X, SLICE, smv, baseIdx, G);
            } else {
                mom_scatter<true, true>(w, in, s, coef, X, SLICE, smv, baseIdx, G);
            }
        }
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int jj = 0; jj < 3; ++jj)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const uint32_t cidx = ibase + (uint32_t)k * SLICE + (uint32_t)jj * X + (uint32_t)i;
                    const int q = (k * 9 + jj * 3 + i) * 3;
                    const int32_t a0 = g_sacc[q + 0][threadIdx.x], a1 = g_sacc[q + 1][threadIdx.x],
                                  a2 = g_sacc[q + 2][threadIdx.x];
                    if (cidx < G) {
                        if (a0) atomicAdd(smv + 3ull * cidx + 0, a0);
                        if (a1) atomicAdd(smv + 3ull * cidx + 1, a1);
                        if (a2) atomicAdd(smv + 3ull * cidx + 2, a2);
                    }
                }
    }
}

// ---------------------------------------------------------------------------
// G2P (shaders.js:579-705), item-major, + binning of the new positions and
// the diffuse spawn decision (shaders.js:800-855).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool estimate_normal_f(const float* __restrict__ cmf, const SceneDesc& sd, float px,
                                                  float py, float pz, f3& n) {
    const int32_t X = sd.X, Y = sd.Y, Z = sd.Z;
    const int32_t gx = __float2int_rz(floorf(px)), gy = __float2int_rz(floorf(py)), gz = __float2int_rz(floorf(pz));
    if (gx < 1 || gx >= X - 1 || gy < 1 || gy >= Y - 1 || gz < 1 || gz >= Z - 1) return false;
    const uint32_t idxL = (uint32_t)((gz * Y + gy) * X + (gx - 1));
    const uint32_t idxR = (uint32_t)((gz * Y + gy) * X + (gx + 1));
    const uint32_t idxD = (uint32_t)((gz * Y + (gy - 1)) * X + gx);
    const uint32_t idxU = (uint32_t)((gz * Y + (gy + 1)) * X + gx);
    const uint32_t idxB = (uint32_t)(((gz - 1) * Y + gy) * X + gx);
    const uint32_t idxF = (uint32_t)(((gz + 1) * Y + gy) * X + gx);
    const f3 vv = mk(cmf[idxL] - cmf[idxR], cmf[idxD] - cmf[idxU], cmf[idxB] - cmf[idxF]);
    const float len = len3(vv);
    if (len < 1e-6f) return false;
    n = mk(__fdiv_rn(vv.x, len), __fdiv_rn(vv.y, len), __fdiv_rn(vv.z, len));
    return true;
}

// Spawn decision + staging (shaders.js:800-855), out of line: most particles
// fail the density test that the caller applies first.
__device__ __noinline__ void spawn_eval(uint32_t id, f3 np, f3 nv, float m, float density, const SceneDesc& sd,
                                        const float* __restrict__ cmf, const DiffuseView& dv) {
    const mpm_gen_params& gen = *dv.gen;
    const f3 vel = nv;
    const float speed2 = dot3(vel, vel);
    const float speed = __fsqrt_rn(speed2);
    const float ke = 0.5f * m * speed2;
    const float rest = sd.P.rest_density;
    float pressure = sd.P.stiffness * (eos_pow(__fdiv_rn(density, rest), sd.P.eos_power) - 1.0f);
    const float pFloor = density > rest * kCohesionGate ? kCohesionPressure : 0.0f;
    pressure = fmaxf(pressure, pFloor);
    const float trappedAir = fmaxf(0.0f, pressure - gen.pressure_threshold);
    f3 nrm;
    const bool ok = estimate_normal_f(cmf, sd, np.x, np.y, np.z, nrm);
    float waveCrest = 0.0f;
    if (speed > 1e-4f && ok) {
        const f3 vs = mk(__fdiv_rn(vel.x, speed), __fdiv_rn(vel.y, speed), __fdiv_rn(vel.z, speed));
        const float dotVal = dot3(vs, nrm);
        if (dotVal > gen.crest_dot_threshold) waveCrest = dotVal * speed;
    }
    const float score = ke + trappedAir * 2.0f + waveCrest * 1.5f;
    if (score < gen.ke_threshold) return;
    const uint32_t randSeed = id * 9781u + gen.seed;
    const float spawnChance = fminf(1.0f, (score - gen.ke_threshold) * gen.spawn_rate_k * sd.P.dt);
    if (diffuse_rand(randSeed) > spawnChance) return;
    const float jitter = 0.3f;
    const float jx = (diffuse_rand(randSeed + 1u) - 0.5f) * jitter * speed;
    const float jy = (diffuse_rand(randSeed + 2u) - 0.5f) * jitter * speed;
    const float jz = (diffuse_rand(randSeed + 3u) - 0.5f) * jitter * speed;
    uint32_t ptype = MPM_DIFFUSE_FOAM;
    if (density < gen.density_spray_max) ptype = MPM_DIFFUSE_SPRAY;
    const float lifetime =
        ptype == MPM_DIFFUSE_FOAM ? gen.lifetime_foam * fminf(1.0f, __fdiv_rn(score, gen.ke_threshold)) : 999.0f;
    mpm_diffuse_particle r;
    r.pos[0] = np.x; r.pos[1] = np.y; r.pos[2] = np.z; r.pos[3] = 0.0f;
    r.vel[0] = vel.x + jx; r.vel[1] = vel.y + jy; r.vel[2] = vel.z + jz; r.vel[3] = 0.0f;
    r.ptype = ptype; r.alive = 1u; r.lifetime = lifetime; r._pad = 0.0f;
    dv.staging[id] = r;
    atomicOr(&dv.spawn_bits[id >> 5], 1u << (id & 31u));
}

// G2P for one particle given its gathered grid velocity (shaders.js:636-700).
__device__ __forceinline__ void g2p_finish(const float4 q, float gvx, float gvy, float gvz, const mpm_params& P,
                                           const mpm_wall_params& W, f3& np, f3& nv) {
    const float dt = P.dt, lk = P.lookahead_k, ws = P.wall_stiffness;
    np = mk(q.x + dt * gvx, q.y + dt * gvy, q.z + dt * gvz);
    nv = mk(gvx, gvy, gvz);
    const float floorZoneY = P.hard_min + kFloorBand;
    const float xny = np.y + nv.y * dt * lk;
    if (xny < floorZoneY) {
        const float distBelowFloor = floorZoneY - xny;
        const float blend = wclamp(__fdiv_rn(distBelowFloor, kFloorBand), 0.0f, 1.0f);
        nv.y += ws * blend * distBelowFloor;
    }
    const uint32_t nw = wall_count_of(W.count_pad[0]);
    for (uint32_t wi = 0; wi < nw; ++wi) {
        const WallD w = load_wall(W.walls[wi]);
        const f3 xnw = mk(np.x + nv.x * dt * lk, np.y + nv.y * dt * lk, np.z + nv.z * dt * lk);
        const f3 lxn = wall_to_local(xnw, w);
        if (inside_open(lxn, w.mn, w.mx)) {
            f3 nl;
            const float sw = wall_sdf_normal(lxn, w.mn, w.mx, nl);
            const float dist = -sw;
            const float blend = wclamp(__fdiv_rn(dist, P.wall_min), 0.0f, 1.0f);
            const f3 nwd = wall_to_world_dir(nl, w);
            const float sc = ws * blend * dist;
            nv = mk(nv.x + nwd.x * sc, nv.y + nwd.y * sc, nv.z + nwd.z * sc);
        }
        const f3 lnp = wall_to_local(np, w);
        if (inside_open(lnp, w.mn, w.mx)) {
            f3 nl;
            const float sw = wall_sdf_normal(lnp, w.mn, w.mx, nl);
            const f3 nn = wall_to_world_dir(nl, w);
            const float mm = fmaxf(sw, -0.5f);
            np = mk(np.x - nn.x * mm, np.y - nn.y * mm, np.z - nn.z * mm);
            const float vn = dot3(sub(nv, wall_vel_at(np, w)), nn);
            if (vn < 0.0f) nv = mk(nv.x - vn * nn.x, nv.y - vn * nn.y, nv.z - vn * nn.z);
        }
    }
    const float hmin = P.hard_min;
    if (np.x < hmin) { np.x = hmin; nv.x = 0.0f; }
    if (np.x > P.hard_max_x) { np.x = P.hard_max_x; nv.x = 0.0f; }
    if (np.y < hmin) { np.y = hmin; nv.y = 0.0f; }
    if (np.y > P.hard_max_y) { np.y = P.hard_max_y; nv.y = 0.0f; }
    if (np.z < hmin) { np.z = hmin; nv.z = 0.0f; }
    if (np.z > P.hard_max_z) { np.z = P.hard_max_z; nv.z = 0.0f; }
}

// G2P gather for a particle outside its item's cell (positions outside the
// grid): the reference's linear stencil index with a bounds guard.
__device__ __noinline__ void g2p_gather_direct(const PW& w, const float4 q, const float* __restrict__ mvf, uint32_t X,
                                               uint32_t Y, uint32_t G, float& gvx, float& gvy, float& gvz,
                                               float* B) {
    const uint32_t SLICE = X * Y;
    const int32_t bx = w.cx - 1, by = w.cy - 1, bz = w.cz - 1;
    const uint32_t baseIdx = (uint32_t)((bz * (int32_t)Y + by) * (int32_t)X + bx);
    for (int k = 0; k < 3; ++k) {
        const float wzk = w.wz[k];
        const float dzk = __int2float_rn(bz + k) - q.z + 0.5f;
        for (int jj = 0; jj < 3; ++jj) {
            const float wyzk = w.wy[jj] * wzk;
            const float dyj = __int2float_rn(by + jj) - q.y + 0.5f;
            for (int i = 0; i < 3; ++i) {
                const float ww = w.wx[i] * wyzk;
                const float dxi = __int2float_rn(bx + i) - q.x + 0.5f;
                const uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)jj * X + (uint32_t)i;
                float cvx = 0.0f, cvy = 0.0f, cvz = 0.0f;
                if (cidx < G) {
                    const float* c = mvf + 3ull * cidx;
                    cvx = c[0]; cvy = c[1]; cvz = c[2];
                }
                const float wvx = ww * cvx, wvy = ww * cvy, wvz = ww * cvz;
                gvx += wvx; gvy += wvy; gvz += wvz;
                B[0] += wvx * dxi; B[1] += wvx * dyj; B[2] += wvx * dzk;
                B[3] += wvy * dxi; B[4] += wvy * dyj; B[5] += wvy * dzk;
                B[6] += wvz * dxi; B[7] += wvz * dyj; B[8] += wvz * dzk;
            }
        }
    }
}

__global__ void __launch_bounds__(kItemThreads, MPM_G2P_LB) k_g2p_items(WorldView v,
                                                                         const float4* __restrict__ posm,
                                                                         const float4* __restrict__ velid,
                                                                         const float* __restrict__ mvf,
                                                                         const float* __restrict__ cmf,
                                                                         float4* __restrict__ posm_out,
                                                                         float4* __restrict__ velid_out,
                                                                         float* __restrict__ aff_out, DiffuseView dv) {
    __shared__ ItemTables tabs;
    load_tables(v, tabs);
    const uint32_t nitems = v.ctrl->total_items;
    const size_t plane = v.npos;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < nitems; g += gridDim.x * blockDim.x) {
        const ItemRef it = item_ref(v, tabs, g);
        if (!it.valid) {
            // padding lane: mark its positions as holes for the next binning and the export
            for (uint32_t kk = 0; kk < it.b; ++kk) {
                const uint32_t pos = it.pbase + kk * 32u;
                if (pos < v.npos) {
                    v.key[pos] = kHole;
                    velid_out[pos] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(kHole));
                }
            }
            continue;
        }
        const SceneDesc& sd = v.scenes[it.scene];
        const uint32_t X = sd.X, SLICE = sd.X * sd.Y, G = sd.G;
        const float* smvf = mvf + 3ull * sd.cell_base;
        int32_t ix, iy, iz;
        cell_xyz(sd, it.cell, ix, iy, iz);
        const uint32_t item_tile = tile_of(sd, ix, iy, iz);
        mark_occupied(v, item_tile);
        const uint32_t ibase = (uint32_t)(((iz - 1) * (int32_t)sd.Y + (iy - 1)) * (int32_t)X + (ix - 1));
        float cv[81];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const uint32_t cidx = ibase + (uint32_t)k * SLICE + (uint32_t)j * X + (uint32_t)i;
                    const int q = (k * 9 + j * 3 + i) * 3;
                    if (cidx < G) {
                        const float* c = smvf + 3ull * cidx;
                        cv[q + 0] = c[0]; cv[q + 1] = c[1]; cv[q + 2] = c[2];
                    } else {
                        cv[q + 0] = 0.0f; cv[q + 1] = 0.0f; cv[q + 2] = 0.0f;
                    }
                }
        const bool spawn_scene = dv.enabled && it.scene == dv.scene;
        uint32_t slot_n = it.b > 1 ? v.perm[it.pbase + 32u] : 0u;
        float4 q_c, vi_c;
        {
            const uint32_t slot = v.perm[it.pbase];
            q_c = posm[slot];
            vi_c = velid[slot];
        }
        for (uint32_t kk = 0; kk < it.b; ++kk) {
            const uint32_t pos = it.pbase + kk * 32u;
            float4 q_n = q_c, vi_n = vi_c;
            uint32_t slot_nn = slot_n;
            if (kk + 1 < it.b) {
                q_n = posm[slot_n];
                vi_n = velid[slot_n];
                if (kk + 2 < it.b) slot_nn = v.perm[pos + 64u];
            }
            const float4 q = q_c;
            const float4 vi = vi_c;
            q_c = q_n;
            vi_c = vi_n;
            slot_n = slot_nn;
            const PW w = particle_weights(q.x, q.y, q.z);
            const bool same = (w.cx == ix && w.cy == iy && w.cz == iz);
            float gvx = 0.0f, gvy = 0.0f, gvz = 0.0f;
            float B[9] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
            if (same) {
                const int32_t bx = w.cx - 1, by = w.cy - 1, bz = w.cz - 1;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float wzk = w.wz[k];
                    const float dzk = __int2float_rn(bz + k) - q.z + 0.5f;
#pragma unroll
                    for (int jj = 0; jj < 3; ++jj) {
                        const float wyzk = w.wy[jj] * wzk;
                        const float dyj = __int2float_rn(by + jj) - q.y + 0.5f;
#pragma unroll
                        for (int i = 0; i < 3; ++i) {
                            const float ww = w.wx[i] * wyzk;
                            const float dxi = __int2float_rn(bx + i) - q.x + 0.5f;
                            const int qq = (k * 9 + jj * 3 + i) * 3;
                            const float wvx = ww * cv[qq + 0], wvy = ww * cv[qq + 1], wvz = ww * cv[qq + 2];
                            gvx += wvx; gvy += wvy; gvz += wvz;
                            B[0] += wvx * dxi; B[1] += wvx * dyj; B[2] += wvx * dzk;
                            B[3] += wvy * dxi; B[4] += wvy * dyj; B[5] += wvy * dzk;
                            B[6] += wvz * dxi; B[7] += wvz * dyj; B[8] += wvz * dzk;
                        }
                    }
                }
            } else {
                g2p_gather_direct(w, q, smvf, X, sd.Y, G, gvx, gvy, gvz, B);
            }
#pragma unroll
            for (int e = 0; e < 9; ++e) aff_out[e * plane + pos] = B[e] * 4.0f;
            f3 np, nv;
            g2p_finish(q, gvx, gvy, gvz, sd.P, sd.W, np, nv);
            posm_out[pos] = make_float4(np.x, np.y, np.z, q.w);
            velid_out[pos] = make_float4(nv.x, nv.y, nv.z, vi.w);
            // binning of the new position
            int32_t cx, cy, cz;
            bin_cell(sd, np.x, np.y, np.z, cx, cy, cz);
            const uint32_t c = sd.cell_base + local_cell(sd, cx, cy, cz);
            v.key[pos] = c;
            if (c != it.cell) {
                const uint32_t t = tile_of(sd, cx, cy, cz);
                if (t != item_tile) mark_occupied(v, t);
            }
            if (spawn_scene) {
                const uint32_t id = __float_as_uint(vi.w) - sd.id_base;
                const float density = v.dens[pos];
                // spawn_record's first test (shaders.js:806), checked inline
                if (id < sd.n && density > 0.0f && density <= dv.gen->density_bubble_min)
                    spawn_eval(id, np, nv, q.w, density, sd, cmf + sd.cell_base, dv);
            }
        }
    }
}

inline uint32_t cdiv(uint64_t a, uint32_t b) { return (uint32_t)((a + b - 1) / b); }

}  // namespace

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
// Capacities derived from the requested particle / cell / scene counts.
static void world_plan(World& w, uint32_t particle_cap, uint64_t cell_cap, uint32_t scene_cap) {
    w.pcap = particle_cap;
    w.npos = particle_cap + kPosSlack;
    w.cell_cap = cell_cap;
    // tiles: a scene pads its grid to whole 16x8x8 tiles; for edges >= 32 cells the padding is
    // below 3x, and scenes of fewer than 64 tiles fit in the per-scene slack
    w.tile_cap = (uint32_t)(3 * (cell_cap / kTileCells)) + 64u * scene_cap + 64u;
    w.id_cap = particle_cap;
    w.scene_cap = scene_cap;
    uint32_t off = 0;
    w.cap_off[0] = 0;
    for (int b = 1; b <= kMaxL; ++b) {
        w.cap_off[b] = off;
        off += w.npos / b + 1;
    }
    w.cap_off[kMaxL + 1] = off;
}

// Every device array of a world with its size (one list for allocation,
// release and the footprint).
template <class F> static void world_arrays(World& w, F&& f) {
    const size_t P = w.npos, C = w.cell_cap ? w.cell_cap : 1, T = w.tile_cap;
    for (int b = 0; b < 2; ++b) {
        f(w.posm[b], P * 16);
        f(w.velid[b], P * 16);
        f(w.aff[b], P * 36);
        f(w.grid_i32[b], C * 16);
    }
    f(w.dens, P * 4);
    f(w.cell_count, (C + 1) * 4);
    f(w.cell_info, C * 16);
    f(w.bucket_items, (size_t)w.cap_off[kMaxL + 1] * 8);
    f(w.key, P * 4);
    f(w.rank, P * 4);
    f(w.perm, P * 4);
    f(w.tile_flags, T * 4);
    f(w.tile_occ, T * 4);
    f(w.tile_hist, (size_t)kMaxL * T * 4);
    f(w.tile_base, (size_t)kMaxL * T * 4);
    f(w.tile_chunk, (size_t)kMaxL * ((T + 1023) / 1024 + 1) * 4);
    f(w.tile_occ_list, T * 4);
    f(w.tile_grid_list, T * 4);
    f(w.tile_scene, T * 4);
    f(w.ctrl, sizeof(Ctrl));
    f(w.cmf, C * 4);
    f(w.mvf, C * 12);
    f(w.d_scenes, (size_t)w.scene_cap * sizeof(SceneDesc));
}

uint64_t world_footprint(uint32_t particle_cap, uint64_t cell_cap, uint32_t scene_cap) {
    World w;
    world_plan(w, particle_cap, cell_cap, scene_cap);
    uint64_t total = 0;
    world_arrays(w, [&](auto*& p, size_t bytes) {
        (void)p;
        total += (bytes + 511) & ~(uint64_t)511;   // allocation granularity
    });
    return total;
}

cudaError_t world_alloc(World& w, int device, cudaStream_t stream, uint32_t particle_cap, uint64_t cell_cap,
                        uint32_t scene_cap) {
    w.device = device;
    w.stream = stream;
    world_plan(w, particle_cap, cell_cap, scene_cap);
    w.cells.reset(cell_cap);
    w.tiles.reset(w.tile_cap);
    w.ids.reset(particle_cap ? particle_cap : 1);
    w.scenes.assign(scene_cap, SceneRec());
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    w.sms = (uint32_t)sms;
    w.item_blocks = (uint32_t)sms * 8;
    w.grid_blocks = (uint32_t)sms * 8;
    w.bin_blocks = (uint32_t)sms * 2;
    w.pos_blocks = std::min<uint32_t>(cdiv(w.npos, 256), (uint32_t)sms * 16);
    const size_t P = w.npos, C = cell_cap ? cell_cap : 1, T = w.tile_cap;
    cudaError_t e = cudaSuccess;
    w.device_bytes = 0;
    world_arrays(w, [&](auto*& p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc((void**)&p, bytes ? bytes : 16);
        if (e == cudaSuccess) w.device_bytes += bytes;
    });
    if (e != cudaSuccess) return e;
    w.h_scenes.assign(scene_cap, SceneDesc{});
    w.h_tile_scene.assign(T, kHole);
    // zero everything the sparse passes rely on being zero
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) e = cudaMemsetAsync(w.grid_i32[b], 0, C * 16, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.cmf, 0, C * 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.mvf, 0, C * 12, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.cell_count, 0, (C + 1) * 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.tile_flags, 0, T * 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.tile_occ, 0, T * 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.dens, 0, P * 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.ctrl, 0, sizeof(Ctrl), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.key, 0xFF, P * 4, stream);
    // every permutation entry always names a valid position, even if a bug left one unwritten
    if (e == cudaSuccess) e = cudaMemsetAsync(w.perm, 0, P * 4, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(w.tile_scene, w.h_tile_scene.data(), T * 4, cudaMemcpyHostToDevice,
                                              stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    w.cm_current = w.grid_i32[0];
    return e;
}

void world_free(World& w) {
    if (w.stream) cudaStreamSynchronize(w.stream);
    for (int b = 0; b < 2; ++b)
        if (w.graph[b]) cudaGraphExecDestroy(w.graph[b]);
    world_arrays(w, [](auto*& p, size_t) {
        if (p) cudaFree((void*)p);
        p = nullptr;
    });
    w = World();
}

void world_set_launch_shape(World& w, uint32_t item_blocks, uint32_t grid_blocks) {
    if (item_blocks == w.item_blocks && grid_blocks == w.grid_blocks) return;
    w.item_blocks = item_blocks;
    w.grid_blocks = grid_blocks;
    w.generation++;   // captured graphs hold the old shape
}

static void fill_desc(World& w, int slot) {
    const SceneRec& r = w.scenes[slot];
    SceneDesc& d = w.h_scenes[slot];
    std::memset(&d, 0, sizeof d);
    d.X = r.X; d.Y = r.Y; d.Z = r.Z; d.G = r.G;
    d.cell_base = r.cell_base; d.tile_base = r.tile_base;
    d.ntx = cdiv(r.X, kTileX); d.nty = cdiv(r.Y, kTileY); d.ntz = cdiv(r.Z, kTileZ);
    d.id_base = r.id_base; d.n = r.n; d.flags = r.live ? 1u : 0u;
    for (int i = 0; i < 6; ++i) d.hand_box[i] = r.hand_box[i];
    d.P = r.P;
    d.W = r.W;
    d.H = r.H;
}

cudaError_t world_upload_table(World& w) {
    if (!w.table_dirty) return cudaSuccess;
    int hi = 0;
    for (int i = 0; i < (int)w.scene_cap; ++i)
        if (w.scenes[i].live) hi = i + 1;
    for (int i = 0; i < hi; ++i) fill_desc(w, i);
    cudaError_t e = cudaSuccess;
    // pageable source: the copy is staged before the call returns, so the host
    // table can change again right away without racing the queued copy
    if (hi) e = cudaMemcpyAsync(w.d_scenes, w.h_scenes.data(), (size_t)hi * sizeof(SceneDesc),
                                cudaMemcpyHostToDevice, w.stream);
    if (e == cudaSuccess) w.table_dirty = false;
    return e;
}

void world_set_uniforms(World& w, int slot, const mpm_params& P, const mpm_wall_params& W,
                        const mpm_hand_params* H, int hand_active, const int32_t* dims) {
    SceneRec& r = w.scenes[slot];
    const SceneRec before = r;
    r.P = P;
    r.P.particle_num = r.n;
    r.W = W;
    // APPLY_HAND runs iff active with a non-empty dispatch box and is_on; it may
    // write the cells of its 4x4x4-rounded dispatch box clipped to bbox_max.
    const bool on = H && hand_active && dims && dims[0] > 0 && dims[1] > 0 && dims[2] > 0 && H->is_on != 0u;
    if (on) {
        r.H = *H;
        r.hand_box[0] = H->bbox_min_x;
        r.hand_box[1] = H->bbox_min_y;
        r.hand_box[2] = H->bbox_min_z;
        r.hand_box[3] = std::min(H->bbox_min_x + (dims[0] + 3) / 4 * 4 - 1, H->bbox_max_x);
        r.hand_box[4] = std::min(H->bbox_min_y + (dims[1] + 3) / 4 * 4 - 1, H->bbox_max_y);
        r.hand_box[5] = std::min(H->bbox_min_z + (dims[2] + 3) / 4 * 4 - 1, H->bbox_max_z);
    } else {
        r.H = mpm_hand_params{};
        r.hand_box[0] = r.hand_box[1] = r.hand_box[2] = 1;
        r.hand_box[3] = r.hand_box[4] = r.hand_box[5] = 0;
    }
    if (std::memcmp(&before.P, &r.P, sizeof r.P) || std::memcmp(&before.W, &r.W, sizeof r.W) ||
        std::memcmp(&before.H, &r.H, sizeof r.H) || std::memcmp(before.hand_box, r.hand_box, sizeof r.hand_box))
        w.table_dirty = true;
}

cudaError_t world_add_scene(World& w, uint32_t X, uint32_t Y, uint32_t Z, const mpm_params& P,
                            const mpm_wall_params& W, const float4* pos, const float4* vel, const float* aff,
                            const float* mass, uint32_t n, int* slot_out) {
    int slot = -1;
    for (int i = 0; i < (int)w.scene_cap; ++i)
        if (!w.scenes[i].live) { slot = i; break; }
    if (slot < 0) return cudaErrorMemoryAllocation;
    if ((uint64_t)w.n_total + n > w.pcap) return cudaErrorMemoryAllocation;
    // the new particles go at the host-side bound of the layout end (holes of
    // removed scenes stay until the next substep compacts them away)
    const uint32_t h_total = w.pos_bound;
    if ((uint64_t)h_total + n > w.npos) return cudaErrorNotReady;
    cudaError_t e = cudaSuccess;
    const uint64_t G = (uint64_t)X * Y * Z;
    const uint32_t nt = cdiv(X, kTileX) * cdiv(Y, kTileY) * cdiv(Z, kTileZ);
    uint64_t cb, tb, ib;
    if (!w.cells.alloc(G, cb)) return cudaErrorMemoryAllocation;
    if (!w.tiles.alloc(nt, tb)) { w.cells.release(cb, G); return cudaErrorMemoryAllocation; }
    if (!w.ids.alloc(n ? n : 1, ib)) {
        w.cells.release(cb, G);
        w.tiles.release(tb, nt);
        return cudaErrorMemoryAllocation;
    }
    SceneRec& r = w.scenes[slot];
    r = SceneRec();
    r.live = true;
    r.X = X; r.Y = Y; r.Z = Z; r.G = (uint32_t)G;
    r.cell_base = (uint32_t)cb; r.tile_base = (uint32_t)tb; r.ntiles = nt;
    r.id_base = (uint32_t)ib; r.n = n; r.id_cap = n ? n : 1;
    world_set_uniforms(w, slot, P, W, nullptr, 0, nullptr);
    w.generation++;
    for (uint32_t t = 0; t < nt; ++t) w.h_tile_scene[tb + t] = (uint32_t)slot;
    e = cudaMemcpyAsync(w.tile_scene + tb, w.h_tile_scene.data() + tb, (size_t)nt * 4, cudaMemcpyHostToDevice,
                        w.stream);
    if (e == cudaSuccess) e = world_upload_table(w);
    if (e != cudaSuccess) return e;
    if (n) {
        const WorldView v = w.view();
        k_extend<<<std::max(1u, std::min<uint32_t>(cdiv(h_total, 256), w.pos_blocks)), 256, 0, w.stream>>>(v, h_total);
        k_import<<<cdiv(n, 256), 256, 0, w.stream>>>(v, (uint32_t)slot, h_total, pos, vel, aff, mass,
                                                     w.posm[w.cur], w.velid[w.cur], w.aff[w.cur], n);
        k_set_total<<<1, 1, 0, w.stream>>>(w.ctrl, h_total + n);
        w.launches += 3;
        e = cudaGetLastError();
        w.pos_bound = h_total + n;
    }
    w.n_total += n;
    *slot_out = slot;
    return e;
}

void world_scene_grid(const World& w, int slot, int32_t** cm, int32_t** mv, float** cmf, float** mvf) {
    const SceneRec& r = w.scenes[slot];
    if (cm) *cm = w.cm_current + r.cell_base;
    if (mv) *mv = w.cm_current + w.cell_cap + 3ull * r.cell_base;
    if (cmf) *cmf = w.cmf + r.cell_base;
    if (mvf) *mvf = w.mvf + 3ull * r.cell_base;
}

cudaError_t world_remove_scene(World& w, int slot) {
    if (slot < 0 || slot >= (int)w.scene_cap || !w.scenes[slot].live) return cudaErrorInvalidValue;
    SceneRec& r = w.scenes[slot];
    const WorldView v = w.view();
    if (r.n) {
        k_remove<<<w.pos_blocks, 256, 0, w.stream>>>(v, w.velid[w.cur], r.id_base, r.n);
        w.launches++;
    }
    // zero the scene's grid region (both i32 buffers, decoded mirrors) and free its ranges
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        e = cudaMemsetAsync(w.grid_i32[b] + r.cell_base, 0, (size_t)r.G * 4, w.stream);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(w.grid_i32[b] + w.cell_cap + 3ull * r.cell_base, 0, (size_t)r.G * 12, w.stream);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(w.cmf + r.cell_base, 0, (size_t)r.G * 4, w.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.mvf + 3ull * r.cell_base, 0, (size_t)r.G * 12, w.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.tile_flags + r.tile_base, 0, (size_t)r.ntiles * 4, w.stream);
    for (uint32_t t = 0; t < r.ntiles; ++t) w.h_tile_scene[r.tile_base + t] = kHole;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(w.tile_scene + r.tile_base, w.h_tile_scene.data() + r.tile_base, (size_t)r.ntiles * 4,
                            cudaMemcpyHostToDevice, w.stream);
    w.cells.release(r.cell_base, r.G);
    w.tiles.release(r.tile_base, r.ntiles);
    w.ids.release(r.id_base, r.id_cap);
    w.n_total -= r.n;
    if (w.n_total == 0 && e == cudaSuccess) {   // every position is a hole: restart the layout
        k_set_total<<<1, 1, 0, w.stream>>>(w.ctrl, 0u);
        w.launches++;
        w.pos_bound = 0;
    }
    r = SceneRec();
    w.table_dirty = true;
    w.generation++;
    if (e == cudaSuccess) e = cudaGetLastError();
    return e;
}

cudaError_t world_export_scene(World& w, int slot, float4* pos, float4* vel, float* aff, float* mass, float* dens) {
    const SceneRec& r = w.scenes[slot];
    if (!r.live || r.n == 0) return cudaSuccess;
    const WorldView v = w.view();
    k_export<<<w.pos_blocks, 256, 0, w.stream>>>(v, w.posm[w.cur], w.velid[w.cur], w.aff[w.cur], w.dens,
                                                      r.id_base, r.n, pos, vel, aff, mass,
                                                      w.dens_valid ? dens : nullptr);
    w.launches++;
    return cudaGetLastError();
}

// Enqueues one substep of all scenes on w.stream (capturable when ds is null).
static cudaError_t enqueue_substep(World& w, Scene* ds) {
    const WorldView v = w.view();
    cudaStream_t st = w.stream;
    const int cur = w.cur, nxt = cur ^ 1;
    int32_t* cm = w.grid_i32[w.gbuf];
    int32_t* mv = cm + w.cell_cap;
    int32_t* cm_n = w.grid_i32[w.gbuf ^ 1];
    int32_t* mv_n = cm_n + w.cell_cap;
    const uint32_t nposb = w.pos_blocks;
    const uint32_t ntb = cdiv(v.ntiles ? v.ntiles : 1, 256);
    DiffuseView dv{};
    mpm_gen_params* gen_dev = nullptr;
    if (ds && ds->diffuse.enabled) {
        dv.enabled = 1;
        dv.scene = (uint32_t)ds->world_slot;
        dv.gen = ds->diffuse.gen_dev;
        dv.staging = ds->diffuse.staging;
        dv.spawn_bits = ds->diffuse.spawn_bits;
        gen_dev = ds->diffuse.gen_dev;
    }
    Scene* prof = ds;
    cudaError_t e;
    {
        Phase ph(prof, MPM_PHASE_SORT);
        e = cudaMemsetAsync(w.ctrl, 0, kCtrlZeroBytes, st);
        if (e != cudaSuccess) return e;
        k_count<<<nposb, 256, 0, st>>>(v);
        k_tiles_occ<<<ntb, 256, 0, st>>>(v);
        k_bin_cells<<<w.bin_blocks, kTileCells, 0, st>>>(v);
        k_tiles_grid<<<ntb, 256, 0, st>>>(v);
        k_tile_scan_local<<<dim3(v.nchunks, kMaxL), 1024, 0, st>>>(v);
        k_tile_scan_chunks<<<kMaxL, 1024, 0, st>>>(v);
        k_bucket_scan<<<1, 32, 0, st>>>(w.ctrl, gen_dev);
        k_scatter<<<nposb, 256, 0, st>>>(v);
        w.launches += 8;
    }
    {
        Phase ph(prof, MPM_PHASE_P2G_MASS);
        k_p2g_mass_items<<<w.item_blocks, kItemThreads, 0, st>>>(v, w.posm[cur], cm);
        w.launches++;
    }
    {
        Phase ph(prof, MPM_PHASE_DECODE_MASS);
        k_decode_tiles<<<w.grid_blocks, 256, 0, st>>>(v, cm, w.cmf);
        w.launches++;
    }
    {
        Phase ph(prof, MPM_PHASE_P2G_MOM);
        k_p2g_mom_items<<<w.item_blocks, kItemThreads, 0, st>>>(v, w.posm[cur], w.velid[cur], w.aff[cur], w.cmf, mv,
                                                                w.dens);
        w.launches++;
    }
    {
        Phase ph(prof, MPM_PHASE_UPDATE_GRID);   // includes APPLY_HAND
        k_update_tiles<<<w.grid_blocks, 256, 0, st>>>(v, cm, mv, w.mvf, cm_n, mv_n);
        w.launches++;
    }
    if (dv.enabled) {
        const uint32_t n = w.scenes[dv.scene].n;
        e = cudaMemsetAsync(dv.spawn_bits, 0, ((size_t)(n + 31) / 32) * 4, st);
        if (e != cudaSuccess) return e;
    }
    {
        Phase ph(prof, MPM_PHASE_G2P);
        k_g2p_items<<<w.item_blocks, kItemThreads, 0, st>>>(v, w.posm[cur], w.velid[cur], w.mvf, w.cmf, w.posm[nxt],
                                                            w.velid[nxt], w.aff[nxt], dv);
        w.launches++;
    }
    w.cur = nxt;
    w.gbuf ^= 1;
    w.cm_current = cm;
    w.dens_valid = true;
    w.pos_bound = std::min<uint64_t>((uint64_t)w.n_total + kPosSlack, w.npos);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (dv.enabled) {
        ds->diffuse.seed += 1u;   // mirrors the device-side bump in k_bucket_scan
        e = launch_diffuse(*ds, false);
    }
    return e;
}

cudaError_t world_substep(World& w, Scene* ds, bool use_graph) {
    cudaError_t e = world_upload_table(w);
    if (e != cudaSuccess) return e;
    const bool diffuse = ds && ds->diffuse.enabled;
    const bool profiling = ds && ds->profile;
    if (!use_graph || diffuse || profiling) return enqueue_substep(w, ds);
    const int p = w.cur;   // cur and gbuf flip together: one graph per parity
    if (!w.graph[p] || w.graph_gen[p] != w.generation) {
        if (w.graph[p]) {
            cudaGraphExecDestroy(w.graph[p]);
            w.graph[p] = nullptr;
        }
        const int cur0 = w.cur, gbuf0 = w.gbuf;
        int32_t* cmc0 = w.cm_current;
        const bool dv0 = w.dens_valid;
        const uint64_t l0 = w.launches;
        cudaGraph_t g = nullptr;
        e = cudaStreamBeginCapture(w.stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        const cudaError_t e2 = enqueue_substep(w, nullptr);
        e = cudaStreamEndCapture(w.stream, &g);
        if (e2 != cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&w.graph[p], g, 0);
        if (g) cudaGraphDestroy(g);
        // capture only recorded the work: restore the host state the enqueue advanced
        w.graph_kernels[p] = w.launches - l0;
        w.cur = cur0;
        w.gbuf = gbuf0;
        w.cm_current = cmc0;
        w.dens_valid = dv0;
        w.launches = l0;
        if (e != cudaSuccess) {
            w.graph[p] = nullptr;
            return e;
        }
        w.graph_gen[p] = w.generation;
    }
    e = cudaGraphLaunch(w.graph[p], w.stream);
    if (e != cudaSuccess) return e;
    // host mirror of what the graph does
    w.launches += w.graph_kernels[p];
    w.pos_bound = std::min<uint64_t>((uint64_t)w.n_total + kPosSlack, w.npos);
    w.cm_current = w.grid_i32[w.gbuf];
    w.cur ^= 1;
    w.gbuf ^= 1;
    w.dens_valid = true;
    return cudaSuccess;
}

}  // namespace mpm
