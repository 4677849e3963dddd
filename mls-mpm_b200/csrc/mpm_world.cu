// mpm_world.cu — the binned MLS-MPM substep over a world of scenes.
//
// Same arithmetic as mpm_kernels.cu (and so the same bits), organised for
// the B200:
//   * Particles are sorted by (tile, cell) every substep (counting sort: the
//     rank of each particle in its new cell is taken in G2P, then a scan per
//     16x8x8-cell tile and a two-level scan over tiles) and each tile's
//     particles are cut into chunks of up to kChunk consecutive particles
//     (kChunkSmall in worlds too small to fill the chunk kernels' grid).
//     The new layout reads the previous one through a permutation (new
//     position -> previous position), which stays nearly coalesced because
//     the order changes little between substeps.
//   * P2G_MASS, P2G_MOM and G2P run one 256-thread block per chunk, two
//     particles per thread.  A chunk's cells form a box inside its tile; P2G
//     sums the i32 contributions of the box plus a one-cell halo in shared
//     memory (integer adds commute, so the bits equal the reference's global
//     atomics) and flushes each halo cell to the grid with one atomic.  G2P
//     stages the halo's grid velocities in shared memory and gathers from
//     there.  The halo arrays use fixed strides, so a particle's 27 stencil
//     offsets are compile-time immediates; the contribution loops are written
//     out through template indices.  Particles whose stencil leaves the halo
//     or the grid take a direct path with the reference's own indexing.
//   * Latency hiding: each block keeps its chunk's scene descriptor in shared
//     memory, loads the next chunk's header (packed by P2G_MASS) a chunk
//     ahead, and P2G_MOM copies the next chunk's halo masses (cp.async) and
//     loads its first particle while the current chunk runs.
//   * Scenes: cells, tiles and particle ids of every scene are ranges of the
//     world's arrays; a tile maps to its scene, and each kernel reads the
//     scene's grid dims, params, walls and hand from the device scene table.
//     All scenes advance in one launch per kernel.
//   * The grid is processed per tile and only for tiles a particle stencil
//     touches now or touched last substep (cells elsewhere are zero, as the
//     reference's CLEAR/DECODE/UPDATE would leave them).  The i32 grid is
//     double-buffered: UPDATE_GRID of substep s reads buffer s%2 and zeroes
//     buffer (s+1)%2, which is the CLEAR of s+1.  APPLY_HAND runs inside the
//     UPDATE_GRID pass.
//   * The diffuse spawn decision runs in the G2P epilogue (post-G2P pos/vel,
//     this substep's density), staging records by particle id; G2P also
//     counts the spawners per group of ids for the free-list ranking.
//   * A substep (diffuse update included) is captured once per layout parity
//     as a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "mpm_alloc.h"
#include "mpm_device.cuh"
#include "mpm_kernels.h"
#include "mpm_scene.h"
#include "mpm_world.h"

// MPM_MIRROR_KEEP (default): the render mirrors' stores carry an L2
// evict-last hint (measured: G2P with the mirrors 93.6 -> 85.9 us at 1M).
#ifndef MPM_MIRROR_KEEP
#define MPM_MIRROR_KEEP 1
#endif

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
    v.ngroups = (v.ntiles + 1023u) / 1024u;
    if (v.ngroups == 0) v.ngroups = 1;
    v.chunk_cap = chunk_cap;
    v.chunk = chunk;
    v.scenes = scenes_dev(cur);
    v.tile_scene = tile_scene;
    v.cell_count = cell_count; v.cell_start = cell_start;
    v.key = key; v.rank = rank; v.perm = perm;
    v.tile_flags = tile_flags; v.tile_occ = tile_occ; v.tile_cnt = tile_cnt;
    v.tile_pstart = tile_pstart; v.tile_cstart = tile_cstart;
    v.group_pstart = group_pstart; v.group_cstart = group_cstart;
    v.chunk_info = chunk_info; v.chunk_last = chunk_last; v.chunk_hdr = chunk_hdr; v.chunk_geo = chunk_geo;
    v.tile_occ_list = tile_occ_list; v.tile_grid_list = tile_grid_list;
    v.ctrl = ctrl; v.dens = dens;
    v.health = health;
    return v;
}

namespace {

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
// Binning: particles sorted by (tile, cell), tiles cut into chunks
// ---------------------------------------------------------------------------

// Rank of every particle of the current state within its binning cell.
__global__ void k_count(WorldView v) {
    const uint32_t total = v.ctrl->total_pos;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const uint32_t c = v.key[i];
        if (c != kHole) v.rank[i] = atomicAdd(&v.cell_count[c], 1u);
    }
}
// k_count for the positions [p0, p1) of a scene just imported behind counted
// ones: their ranks continue the counts G2P left for the next binning.
__global__ void k_count_range(WorldView v, uint32_t p0, uint32_t p1) {
    for (uint32_t i = p0 + blockIdx.x * blockDim.x + threadIdx.x; i < p1; i += gridDim.x * blockDim.x) {
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


// One block per occupied tile, one thread per cell (local order x fastest,
// then y, then z): exclusive scan of the cell counts inside the tile ->
// cell_start (tile-local), tile total -> tile_cnt.  Also marks every tile the
// particles' 3x3x3 stencils touch (bit 1).
__device__ void tiles_fold(const WorldView& v, mpm_gen_params* gen);

__global__ void __launch_bounds__(kTileCells) k_bin_cells(WorldView v, mpm_gen_params* gen, int fold) {
    __shared__ uint32_t ws[33];
    __shared__ uint32_t dirs;
    const uint32_t nocc = v.ctrl->n_occ;
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
        const uint32_t cnt = inside ? v.cell_count[c] : 0u;
        if (threadIdx.x == 0) dirs = 0u;
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
        if ((threadIdx.x & 31) == 0 && wm) atomicOr(&dirs, wm);
        uint32_t total;
        const uint32_t local = block_exclusive_scan_1024(cnt, ws, total);   // also orders the dirs updates
        if (cnt) v.cell_start[c] = local;
        if (threadIdx.x == 0) v.tile_cnt[t] = total;
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
    }
    if (!fold) return;
    // the last block to finish runs the per-tile passes (block-uniform test)
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&v.ctrl->bins_done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    tiles_fold(v, gen);
}

// Grid-tile list (stencil tiles of this substep or the last one, plus the
// hand boxes); shifts the flags for the next substep.
// (The flags are read past L1: in the folded form other blocks of the same
// kernel have just set their bit 1.)
__device__ __forceinline__ void tile_grid_entry(const WorldView& v, uint32_t t) {
    const uint32_t scene = v.tile_scene[t];
    const uint32_t f = __ldcg(v.tile_flags + t);
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

__global__ void k_tiles_grid(WorldView v) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < v.ntiles) tile_grid_entry(v, t);
}


// Two-level exclusive scan over all tiles in index order of the particle
// counts and the chunk counts of the occupied tiles.  Level 1, one block per
// group of 1024 tiles: prefixes inside the group, group totals.
__global__ void __launch_bounds__(1024) k_tile_scan_local(WorldView v) {
    __shared__ uint32_t ws[33];
    const uint32_t g = blockIdx.x;
    const uint32_t t = g * 1024u + threadIdx.x;
    const uint32_t np = (t < v.ntiles && v.tile_occ[t]) ? v.tile_cnt[t] : 0u;
    const uint32_t nc = (np + v.chunk - 1) / v.chunk;
    uint32_t tp, tc;
    const uint32_t rp = block_exclusive_scan_1024(np, ws, tp);
    const uint32_t rc = block_exclusive_scan_1024(nc, ws, tc);
    if (t < v.ntiles) {
        v.tile_pstart[t] = rp;
        v.tile_cstart[t] = rc;
    }
    if (threadIdx.x == 0) {
        v.group_pstart[g] = tp;
        v.group_cstart[g] = tc;
    }
}

// Level 2, one block: exclusive scan of the group totals; the layout size and
// chunk count go to ctrl.  Also advances the diffuse seed (diffuse-gpu.js:149).
__global__ void __launch_bounds__(1024) k_tile_scan_top(WorldView v, mpm_gen_params* gen) {
    __shared__ uint32_t ws[33];
    uint32_t cp = 0, cc = 0;
    for (uint32_t g0 = 0; g0 < v.ngroups; g0 += 1024) {
        const uint32_t g = g0 + threadIdx.x;
        const uint32_t xp = g < v.ngroups ? v.group_pstart[g] : 0u;
        const uint32_t xc = g < v.ngroups ? v.group_cstart[g] : 0u;
        uint32_t tp, tc;
        const uint32_t rp = block_exclusive_scan_1024(xp, ws, tp);
        const uint32_t rc = block_exclusive_scan_1024(xc, ws, tc);
        if (g < v.ngroups) {
            v.group_pstart[g] = cp + rp;
            v.group_cstart[g] = cc + rc;
        }
        cp += tp;
        cc += tc;
    }
    if (threadIdx.x == 0) {
        v.ctrl->prev_total_pos = v.ctrl->total_pos;
        v.ctrl->total_pos = min(cp, v.npos);
        v.ctrl->total_chunks = min(cc, v.chunk_cap);
        if (gen) gen->seed = gen->seed + 1u;
    }
}

// Tiles of a world small enough for one block to finish the binning's
// per-tile passes: the last k_bin_cells block to finish builds the grid-tile
// list and scans the tile counts itself instead of three more launches.
constexpr uint32_t kFoldTiles = 4096;

// The grid-tile list and the exclusive scans of the particle and chunk counts
// over all tiles (tile_pstart/tile_cstart global, group offsets 0), the layout
// totals and the diffuse seed bump: the work of k_tiles_grid,
// k_tile_scan_local and k_tile_scan_top, by one 1024-thread block.
__device__ void tiles_fold(const WorldView& v, mpm_gen_params* gen) {
    __shared__ uint32_t ws[33];
    for (uint32_t t = threadIdx.x; t < v.ntiles; t += blockDim.x) tile_grid_entry(v, t);
    uint32_t cp = 0, cc = 0;
    for (uint32_t t0 = 0; t0 < v.ntiles; t0 += 1024) {
        const uint32_t t = t0 + threadIdx.x;
        // tile counts written by the other blocks of k_bin_cells: read past L1
        const uint32_t np = (t < v.ntiles && v.tile_occ[t]) ? __ldcg(v.tile_cnt + t) : 0u;
        const uint32_t nc = (np + v.chunk - 1) / v.chunk;
        uint32_t tp, tc;
        const uint32_t rp = block_exclusive_scan_1024(np, ws, tp);
        const uint32_t rc = block_exclusive_scan_1024(nc, ws, tc);
        if (t < v.ntiles) {
            v.tile_pstart[t] = cp + rp;
            v.tile_cstart[t] = cc + rc;
        }
        cp += tp;
        cc += tc;
    }
    for (uint32_t g = threadIdx.x; g < v.ngroups; g += blockDim.x) {
        v.group_pstart[g] = 0u;
        v.group_cstart[g] = 0u;
    }
    if (threadIdx.x == 0) {
        v.ctrl->prev_total_pos = v.ctrl->total_pos;
        v.ctrl->total_pos = min(cp, v.npos);
        v.ctrl->total_chunks = min(cc, v.chunk_cap);
        if (gen) gen->seed = gen->seed + 1u;
    }
}

// One block per occupied tile, one thread per cell: cell_start becomes the
// global first position, the counts are cleared, and the tile's chunks are
// written: (tile, first position, end position, first local cell) and the
// last local cell, each by the thread whose cell holds that particle.
__global__ void __launch_bounds__(kTileCells) k_tile_finish(WorldView v) {
    const uint32_t nocc = v.ctrl->n_occ;
    for (uint32_t ti = blockIdx.x; ti < nocc; ti += gridDim.x) {
        const uint32_t t = v.tile_occ_list[ti];
        const uint32_t scene = v.tile_scene[t];
        const SceneDesc& sd = v.scenes[scene];
        const uint32_t lt = t - sd.tile_base;
        const uint32_t tx = lt % sd.ntx, ty = (lt / sd.ntx) % sd.nty, tz = lt / (sd.ntx * sd.nty);
        const uint32_t lid = threadIdx.x;
        const uint32_t x = tx * kTileX + lid % kTileX, y = ty * kTileY + (lid / kTileX) % kTileY,
                       z = tz * kTileZ + lid / (kTileX * kTileY);
        if (x >= sd.X || y >= sd.Y || z >= sd.Z) continue;
        const uint32_t c = sd.cell_base + local_cell(sd, x, y, z);
        const uint32_t cnt = v.cell_count[c];
        if (cnt == 0) continue;
        const uint32_t base_p = v.tile_pstart[t] + v.group_pstart[t >> 10];
        const uint32_t base_c = v.tile_cstart[t] + v.group_cstart[t >> 10];
        const uint32_t total = v.tile_cnt[t];
        const uint32_t a = v.cell_start[c];
        v.cell_start[c] = base_p + a;
        v.cell_count[c] = 0u;
        const uint32_t C = v.chunk;
        for (uint32_t j = a / C; j <= (a + cnt - 1) / C; ++j) {
            const uint32_t ci = base_c + j;
            if (ci >= v.chunk_cap) break;
            const uint32_t f = j * C;
            const uint32_t e = min(f + C, total);
            if (f >= a) {
                v.chunk_info[ci] = make_uint4(t, base_p + f, base_p + e, lid);
                v.chunk_geo[ci] = make_uint4(scene, tx, ty, tz);
            }
            if (e - 1 < a + cnt) v.chunk_last[ci] = lid;
        }
    }
}

// perm[new position] = previous position for every particle.
__global__ void k_scatter(WorldView v) {
    const uint32_t total = v.ctrl->prev_total_pos;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const uint32_t c = v.key[i];
        if (c == kHole) continue;
        const uint32_t pos = v.cell_start[c] + v.rank[i];
        if (pos < v.npos) v.perm[pos] = i;
    }
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

// encode() without the clamp, for values already known to lie in +-20000.
__device__ __forceinline__ int32_t encode_unclamped(float v) { return __float2int_rz(v * kFixed); }

// ---------------------------------------------------------------------------
// Paired f32 arithmetic (add/mul.rn.f32x2): two independent lanes per
// instruction, each lane rounded exactly as the scalar operation.  One rule
// keeps every result bit-identical to the scalar sequence: a paired add never
// takes a paired product directly as an operand (ptxas contracts that pair
// into a fused multiply-add, which rounds once; measured on sm_100a, where a
// paired product feeding scalar adds, or scalar products feeding a paired
// add, stay separately rounded).  pmul: paired product; smul: two scalar
// products as a pair; padd: paired add (operands never from pmul); sadd: two
// scalar adds (for a pmul operand).  MPM_G2P_PACKED / MPM_MOM_PACKED select
// the paired forms per kernel (on by default; 0 builds the scalar forms,
// which give the same bits).
// ---------------------------------------------------------------------------
#ifndef MPM_G2P_PACKED
#define MPM_G2P_PACKED 1
#endif
#ifndef MPM_MOM_PACKED
#define MPM_MOM_PACKED 1
#endif
#if MPM_G2P_PACKED || MPM_MOM_PACKED
__device__ __forceinline__ unsigned long long pk2(float a, float b) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float2 up2(unsigned long long r) {
    float2 o;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(o.x), "=f"(o.y) : "l"(r));
    return o;
}
__device__ __forceinline__ float2 pmul(float2 a, float2 b) {
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a.x, a.y)), "l"(pk2(b.x, b.y)));
    return up2(r);
}
__device__ __forceinline__ float2 smul(float2 a, float2 b) { return make_float2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) {
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a.x, a.y)), "l"(pk2(b.x, b.y)));
    return up2(r);
}
__device__ __forceinline__ float2 sadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
#endif


// ---------------------------------------------------------------------------
// Chunks: the halo box of a chunk's cells in shared memory
// ---------------------------------------------------------------------------
// Lane order of the P2G chunk kernels: lane l of warp w has offset 8*l + w
// (8 warps per block), which chunk_slot scales to a particle of the chunk, so
// neighbouring lanes sit in different cells and the lanes of one shared
// atomic rarely share an address.  (Adding same-cell lanes with a warp
// reduction first was measured slower, both per cell with match + redux and
// for warp passes in at most two cells.)
__device__ __forceinline__ uint32_t chunk_lane_offset() {
    return (threadIdx.x & 31u) * (kChunkThreads / 32) + (threadIdx.x >> 5);
}

// Position within a chunk of kC particles of this thread's particle in pass
// r.  MPM_P2G_SPREAD (default): a thread's passes take neighbouring particles
// and the lanes of a warp spread over the whole chunk, so in dense cells fewer
// lanes of one shared atomic share its address (results do not depend on it;
// measured -1% on the 1M dam break, -2.3% on the batched mix with its
// overpacked blocks).  0: lanes spread over one pass of kChunkThreads.
#ifndef MPM_P2G_SPREAD
#define MPM_P2G_SPREAD 1
#endif
template <uint32_t kC>
__device__ __forceinline__ uint32_t chunk_slot(int r) {
#if MPM_P2G_SPREAD
    return (uint32_t)r + (kC / kChunkThreads) * chunk_lane_offset();
#else
    return (uint32_t)r * kChunkThreads + chunk_lane_offset();
#endif
}

struct ChunkHdr {
    uint32_t scene, first, end;
    int32_t ox, oy, oz;      // scene-local cell at halo index 0
    int32_t hx, hy, hz;      // halo dims
};

// The box of the local cells [lo, hi] (x fastest, then y, then z) plus one
// cell on every side.
// The chunk's header from its three independent words: chunk_info (tile,
// first, end, first local cell), chunk_last (last local cell) and chunk_geo
// (scene, tile coordinates).
__device__ __forceinline__ void chunk_header_from(const uint4 ci, uint32_t hi, const uint4 geo, ChunkHdr& h) {
    const uint32_t lo = ci.w;
    const int32_t tx = (int32_t)geo.y, ty = (int32_t)geo.z, tz = (int32_t)geo.w;
    constexpr uint32_t kRow = kTileX, kSlab = kTileX * kTileY;
    int32_t x0 = 0, x1 = kTileX - 1, y0 = 0, y1 = kTileY - 1;
    const int32_t z0 = (int32_t)(lo / kSlab), z1 = (int32_t)(hi / kSlab);
    if (z0 == z1) {
        y0 = (int32_t)((lo / kRow) % kTileY);
        y1 = (int32_t)((hi / kRow) % kTileY);
        if (y0 == y1) {
            x0 = (int32_t)(lo % kRow);
            x1 = (int32_t)(hi % kRow);
        }
    }
    h.scene = geo.x;
    h.first = ci.y;
    h.end = ci.z;
    h.ox = tx * kTileX + x0 - 1;
    h.oy = ty * kTileY + y0 - 1;
    h.oz = tz * kTileZ + z0 - 1;
    h.hx = x1 - x0 + 3;
    h.hy = y1 - y0 + 3;
    h.hz = z1 - z0 + 3;
}

// Asynchronous 16-byte global -> shared copy (cp.async); src_bytes 0 writes
// zeros.  cp_async_wait waits for all of this thread's copies.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, uint32_t src_bytes) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes) : "memory");
}
// Asynchronous 4-byte global -> shared copy; src_bytes 0 writes a zero.
__device__ __forceinline__ void cp_async4z(void* smem, const void* gmem, uint32_t src_bytes) {
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// ChunkHdr packed in two 16-byte words (box dims below 256).
__device__ __forceinline__ void pack_header(const ChunkHdr& h, uint4* dst) {
    dst[0] = make_uint4(h.scene, h.first, h.end, (uint32_t)h.hx | ((uint32_t)h.hy << 8) | ((uint32_t)h.hz << 16));
    dst[1] = make_uint4((uint32_t)h.ox, (uint32_t)h.oy, (uint32_t)h.oz, 0u);
}
__device__ __forceinline__ ChunkHdr unpack_header(const uint4 a, const uint4 b) {
    ChunkHdr h;
    h.scene = a.x;
    h.first = a.y;
    h.end = a.z;
    h.hx = (int32_t)(a.w & 0xFFu);
    h.hy = (int32_t)((a.w >> 8) & 0xFFu);
    h.hz = (int32_t)((a.w >> 16) & 0xFFu);
    h.ox = (int32_t)b.x;
    h.oy = (int32_t)b.y;
    h.oz = (int32_t)b.z;
    return h;
}

// Each block of the chunk kernels keeps its chunk's scene descriptor in
// shared memory, so per-particle reads of grid dims and uniforms are shared
// loads; the next chunk's descriptor is copied while the current one runs.
static_assert(sizeof(SceneDesc) % 16 == 0, "SceneDesc copy in 16-byte words");

// Starts copying scene `scene`'s descriptor into shared memory (cp.async,
// 16-byte words); the block's next cp_async_wait and barrier make it visible.
__device__ __forceinline__ void copy_scene_async(const WorldView& v, uint32_t scene, SceneDesc& dst) {
    constexpr int kWords = (int)(sizeof(SceneDesc) / 16);
    if (threadIdx.x < kWords)
        cp_async16(reinterpret_cast<uint4*>(&dst) + threadIdx.x, reinterpret_cast<const uint4*>(v.scenes + scene) + threadIdx.x,
                   16u);
}

// The same, issued by one thread (36 copies); its own cp_async_wait and the
// next barrier make it visible.
__device__ __forceinline__ void copy_scene_async_one(const WorldView& v, uint32_t scene, SceneDesc& dst) {
    constexpr int kWords = (int)(sizeof(SceneDesc) / 16);
#pragma unroll 4
    for (int i = 0; i < kWords; ++i)
        cp_async16(reinterpret_cast<uint4*>(&dst) + i, reinterpret_cast<const uint4*>(v.scenes + scene) + i, 16u);
}

// True when the particle's 3x3x3 stencil lies in the chunk's halo box and in
// the grid (then shared-memory accumulation / gathering is exact); otherwise
// the particle takes the direct path with the reference's indexing.
__device__ __forceinline__ bool in_halo(const PW& w, const ChunkHdr& h, const SceneDesc& sd) {
    return w.cx - 1 >= h.ox && w.cy - 1 >= h.oy && w.cz - 1 >= h.oz && w.cx + 1 < h.ox + h.hx &&
           w.cy + 1 < h.oy + h.hy && w.cz + 1 < h.oz + h.hz && w.cx >= 1 && w.cy >= 1 && w.cz >= 1 &&
           w.cx + 1 < (int32_t)sd.X && w.cy + 1 < (int32_t)sd.Y && w.cz + 1 < (int32_t)sd.Z;
}

// Shared halo arrays use the strides of the largest box (a tile plus its
// halo) whatever the chunk's box, so the 27 stencil offsets of a particle are
// compile-time constants.
constexpr int kHX = kTileX + 2, kHXY = (kTileX + 2) * (kTileY + 2);
static_assert(kHXY * (kTileZ + 2) == kHaloCells, "halo strides");

// Halo slot of the stencil base (cx-1, cy-1, cz-1).
__device__ __forceinline__ int halo_base(const ChunkHdr& h, int32_t cx, int32_t cy, int32_t cz) {
    return (cz - 1 - h.oz) * kHXY + (cy - 1 - h.oy) * kHX + (cx - 1 - h.ox);
}

// Slots of the halo arrays that the chunk's box spans: [0, halo_span(h)).
// Loops over them divide by compile-time strides only.
__device__ __forceinline__ int halo_span(const ChunkHdr& h) { return h.hz * kHXY; }

// Slot s as a cell of the chunk's box inside the grid: its scene-local cell,
// or false for a slot outside the box or a box cell outside the grid.
__device__ __forceinline__ bool halo_cell(const ChunkHdr& h, const SceneDesc& sd, int s, uint32_t& cell) {
    const int dz = s / kHXY, r = s - dz * kHXY, dy = r / kHX, dx = r - dy * kHX;
    if (dx >= h.hx || dy >= h.hy) return false;
    const int32_t x = h.ox + dx, y = h.oy + dy, z = h.oz + dz;
    if (x < 0 || y < 0 || z < 0 || x >= (int32_t)sd.X || y >= (int32_t)sd.Y || z >= (int32_t)sd.Z) return false;
    cell = local_cell(sd, x, y, z);
    return true;
}

// The 27 P2G_MASS contributions of one particle into the shared halo at base
// slot hb, written out through template indices (immediate offsets, no
// per-cell control flow).  kClamp: encode with its clamp.
template <bool kClamp, int K, int J, int I>
__device__ __forceinline__ void mass_cell(const PW& w, float m, int32_t* a) {
    const float x = w.wx[I] * w.wy[J] * w.wz[K] * m;
    atomicAdd(a + (K * kHXY + J * kHX + I), kClamp ? encode(x) : encode_unclamped(x));
}
template <bool kClamp, int K, int J>
__device__ __forceinline__ void mass_row(const PW& w, float m, int32_t* a) {
    mass_cell<kClamp, K, J, 0>(w, m, a);
    mass_cell<kClamp, K, J, 1>(w, m, a);
    mass_cell<kClamp, K, J, 2>(w, m, a);
}
template <bool kClamp>
__device__ __forceinline__ void mass_contrib_shared(const PW& w, float m, int32_t* a) {
    mass_row<kClamp, 0, 0>(w, m, a);
    mass_row<kClamp, 0, 1>(w, m, a);
    mass_row<kClamp, 0, 2>(w, m, a);
    mass_row<kClamp, 1, 0>(w, m, a);
    mass_row<kClamp, 1, 1>(w, m, a);
    mass_row<kClamp, 1, 2>(w, m, a);
    mass_row<kClamp, 2, 0>(w, m, a);
    mass_row<kClamp, 2, 1>(w, m, a);
    mass_row<kClamp, 2, 2>(w, m, a);
}

// ---------------------------------------------------------------------------
// P2G_MASS (shaders.js:242-274): one block per chunk, one thread per particle
// ---------------------------------------------------------------------------
template <uint32_t kC>
__global__ void __launch_bounds__(kChunkThreads) k_p2g_mass_chunks(WorldView v, const float4* __restrict__ posm,
                                                                   int32_t* __restrict__ cm) {
    constexpr int kPer = kC / kChunkThreads;
    __shared__ int32_t acc[kHaloCells];
    const uint32_t nch = v.ctrl->total_chunks;
    __shared__ ChunkHdr hs;
    // scene descriptors of this chunk and the next (thread 0 copies the next
    // one while this chunk runs)
    __shared__ SceneDesc ssd[2];
    int sb = 0;                                      // ssd[sb]: this chunk's scene
    uint32_t ss_nxt = kHole;                         // thread 0: scene held in ssd[sb ^ 1]
    // thread 0: the next chunk's header words, loaded while this chunk runs
    uint4 nci = make_uint4(0u, 0u, 0u, 0u), ngeo = nci;
    uint32_t nlast = 0;
    if (threadIdx.x == 0 && blockIdx.x < nch) {
        const uint4 g0 = v.chunk_geo[blockIdx.x];
        chunk_header_from(v.chunk_info[blockIdx.x], v.chunk_last[blockIdx.x], g0, hs);
        copy_scene_async_one(v, g0.x, ssd[0]);
        cp_async_wait();
    }
    // the accumulators start at zero and every flush zeroes what it read
    for (int i = threadIdx.x; i < kHaloCells; i += blockDim.x) acc[i] = 0;
    __syncthreads();
    for (uint32_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
        const ChunkHdr h = hs;
        const uint32_t nxt = ch + gridDim.x;
        if (threadIdx.x == 0) {
            pack_header(h, v.chunk_hdr + 2ull * ch);   // for P2G_MOM and G2P
            if (nxt < nch) {
                nci = v.chunk_info[nxt];
                nlast = v.chunk_last[nxt];
                ngeo = v.chunk_geo[nxt];
            }
        }
        // this thread's particles, all loads issued before the first is used
        float4 q[kPer];
#pragma unroll
        for (int r = 0; r < kPer; ++r) {
            const uint32_t p = h.first + chunk_slot<kC>(r);
            q[r] = p < h.end ? posm[v.perm[p]] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        const int hn = halo_span(h);
        const SceneDesc& sd = ssd[sb];
#pragma unroll
        for (int r = 0; r < kPer; ++r) {
            const bool valid = h.first + chunk_slot<kC>(r) < h.end;
            const PW w = particle_weights(q[r].x, q[r].y, q[r].z);
            const bool fast = valid && in_halo(w, h, sd);
            const int hb = halo_base(h, w.cx, w.cy, w.cz);
            if (fast) {
                // weight <= 0.4219: for |mass| < 47000 encode's clamp is the identity
                const bool safe = fabsf(q[r].w) < 47000.0f;
                if (safe) {
                    mass_contrib_shared<false>(w, q[r].w, acc + hb);
                } else {
                    // health: encode's clamp may engage (a weight times |mass| >= 20000 needs |mass| >= 47000)
                    atomicOr(&v.health[h.scene], MPM_HEALTH_SATURATED);
                    mass_contrib_shared<true>(w, q[r].w, acc + hb);
                }
            } else if (valid) {
                // health: every position that is NaN or infinite takes this path
                // (its cell is 0 or saturated, outside every halo); it never heals
                if (!(fabsf(q[r].x + q[r].y + q[r].z) <= 3.0e38f)) atomicOr(&v.health[h.scene], MPM_HEALTH_NONFINITE);
                // stencil outside the halo or the grid: bounds-checked global atomics
                const int32_t X = sd.X, Y = sd.Y, Z = sd.Z;
                int32_t* scm = cm + sd.cell_base;
                for (int kk = 0; kk < 3; ++kk)
                    for (int j = 0; j < 3; ++j)
                        for (int i = 0; i < 3; ++i) {
                            const int32_t xx = w.cx - 1 + i, yy = w.cy - 1 + j, zz = w.cz - 1 + kk;
                            if (xx < 0 || xx >= X || yy < 0 || yy >= Y || zz < 0 || zz >= Z) continue;
                            const float ww = w.wx[i] * w.wy[j] * w.wz[kk];
                            const int32_t e = encode(ww * q[r].w);
                            if (at_clamp(e)) atomicOr(&v.health[h.scene], MPM_HEALTH_SATURATED);
                            atomicAdd(&scm[(zz * Y + yy) * X + xx], e);
                        }
            }
        }
        __syncthreads();
        // every thread holds this chunk's header: the next one can replace it
        if (threadIdx.x == 0 && nxt < nch) {
            chunk_header_from(nci, nlast, ngeo, hs);
            if (ngeo.x != ss_nxt) {
                copy_scene_async_one(v, ngeo.x, ssd[sb ^ 1]);
                ss_nxt = ngeo.x;
            }
        }
        int32_t* scm = cm + sd.cell_base;
        for (int i = threadIdx.x; i < hn; i += blockDim.x) {
            const int32_t a = acc[i];
            if (a == 0) continue;
            acc[i] = 0;
            uint32_t cell;
            if (halo_cell(h, sd, i, cell)) atomicAdd(&scm[cell], a);
        }
        if (threadIdx.x == 0) {
            cp_async_wait();
            ss_nxt = h.scene;   // after the swap ssd[sb ^ 1] holds this chunk's scene
        }
        __syncthreads();
        sb ^= 1;
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
                                                      float4* __restrict__ vel4, int32_t* __restrict__ cm_next,
                                                      int32_t* __restrict__ mv_next) {
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
        vel4[idx] = make_float4(vx, vy, vz, 0.0f);
    }
}


// ---------------------------------------------------------------------------
// P2G_MOM (shaders.js:276-371): one block per chunk, one thread per particle
// ---------------------------------------------------------------------------
struct MomIn {
    float vx, vy, vz, m;
    float a00, a01, a02, a10, a11, a12, a20, a21, a22;
};

// The 81 encoded momentum contributions of one particle (shaders.js:340-370),
// handed to sink(k, j, i, ex, ey, ez).  Every value is the reference's own
// expression, (C d) = (c0 dx + c1 dy) + c2 dz and (S d) likewise, with the
// products along the third axis and the (dx, dy) partial sums computed once
// and reused (the same roundings, fewer instructions).  kClamp: full encode;
// without it the caller has bounded every value inside +-20000, where the
// clamp is the identity.
template <bool kClamp, class Sink>
__device__ __forceinline__ void mom_contrib(const PW& w, const MomIn& in, const float* s, float coef, Sink&& sink) {
    const float s00 = s[0], s11 = s[1], s22 = s[2], s01 = s[3], s02 = s[4], s12 = s[5];
    const float dxs[3] = {-w.fx - 1.0f, -w.fx, 1.0f - w.fx};
    const float dys[3] = {-w.fy - 1.0f, -w.fy, 1.0f - w.fy};
    const float dzs[3] = {-w.fz - 1.0f, -w.fz, 1.0f - w.fz};
    float qz[3][3], fz[3][3];   // [component][k]: C[c][2] dz_k and S[c][2] dz_k
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        qz[0][k] = in.a02 * dzs[k];
        qz[1][k] = in.a12 * dzs[k];
        qz[2][k] = in.a22 * dzs[k];
        fz[0][k] = s02 * dzs[k];
        fz[1][k] = s12 * dzs[k];
        fz[2][k] = s22 * dzs[k];
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const float dxi = dxs[i], dyj = dys[j];
            const float qx = in.a00 * dxi + in.a01 * dyj;
            const float qy = in.a10 * dxi + in.a11 * dyj;
            const float qzz = in.a20 * dxi + in.a21 * dyj;
            const float gx = s00 * dxi + s01 * dyj;
            const float gy = s01 * dxi + s11 * dyj;
            const float gz = s02 * dxi + s12 * dyj;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float ww = w.wx[i] * (w.wy[j] * w.wz[k]);
                const float Qx = qx + qz[0][k];
                const float Qy = qy + qz[1][k];
                const float Qz = qzz + qz[2][k];
                const float fxf = coef * (gx + fz[0][k]);
                const float fyf = coef * (gy + fz[1][k]);
                const float fzf = coef * (gz + fz[2][k]);
                const float vx = ww * (in.m * (in.vx + Qx) + fxf);
                const float vy = ww * (in.m * (in.vy + Qy) + fyf);
                const float vz = ww * (in.m * (in.vz + Qz) + fzf);
                sink(k, j, i, kClamp ? encode(vx) : encode_unclamped(vx), kClamp ? encode(vy) : encode_unclamped(vy),
                     kClamp ? encode(vz) : encode_unclamped(vz));
            }
        }
    }
}

// The shared-halo form of mom_contrib with every loop written out at compile
// time (template indices): the 81 contributions go straight into the three
// accumulator arrays at base slot hb with immediate offsets.
struct MomTerms {
    float dxs[3], dys[3];
    float qz[3][3], fz[3][3];   // [component][k]
    float s00, s11, s01, s02, s12;
    float coef;
};

template <bool kClamp, int K, int J, int I>
__device__ __forceinline__ void mom_cell(const PW& w, const MomIn& in, const MomTerms& t, float qx, float qy,
                                         float qzz, float gx, float gy, float gz, int32_t* a0, int32_t* a1,
                                         int32_t* a2) {
    const float ww = w.wx[I] * (w.wy[J] * w.wz[K]);
    const float Qx = qx + t.qz[0][K];
    const float Qy = qy + t.qz[1][K];
    const float Qz = qzz + t.qz[2][K];
    const float fxf = t.coef * (gx + t.fz[0][K]);
    const float fyf = t.coef * (gy + t.fz[1][K]);
    const float fzf = t.coef * (gz + t.fz[2][K]);
    const float vx = ww * (in.m * (in.vx + Qx) + fxf);
    const float vy = ww * (in.m * (in.vy + Qy) + fyf);
    const float vz = ww * (in.m * (in.vz + Qz) + fzf);
    constexpr int o = K * kHXY + J * kHX + I;
    atomicAdd(a0 + o, kClamp ? encode(vx) : encode_unclamped(vx));
    atomicAdd(a1 + o, kClamp ? encode(vy) : encode_unclamped(vy));
    atomicAdd(a2 + o, kClamp ? encode(vz) : encode_unclamped(vz));
}

template <bool kClamp, int J, int I>
__device__ __forceinline__ void mom_column(const PW& w, const MomIn& in, const MomTerms& t, int32_t* a0,
                                           int32_t* a1, int32_t* a2) {
    const float dxi = t.dxs[I], dyj = t.dys[J];
    const float qx = in.a00 * dxi + in.a01 * dyj;
    const float qy = in.a10 * dxi + in.a11 * dyj;
    const float qzz = in.a20 * dxi + in.a21 * dyj;
    const float gx = t.s00 * dxi + t.s01 * dyj;
    const float gy = t.s01 * dxi + t.s11 * dyj;
    const float gz = t.s02 * dxi + t.s12 * dyj;
    mom_cell<kClamp, 0, J, I>(w, in, t, qx, qy, qzz, gx, gy, gz, a0, a1, a2);
    mom_cell<kClamp, 1, J, I>(w, in, t, qx, qy, qzz, gx, gy, gz, a0, a1, a2);
    mom_cell<kClamp, 2, J, I>(w, in, t, qx, qy, qzz, gx, gy, gz, a0, a1, a2);
}

template <bool kClamp>
__device__ __forceinline__ void mom_contrib_shared(const PW& w, const MomIn& in, const float* s, float coef,
                                                   int32_t (*acc)[kHaloCells], int hb) {
    MomTerms t;
    t.s00 = s[0]; t.s11 = s[1]; t.s01 = s[3]; t.s02 = s[4]; t.s12 = s[5];
    const float s22 = s[2];
    t.coef = coef;
    t.dxs[0] = -w.fx - 1.0f; t.dxs[1] = -w.fx; t.dxs[2] = 1.0f - w.fx;
    t.dys[0] = -w.fy - 1.0f; t.dys[1] = -w.fy; t.dys[2] = 1.0f - w.fy;
    const float dzs[3] = {-w.fz - 1.0f, -w.fz, 1.0f - w.fz};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        t.qz[0][k] = in.a02 * dzs[k];
        t.qz[1][k] = in.a12 * dzs[k];
        t.qz[2][k] = in.a22 * dzs[k];
        t.fz[0][k] = t.s02 * dzs[k];
        t.fz[1][k] = t.s12 * dzs[k];
        t.fz[2][k] = s22 * dzs[k];
    }
    int32_t* a0 = &acc[0][hb];
    int32_t* a1 = &acc[1][hb];
    int32_t* a2 = &acc[2][hb];
    mom_column<kClamp, 0, 0>(w, in, t, a0, a1, a2);
    mom_column<kClamp, 0, 1>(w, in, t, a0, a1, a2);
    mom_column<kClamp, 0, 2>(w, in, t, a0, a1, a2);
    mom_column<kClamp, 1, 0>(w, in, t, a0, a1, a2);
    mom_column<kClamp, 1, 1>(w, in, t, a0, a1, a2);
    mom_column<kClamp, 1, 2>(w, in, t, a0, a1, a2);
    mom_column<kClamp, 2, 0>(w, in, t, a0, a1, a2);
    mom_column<kClamp, 2, 1>(w, in, t, a0, a1, a2);
    mom_column<kClamp, 2, 2>(w, in, t, a0, a1, a2);
}

#if MPM_MOM_PACKED
// mom_contrib_shared with the x and y components paired (paired f32 lanes):
// each of the 81 values is the reference's own expression, as in mom_cell.
struct MomTerms2 {
    float dxs[3], dys[3];
    float2 qz2[3], fz2[3];   // (x, y) lanes of C[.][2] dz_k and S[.][2] dz_k (scalar products)
    float qzz[3], fzz[3];    // z lane
    float2 axy0, axy1;       // (a00, a10), (a01, a11)
    float2 sxy0, sxy1;       // (s00, s01), (s01, s11)
    float a20, a21, s02, s12, coef;
    float2 vxy, mm, cc;      // (vx, vy), (m, m), (coef, coef)
};

template <bool kClamp, int K, int J, int I>
__device__ __forceinline__ void mom_cell2(const PW& w, const MomIn& in, const MomTerms2& t, float2 qxy, float qzz,
                                          float2 gxy, float gz, int32_t* a0, int32_t* a1, int32_t* a2) {
    const float ww = w.wx[I] * (w.wy[J] * w.wz[K]);
    // x and y: w * (m * (v + Q) + coef * (G + S dz))
    const float2 vq = padd(t.vxy, padd(qxy, t.qz2[K]));
    const float2 tm = pmul(t.mm, vq);
    const float2 f = pmul(t.cc, padd(gxy, t.fz2[K]));
    const float2 r = pmul(make_float2(ww, ww), sadd(tm, f));
    int32_t ex, ey;
    if (kClamp) {
        ex = encode(r.x);
        ey = encode(r.y);
    } else {
        const float2 e = pmul(r, make_float2(kFixed, kFixed));
        ex = __float2int_rz(e.x);
        ey = __float2int_rz(e.y);
    }
    // z as mom_cell
    const float Qz = qzz + t.qzz[K];
    const float fzf = t.coef * (gz + t.fzz[K]);
    const float vz = ww * (in.m * (in.vz + Qz) + fzf);
    constexpr int o = K * kHXY + J * kHX + I;
    atomicAdd(a0 + o, ex);
    atomicAdd(a1 + o, ey);
    atomicAdd(a2 + o, kClamp ? encode(vz) : encode_unclamped(vz));
}

template <bool kClamp, int J, int I>
__device__ __forceinline__ void mom_column2(const PW& w, const MomIn& in, const MomTerms2& t, int32_t* a0,
                                            int32_t* a1, int32_t* a2) {
    const float dxi = t.dxs[I], dyj = t.dys[J];
    const float2 dx2 = make_float2(dxi, dxi), dy2 = make_float2(dyj, dyj);
    // (a00 dxi + a01 dyj, a10 dxi + a11 dyj) and (s00 dxi + s01 dyj, s01 dxi + s11 dyj)
    const float2 qxy = padd(smul(t.axy0, dx2), smul(t.axy1, dy2));
    const float qzz = t.a20 * dxi + t.a21 * dyj;
    const float2 gxy = padd(smul(t.sxy0, dx2), smul(t.sxy1, dy2));
    const float gz = t.s02 * dxi + t.s12 * dyj;
    mom_cell2<kClamp, 0, J, I>(w, in, t, qxy, qzz, gxy, gz, a0, a1, a2);
    mom_cell2<kClamp, 1, J, I>(w, in, t, qxy, qzz, gxy, gz, a0, a1, a2);
    mom_cell2<kClamp, 2, J, I>(w, in, t, qxy, qzz, gxy, gz, a0, a1, a2);
}

template <bool kClamp>
__device__ __forceinline__ void mom_contrib_shared2(const PW& w, const MomIn& in, const float* s, float coef,
                                                    int32_t (*acc)[kHaloCells], int hb) {
    MomTerms2 t;
    const float s00 = s[0], s11 = s[1], s22 = s[2], s01 = s[3], s02 = s[4], s12 = s[5];
    t.dxs[0] = -w.fx - 1.0f; t.dxs[1] = -w.fx; t.dxs[2] = 1.0f - w.fx;
    t.dys[0] = -w.fy - 1.0f; t.dys[1] = -w.fy; t.dys[2] = 1.0f - w.fy;
    const float dzs[3] = {-w.fz - 1.0f, -w.fz, 1.0f - w.fz};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float2 dz2 = make_float2(dzs[k], dzs[k]);
        t.qz2[k] = smul(make_float2(in.a02, in.a12), dz2);   // scalar: each feeds paired adds
        t.qzz[k] = in.a22 * dzs[k];
        t.fz2[k] = smul(make_float2(s02, s12), dz2);
        t.fzz[k] = s22 * dzs[k];
    }
    t.axy0 = make_float2(in.a00, in.a10);
    t.axy1 = make_float2(in.a01, in.a11);
    t.sxy0 = make_float2(s00, s01);
    t.sxy1 = make_float2(s01, s11);
    t.a20 = in.a20; t.a21 = in.a21; t.s02 = s02; t.s12 = s12; t.coef = coef;
    t.vxy = make_float2(in.vx, in.vy);
    t.mm = make_float2(in.m, in.m);
    t.cc = make_float2(coef, coef);
    int32_t* a0 = &acc[0][hb];
    int32_t* a1 = &acc[1][hb];
    int32_t* a2 = &acc[2][hb];
    mom_column2<kClamp, 0, 0>(w, in, t, a0, a1, a2);
    mom_column2<kClamp, 0, 1>(w, in, t, a0, a1, a2);
    mom_column2<kClamp, 0, 2>(w, in, t, a0, a1, a2);
    mom_column2<kClamp, 1, 0>(w, in, t, a0, a1, a2);
    mom_column2<kClamp, 1, 1>(w, in, t, a0, a1, a2);
    mom_column2<kClamp, 1, 2>(w, in, t, a0, a1, a2);
    mom_column2<kClamp, 2, 0>(w, in, t, a0, a1, a2);
    mom_column2<kClamp, 2, 1>(w, in, t, a0, a1, a2);
    mom_column2<kClamp, 2, 2>(w, in, t, a0, a1, a2);
}
#endif

// Density of one particle from the staged halo masses (shaders.js:305-313):
// the reference's k, j, i summation order, written out through template
// indices.
template <int K, int J, int I>
__device__ __forceinline__ void density_term(const PW& w, const float* m, float& d) {
    d += w.wx[I] * w.wy[J] * w.wz[K] * m[K * kHXY + J * kHX + I];
}
template <int K, int J>
__device__ __forceinline__ void density_row(const PW& w, const float* m, float& d) {
    density_term<K, J, 0>(w, m, d);
    density_term<K, J, 1>(w, m, d);
    density_term<K, J, 2>(w, m, d);
}
__device__ __forceinline__ float density_shared(const PW& w, const float* m) {
    float d = 0.0f;
    density_row<0, 0>(w, m, d);
    density_row<0, 1>(w, m, d);
    density_row<0, 2>(w, m, d);
    density_row<1, 0>(w, m, d);
    density_row<1, 1>(w, m, d);
    density_row<1, 2>(w, m, d);
    density_row<2, 0>(w, m, d);
    density_row<2, 1>(w, m, d);
    density_row<2, 2>(w, m, d);
    return d;
}

// P2G_MOM for one particle whose inputs are loaded.
__device__ __forceinline__ void mom_particle(const WorldView& v, const ChunkHdr& h, const SceneDesc& sd, bool valid,
                                             uint32_t p, const float4 pm, const float4 vi, const float* a,
                                             const float* mh, int32_t (*acc)[kHaloCells],
                                             const float* __restrict__ scmf, int32_t* __restrict__ smv,
                                             float* __restrict__ dens, uint32_t* __restrict__ health) {
    const uint32_t X = sd.X, SLICE = sd.X * sd.Y, G = sd.G;
    const PW w = particle_weights(pm.x, pm.y, pm.z);
    const bool fast = valid && in_halo(w, h, sd);
    const int hb = halo_base(h, w.cx, w.cy, w.cz);
    const uint32_t baseIdx = (uint32_t)(((w.cz - 1) * (int32_t)sd.Y + (w.cy - 1)) * (int32_t)X + (w.cx - 1));
    // density (shaders.js:305-313), k, j, i order
    float density = 0.0f;
    if (fast) {
        density = density_shared(w, mh + hb);
    } else if (valid) {
        for (int k = 0; k < 3; ++k)
            for (int jj = 0; jj < 3; ++jj)
                for (int i = 0; i < 3; ++i) {
                    const uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)jj * X + (uint32_t)i;
                    const float cmass = cidx < G ? scmf[cidx] : 0.0f;
                    density += w.wx[i] * w.wy[jj] * w.wz[k] * cmass;
                }
    }
    if (valid) dens[p] = density;
    const bool live = valid && density > 1e-8f;   // shaders.js:315
    // stress (shaders.js:325-338)
    const float rest = sd.P.rest_density;
    const MomIn in{vi.x, vi.y, vi.z, pm.w, a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8]};
    const float vol = __fdiv_rn(in.m, fmaxf(density, rest * 0.15f));
    float pressure = sd.P.stiffness * (eos_pow(__fdiv_rn(density, rest), sd.P.eos_power) - 1.0f);
    const float pFloor = density > rest * kCohesionGate ? kCohesionPressure : 0.0f;
    pressure = fmaxf(pressure, pFloor);
    const float visc = sd.P.viscosity;
    float s[6];
    s[0] = -pressure + visc * (in.a00 + in.a00);
    s[1] = -pressure + visc * (in.a11 + in.a11);
    s[2] = -pressure + visc * (in.a22 + in.a22);
    s[3] = visc * (in.a01 + in.a10);
    s[4] = visc * (in.a02 + in.a20);
    s[5] = visc * (in.a12 + in.a21);
    const float coef = -vol * 4.0f * sd.P.dt;
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
    // health: the bound says encode's clamp may engage (a contribution may reach 20000)
    if (live && !safe) atomicOr(health, MPM_HEALTH_SATURATED);
    if (live && fast) {
#if MPM_MOM_PACKED
        if (safe) mom_contrib_shared2<false>(w, in, s, coef, acc, hb);
        else mom_contrib_shared2<true>(w, in, s, coef, acc, hb);
#else
        if (safe) mom_contrib_shared<false>(w, in, s, coef, acc, hb);
        else mom_contrib_shared<true>(w, in, s, coef, acc, hb);
#endif
    } else if (live) {
        auto sink = [&](int k, int j, int i, int32_t ex, int32_t ey, int32_t ez) {
            const uint32_t cidx = baseIdx + (uint32_t)k * SLICE + (uint32_t)j * X + (uint32_t)i;
            if (cidx < G) {
                atomicAdd(smv + 3ull * cidx + 0, ex);
                atomicAdd(smv + 3ull * cidx + 1, ey);
                atomicAdd(smv + 3ull * cidx + 2, ez);
            }
        };
        mom_contrib<true>(w, in, s, coef, sink);
    }
}

#ifndef MPM_G2P_MINB
#define MPM_G2P_MINB 4
#endif

#ifndef MPM_MOM_MINB
#define MPM_MOM_MINB 2
#endif

// P2G_MOM, software-pipelined across the block's chunks: while chunk c runs,
// the halo masses of the block's next chunk are copied into the other
// staging buffer (cp.async) and its first particle's inputs are loaded; the
// accumulators are zeroed by the flush that reads them.
__device__ __forceinline__ void stage_masses_async(const WorldView& v, const ChunkHdr& hh,
                                                   const float* __restrict__ cmf, float* buf) {
    const SceneDesc& nsd = v.scenes[hh.scene];
    const float* src = cmf + nsd.cell_base;
    const int hn = halo_span(hh);
    for (int i = threadIdx.x; i < hn; i += blockDim.x) {
        uint32_t cell;
        const bool in = halo_cell(hh, nsd, i, cell);
        cp_async4z(buf + i, in ? (const void*)(src + cell) : (const void*)src, in ? 4u : 0u);
    }
}

__device__ __forceinline__ void mom_load(const WorldView& v, uint32_t p, bool valid, const float4* __restrict__ posm,
                                         const float4* __restrict__ velid, const float* __restrict__ aff,
                                         size_t plane, float4& pm, float4& vi, float* a) {
    const uint32_t slot = valid ? v.perm[p] : 0u;
    if (valid) {
        pm = posm[slot];
        vi = velid[slot];
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) a[e] = valid ? aff[e * plane + slot] : 0.0f;
}

template <uint32_t kC>
__global__ void __launch_bounds__(kChunkThreads, MPM_MOM_MINB) k_p2g_mom_chunks(WorldView v, const float4* __restrict__ posm,
                                                                   const float4* __restrict__ velid,
                                                                   const float* __restrict__ aff,
                                                                   const float* __restrict__ cmf,
                                                                   int32_t* __restrict__ mv,
                                                                   float* __restrict__ dens) {
    constexpr int kPer = kC / kChunkThreads;
    __shared__ float mh[2][kHaloCells];
    __shared__ int32_t acc[3][kHaloCells];
    __shared__ ChunkHdr hdr[2];
    // the scene descriptors of the current chunk and of the next one, which is
    // copied while the current chunk runs (no wait when the scene changes)
    __shared__ SceneDesc ssd[2];
    const uint32_t nch = v.ctrl->total_chunks;
    const uint32_t G = gridDim.x;
    if (blockIdx.x >= nch) return;   // block-uniform
    const size_t plane = v.npos;
    uint4 nh0 = make_uint4(0u, 0u, 0u, 0u), nh1 = nh0;   // thread 0: the words of the chunk two ahead
    if (threadIdx.x == 0) {
        const uint32_t c0 = blockIdx.x, c1 = c0 + G;
        hdr[0] = unpack_header(v.chunk_hdr[2ull * c0], v.chunk_hdr[2ull * c0 + 1]);
        if (c1 < nch) hdr[1] = unpack_header(v.chunk_hdr[2ull * c1], v.chunk_hdr[2ull * c1 + 1]);
    }
    for (int i = threadIdx.x; i < kHaloCells; i += blockDim.x) {
        acc[0][i] = 0;
        acc[1][i] = 0;
        acc[2][i] = 0;
    }
    __syncthreads();
    copy_scene_async(v, hdr[0].scene, ssd[0]);
    uint32_t ss_cur = hdr[0].scene, ss_nxt = kHole;   // scenes held in ssd[b], ssd[b ^ 1]
    stage_masses_async(v, hdr[0], cmf, mh[0]);
    // the first particle's inputs
    uint32_t p = hdr[0].first + chunk_slot<kC>(0);
    bool valid = p < hdr[0].end;
    float4 pm = make_float4(0.0f, 0.0f, 0.0f, 0.0f), vi = pm;
    float a[9];
    mom_load(v, p, valid, posm, velid, aff, plane, pm, vi, a);
    cp_async_wait();
    __syncthreads();
    int b = 0;
    for (uint32_t ch = blockIdx.x; ch < nch; ch += G) {
        const ChunkHdr h = hdr[b];
        const uint32_t nxt = ch + G, nxt2 = nxt + G;
        if (threadIdx.x == 0 && nxt2 < nch) {
            nh0 = v.chunk_hdr[2ull * nxt2];
            nh1 = v.chunk_hdr[2ull * nxt2 + 1];
        }
        const SceneDesc& sd = ssd[b];
        const float* scmf = cmf + sd.cell_base;
        int32_t* smv = mv + 3ull * sd.cell_base;
        // the next chunk's halo masses (and scene descriptor), copied while this chunk runs
        const bool has_next = nxt < nch;
        if (has_next) {
            stage_masses_async(v, hdr[b ^ 1], cmf, mh[b ^ 1]);
            const uint32_t ns = hdr[b ^ 1].scene;
            if (ns != ss_nxt) {
                copy_scene_async(v, ns, ssd[b ^ 1]);
                ss_nxt = ns;
            }
        }
        const uint32_t next_first = has_next ? hdr[b ^ 1].first : 0u, next_end = has_next ? hdr[b ^ 1].end : 0u;
#pragma unroll 1
        for (int r = 0; r < kPer; ++r) {
            // inputs of this thread's next particle: the next one of this
            // chunk, or the first one of the block's next chunk
            uint32_t pn;
            bool vn;
            if (r + 1 < kPer) {
                pn = p + (chunk_slot<kC>(1) - chunk_slot<kC>(0));   // the pass stride
                vn = pn < h.end;
            } else {
                pn = next_first + chunk_slot<kC>(0);
                vn = has_next && pn < next_end;
            }
            float4 pmn = make_float4(0.0f, 0.0f, 0.0f, 0.0f), vin = pmn;
            float an[9];
            mom_load(v, pn, vn, posm, velid, aff, plane, pmn, vin, an);
            mom_particle(v, h, sd, valid, p, pm, vi, a, mh[b], acc, scmf, smv, dens, v.health + h.scene);
            p = pn;
            valid = vn;
            pm = pmn;
            vi = vin;
#pragma unroll
            for (int e = 0; e < 9; ++e) a[e] = an[e];
        }
        __syncthreads();
        // hdr[b] is free: the header two chunks ahead goes there
        if (threadIdx.x == 0 && nxt2 < nch) hdr[b] = unpack_header(nh0, nh1);
        const int hn = halo_span(h);
        for (int i = threadIdx.x; i < hn; i += blockDim.x) {
            const int32_t a0 = acc[0][i], a1 = acc[1][i], a2 = acc[2][i];
            if ((a0 | a1 | a2) == 0) continue;
            acc[0][i] = 0;
            acc[1][i] = 0;
            acc[2][i] = 0;
            uint32_t cell;
            if (halo_cell(h, sd, i, cell)) {
                int32_t* d = smv + 3ull * cell;
                if (a0) atomicAdd(d + 0, a0);
                if (a1) atomicAdd(d + 1, a1);
                if (a2) atomicAdd(d + 2, a2);
            }
        }
        cp_async_wait();
        __syncthreads();
        b ^= 1;
        const uint32_t t = ss_cur;
        ss_cur = ss_nxt;
        ss_nxt = t;
    }
}

// ---------------------------------------------------------------------------
// G2P (shaders.js:579-705): one block per chunk, one thread per particle,
// + binning of the new positions and the diffuse spawn decision (shaders.js:800-855).
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

// Out-of-line functions for G2P's rare paths (keeps their registers out of
// the common path).
#define MPM_G2P_RARE __noinline__
// The spawn test's terms that need no neighbour data (shaders.js:807-815):
// speed, kinetic energy and trapped air.
struct SpawnPre {
    float speed, ke, trappedAir;
};

__device__ __forceinline__ SpawnPre spawn_pre(f3 vel, float m, float density, const SceneDesc& sd,
                                              float pressure_threshold) {
    SpawnPre r;
    const float speed2 = dot3(vel, vel);
    r.speed = __fsqrt_rn(speed2);
    r.ke = 0.5f * m * speed2;
    const float rest = sd.P.rest_density;
    float pressure = sd.P.stiffness * (eos_pow(__fdiv_rn(density, rest), sd.P.eos_power) - 1.0f);
    const float pFloor = density > rest * kCohesionGate ? kCohesionPressure : 0.0f;
    pressure = fmaxf(pressure, pFloor);
    r.trappedAir = fmaxf(0.0f, pressure - pressure_threshold);
    return r;
}

// True when the score cannot reach ke_threshold whatever the wave-crest term:
// that term is dotVal * speed with dotVal the dot product of two unit vectors
// (below 1.0001 after rounding), and every operation is rounded monotonically,
// so the score evaluated with 1.0001 * speed in its place bounds the real one.
__device__ __forceinline__ bool spawn_hopeless(const SpawnPre& s, float ke_threshold) {
    return (s.ke + s.trappedAir * 2.0f) + (1.0001f * s.speed) * 1.5f < ke_threshold;
}

// Spawn decision + staging (shaders.js:800-855) of a particle that passed the
// density and score-bound tests.  Inline: as an out-of-line call its register
// saves cost the common path more (G2P 78.0 vs 75.2 us at 1M particles) than
// the inlined code does.
__device__ __forceinline__ void spawn_eval(uint32_t id, f3 np, f3 nv, float density, SpawnPre pre,
                                        const SceneDesc& sd, const float* __restrict__ cmf,
                                        const mpm_gen_params* __restrict__ genp,
                                        mpm_diffuse_particle* __restrict__ staging,
                                        uint32_t* __restrict__ spawn_bits, uint32_t* __restrict__ group_counts) {
    const mpm_gen_params& gen = *genp;
    const f3 vel = nv;
    const float speed = pre.speed, ke = pre.ke, trappedAir = pre.trappedAir;
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
    staging[id] = r;
    atomicOr(&spawn_bits[id >> 5], 1u << (id & 31u));
    atomicAdd(&group_counts[id / kGroupIds], 1u);
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

// G2P gather for a particle whose stencil leaves the halo box or the grid:
// the reference's linear stencil index with a bounds guard.
struct G2PSum {
    float gv[3];
    float B[9];
};

// Returned by value: a pointer to the caller's accumulators would keep them
// in local memory on the common (halo) path too.
__device__ MPM_G2P_RARE G2PSum g2p_gather_direct(const PW w, const float4 q, const float4* __restrict__ vel4,
                                                 uint32_t X, uint32_t Y, uint32_t G) {
    G2PSum r;
    float& gvx = r.gv[0];
    float& gvy = r.gv[1];
    float& gvz = r.gv[2];
    float* B = r.B;
    gvx = gvy = gvz = 0.0f;
#pragma unroll
    for (int e = 0; e < 9; ++e) B[e] = 0.0f;
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
                    const float4 c = vel4[cidx];
                    cvx = c.x; cvy = c.y; cvz = c.z;
                }
                const float wvx = ww * cvx, wvy = ww * cvy, wvz = ww * cvz;
                gvx += wvx; gvy += wvy; gvz += wvz;
                B[0] += wvx * dxi; B[1] += wvx * dyj; B[2] += wvx * dzk;
                B[3] += wvy * dxi; B[4] += wvy * dyj; B[5] += wvy * dzk;
                B[6] += wvz * dxi; B[7] += wvz * dyj; B[8] += wvz * dzk;
            }
        }
    }
    return r;
}


// Where G2P writes: the new state, the binning key and tile marks, and the
// diffuse spawn staging.
struct G2POut {
    float4* posm;
    float4* velid;
    float* aff;
    size_t plane;
    uint32_t* key;
    uint32_t* rank;
    uint32_t* cell_count;
    uint32_t* tile_flags;
    const float* dens;
    const float* cmf;                    // scene's decoded cell masses
    const mpm_gen_params* gen;           // null: no spawning for this scene
    float bubble_min;                    // gen->density_bubble_min
    float pressure_threshold;            // gen->pressure_threshold
    float ke_threshold;                  // gen->ke_threshold
    mpm_diffuse_particle* staging;
    uint32_t* spawn_bits;
    uint32_t* group_counts;
};

// G2P epilogue of one particle (shaders.js:631-700): affine, advection and
// boundary handling, the new state at position p, its binning key and tile
// mark, and the diffuse spawn decision.  Returns the particle's rank within
// its new binning cell (the caller stores it at rank[p], as late as it can,
// so the atomic's round trip overlaps later work).
__device__ __forceinline__ uint32_t g2p_store(const G2POut& o, const SceneDesc& sd, uint32_t p, const float4 q,
                                              const float4 vi, float density, float gvx, float gvy, float gvz,
                                              const float* B, const RefOut& ro, bool mirror) {
#pragma unroll
    for (int e = 0; e < 9; ++e) o.aff[e * o.plane + p] = B[e] * 4.0f;
    f3 np, nv;
    g2p_finish(q, gvx, gvy, gvz, sd.P, sd.W, np, nv);
    o.posm[p] = make_float4(np.x, np.y, np.z, q.w);
    o.velid[p] = make_float4(nv.x, nv.y, nv.z, vi.w);
    if (mirror) {   // particle_pos/vel (shaders.js:703-704) and particle_density (shaders.js:314) by id
        const uint32_t id = __float_as_uint(vi.w) - sd.id_base;
        if (id < sd.n) {
#if MPM_MIRROR_KEEP
            // the scattered 16- and 4-byte writes by id fill 32-byte sectors
            // half or an eighth at a time: an evict-last hint keeps their L2
            // lines until the rest of each sector has been written
            uint64_t pol;
// share of the mirror lines given the evict-last priority (the rest keep
// their place): G2P with the mirrors 87.4 / 84.3 / 84.1 us at 1M for 1.0 /
// 0.75 / 0.5, and 490 / 492 / 495 us at 8M
#ifndef MPM_MIRROR_FRAC
#define MPM_MIRROR_FRAC "0.75"
#endif
            asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, " MPM_MIRROR_FRAC ";" : "=l"(pol));
            asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(ro.pos + id), "f"(np.x),
                         "f"(np.y), "f"(np.z), "f"(0.0f), "l"(pol) : "memory");
            asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(ro.vel + id), "f"(nv.x),
                         "f"(nv.y), "f"(nv.z), "f"(0.0f), "l"(pol) : "memory");
            asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(ro.dens + id), "f"(density), "l"(pol)
                         : "memory");
#else
            ro.pos[id] = make_float4(np.x, np.y, np.z, 0.0f);
            ro.vel[id] = make_float4(nv.x, nv.y, nv.z, 0.0f);
            ro.dens[id] = density;
#endif
        }
    }
    // binning of the new position
    int32_t cx, cy, cz;
    bin_cell(sd, np.x, np.y, np.z, cx, cy, cz);
    const uint32_t key = sd.cell_base + local_cell(sd, cx, cy, cz);
    o.key[p] = key;
    // the rank within the cell for the next substep's binning (k_count's work)
    const uint32_t rank = atomicAdd(&o.cell_count[key], 1u);
    // occupied-tile mark: one fire-and-forget OR per distinct tile of the
    // active lanes (consecutive positions mostly share one tile)
    {
        const uint32_t t = tile_of(sd, cx, cy, cz);
        const unsigned act = __activemask();
        const unsigned same = __match_any_sync(act, t);
        if ((threadIdx.x & 31u) == (uint32_t)(__ffs(same) - 1)) atomicOr(&o.tile_flags[t], 1u);
    }
    if (o.gen) {
        const uint32_t id = __float_as_uint(vi.w) - sd.id_base;
        // spawn_record's first test (shaders.js:806), checked inline
        if (id < sd.n && density > 0.0f && density <= o.bubble_min) {
            const SpawnPre pre = spawn_pre(nv, q.w, density, sd, o.pressure_threshold);
            if (!spawn_hopeless(pre, o.ke_threshold))
                spawn_eval(id, np, nv, density, pre, sd, o.cmf, o.gen, o.staging, o.spawn_bits, o.group_counts);
        }
    }
    return rank;
}

// G2P of a particle whose stencil leaves the halo box or the grid (rare): the
// reference's linear stencil index with a bounds guard, then the epilogue.
__device__ __noinline__ void g2p_direct_particle(const G2POut o, const SceneDesc* sdp, uint32_t p, const float4 q,
                                                 const float4 vi, const float4* __restrict__ vel4, const RefOut ro,
                                                 bool mirror) {
    const SceneDesc& sd = *sdp;
    const PW w = particle_weights(q.x, q.y, q.z);
    const G2PSum r = g2p_gather_direct(w, q, vel4, sd.X, sd.Y, sd.G);
    o.rank[p] = g2p_store(o, sd, p, q, vi, o.dens[p], r.gv[0], r.gv[1], r.gv[2], r.B, ro, mirror);
}

#if MPM_G2P_PACKED
// The 27-cell gather of G2P (shaders.js:606-629) with the x and y lanes of
// each accumulation paired: (gvx, gvy), (B00, B10), (B01, B11), (B02, B12),
// (B20, B21); every element keeps the reference's products and summation
// order.  vb: the staged halo at the stencil base.
__device__ __forceinline__ void g2p_gather_packed(const PW& w, const float4 q, const float4* vb, float& gvx,
                                                  float& gvy, float& gvz, float* B) {
    const int32_t bx = w.cx - 1, by = w.cy - 1, bz = w.cz - 1;
    float2 gxy = make_float2(0.0f, 0.0f), b0 = gxy, b1 = gxy, b2 = gxy, b3 = gxy;
    float gz = 0.0f, b22 = 0.0f;
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
                const float4 c = vb[k * kHXY + jj * kHX + i];
                const float2 wvxy = pmul(make_float2(ww, ww), make_float2(c.x, c.y));
                const float wvz = ww * c.z;
                gxy = sadd(gxy, wvxy);
                gz += wvz;
                b0 = sadd(b0, pmul(wvxy, make_float2(dxi, dxi)));
                b1 = sadd(b1, pmul(wvxy, make_float2(dyj, dyj)));
                b2 = sadd(b2, pmul(wvxy, make_float2(dzk, dzk)));
                b3 = padd(b3, smul(make_float2(wvz, wvz), make_float2(dxi, dyj)));
                b22 += wvz * dzk;
            }
        }
    }
    gvx = gxy.x; gvy = gxy.y; gvz = gz;
    B[0] = b0.x; B[1] = b1.x; B[2] = b2.x;
    B[3] = b0.y; B[4] = b1.y; B[5] = b2.y;
    B[6] = b3.x; B[7] = b3.y; B[8] = b22;
}
#endif

template <uint32_t kC>
__global__ void __launch_bounds__(kChunkThreads, MPM_G2P_MINB) k_g2p_chunks(WorldView v, const float4* __restrict__ posm,
                                                              const float4* __restrict__ velid,
                                                              const float4* __restrict__ vel4,
                                                              const float* __restrict__ cmf,
                                                              float4* __restrict__ posm_out,
                                                              float4* __restrict__ velid_out,
                                                              float* __restrict__ aff_out, DiffuseView dv,
                                                              RefOut ro) {
    constexpr int kPer = kC / kChunkThreads;
    __shared__ float4 vh[kHaloCells];   // staged grid velocities (x, y, z, 0)
    __shared__ uint4 nhs[2];              // the next chunk's header words
    const uint32_t nch = v.ctrl->total_chunks;
    const size_t plane = v.npos;
    __shared__ ChunkHdr hs;
    // scene descriptors of this chunk and the next (thread 0 copies the next
    // one while this chunk runs)
    __shared__ SceneDesc ssd[2];
    int sb = 0;                 // ssd[sb]: this chunk's scene
    uint32_t ss_nxt = kHole;    // thread 0: scene held in ssd[sb ^ 1]
    // rank of the last particle whose atomic is still in flight
    uint32_t pend_p = kHole, pend_rank = 0;
    const float bubble_min = dv.enabled ? dv.gen->density_bubble_min : 0.0f;
    const float pressure_threshold = dv.enabled ? dv.gen->pressure_threshold : 0.0f;
    const float ke_threshold = dv.enabled ? dv.gen->ke_threshold : 0.0f;
    // the per-substep counters of the binning and the grid passes are read
    // no more in this substep: clear them for the next one
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        v.ctrl->n_occ = 0u;
        v.ctrl->n_grid = 0u;
        v.ctrl->bins_done = 0u;
    }
    // chunk headers: the next one's words are copied while this chunk runs
    if (threadIdx.x == 0 && blockIdx.x < nch) {
        hs = unpack_header(v.chunk_hdr[2ull * blockIdx.x], v.chunk_hdr[2ull * blockIdx.x + 1]);
        copy_scene_async_one(v, hs.scene, ssd[0]);
        cp_async_wait();
    }
    __syncthreads();
    for (uint32_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
        const ChunkHdr h = hs;
        const uint32_t nxt = ch + gridDim.x;
        if (threadIdx.x == 0 && nxt < nch) {
            cp_async16(&nhs[0], v.chunk_hdr + 2ull * nxt, 16u);
            cp_async16(&nhs[1], v.chunk_hdr + 2ull * nxt + 1, 16u);
        }
        const SceneDesc& sd = ssd[sb];
        // this thread's particles, in flight while the halo is staged
        float4 qs[kPer];
        float ids[kPer], dns[kPer];
#pragma unroll
        for (int r = 0; r < kPer; ++r) {
            const uint32_t p = h.first + r * kChunkThreads + threadIdx.x;
            qs[r] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            ids[r] = 0.0f;
            dns[r] = 0.0f;
            if (p < h.end) {
                const uint32_t slot = v.perm[p];
                qs[r] = posm[slot];
                ids[r] = velid[slot].w;
                dns[r] = v.dens[p];
            }
        }
        const int hn = halo_span(h);
        const float4* svel = vel4 + sd.cell_base;
        for (int i = threadIdx.x; i < hn; i += blockDim.x) {
            uint32_t cell;
            const bool in = halo_cell(h, sd, i, cell);
            cp_async16(&vh[i], in ? (const void*)(svel + cell) : (const void*)svel, in ? 16u : 0u);
        }
        cp_async_wait();
        __syncthreads();
        // every thread holds this chunk's header: the next one can replace it
        if (threadIdx.x == 0 && nxt < nch) {
            cp_async_wait();
            hs = unpack_header(nhs[0], nhs[1]);
            if (hs.scene != ss_nxt) {
                copy_scene_async_one(v, hs.scene, ssd[sb ^ 1]);
                ss_nxt = hs.scene;
            }
        }
        const bool spawn_scene = dv.enabled && h.scene == dv.scene;
        const bool mirror = ro.enabled && h.scene == ro.scene;
        const G2POut out{posm_out, velid_out, aff_out, plane, v.key, v.rank, v.cell_count, v.tile_flags, v.dens,
                         cmf + sd.cell_base, spawn_scene ? dv.gen : nullptr, bubble_min, pressure_threshold,
                         ke_threshold, dv.staging, dv.spawn_bits, dv.group_counts};
#pragma unroll 1
        for (int r = 0; r < kPer; ++r) {
            const uint32_t p = h.first + r * kChunkThreads + threadIdx.x;
            if (p >= h.end) break;
            const float4 q = qs[r];
            const float4 vi = make_float4(0.0f, 0.0f, 0.0f, ids[r]);
            const PW w = particle_weights(q.x, q.y, q.z);
            if (!in_halo(w, h, sd)) {
                g2p_direct_particle(out, &sd, p, q, vi, svel, ro, mirror);
                continue;
            }
            float gvx = 0.0f, gvy = 0.0f, gvz = 0.0f;
            float B[9] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
#if MPM_G2P_PACKED
            g2p_gather_packed(w, q, vh + halo_base(h, w.cx, w.cy, w.cz), gvx, gvy, gvz, B);
#else
            {
                const int32_t bx = w.cx - 1, by = w.cy - 1, bz = w.cz - 1;
                const int hb = halo_base(h, w.cx, w.cy, w.cz);
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
                            const float4 c = vh[hb + k * kHXY + jj * kHX + i];
                            const float wvx = ww * c.x, wvy = ww * c.y, wvz = ww * c.z;
                            gvx += wvx; gvy += wvy; gvz += wvz;
                            B[0] += wvx * dxi; B[1] += wvx * dyj; B[2] += wvx * dzk;
                            B[3] += wvy * dxi; B[4] += wvy * dyj; B[5] += wvy * dzk;
                            B[6] += wvz * dxi; B[7] += wvz * dyj; B[8] += wvz * dzk;
                        }
                    }
                }
            }
#endif
            const uint32_t rk = g2p_store(out, sd, p, q, vi, dns[r], gvx, gvy, gvz, B, ro, mirror);
            // the previous particle's rank: its atomic has long returned
            if (pend_p != kHole) v.rank[pend_p] = pend_rank;
            pend_p = p;
            pend_rank = rk;
        }
        if (threadIdx.x == 0) {
            cp_async_wait();      // the next chunk's scene descriptor
            ss_nxt = h.scene;     // after the swap ssd[sb ^ 1] holds this chunk's scene
        }
        __syncthreads();
        sb ^= 1;
    }
    if (pend_p != kHole) v.rank[pend_p] = pend_rank;
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
    // every occupied tile has at most one partial chunk
    w.chunk_cap = w.npos / kChunkSmall + w.tile_cap + 1;   // room for the smaller chunks
}

// Every device array of a world with its size (one list for allocation,
// release and the footprint).
template <class F> static void world_arrays(World& w, F&& f) {
    const size_t P = w.npos, C = w.cell_cap ? w.cell_cap : 1, T = w.tile_cap;
    const size_t NG = (T + 1023) / 1024 + 1;
    for (int b = 0; b < 2; ++b) {
        f(w.posm[b], P * 16);
        f(w.velid[b], P * 16);
        f(w.aff[b], P * 36);
        f(w.grid_i32[b], C * 16);
    }
    f(w.dens, P * 4);
    f(w.cell_count, (C + 1) * 4);
    f(w.cell_start, C * 4);
    f(w.key, P * 4);
    f(w.rank, P * 4);
    f(w.perm, P * 4);
    f(w.tile_flags, T * 4);
    f(w.tile_occ, T * 4);
    f(w.tile_cnt, T * 4);
    f(w.tile_pstart, T * 4);
    f(w.tile_cstart, T * 4);
    f(w.group_pstart, NG * 4);
    f(w.group_cstart, NG * 4);
    f(w.chunk_info, (size_t)w.chunk_cap * 16);
    f(w.chunk_last, (size_t)w.chunk_cap * 4);
    f(w.chunk_hdr, (size_t)w.chunk_cap * 32);
    f(w.chunk_geo, (size_t)w.chunk_cap * 16);
    f(w.tile_occ_list, T * 4);
    f(w.tile_grid_list, T * 4);
    f(w.tile_scene, T * 4);
    f(w.ctrl, sizeof(Ctrl));
    f(w.cmf, C * 4);
    f(w.mvf, C * 12);
    f(w.vel4, C * 16);
    f(w.d_scenes, 2 * (size_t)w.scene_cap * sizeof(SceneDesc));
    f(w.health, (size_t)(w.scene_cap ? w.scene_cap : 1) * 4);
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
    w.item_blocks = (uint32_t)sms * 4;
    w.grid_blocks = (uint32_t)sms * 8;
    w.bin_blocks = (uint32_t)sms * 2;
    w.pos_blocks = std::min<uint32_t>(cdiv(w.npos, 256), (uint32_t)sms * 16);
    const size_t P = w.npos, C = cell_cap ? cell_cap : 1, T = w.tile_cap;
    cudaError_t e = cudaSuccess;
    w.device_bytes = 0;
    world_arrays(w, [&](auto*& p, size_t bytes) {
        if (e == cudaSuccess) e = dmalloc(&p, bytes);
        if (e == cudaSuccess) w.device_bytes += bytes;
    });
    if (e != cudaSuccess) return e;
    w.h_scenes.assign(scene_cap, SceneDesc{});
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        e = cudaMallocHost((void**)&w.h_stage[b], (size_t)scene_cap * sizeof(SceneDesc));
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w.stage_ev[b], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w.sub_done[b], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&w.tbl_side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w.tbl_ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
    w.h_tile_scene.assign(T, kHole);
    // zero everything the sparse passes rely on being zero
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) e = cudaMemsetAsync(w.grid_i32[b], 0, C * 16, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.cmf, 0, C * 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.mvf, 0, C * 12, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.vel4, 0, C * 16, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.cell_count, 0, (C + 1) * 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.tile_flags, 0, T * 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.tile_occ, 0, T * 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.dens, 0, P * 4, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.ctrl, 0, sizeof(Ctrl), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.health, 0, (size_t)(scene_cap ? scene_cap : 1) * 4, stream);
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
    if (w.tbl_side) cudaStreamSynchronize(w.tbl_side);
    for (int b = 0; b < 2; ++b) {
        if (w.h_stage[b]) cudaFreeHost(w.h_stage[b]);
        if (w.stage_ev[b]) cudaEventDestroy(w.stage_ev[b]);
        if (w.sub_done[b]) cudaEventDestroy(w.sub_done[b]);
        w.h_stage[b] = nullptr;
        w.stage_ev[b] = nullptr;
        w.sub_done[b] = nullptr;
    }
    if (w.tbl_ev) cudaEventDestroy(w.tbl_ev);
    if (w.tbl_side) cudaStreamDestroy(w.tbl_side);
    for (int b = 0; b < World::kGraphs; ++b)
        if (w.graph[b]) cudaGraphExecDestroy(w.graph[b]);
    world_arrays(w, [](auto*& p, size_t) {
        dfree(p);
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

static int table_entries(const World& w) {
    int hi = 0;
    for (int i = 0; i < (int)w.scene_cap; ++i)
        if (w.scenes[i].live) hi = i + 1;
    return hi;
}

// The host table from the scene records, when they changed: both device
// copies are then behind.
static void refresh_host_table(World& w) {
    if (!w.table_dirty) return;
    const int hi = table_entries(w);
    for (int i = 0; i < hi; ++i) fill_desc(w, i);
    w.table_dirty = false;
    w.tbl_dirty[0] = w.tbl_dirty[1] = true;
}

// Copies the host table into device copy c on stream st, through pinned
// staging (an upload from pageable memory would first wait for all work
// queued on the stream); a staging buffer is reused only once the copy that
// last read it has run.
static cudaError_t upload_copy(World& w, int c, cudaStream_t st) {
    const int hi = table_entries(w);
    cudaError_t e = cudaSuccess;
    if (hi) {
        const int b = w.stage_i;
        w.stage_i ^= 1;
        e = cudaEventSynchronize(w.stage_ev[b]);
        if (e == cudaSuccess) {
            std::memcpy(w.h_stage[b], w.h_scenes.data(), (size_t)hi * sizeof(SceneDesc));
            e = cudaMemcpyAsync(w.scenes_dev(c), w.h_stage[b], (size_t)hi * sizeof(SceneDesc),
                                cudaMemcpyHostToDevice, st);
        }
        if (e == cudaSuccess) e = cudaEventRecord(w.stage_ev[b], st);
    }
    if (e == cudaSuccess) w.tbl_dirty[c] = false;
    return e;
}

// Outside a substep: both copies in stream order, so the kernels about to be
// launched and every later substep see the current table.
cudaError_t world_upload_table(World& w) {
    refresh_host_table(w);
    cudaError_t e = cudaSuccess;
    for (int c = 0; c < 2 && e == cudaSuccess; ++c)
        if (w.tbl_dirty[c]) {
            e = upload_copy(w, c, w.stream);
            if (e == cudaSuccess) w.tbl_outside[c] = false;
        }
    return e;
}

// Before a substep of parity cur: its copy of the table.  When nothing but
// the substep two back (same parity) has read that copy since it was last
// written, the copy is made on a side stream after that substep, beside the
// substep now running, and this one waits for it; a copy made between two
// substeps in stream order would leave the GPU idle for its round trip
// (uniforms change every frame: the hand, walls).
static cudaError_t upload_table_for_substep(World& w) {
    refresh_host_table(w);
    const int c = w.cur;
    if (!w.tbl_dirty[c]) return cudaSuccess;
    if (w.tbl_outside[c]) {
        const cudaError_t e = upload_copy(w, c, w.stream);
        if (e == cudaSuccess) w.tbl_outside[c] = false;
        return e;
    }
    cudaError_t e = cudaStreamWaitEvent(w.tbl_side, w.sub_done[c], 0);
    if (e == cudaSuccess) e = upload_copy(w, c, w.tbl_side);
    if (e == cudaSuccess) e = cudaEventRecord(w.tbl_ev, w.tbl_side);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(w.stream, w.tbl_ev, 0);
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
    if (e == cudaSuccess) e = cudaMemsetAsync(w.health + slot, 0, 4, w.stream);   // a new scene starts healthy
    if (e == cudaSuccess) e = world_upload_table(w);
    if (e != cudaSuccess) return e;
    if (n) {
        const WorldView v = w.view();
        k_extend<<<std::max(1u, std::min<uint32_t>(cdiv(h_total, 256), w.pos_blocks)), 256, 0, w.stream>>>(v, h_total);
        k_import<<<cdiv(n, 256), 256, 0, w.stream>>>(v, (uint32_t)slot, h_total, pos, vel, aff, mass,
                                                     w.posm[w.cur], w.velid[w.cur], w.aff[w.cur], n);
        k_set_total<<<1, 1, 0, w.stream>>>(w.ctrl, h_total + n);
        w.launches += 3;
        w.tbl_outside[w.cur] = true;
        // the other positions keep the ranks G2P counted: count only the new
        // ones (before any count, the next substep counts everything)
        if (w.counted) {
            k_count_range<<<std::min<uint32_t>(cdiv(n, 256), w.pos_blocks), 256, 0, w.stream>>>(v, h_total,
                                                                                             h_total + n);
            w.launches++;
        }
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

cudaError_t world_read_health(World& w, int slot, uint32_t* flags, bool clear) {
    *flags = 0;
    if (slot < 0 || slot >= (int)w.scene_cap) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemcpyAsync(flags, w.health + slot, 4, cudaMemcpyDeviceToHost, w.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(w.stream);
    if (e == cudaSuccess && clear && *flags) e = cudaMemsetAsync(w.health + slot, 0, 4, w.stream);
    return e;
}

cudaError_t world_remove_scene(World& w, int slot) {
    if (slot < 0 || slot >= (int)w.scene_cap || !w.scenes[slot].live) return cudaErrorInvalidValue;
    SceneRec& r = w.scenes[slot];
    const WorldView v = w.view();
    if (r.n) {
        k_remove<<<w.pos_blocks, 256, 0, w.stream>>>(v, w.velid[w.cur], r.id_base, r.n);
        w.launches++;
        w.tbl_outside[w.cur] = true;
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
    if (e == cudaSuccess) e = cudaMemsetAsync(w.vel4 + r.cell_base, 0, (size_t)r.G * 16, w.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.tile_flags + r.tile_base, 0, (size_t)r.ntiles * 4, w.stream);
    // the counts G2P left in the scene's cells: the other scenes' counts and
    // ranks stay valid, so no recount is needed
    if (e == cudaSuccess) e = cudaMemsetAsync(w.cell_count + r.cell_base, 0, (size_t)r.G * 4, w.stream);
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
    w.tbl_outside[w.cur] = true;
    return cudaGetLastError();
}

// Enqueues one substep of all scenes on w.stream.  ds: the single-scene owner
// (its diffuse update runs when enabled, its profiler times the phases; null
// in a graph capture without diffuse, and for batches); ro: the owner's
// reference-layout mirrors.
// tail_in: ds's deferred diffuse tail of the previous substep runs on its side
// stream beside this substep's first passes; defer: this substep's tail is
// left pending (else it runs at the end, in stream order).
static cudaError_t enqueue_substep(World& w, Scene* ds, const RefOut& ro, bool tail_in, bool defer) {
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
        dv.group_counts = ds->diffuse.block_counts;
        gen_dev = ds->diffuse.gen_dev;
    }
    Scene* prof = ds;
    cudaError_t e;
    if (tail_in) {
        // DiffuseGPU.step of the previous substep (spawn pass, ADVECT, kill pass)
        // reads the pool, the free list, vel4 and its own copy of the uniforms,
        // none of which the binning, P2G_MASS, DECODE_MASS or P2G_MOM touch
        DiffuseState& d = ds->diffuse;
        e = cudaEventRecord(d.fork_ev, st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(d.side, d.fork_ev, 0);
        if (e == cudaSuccess) e = launch_diffuse(*ds, false, d.tail_P, d.tail_W, d.side);
        if (e == cudaSuccess) e = cudaEventRecord(d.join_ev, d.side);
        if (e != cudaSuccess) return e;
        d.tail_pending = false;
    }
    {
        Phase ph(prof, MPM_PHASE_SORT);
        if (!w.counted) {
            // nothing counted yet (a new world, or positions edited in place): count all
            e = cudaMemsetAsync(w.cell_count, 0, ((size_t)w.cell_cap + 1) * 4, st);
            if (e != cudaSuccess) return e;
            k_count<<<nposb, 256, 0, st>>>(v);
            w.launches++;
        }
        k_tiles_occ<<<ntb, 256, 0, st>>>(v);
        if (v.ntiles <= kFoldTiles) {
            // the last binning block builds the grid list and scans the tiles
            k_bin_cells<<<w.bin_blocks, kTileCells, 0, st>>>(v, gen_dev, 1);
            w.launches += 1;
        } else {
            k_bin_cells<<<w.bin_blocks, kTileCells, 0, st>>>(v, gen_dev, 0);
            k_tiles_grid<<<ntb, 256, 0, st>>>(v);
            k_tile_scan_local<<<v.ngroups, 1024, 0, st>>>(v);
            k_tile_scan_top<<<1, 1024, 0, st>>>(v, gen_dev);
            w.launches += 4;
        }
        k_tile_finish<<<w.bin_blocks, kTileCells, 0, st>>>(v);
        k_scatter<<<nposb, 256, 0, st>>>(v);
        w.launches += 3;
    }
    {
        Phase ph(prof, MPM_PHASE_P2G_MASS);
        if (w.chunk == kChunkSmall)
            k_p2g_mass_chunks<kChunkSmall><<<w.item_blocks, kChunkThreads, 0, st>>>(v, w.posm[cur], cm);
        else
            k_p2g_mass_chunks<kChunk><<<w.item_blocks, kChunkThreads, 0, st>>>(v, w.posm[cur], cm);
        w.launches++;
    }
    {
        Phase ph(prof, MPM_PHASE_DECODE_MASS);
        k_decode_tiles<<<w.grid_blocks, 256, 0, st>>>(v, cm, w.cmf);
        w.launches++;
    }
    {
        Phase ph(prof, MPM_PHASE_P2G_MOM);
        if (w.chunk == kChunkSmall)
            k_p2g_mom_chunks<kChunkSmall><<<w.item_blocks, kChunkThreads, 0, st>>>(v, w.posm[cur], w.velid[cur],
                                                                                 w.aff[cur], w.cmf, mv, w.dens);
        else
            k_p2g_mom_chunks<kChunk><<<w.item_blocks, kChunkThreads, 0, st>>>(v, w.posm[cur], w.velid[cur],
                                                                            w.aff[cur], w.cmf, mv, w.dens);
        w.launches++;
    }
    // the tail's ADVECT reads vel4 and its spawn pass the spawn bits that
    // UPDATE_GRID and G2P are about to rewrite
    if (tail_in) {
        e = cudaStreamWaitEvent(st, ds->diffuse.join_ev, 0);
        if (e != cudaSuccess) return e;
    }
    {
        Phase ph(prof, MPM_PHASE_UPDATE_GRID);   // includes APPLY_HAND
        k_update_tiles<<<w.grid_blocks, 256, 0, st>>>(v, cm, mv, w.mvf, w.vel4, cm_n, mv_n);
        w.launches++;
    }
    // (the spawn bits and group counts G2P adds to were cleared by the
    // previous substep's kill pass)
    {
        Phase ph(prof, MPM_PHASE_G2P);
        if (w.chunk == kChunkSmall)
            k_g2p_chunks<kChunkSmall><<<w.item_blocks, kChunkThreads, 0, st>>>(v, w.posm[cur], w.velid[cur], w.vel4,
                                                                             w.cmf, w.posm[nxt], w.velid[nxt],
                                                                             w.aff[nxt], dv, ro);
        else
            k_g2p_chunks<kChunk><<<w.item_blocks, kChunkThreads, 0, st>>>(v, w.posm[cur], w.velid[cur], w.vel4,
                                                                        w.cmf, w.posm[nxt], w.velid[nxt],
                                                                        w.aff[nxt], dv, ro);
        w.launches++;
    }
    w.cur = nxt;
    w.gbuf ^= 1;
    w.cm_current = cm;
    w.dens_valid = true;
    w.counted = true;   // G2P ranked every new position in its cell
    w.pos_bound = w.n_total;   // the layout after a substep is dense
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (dv.enabled) {
        ds->diffuse.seed += 1u;   // mirrors the device-side bump in k_tile_scan_top
        const SceneDesc* sd_dev = w.scenes_dev(cur) + dv.scene;
        if (defer) {
            // this substep's uniforms for its deferred tail (the scene table may
            // be rewritten before the tail runs)
            DiffuseState& d = ds->diffuse;
            e = cudaMemcpyAsync(d.tail_P, &sd_dev->P, sizeof(mpm_params), cudaMemcpyDeviceToDevice, st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(d.tail_W, &sd_dev->W, sizeof(mpm_wall_params), cudaMemcpyDeviceToDevice, st);
            if (e == cudaSuccess) d.tail_pending = true;
        } else {
            e = launch_diffuse(*ds, false, &sd_dev->P, &sd_dev->W);
        }
    }
    return e;
}

cudaError_t world_flush_diffuse(Scene& s) {
    DiffuseState& d = s.diffuse;
    if (!d.tail_pending) return cudaSuccess;
    d.tail_pending = false;
    return launch_diffuse(s, false, d.tail_P, d.tail_W, s.stream);
}

cudaError_t world_substep(World& w, Scene* ds, bool use_graph) {
    RefOut ro{};
    if (ds && ds->mirror && ds->world_slot >= 0) {
        ro.enabled = 1;
        ro.scene = (uint32_t)ds->world_slot;
        ro.pos = ds->pos;
        ro.vel = ds->vel;
        ro.dens = ds->dens;
    }
    // chunk size: one pass per chunk when full-size chunks would leave blocks
    // of the chunk kernels idle (a new size means new captured graphs)
    const uint32_t chunk = (uint64_t)w.n_total < (uint64_t)w.item_blocks * kChunk ? kChunkSmall : kChunk;
    if (chunk != w.chunk) {
        w.chunk = chunk;
        w.generation++;
    }
    cudaError_t e = upload_table_for_substep(w);
    if (e != cudaSuccess) return e;
    const int parity = w.cur;   // the table copy this substep reads
    const bool diffuse = ds && ds->diffuse.enabled;
    const bool profiling = ds && ds->profile;
    if (profiling && diffuse && ds->diffuse.tail_pending) {
        // phases are timed on the scene stream: no tail beside them
        e = world_flush_diffuse(*ds);
        if (e != cudaSuccess) return e;
    }
    const bool tail_in = diffuse && ds->diffuse.tail_pending;
    const bool defer = diffuse && !profiling;
    // a substep that must recount runs eagerly; the captured graphs never count
    if (!use_graph || profiling || !w.counted) {
        e = enqueue_substep(w, ds, ro, tail_in, defer);
        if (e == cudaSuccess) e = cudaEventRecord(w.sub_done[parity], w.stream);
        return e;
    }
    // the diffuse update joins the graph: its kernels read the uniforms from
    // device copies and the advect parameters from a device copy
    Scene* dsc = diffuse ? ds : nullptr;
    const int p = 2 * w.cur + (tail_in ? 1 : 0);   // cur and gbuf flip together: graphs per parity
    const bool mirror = ro.enabled != 0;
    if (!w.graph[p] || w.graph_gen[p] != w.generation || w.graph_diffuse[p] != diffuse ||
        w.graph_mirror[p] != mirror) {
        if (w.graph[p]) {
            cudaGraphExecDestroy(w.graph[p]);
            w.graph[p] = nullptr;
        }
        const int cur0 = w.cur, gbuf0 = w.gbuf;
        int32_t* cmc0 = w.cm_current;
        const bool dv0 = w.dens_valid;
        const uint64_t l0 = w.launches;
        const uint64_t sl0 = dsc ? dsc->launches : 0;
        const uint32_t seed0 = dsc ? dsc->diffuse.seed : 0;
        const uint64_t passes0 = dsc ? dsc->diffuse.passes : 0;
        const bool pending0 = dsc ? dsc->diffuse.tail_pending : false;
        const bool written0 = dsc ? dsc->diffuse.top_written : false;
        cudaGraph_t g = nullptr;
        e = cudaStreamBeginCapture(w.stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        const cudaError_t e2 = enqueue_substep(w, dsc, ro, tail_in, defer);
        e = cudaStreamEndCapture(w.stream, &g);
        if (e2 != cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&w.graph[p], g, 0);
        if (g) cudaGraphDestroy(g);
        // capture only recorded the work: restore the host state the enqueue advanced
        w.graph_kernels[p] = w.launches - l0 + (dsc ? dsc->launches - sl0 : 0);
        w.cur = cur0;
        w.gbuf = gbuf0;
        w.cm_current = cmc0;
        w.dens_valid = dv0;
        w.launches = l0;
        if (dsc) {
            dsc->launches = sl0;
            dsc->diffuse.seed = seed0;
            dsc->diffuse.passes = passes0;
            dsc->diffuse.tail_pending = pending0;
            dsc->diffuse.top_written = written0;
        }
        if (e != cudaSuccess) {
            w.graph[p] = nullptr;
            return e;
        }
        w.graph_gen[p] = w.generation;
        w.graph_diffuse[p] = diffuse;
        w.graph_mirror[p] = mirror;
    }
    e = cudaGraphLaunch(w.graph[p], w.stream);
    if (e == cudaSuccess) e = cudaEventRecord(w.sub_done[parity], w.stream);
    if (e != cudaSuccess) return e;
    // host mirror of what the graph does
    w.launches += w.graph_kernels[p];
    if (dsc) {
        dsc->diffuse.seed += 1u;
        if (tail_in) {
            dsc->diffuse.passes += 1u;   // the previous substep's kill pass ran in the graph
            dsc->diffuse.top_written = false;
        }
        dsc->diffuse.tail_pending = true;   // this substep's tail waits for the next one
    }
    w.pos_bound = w.n_total;   // the layout after a substep is dense
    w.cm_current = w.grid_i32[w.gbuf];
    w.cur ^= 1;
    w.gbuf ^= 1;
    w.dens_valid = true;
    return cudaSuccess;
}

}  // namespace mpm
