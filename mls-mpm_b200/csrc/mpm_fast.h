// mpm_fast.h — state and launchers of the binned, item-major engine.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/mpm_types.h"

namespace mpm {

// Grid tile (cells) used by the sparse grid passes and the binning.
constexpr int kTileX = 16, kTileY = 8, kTileZ = 8;
constexpr int kTileCells = kTileX * kTileY * kTileZ;   // 1024: one thread per cell in k_bin_cells

// A cell's particles are split into work items of at most kMaxL particles;
// items are grouped by length into buckets 1..kMaxL so that the 32 lanes of a
// warp always run the same number of iterations.
constexpr int kMaxL = 16;
// Positions lost to padding the last warp of each bucket: 31 * (1 + ... + kMaxL).
constexpr uint32_t kPosSlack = 31u * (kMaxL * (kMaxL + 1) / 2) + 64u;
constexpr uint32_t kHole = 0xFFFFFFFFu;   // key / id of a padding position

// Small device-side control block.  The first kCtrlZeroBytes are cleared at
// the start of every substep.
struct Ctrl {
    uint32_t n_occ, n_grid, pad0, pad1;
    uint32_t tail_cnt[kMaxL + 1];            // items of overpacked cells per length (unordered)
    uint32_t pad2[64 - 4 - (kMaxL + 1)];
    // persistent
    uint32_t bucket_reg[kMaxL + 2];          // ordered items per length (one per cell with 1..kMaxL particles)
    uint32_t bucket_cnt[kMaxL + 2];          // ordered + tail items per length
    uint32_t item_off[kMaxL + 2];            // first padded item index of each bucket
    uint32_t pos_off[kMaxL + 2];             // first position of each bucket
    uint32_t total_items, total_pos, prev_total_pos, pad3;
};
constexpr size_t kCtrlZeroBytes = 64 * 4;

// Everything the device kernels of the binned engine need (passed by value).
struct FastView {
    uint32_t n;                // particles
    uint32_t npos;             // capacity of the position space
    uint32_t X, Y, Z;
    uint64_t G;
    uint32_t ntx, nty, ntz, ntiles;
    uint32_t cap_off[kMaxL + 2];   // start of each bucket's item list in bucket_items
    uint32_t* cell_count;      // G + 1, zero outside binning
    uint4* cell_info;          // G: (L | Llast<<8 | q<<16, first item idx, last item idx, 0)
    uint32_t* bucket_items;    // cell of each item, per bucket
    uint32_t* key;             // npos: binning cell of each position of the current state (kHole)
    uint32_t* rank;            // npos: rank within the cell
    uint32_t* perm;            // npos: position -> position of the previous layout
    uint32_t* tile_flags;      // ntiles
    uint32_t* tile_occ;        // ntiles: 1 if the tile holds particles this substep
    uint32_t* tile_hist;       // kMaxL x ntiles: ordered items per (length, tile)
    uint32_t* tile_base;       // kMaxL x ntiles: exclusive scan of tile_hist over tiles
    uint32_t* tile_occ_list;   // ntiles
    uint32_t* tile_grid_list;  // ntiles
    Ctrl* ctrl;
    float* dens;               // npos, layout of the last substep
};

struct DiffuseView {
    int enabled;
    mpm_gen_params gen;
    mpm_diffuse_particle* staging;   // by particle id
    uint32_t* spawn_bits;            // by particle id
    const float* cmf;
};

struct FastEngine {
    uint32_t X = 0, Y = 0, Z = 0;
    uint64_t G = 0;
    uint32_t ntx = 0, nty = 0, ntz = 0, ntiles = 0;
    uint32_t capacity = 0, n = 0, npos = 0;
    uint32_t item_blocks = 0;       // grid size of the item kernels
    uint32_t grid_blocks = 0;       // grid size of the tile passes
    uint32_t bin_blocks = 0;        // grid size of the binning kernel
    uint32_t cap_off[kMaxL + 2] = {};
    int gbuf = 0;                   // i32 grid buffer the next substep accumulates into
    bool dens_valid = false;
    uint64_t launches = 0;

    // posm/velid/aff[cur]: the state after the last substep (in that substep's layout)
    int cur = 0;
    float4* posm[2] = {nullptr, nullptr};    // (x, y, z, mass)
    float4* velid[2] = {nullptr, nullptr};   // (vx, vy, vz, id bits)
    float* aff[2] = {nullptr, nullptr};      // 9 planes of npos floats
    float* dens = nullptr;
    uint32_t* cell_count = nullptr;
    uint4* cell_info = nullptr;
    uint32_t* bucket_items = nullptr;
    uint32_t* key = nullptr;
    uint32_t* rank = nullptr;
    uint32_t* perm = nullptr;
    uint32_t* tile_flags = nullptr;
    uint32_t* tile_occ = nullptr;
    uint32_t* tile_hist = nullptr;
    uint32_t* tile_base = nullptr;
    uint32_t* tile_occ_list = nullptr;
    uint32_t* tile_grid_list = nullptr;
    Ctrl* ctrl = nullptr;
    int32_t* grid_i32[2] = {nullptr, nullptr};   // each [cm: G][mv: 3G]
    int32_t* cm_current = nullptr;               // buffer holding the last substep's P2G sums

    FastView view() const {
        FastView v;
        v.n = n;
        v.npos = npos;
        v.X = X; v.Y = Y; v.Z = Z; v.G = G;
        v.ntx = ntx; v.nty = nty; v.ntz = ntz; v.ntiles = ntiles;
        for (int b = 0; b < kMaxL + 2; ++b) v.cap_off[b] = cap_off[b];
        v.cell_count = cell_count; v.cell_info = cell_info; v.bucket_items = bucket_items;
        v.key = key; v.rank = rank; v.perm = perm;
        v.tile_flags = tile_flags; v.tile_occ = tile_occ; v.tile_hist = tile_hist; v.tile_base = tile_base; v.tile_occ_list = tile_occ_list; v.tile_grid_list = tile_grid_list;
        v.ctrl = ctrl; v.dens = dens;
        return v;
    }
};

struct Scene;

cudaError_t fast_alloc(FastEngine& f, uint32_t X, uint32_t Y, uint32_t Z, uint32_t capacity, int device);
void fast_free(FastEngine& f);
cudaError_t fast_import(FastEngine& f, const float4* pos, const float4* vel, const float* aff, const float* mass,
                        uint32_t n, cudaStream_t st);
cudaError_t fast_export(FastEngine& f, float4* pos, float4* vel, float* aff, float* mass, float* dens,
                        cudaStream_t st);
cudaError_t fast_substep(Scene& s);

}  // namespace mpm
