// mpm_fast.h — state and launchers of the binned, item-major engine.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/mpm_types.h"

namespace mpm {

// Grid tile (cells) used by the sparse grid passes and the binning.
constexpr int kTileX = 16, kTileY = 8, kTileZ = 8;
constexpr int kTileCells = kTileX * kTileY * kTileZ;   // 1024: one thread per cell in k_bin_tiles

// counters[] slots (device), zeroed at the start of every substep
constexpr int kCntOcc = 0;      // occupied tiles listed
constexpr int kCntGrid = 1;     // grid tiles listed
constexpr int kCntSorted = 2;   // particles placed
constexpr int kCntItems = 3;    // work items emitted

// Everything the device kernels of the binned engine need (passed by value).
struct FastView {
    uint32_t n;                // particles in the state
    uint32_t X, Y, Z;
    uint64_t G;
    uint32_t ntx, nty, ntz, ntiles;
    uint32_t* cell_count;      // G + 1, zero outside binning
    uint32_t* cell_start;      // G
    uint32_t* key;             // N: binning cell of each slot of the current state
    uint32_t* rank;            // N: rank within the cell
    uint32_t* perm;            // N: sorted position -> slot of the current state
    uint4* items;              // N: (cell, begin, len, 0)
    uint32_t* tile_flags;      // ntiles
    uint32_t* tile_occ_list;   // ntiles
    uint32_t* tile_grid_list;  // ntiles
    uint32_t* counters;        // 16
    float* dens;               // N, sorted order of the last substep
};

struct DiffuseView {
    int enabled;
    mpm_gen_params gen;
    mpm_diffuse_particle* staging;   // by particle id
    uint32_t* spawn_bits;            // by particle id
    const float* cmf;
};

struct HandLaunch {
    int active;
    mpm_hand_params h;
    int32_t dims[3];
    // tile marking box (cells); x0 > x1 when inactive
    int32_t x0, y0, z0, x1, y1, z1;
};

struct FastEngine {
    uint32_t X = 0, Y = 0, Z = 0;
    uint64_t G = 0;
    uint32_t ntx = 0, nty = 0, ntz = 0, ntiles = 0;
    uint32_t capacity = 0, n = 0;
    uint32_t chunk = 8;             // max particles per work item (tuned)
    uint32_t item_blocks = 0;       // grid size of the item kernels
    uint32_t grid_blocks = 0;       // grid size of the tile passes
    uint32_t bin_blocks = 0;        // grid size of the binning kernel
    int cur = 0;                    // current particle state buffer
    int gbuf = 0;                   // i32 grid buffer the next substep accumulates into
    bool dens_valid = false;
    uint64_t launches = 0;

    float4* posm[2] = {nullptr, nullptr};
    float4* velid[2] = {nullptr, nullptr};
    float* aff[2] = {nullptr, nullptr};
    float* dens = nullptr;
    uint32_t* cell_count = nullptr;
    uint32_t* cell_start = nullptr;
    uint32_t* key = nullptr;
    uint32_t* rank = nullptr;
    uint32_t* perm = nullptr;
    uint4* items = nullptr;
    uint32_t* tile_flags = nullptr;
    uint32_t* tile_occ_list = nullptr;
    uint32_t* tile_grid_list = nullptr;
    uint32_t* counters = nullptr;
    int32_t* grid_i32[2] = {nullptr, nullptr};   // each [cm: G][mv: 3G]
    int32_t* cm_current = nullptr;               // buffer holding the last substep's P2G sums

    FastView view() const {
        FastView v;
        v.n = n;
        v.X = X; v.Y = Y; v.Z = Z; v.G = G;
        v.ntx = ntx; v.nty = nty; v.ntz = ntz; v.ntiles = ntiles;
        v.cell_count = cell_count; v.cell_start = cell_start; v.key = key; v.rank = rank; v.perm = perm;
        v.items = items; v.tile_flags = tile_flags; v.tile_occ_list = tile_occ_list;
        v.tile_grid_list = tile_grid_list; v.counters = counters; v.dens = dens;
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
